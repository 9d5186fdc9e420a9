// Batched log-Pfaffian (blocked Parlett-Reid LTL^T with partial pivoting), the pairing
// gather, and the combination of symmetry images.
//
// One CTA (256 threads) per antisymmetric n x n matrix, n even, n <= 256; FP32 (two CTAs per
// SM at n = 224) or FP64 (one CTA per SM, used to recompute ill-conditioned items).  The strict
// lower triangle lives in shared memory (row i at offset i (i - 1) / 2) and thread t owns
// physical row t.  A pivot does not move data: it swaps the logical labels of two physical rows,
// so an elimination step costs two block barriers.  Panel columns are formed lazily (stored
// column plus the panel's rank-2 terms U V^T - V U^T); at the end of a panel of NB steps the
// active rows are listed in physical order and the trailing triangle receives the rank-2NB
// update, one warp per row and one lane per column, the column's U/V in registers and the row's
// U/V broadcast.  The Pfaffian is the product of the pivots A[k, k+1] times the parity of the
// relabelling, accumulated in FP64 as mantissa and exponent.  The ratio of the largest to the
// smallest pivot magnitude estimates the condition number; above cond_tau the item is flagged
// NH_FLAG_GROWTH (near-nodal) for the FP64 recompute.
//
// Replaces fermix.slogpf (code/backflow/models.py:210) and, in the gather mode, the Pallas
// pairing kernel pfsbp_pairing_fwd (code/backflow/pf_kernel.py:156-190) whose formula it
// follows: F[p, q] = sum_a (Y[p, a] Y[q, a]) Wt[2 s_p + s_q, r(p, q), a] with the product of
// the features formed first, so that F[q, p] = -F[p, q] holds bit for bit.
#include <math.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "nh_cnn_item.cuh"
#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kWarps = kNumThreads / 32;

template <typename T>
struct Vec;
template <>
struct Vec<float> {
  static constexpr int k = 4;
};
template <>
struct Vec<double> {
  static constexpr int k = 2;
};

__device__ __forceinline__ float tfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double tfma(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ void ldg16(const float* p, float* o) {
  float4 v = __ldg(reinterpret_cast<const float4*>(p));
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}
__device__ __forceinline__ void ldg16(const double* p, double* o) {
  double2 v = __ldg(reinterpret_cast<const double2*>(p));
  o[0] = v.x;
  o[1] = v.y;
}
__device__ __forceinline__ void lds16(const float* p, float* o) {
  float4 v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}
__device__ __forceinline__ void lds16(const double* p, double* o) {
  double2 v = *reinterpret_cast<const double2*>(p);
  o[0] = v.x;
  o[1] = v.y;
}

struct PfArgs {
  int n;
  int mode;  // 0: F dense FP32 (items, n, n) in global memory; 1: gather from Y / idx / Wt
  const float* F;
  const void* Y;       // (slots, n, D) of T
  const int32_t* idx;  // (slots, n)
  const void* Wt;      // (4, N, D) of T
  int Lx, Ly;
  const int32_t* count_dev;  // work count on the device (times count_mult) or null
  int count_mult;
  int n_slots;               // host count, upper bound when count_dev is set
  const int32_t* slot_item;  // slot -> item, null: identity
  const float* item_sign;    // (items,) or null
  float* sign;               // (items,)
  double* logabs;            // (items,)
  int32_t* flags;            // (items,) or null
  double cond_tau;           // flag NH_FLAG_GROWTH when max|piv| > cond_tau min|piv| (0: off)
  int flag_or;               // OR-ed into every written flag
  void* tri;                 // large n: per-CTA lower triangles of T in global memory
  uint16_t* perm;            // or null: per item, logical -> physical row, then the parity
  double refine_tau;         // set kFlagNeedRefine when max|piv| > refine_tau min|piv| (0: off)
  float* ratio;              // or null: per item, max|piv| / min|piv| (inf for a zero pivot)
  // mode 2 (features in the kernel): item = c * G + g of the configuration list; the CNN's
  // occupied rows at byte y_off and their modes at idx_off of shared memory; rows >= tail_row
  // of the triangle overlap the rows and are gathered through registers first.
  ConfigList cl;
  const float* cnn_w;   // packed weights [l][ci][tap][co]
  const float* cnn_b;
  int C, layers;
  int y_off, idx_off, tail_row;
  float* item_sign_out;  // (items,) the item signs the CNN phase computes
  int32_t* queue;        // mode 2: work counter (zero before the launch)
};

// Shared-memory layout of the in-kernel CNN phase (mode 2): simg, occl (2N ints each), scan
// scratch (4 Lx + 32 ints), activation planes A and B (C (N + 1) floats each), staged weights
// (C * C * 9) and biases (C).  Returns the end of the activation planes; *end the whole extent.
__host__ __device__ inline size_t cnn_phase_layout(int N, int C, int Lx, size_t* end) {
  const size_t ints = 4 * (size_t)N + 4 * Lx + 32;
  const size_t act0 = (sizeof(int) * ints + 15) & ~(size_t)15;
  const size_t act_end = act0 + sizeof(float) * 2 * (size_t)C * (N + 1);
  const size_t w0 = (act_end + 15) & ~(size_t)15;
  *end = w0 + sizeof(float) * ((size_t)C * C * 9 + C);
  return act_end;
}

// A mode m (spin s = m >= N, site x Ly + y) packed as s << 16 | x << 8 | y for the gather from
// shared memory (no division per element).
__device__ __forceinline__ int pack_mode(int m, int N, int Ly) {
  const int s = m >= N ? 1 : 0, site = m - s * N, x = site / Ly;
  return (s << 16) | (x << 8) | (site - x * Ly);
}

// F[p][q] (p > q) of the item from occupied rows Y (n, D, chunk-swizzled: swz_index) and packed
// modes (pack_mode) in shared memory, the same arithmetic as pair_value:
// sum_a (Y[p, a] Y[q, a]) Wt[2 s_p + s_q, r(p, q), a] in order of a.
template <int D>
__device__ __forceinline__ float pair_smem(const float* yp, int cp, const float* __restrict__ Ys,
                                           const int* __restrict__ ids, int q, int N, int Lx,
                                           int Ly, const float* __restrict__ Wt) {
  const int cq = ids[q];
  int dx = ((cp >> 8) & 0xff) - ((cq >> 8) & 0xff), dy = (cp & 0xff) - (cq & 0xff);
  dx += dx < 0 ? Lx : 0;
  dy += dy < 0 ? Ly : 0;
  const float* wrow = Wt + ((size_t)(2 * (cp >> 16) + (cq >> 16)) * N + dx * Ly + dy) * D;
  float acc = 0.0f;
#pragma unroll
  for (int a0 = 0; a0 < D; a0 += 4) {
    const float4 w = __ldg(reinterpret_cast<const float4*>(wrow + a0));
    const float4 v = *reinterpret_cast<const float4*>(Ys + swz_index<float, D>(q, a0));
    acc = fmaf(yp[a0] * v.x, w.x, acc);
    acc = fmaf(yp[a0 + 1] * v.y, w.y, acc);
    acc = fmaf(yp[a0 + 2] * v.z, w.z, acc);
    acc = fmaf(yp[a0 + 3] * v.w, w.w, acc);
  }
  return acc;
}

__device__ __forceinline__ int tri_off(int i) { return (i * (i - 1)) >> 1; }

// Pivot-search key of a magnitude: FP32, rounded up so that no non-zero value becomes zero.
__device__ __forceinline__ float to_key_float(float x) { return x; }
__device__ __forceinline__ float to_key_float(double x) { return __double2float_ru(x); }

template <typename T>
__device__ __forceinline__ T aval(const T* Lw, int i, int j) {
  return i > j ? Lw[tri_off(i) + j] : (i < j ? -Lw[tri_off(j) + i] : T(0));
}

template <typename T, int D>
__device__ __forceinline__ T pair_value(const T* yp, int sp, int xp, int ypos,
                                        const T* __restrict__ Yq, int mq, int N, int Lx, int Ly,
                                        const T* __restrict__ Wt) {
  const int sq = mq >= N ? 1 : 0;
  const int siteq = mq - sq * N;
  const int xq = siteq / Ly, yq = siteq - xq * Ly;
  int dx = xp - xq, dy = ypos - yq;
  dx += dx < 0 ? Lx : 0;
  dy += dy < 0 ? Ly : 0;
  const T* wrow = Wt + ((size_t)(2 * sp + sq) * N + dx * Ly + dy) * D;
  T acc = T(0);
#pragma unroll
  for (int a0 = 0; a0 < D; a0 += Vec<T>::k) {
    T w[Vec<T>::k], q[Vec<T>::k];
    ldg16(wrow + a0, w);
    ldg16(Yq + a0, q);
#pragma unroll
    for (int k = 0; k < Vec<T>::k; ++k) acc = tfma(yp[a0 + k] * q[k], w[k], acc);
  }
  return acc;
}

template <typename T, int D, int WARPS = kWarps>
__device__ void gather_lower(T* Lw, int n, const T* __restrict__ Y, const int32_t* __restrict__ idx,
                             const T* __restrict__ Wt, int Lx, int Ly) {
  const int N = Lx * Ly;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int p = wid; p < n; p += WARPS) {
    const int mp = __ldg(idx + p);
    const int sp = mp >= N ? 1 : 0;
    const int sitep = mp - sp * N;
    const int xp = sitep / Ly, ypos = sitep - xp * Ly;
    T yp[D];
#pragma unroll
    for (int a0 = 0; a0 < D; a0 += Vec<T>::k) ldg16(Y + (size_t)p * D + a0, yp + a0);
    T* row = Lw + tri_off(p);
    int q = lane;
    for (; q + 32 < p; q += 64) {  // two independent elements per lane in flight
      const int mq0 = __ldg(idx + q), mq1 = __ldg(idx + q + 32);
      const T v0 = pair_value<T, D>(yp, sp, xp, ypos, Y + (size_t)q * D, mq0, N, Lx, Ly, Wt);
      const T v1 = pair_value<T, D>(yp, sp, xp, ypos, Y + (size_t)(q + 32) * D, mq1, N, Lx, Ly, Wt);
      row[q] = v0;
      row[q + 32] = v1;
    }
    if (q < p)
      row[q] = pair_value<T, D>(yp, sp, xp, ypos, Y + (size_t)q * D, __ldg(idx + q), N, Lx, Ly, Wt);
  }
}

// Load phase of modes 2 and 3: the item's occupied rows Y (n, D) and packed modes in shared memory
// (mode 2: the CNN of its configuration in shared memory, write_occupied_rows, item sign to
// item_sign_out; mode 3: copied from the global rows a.Y / a.idx of slot), then the gather of
// the lower triangle from them.  Rows of the triangle that overlap Y (tail_row on) are computed
// into registers first and stored after a barrier.
constexpr int kTailRegs = 16;

template <int D>
__device__ void features_to_smem(const PfArgs& a, int item, unsigned char* smem, float* Ys,
                                 int* ids);
template <int D>
__device__ void gather_from_rows(const PfArgs& a, float* Lw, const float* Ys, const int* ids);

template <int D>
__device__ void rows_and_gather(const PfArgs& a, int item, int slot, float* Lw,
                                unsigned char* smem) {
  const int n = a.n;
  const int tid = threadIdx.x;
  float* Ys = reinterpret_cast<float*>(smem + a.y_off);
  int* ids = reinterpret_cast<int*>(smem + a.idx_off);
  if (a.mode == 3) {
    const float4* src = reinterpret_cast<const float4*>(static_cast<const float*>(a.Y) +
                                                        (size_t)slot * n * D);
    constexpr int K = D / 4;  // 16-byte chunks per row, stored swizzled (swz_index)
    const int nv = n * K;
    for (int v0 = tid; v0 < nv; v0 += 4 * kNumThreads) {
      float4 buf[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (v0 + u * kNumThreads < nv) buf[u] = __ldg(src + v0 + u * kNumThreads);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int v = v0 + u * kNumThreads, row = v / K;
        if (v < nv) reinterpret_cast<float4*>(Ys)[row * K + ((v % K) ^ swz_key(row, K))] = buf[u];
      }
    }
    const int N = a.Lx * a.Ly;
    for (int p = tid; p < n; p += kNumThreads)
      ids[p] = pack_mode(__ldg(a.idx + (size_t)slot * n + p), N, a.Ly);
    __syncthreads();
  } else {
    features_to_smem<D>(a, item, smem, Ys, ids);
  }
  gather_from_rows<D>(a, Lw, Ys, ids);
}

template <int D>
__device__ void features_to_smem(const PfArgs& a, int item, unsigned char* smem, float* Ys,
                                 int* ids) {
  const int N = a.Lx * a.Ly, C = a.C, M2 = 2 * N, NS = N + 1;
  const int G = a.cl.G;
  const int c = item / G, g = item - c * G;
  const int smp = a.cl.sample ? a.cl.sample[c] : c;
  const int fr = a.cl.from ? a.cl.from[c] : -1;
  const int to = a.cl.from ? a.cl.to[c] : -1;
  const int8_t* base = a.cl.spins + (int64_t)smp * M2;
  int* simg = reinterpret_cast<int*>(smem);
  int* occl = simg + M2;
  int* wbuf = occl + M2;
  size_t cnn_end;
  const size_t act_end = cnn_phase_layout(N, C, a.Lx, &cnn_end);
  const size_t act0 = act_end - sizeof(float) * 2 * (size_t)C * NS;
  float* actA = reinterpret_cast<float*>(smem + act0);
  float* actB = actA + C * NS;
  float* wsm = reinterpret_cast<float*>(smem + ((act_end + 15) & ~(size_t)15));
  float* bsm = wsm + C * C * 9;
  const float* in = cnn_layers<float>(a.cnn_w, a.cnn_b, a.Lx, a.Ly, C, a.layers, base, fr, to,
                                      g, actA, actB, wsm, bsm, simg);
  const int d = C / 2;
  write_occupied_rows(simg, occl, wbuf, N, a.n, d, g, a.Lx, a.Ly, Ys, ids,
                      a.item_sign_out + item,
                      [&](int sg, int aa, int site) { return in[(sg * d + aa) * NS + site]; },
                      true);
  __syncthreads();
  for (int p = threadIdx.x; p < a.n; p += kNumThreads) ids[p] = pack_mode(ids[p], N, a.Ly);
  __syncthreads();
}

template <int D>
__device__ void gather_from_rows(const PfArgs& a, float* Lw, const float* Ys, const int* ids) {
  const int n = a.n, N = a.Lx * a.Ly;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const float* Wt = static_cast<const float*>(a.Wt);
  // rows below tail_row: straight into the triangle, warp <-> row, lane <-> two columns in flight
  for (int p = wid; p < a.tail_row; p += kNumThreads / 32) {
    float yp[D];
#pragma unroll
    for (int a0 = 0; a0 < D; a0 += 4) {
      const float4 v = *reinterpret_cast<const float4*>(Ys + swz_index<float, D>(p, a0));
      yp[a0] = v.x;
      yp[a0 + 1] = v.y;
      yp[a0 + 2] = v.z;
      yp[a0 + 3] = v.w;
    }
    const int mp = ids[p];
    float* row = Lw + ((p * (p - 1)) >> 1);
    int q = lane;
    for (; q + 32 < p; q += 64) {
      const float v0 = pair_smem<D>(yp, mp, Ys, ids, q, N, a.Lx, a.Ly, Wt);
      const float v1 = pair_smem<D>(yp, mp, Ys, ids, q + 32, N, a.Lx, a.Ly, Wt);
      row[q] = v0;
      row[q + 32] = v1;
    }
    if (q < p) row[q] = pair_smem<D>(yp, mp, Ys, ids, q, N, a.Lx, a.Ly, Wt);
  }
  if (a.tail_row < n) {
    // rows tail_row .. n-1 (E elements, at most kTailRegs per thread) through registers
    const int t0 = (a.tail_row * (a.tail_row - 1)) >> 1;
    const int E = ((n * (n - 1)) >> 1) - t0;
    float v[kTailRegs];
#pragma unroll
    for (int k = 0; k < kTailRegs; ++k) {
      const int e = tid + k * kNumThreads;
      v[k] = 0.0f;
      if (e < E) {
        int p = a.tail_row;
        while ((((p + 1) * p) >> 1) - t0 <= e) ++p;
        const int q = e - ((((p * (p - 1)) >> 1)) - t0);
        float yp[D];
#pragma unroll
        for (int a0 = 0; a0 < D; a0 += 4) {
          const float4 y4 = *reinterpret_cast<const float4*>(Ys + swz_index<float, D>(p, a0));
          yp[a0] = y4.x;
          yp[a0 + 1] = y4.y;
          yp[a0 + 2] = y4.z;
          yp[a0 + 3] = y4.w;
        }
        v[k] = pair_smem<D>(yp, ids[p], Ys, ids, q, N, a.Lx, a.Ly, Wt);
      }
    }
    __syncthreads();  // every read of Y is done
#pragma unroll
    for (int k = 0; k < kTailRegs; ++k) {
      const int e = tid + k * kNumThreads;
      if (e < E) Lw[t0 + e] = v[k];
    }
  }
}

// THREADS = 256: the lower triangle lives in shared memory (n <= 256).  THREADS = 1024 (large
// lattices, n <= 1024): one thread per row as well, the triangle in a per-CTA slice of global
// memory (a.tri; L2-resident up to n ~ 500), shared memory holding only the panel and the
// reduction slots.
template <typename T, int NB, int D, int THREADS = kNumThreads>
__global__ void __launch_bounds__(THREADS, THREADS > kNumThreads ? 1 : (sizeof(T) == 4 ? 2 : 1))
    pfaffian_kernel(PfArgs a) {
  static_assert(NB % Vec<T>::k == 0, "panel width must fill 16-byte vectors");
  constexpr int WARPS = THREADS / 32;
  constexpr bool kGlobalTri = THREADS > kNumThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int tri = tri_off(n);
  T* Lw;
  T* Us;  // (n, NB)
  if constexpr (kGlobalTri) {
    Lw = static_cast<T*>(a.tri) + (size_t)blockIdx.x * ((tri + 3) & ~3);
    Us = reinterpret_cast<T*>(smem_raw);
  } else {
    Lw = reinterpret_cast<T*>(smem_raw);
    Us = Lw + ((tri + 3) & ~3);
  }
  T* Vs = Us + n * NB;            // (n, NB)
  // FP32: the winner's signed value shares the key slot (its magnitude is the key); FP64 keeps
  // it separately.  pivs[k/2] = pivot A[k, k+1], negated when that step swapped labels.
  constexpr int kValSlots = sizeof(T) == 4 ? 0 : WARPS;
  T* rval = Vs + n * NB;                 // (warps, FP64 only) candidate signed value
  T* pivs = rval + kValSlots;            // (n / 2) signed pivots, multiplied at the end
  float* rkey = reinterpret_cast<float*>(pivs + ((n / 2 + 3) & ~3));
  int* rt = reinterpret_cast<int*>(rkey + WARPS);  // (warps) trailing update: ballot counts
  int* rlog = rt + WARPS;
  // (warps) packed pivot candidates over rkey and rt: |c| key + 1 (bits 63..32), 0xFFFF - row
  // (31..16), sign of c (15), logical label (14..0): the largest word is the largest |c|, ties
  // to the lowest row.
  unsigned long long* cand = reinterpret_cast<unsigned long long*>(rkey);
  int* alist = rlog + WARPS;                       // (n) active physical rows
  int* misc = alist + n;                            // [0] physical row of logical k, [1] item

  const int n_work = a.count_dev ? (*a.count_dev) * a.count_mult : a.n_slots;
  const T* Ybase = static_cast<const T*>(a.Y);
  const T* Wt = static_cast<const T*>(a.Wt);
  for (int slot = blockIdx.x;; slot += gridDim.x) {
    if (a.queue) {  // dynamic schedule: the next item comes off the work counter
      __syncthreads();
      if (tid == 0) misc[1] = atomicAdd(a.queue, 1);
      __syncthreads();
      slot = misc[1];
    }
    if (slot >= n_work) break;
    const int item = a.slot_item ? a.slot_item[slot] : slot;
    __syncthreads();
    if constexpr (sizeof(T) == 4 && THREADS == kNumThreads && D % 4 == 0) {
      if (a.mode >= 2) rows_and_gather<D>(a, item, slot, Lw, smem_raw);
    }
    if (a.mode == 0) {
      const float* F = a.F + (size_t)item * n * n;
      for (int i = wid; i < n; i += WARPS) {
        const float* src = F + (size_t)i * n;
        T* dst = Lw + tri_off(i);
        for (int j = lane; j < i; j += 32) dst[j] = T(__ldg(src + j));
      }
    } else if (a.mode == 1) {
      gather_lower<T, D, WARPS>(Lw, n, Ybase + (size_t)slot * n * D, a.idx + (size_t)slot * n,
                                Wt, a.Lx, a.Ly);
    }
    // Modes 2 and 3: the rows in shared memory can overlap the factorisation's scratch (misc
    // among it), so every warp's gather reads end before the first scratch write.
    if (a.mode >= 2) __syncthreads();
    if (tid == 0) misc[0] = 0;
    __syncthreads();

    int my_log = tid < n ? tid : -1;
    int flag = 0, swaps = 0;
    bool zero = false;

    for (int k0 = 0; k0 < n - 1 && !zero; k0 += 2 * NB) {
      const int steps = min(NB, (n - k0) >> 1);
      T myU[NB], myV[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        myU[j] = T(0);
        myV[j] = T(0);
      }
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        if (j < steps && !zero) {
          const int k = k0 + 2 * j;
          const int ck = misc[0];
          T c = T(0);
          const bool act = my_log > k;
          if (act) {
            c = aval(Lw, tid, ck);
            if (j > 0) {  // row ck's panel values: 16-byte loads (chunk-swizzled rows, swz_index)
              T vr[NB], ur[NB];
#pragma unroll
              for (int q = 0; q < NB; q += Vec<T>::k) {
                lds16(Vs + swz_index<T, NB>(ck, q), vr + q);
                lds16(Us + swz_index<T, NB>(ck, q), ur + q);
              }
#pragma unroll
              for (int p = 0; p < NB; ++p)
                if (p < j) c += myU[p] * vr[p] - myV[p] * ur[p];
            }
          }
          // Warp max of |c| (rounded up to FP32, NaN as +inf), ties to the lowest row, as one
          // integer reduction: non-negative floats order like their bit patterns, and the key
          // bits + 1 leaves 0 for rows that are no longer active.
          const float mag = isnan(c) ? INFINITY : to_key_float(fabs(c));
          const unsigned key = act ? __float_as_uint(mag) + 1u : 0u;
          const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
          const unsigned hit = __ballot_sync(0xffffffffu, key == kmax);
          if (lane == __ffs(hit) - 1) {
            const unsigned lo = ((0xFFFFu - (unsigned)tid) << 16) |
                                (signbit(c) ? 0x8000u : 0u) | ((unsigned)my_log & 0x7FFFu);
            cand[wid] = ((unsigned long long)kmax << 32) | lo;
            if constexpr (sizeof(T) == 8) rval[wid] = c;  // FP64 keeps the signed value
          }
          __syncthreads();  // (1) pivot candidates
          unsigned long long best = 0;
#pragma unroll
          for (int w = 0; w < WARPS; w += 2) {
            const ulonglong2 q2 = *reinterpret_cast<const ulonglong2*>(cand + w);
            best = q2.x > best ? q2.x : best;
            best = q2.y > best ? q2.y : best;
          }
          const unsigned kbest = (unsigned)(best >> 32);
          const float bk = kbest ? __uint_as_float(kbest - 1u) : -1.0f;
          const int r = 0xFFFF - (int)((best >> 16) & 0xFFFFu);
          const int lr = (int)(best & 0x7FFFu);
          T cr;
          if constexpr (sizeof(T) == 4)
            cr = (best & 0x8000u) ? -bk : bk;  // a NaN candidate comes back as an infinite pivot
          else
            cr = rval[r >> 5];
          if (!(bk > 0.0f)) {
            zero = true;  // exactly singular (or empty) column: pf = 0
          } else {
            if (tid == r)
              my_log = k + 1;
            else if (my_log == k + 1)
              my_log = lr;  // the row that held label k+1 takes the pivot's old label
            const T piv = -cr;
            const bool live = my_log > k + 1;
            T u = T(0), v = T(0);
            if (live) {
              T dv = aval(Lw, tid, r);
              if (j > 0) {
                T vr[NB], ur[NB];
#pragma unroll
                for (int q = 0; q < NB; q += Vec<T>::k) {
                  lds16(Vs + swz_index<T, NB>(r, q), vr + q);
                  lds16(Us + swz_index<T, NB>(r, q), ur + q);
                }
#pragma unroll
                for (int p = 0; p < NB; ++p)
                  if (p < j) dv += myU[p] * vr[p] - myV[p] * ur[p];
              }
              u = dv;
              v = c * (T(1) / piv);
            }
            myU[j] = u;
            myV[j] = v;
            if (tid < n) {
              Us[swz_index<T, NB>(tid, j)] = u;
              Vs[swz_index<T, NB>(tid, j)] = v;
            }
            if (my_log == k + 2) misc[0] = tid;
            if (tid == 0) pivs[k >> 1] = lr != k + 1 ? -piv : piv;
            swaps ^= lr != k + 1 ? 1 : 0;
          }
          __syncthreads();  // (2) panel column written, next column's owner known
        }
      }
      if (zero) break;
      // Trailing update of the active rows: warp <-> row, lane <-> column (32-column blocks).
      const int k_end = k0 + 2 * steps;
      const int m = n - k_end;
      if (m >= 2) {
        const bool on = tid < n && my_log >= k_end;
        const unsigned bal = __ballot_sync(0xffffffffu, on);
        if (lane == 0) rt[wid] = __popc(bal);
        __syncthreads();
        int before = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) before += (w < wid) ? rt[w] : 0;
        if (on) alist[before + __popc(bal & ((1u << lane) - 1u))] = tid;
        __syncthreads();  // (3) active list in physical order
        // Work units: (64-column block cb, group of RT consecutive rows below its diagonal);
        // lane l updates columns 64 cb + l and 64 cb + 32 + l, so each row's broadcast U/V
        // serves 64 elements.  All loads of a unit precede its stores (stores may alias loads).
        constexpr int RT = sizeof(T) == 4 ? 2 : 1;
        int total = 0;
        for (int cb = 0; 64 * cb + 1 < m; ++cb) total += (m - 64 * cb - 1 + RT - 1) / RT;
        int cb = 0, rem = wid, cur_cb = -1, ib0 = 0, ib1 = 0, pb0 = 0, pb1 = 0;
        T ub0[NB], vb0[NB], ub1[NB], vb1[NB];
#pragma unroll
        for (int p = 0; p < NB; ++p) ub0[p] = vb0[p] = ub1[p] = vb1[p] = T(0);
        for (int pi = wid; pi < total; pi += WARPS, rem += WARPS) {
          while (rem >= (m - 64 * cb - 1 + RT - 1) / RT) {
            rem -= (m - 64 * cb - 1 + RT - 1) / RT;
            ++cb;
          }
          const int ia0 = 64 * cb + 1 + rem * RT;
          if (cb != cur_cb) {
            cur_cb = cb;
            ib0 = 64 * cb + lane;
            ib1 = ib0 + 32;
            pb0 = ib0 < m ? alist[ib0] : 0;
            pb1 = ib1 < m ? alist[ib1] : 0;
            // the columns' panel values, 16-byte loads of swizzled rows (conflict-free for
            // consecutive active rows); rows past the end read row 0 and are zeroed
#pragma unroll
            for (int p = 0; p < NB; p += Vec<T>::k) {
              lds16(Us + swz_index<T, NB>(pb0, p), ub0 + p);
              lds16(Vs + swz_index<T, NB>(pb0, p), vb0 + p);
              lds16(Us + swz_index<T, NB>(pb1, p), ub1 + p);
              lds16(Vs + swz_index<T, NB>(pb1, p), vb1 + p);
            }
#pragma unroll
            for (int p = 0; p < NB; ++p) {
              if (ib0 >= m) ub0[p] = vb0[p] = T(0);
              if (ib1 >= m) ub1[p] = vb1[p] = T(0);
            }
          }
          T acc0[RT], acc1[RT], ua[RT][NB], va[RT][NB];
          int off[RT];
          bool ok0[RT], ok1[RT];
#pragma unroll
          for (int rr = 0; rr < RT; ++rr) {
            const int ia = ia0 + rr;
            ok0[rr] = ia < m && ib0 < ia;
            ok1[rr] = ia < m && ib1 < ia;
            const int pa = alist[ia < m ? ia : ia0];
            off[rr] = tri_off(pa);
#pragma unroll
            for (int p = 0; p < NB; p += Vec<T>::k) {
              lds16(Us + swz_index<T, NB>(pa, p), ua[rr] + p);
              lds16(Vs + swz_index<T, NB>(pa, p), va[rr] + p);
            }
          }
#pragma unroll
          for (int rr = 0; rr < RT; ++rr) {
            acc0[rr] = ok0[rr] ? Lw[off[rr] + pb0] : T(0);
            acc1[rr] = ok1[rr] ? Lw[off[rr] + pb1] : T(0);
          }
#pragma unroll
          for (int p = 0; p < NB; ++p) {
            if (p < steps) {
#pragma unroll
              for (int rr = 0; rr < RT; ++rr) {
                acc0[rr] = tfma(ua[rr][p], vb0[p], acc0[rr]);
                acc1[rr] = tfma(ua[rr][p], vb1[p], acc1[rr]);
                acc0[rr] = tfma(-va[rr][p], ub0[p], acc0[rr]);
                acc1[rr] = tfma(-va[rr][p], ub1[p], acc1[rr]);
              }
            }
          }
#pragma unroll
          for (int rr = 0; rr < RT; ++rr) {
            if (ok0[rr]) Lw[off[rr] + pb0] = acc0[rr];
            if (ok1[rr]) Lw[off[rr] + pb1] = acc1[rr];
          }
        }
        __syncthreads();  // (4) trailing triangle updated
      }
    }
    if (tid == 0) {
      // Pfaffian = relabelling parity x product of the pivots, accumulated in FP64 as mantissa
      // and exponent; the pivot ratio flags near-nodal blocks.
      const float* isg = a.mode == 2 ? a.item_sign_out : a.item_sign;
      float s = isg ? isg[item] : 1.0f;
      double la, pmax_all = 0.0, pmin_all = 1.0;
      if (isnan(s)) flag |= NH_FLAG_NONFINITE;  // the CNN could not compute this item
      if (zero) {
        s = 0.0f;
        la = -INFINITY;
        flag |= NH_FLAG_ZERO_PIVOT;
      } else {
        double mant = 1.0;
        int expo = 0;
        double pmin = INFINITY, pmax = 0.0;
        for (int k = 0; k < n / 2; ++k) {
          const double pv = (double)pivs[k];
          if (pv < 0.0) s = -s;
          const double ap = fabs(pv);
          if (!isfinite(ap)) flag |= NH_FLAG_NONFINITE;
          pmin = fmin(pmin, ap);
          pmax = fmax(pmax, ap);
          int e;
          mant = frexp(mant * ap, &e);
          expo += e;
        }
        la = log(mant) + (double)expo * 0.6931471805599453;
        if (!isfinite(la)) flag |= NH_FLAG_NONFINITE;
        if (a.cond_tau > 0.0 && pmax > a.cond_tau * pmin) flag |= NH_FLAG_GROWTH;
        if (a.refine_tau > 0.0 && pmax > a.refine_tau * pmin) flag |= kFlagNeedRefine;
        pmax_all = pmax;
        pmin_all = pmin;
      }
      if (s == 0.0f) la = -INFINITY;
      a.sign[item] = s;
      a.logabs[item] = la;
      if (a.flags) a.flags[item] = flag | a.flag_or;
      if (a.ratio) a.ratio[item] = zero ? INFINITY : (float)(pmax_all / pmin_all);
    }
    // Pivot order for the FP64 refinement: every row's final logical label, and the parity.
    if (a.perm && !zero) {
      uint16_t* pr = a.perm + (size_t)item * perm_stride(n);
      if (tid < n) pr[my_log] = (uint16_t)tid;
      if (tid == 0) pr[n] = (uint16_t)swaps;
    }
  }
}

template <typename T, int NB, int WARPS = kWarps, bool kGlobalTri = false>
size_t pf_smem(int n) {
  const size_t tri = (size_t)n * (n - 1) / 2;
  const size_t val_slots = sizeof(T) == 4 ? 0 : WARPS;
  return sizeof(T) * ((kGlobalTri ? 0 : ((tri + 3) & ~(size_t)3)) + 2 * (size_t)n * NB +
                      val_slots + ((n / 2 + 3) & ~(size_t)3)) +
         sizeof(float) * WARPS + sizeof(int) * (2 * WARPS + (size_t)n + 2);
}

// Raises a kernel's dynamic shared-memory cap to the largest the launches need, never lowering
// it: the plain and the fused launchers share kernel instantiations, and a cap set lower by one
// would make the other's launch fail.  One cap per kernel, under a lock.
template <typename K>
int raise_smem_cap(K* kernel, size_t smem) {
  static std::mutex mu;
  static std::map<const void*, size_t> caps;
  if (smem <= 48 * 1024) return NH_OK;
  std::lock_guard<std::mutex> g(mu);
  size_t& cap = caps[reinterpret_cast<const void*>(kernel)];
  if (smem <= cap) return NH_OK;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return check_cuda(e, "pfaffian kernel shared-memory attribute");
  cap = smem;
  return NH_OK;
}

// Large lattices: 1024 threads, triangle in a.tri; the panel width that fits shared memory.
constexpr int kBigThreads = 1024;
constexpr int kBigNB = 4;

template <typename T, int NB, int D, int THREADS = kNumThreads>
int launch_pf(const PfArgs& a, cudaStream_t st) {
  constexpr bool kGlobalTri = THREADS > kNumThreads;
  const size_t smem = pf_smem<T, NB, THREADS / 32, kGlobalTri>(a.n);
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d needs %zu B of shared memory", a.n, smem);
  if (kGlobalTri && !a.tri)
    return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d needs the large-lattice scratch", a.n);
  if (int rc = raise_smem_cap(pfaffian_kernel<T, NB, D, THREADS>, smem)) return rc;
  const int per_sm = (!kGlobalTri && smem <= 113 * 1024) ? 2 : 1;
  int grid = num_sms() * per_sm;
  if (grid > a.n_slots) grid = a.n_slots;
  if (grid <= 0) return NH_OK;
  ProfScope prof_scope(sizeof(T) == 4 ? NH_K_PFAFFIAN : NH_K_PFAFFIAN64, st);
  pfaffian_kernel<T, NB, D, THREADS><<<grid, THREADS, smem, st>>>(a);
  return check_launch("pfaffian_kernel");
}

// FP32: the widest panel that keeps two CTAs per SM; FP64: one CTA per SM; beyond shared
// memory (FP32 n > 256, FP64 n > 236): the large-lattice kernel.
template <typename T, int D>
int launch_pf_pick(const PfArgs& a, cudaStream_t st) {
  if (a.n <= kNumThreads) {
    if constexpr (sizeof(T) == 4) {
      if (pf_smem<T, 8>(a.n) <= 113 * 1024) return launch_pf<T, 8, D>(a, st);
      return launch_pf<T, 4, D>(a, st);
    } else {
      if (pf_smem<T, 4>(a.n) <= 227 * 1024) return launch_pf<T, 4, D>(a, st);
      if (pf_smem<T, 2>(a.n) <= 227 * 1024) return launch_pf<T, 2, D>(a, st);
    }
  }
  return launch_pf<T, kBigNB, D, kBigThreads>(a, st);
}

template <typename T>
int launch_pf_d(const PfArgs& a, int d, cudaStream_t st) {
  switch (d) {
    case 8: return launch_pf_pick<T, 8>(a, st);
    case 16: return launch_pf_pick<T, 16>(a, st);
    case 32: return launch_pf_pick<T, 32>(a, st);
    default: return fail(NH_ERR_UNSUPPORTED, "amplitude: d=%d (8, 16 or 32)", d);
  }
}

// ------------------------------------------------------------------ standalone gather
template <int D>
__global__ void __launch_bounds__(kNumThreads) pairing_kernel(const float* __restrict__ Y,
                                                              const int32_t* __restrict__ idx,
                                                              const float* __restrict__ Wt,
                                                              int Lx, int Ly, int n, int batch,
                                                              float* __restrict__ F) {
  const int N = Lx * Ly;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int item = blockIdx.x; item < batch; item += gridDim.x) {
    const float* Yi = Y + (size_t)item * n * D;
    const int32_t* ii = idx + (size_t)item * n;
    float* Fi = F + (size_t)item * n * n;
    for (int p = wid; p < n; p += kWarps) {
      const int mp = __ldg(ii + p);
      const int sp = mp >= N ? 1 : 0;
      const int sitep = mp - sp * N;
      const int xp = sitep / Ly, ypos = sitep - xp * Ly;
      float yp[D];
#pragma unroll
      for (int a0 = 0; a0 < D; a0 += 4) ldg16(Yi + (size_t)p * D + a0, yp + a0);
      for (int q = lane; q < n; q += 32) {
        float v = 0.0f;
        if (q != p)
          v = pair_value<float, D>(yp, sp, xp, ypos, Yi + (size_t)q * D, __ldg(ii + q), N, Lx, Ly,
                                   Wt);
        Fi[(size_t)p * n + q] = v;
      }
    }
  }
}

// Shared-memory variant: the Wt table is staged once per CTA and each matrix's occupied features
// once per matrix, rows padded to D + 4 floats (16-byte chunks of 8 consecutive rows fall in
// distinct banks); a warp computes two rows per pass so that each feature row it loads serves
// two outputs.  Same per-element arithmetic as pair_value: F is bit-for-bit that of the fused
// gather and exactly antisymmetric.
template <int D>
__global__ void __launch_bounds__(kNumThreads) pairing_smem_kernel(
    const float* __restrict__ Y, const int32_t* __restrict__ idx, const float* __restrict__ Wt,
    int Lx, int Ly, int n, int batch, float* __restrict__ F) {
  constexpr int DP = D + 4;
  extern __shared__ __align__(16) float psm[];
  const int N = Lx * Ly;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  float* wts = psm;            // (4 N, DP)
  float* ys = wts + 4 * N * DP;  // (n, DP)
  int* info = reinterpret_cast<int*>(ys + n * DP);  // (spin << 16) | (x << 8) | y per row
  for (int e = tid; e < 4 * N * D; e += kNumThreads) {
    const int row = e / D;
    wts[row * DP + (e - row * D)] = __ldg(Wt + e);
  }
  for (int item = blockIdx.x; item < batch; item += gridDim.x) {
    const float* Yi = Y + (size_t)item * n * D;
    const int32_t* ii = idx + (size_t)item * n;
    float* Fi = F + (size_t)item * n * n;
    __syncthreads();
    for (int e = tid; e < n * D; e += kNumThreads) {
      const int row = e / D;
      ys[row * DP + (e - row * D)] = __ldg(Yi + e);
    }
    for (int p = tid; p < n; p += kNumThreads) {
      const int m = __ldg(ii + p);
      const int sp = m >= N ? 1 : 0;
      const int site = m - sp * N;
      const int x = site / Ly;
      info[p] = (sp << 16) | (x << 8) | (site - x * Ly);
    }
    __syncthreads();
    for (int p0 = 2 * wid; p0 < n; p0 += 2 * kWarps) {
      const int np = p0 + 1 < n ? 2 : 1;
      float yp[2][D];
      int sp[2], xp[2], ypos[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int p = h < np ? p0 + h : p0;
#pragma unroll
        for (int a0 = 0; a0 < D; a0 += 4) {
          const float4 v = *reinterpret_cast<const float4*>(ys + p * DP + a0);
          yp[h][a0] = v.x;
          yp[h][a0 + 1] = v.y;
          yp[h][a0 + 2] = v.z;
          yp[h][a0 + 3] = v.w;
        }
        const int inf = info[p];
        sp[h] = inf >> 16;
        xp[h] = (inf >> 8) & 0xFF;
        ypos[h] = inf & 0xFF;
      }
      for (int q = lane; q < n; q += 32) {
        float yq[D];
#pragma unroll
        for (int a0 = 0; a0 < D; a0 += 4) {
          const float4 v = *reinterpret_cast<const float4*>(ys + q * DP + a0);
          yq[a0] = v.x;
          yq[a0 + 1] = v.y;
          yq[a0 + 2] = v.z;
          yq[a0 + 3] = v.w;
        }
        const int inf = info[q];
        const int sq = inf >> 16, xq = (inf >> 8) & 0xFF, yqp = inf & 0xFF;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (h >= np) continue;
          const int p = p0 + h;
          float acc = 0.0f;
          if (q != p) {
            int dx = xp[h] - xq, dy = ypos[h] - yqp;
            dx += dx < 0 ? Lx : 0;
            dy += dy < 0 ? Ly : 0;
            const float* w = wts + ((2 * sp[h] + sq) * N + dx * Ly + dy) * DP;
#pragma unroll
            for (int a0 = 0; a0 < D; a0 += 4) {
              const float4 wv = *reinterpret_cast<const float4*>(w + a0);
              acc = fmaf(yp[h][a0] * yq[a0], wv.x, acc);
              acc = fmaf(yp[h][a0 + 1] * yq[a0 + 1], wv.y, acc);
              acc = fmaf(yp[h][a0 + 2] * yq[a0 + 2], wv.z, acc);
              acc = fmaf(yp[h][a0 + 3] * yq[a0 + 3], wv.w, acc);
            }
          }
          Fi[(size_t)p * n + q] = acc;
        }
      }
    }
  }
}

size_t pairing_smem_bytes(int N, int n, int D) {
  return sizeof(float) * (4 * (size_t)N + n) * (D + 4) + sizeof(int) * (size_t)n;
}

// ------------------------------------------------------------------ image combination
// Also used with G = 1 to copy the per-item results into the caller's arrays.
// Sum over the images of one configuration in FP64: returns sum_g s_g exp(l_g - m) and sets
// *asum to sum_g |.| and *m to the largest log.
__device__ __forceinline__ double image_sum(const float* __restrict__ sg,
                                           const double* __restrict__ la, int c, int G,
                                           double* m_out, double* asum) {
  double m = -INFINITY;
  for (int g = 0; g < G; ++g) {
    const float s = sg[(size_t)c * G + g];
    const double l = la[(size_t)c * G + g];
    if (s != 0.0f && l > m) m = l;
  }
  double tot = 0.0, a = 0.0;
  if (m > -INFINITY)
    for (int g = 0; g < G; ++g) {
      const float s = sg[(size_t)c * G + g];
      if (s != 0.0f) {
        const double t = exp(la[(size_t)c * G + g] - m);
        tot += (double)s * t;
        a += t;
      }
    }
  *m_out = m;
  *asum = a;
  return tot;
}

// FP64-feature selection for projected amplitudes, before the FP64 list is built.  An image's
// error reaches log|psi_P| weighted by its share w_g = eta_g psi_g / psi_P (sum_g w_g = 1,
// sum_g |w_g| = C), and the error of an image with FP32 (or BF16x3) features grows with its
// pivot ratio r_g.  In a configuration whose images cancel (C > cancel_tau > 0) every image
// with |w_g| > kCancelImageFloor is marked (NH_FLAG_GROWTH | NH_FLAG_CANCEL): an FP32 image
// error (at most ~1e-3) of the others adds < 2e-5.  Otherwise, with weighted set, an image is
// marked exactly when |w_g| r_g > cond_tau (its estimated error, up to the features' relative
// accuracy), and unmarked when not; without weighted (cond_tau <= 1, every image already
// marked) the marks stay.
constexpr double kCancelImageFloor = 2e-2;

__global__ void image_mark_kernel(const float* __restrict__ sg, const double* __restrict__ la,
                                  int32_t* __restrict__ fl, const float* __restrict__ ratio,
                                  int G, int n_cfg, const int32_t* n_cfg_dev, double cancel_tau,
                                  double cond_tau, bool weighted) {
  const int n = n_cfg_dev ? *n_cfg_dev : n_cfg;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double m, a;
    const double tot = image_sum(sg, la, c, G, &m, &a);
    if (cancel_tau > 0.0 && a > 0.0 && a > cancel_tau * fabs(tot)) {
      for (int g = 0; g < G; ++g) {
        const size_t i = (size_t)c * G + g;
        if (sg[i] != 0.0f && exp(la[i] - m) > kCancelImageFloor * fabs(tot))
          fl[i] |= NH_FLAG_GROWTH | NH_FLAG_CANCEL;
      }
    } else if (weighted && tot != 0.0) {
      for (int g = 0; g < G; ++g) {
        const size_t i = (size_t)c * G + g;
        const int f = fl[i];
        if ((f & (NH_FLAG_NONFINITE | NH_FLAG_ZERO_PIVOT)) || sg[i] == 0.0f) continue;
        const double w = exp(la[i] - m) / fabs(tot);
        fl[i] = w * (double)ratio[i] > cond_tau ? (f | NH_FLAG_GROWTH) : (f & ~NH_FLAG_GROWTH);
      }
    }
  }
}

__global__ void combine_kernel(const float* __restrict__ sg, const double* __restrict__ la,
                               const int32_t* __restrict__ fl, int G, int n_cfg,
                               const int32_t* n_cfg_dev, float* sign, double* logabs,
                               int32_t* flags, double cancel_tau, const int32_t* err) {
  const int n = n_cfg_dev ? *n_cfg_dev : n_cfg;
  const int timeout = (err && *err) ? NH_FLAG_TIMEOUT : 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    int f = timeout;
    if (fl)
      for (int g = 0; g < G; ++g) f |= fl[(size_t)c * G + g] & kPublicFlags;
    double m, a;
    const double tot = image_sum(sg, la, c, G, &m, &a);
    if (cancel_tau > 0.0 && a > 0.0 && a > cancel_tau * fabs(tot)) f |= NH_FLAG_CANCEL;
    const float so = tot > 0.0 ? 1.0f : (tot < 0.0 ? -1.0f : 0.0f);
    sign[c] = so;
    logabs[c] = so != 0.0f ? log(fabs(tot)) + m - log((double)G) : -INFINITY;
    if (flags) flags[c] = f;
  }
}

// Ordered list of the items whose flags carry a bit of set_mask and none of clear_mask (single
// CTA).
__global__ void __launch_bounds__(1024) flagged_kernel(const int32_t* __restrict__ flags,
                                                       int n_items, const int32_t* count_dev,
                                                       int count_mult, int32_t* list,
                                                       int32_t* count, int set_mask,
                                                       int clear_mask) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int n = count_dev ? (*count_dev) * count_mult : n_items;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    const int f = i < n ? flags[i] : 0;
    const int v = (i < n && (f & set_mask) && !(f & clear_mask)) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, v);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    if (wid == 0) {
      int w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    if (v) list[carry + (wid ? wsum[wid - 1] : 0) + __popc(bal & ((1u << lane) - 1u))] = i;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = carry;
}


// ------------------------------------------------------------------ tensor-memory Pfaffian
// The FP32 matrix lives in tensor memory (one matrix per SM: rows 0-127 in lanes 0-127 of
// columns [0, NP), rows 128-255 in columns [NP, 2 NP), NP = n rounded up to 32); thread t owns
// row t and reads pivot columns with tcgen05.ld.  The panel is the same relabelling Parlett-Reid
// as pfaffian_kernel; at the end of each panel of 8 steps the rank-16 update
// A += U V^T - V U^T runs on the tensor cores as 3xTF32 products (X = X_big + X_small, both
// rounded to TF32): U_b V_b^T + U_b V_s^T + U_s V_b^T - V_b U_b^T - V_b U_s^T - V_s U_b^T, six
// kind::tf32 MMAs (M = 128, N = NP, K = 8) per 128-row tile, the minus signs via the A-negate bit
// of the instruction descriptor.  Accuracy: the accumulation into the FP32 matrix in tensor
// memory, not the operand split, limits this form (a three-way split measured no better); at
// n = 224 log|pf| is within about 2e-4 of FP64, against 1e-4 for the CUDA-core kernel.  Rows and columns of eliminated indices carry U = V = 0 and never
// change again.  The occupied block is gathered into a shared-memory lower triangle first and
// copied into tensor memory with tcgen05.st.

constexpr int kTcNB = 8;
constexpr int kTcOpFloats = 4 * 2048 + 2 * kNumThreads * kTcNB;  // operands + FP32 panel copies
constexpr uint32_t kTcCols = 512;
constexpr long long kTcWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // sm_100 descriptor version; no swizzle, base offset 0
  return d;
}

// kind::tf32 instruction descriptor: FP32 accumulate, TF32 A and B, K-major, M = 128, N = np.
__device__ __forceinline__ uint32_t tf32_idesc(int np, bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) |
         ((uint32_t)(np >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, 1, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc));
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n" : "=r"(r) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31, %32};\n" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31])));
}

__device__ __forceinline__ float tf32_big(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (long long it = 0; it < kTcWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Operand arrays (K-major, no swizzle): element (row t, k) of a 256 x 8 TF32 matrix at
// (k / 4) * 4096 + (t / 8) * 128 + (t % 8) * 16 + (k % 4) * 4 bytes.
__device__ __forceinline__ int opnd_off(int t, int k) {
  return (k >> 2) * 1024 + (t >> 3) * 32 + (t & 7) * 4 + (k & 3);  // in floats
}

template <int D>
__global__ void __launch_bounds__(kNumThreads, 1) pfaffian_tc_kernel(PfArgs a, int32_t* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int tri = tri_off(n);
  const int NP = (n + 31) & ~31;
  const int n_tiles = (n + 127) >> 7;
  float* region = reinterpret_cast<float*>(smem_raw);  // staging triangle, later the operands
  const int region_floats = max((tri + 31) & ~31, kTcOpFloats);
  float* Ub = region;               // 4 operand arrays of 256 x 8 TF32 (8 KB each)
  float* Us = region + 2048;
  float* Vb = region + 4096;
  float* Vs = region + 6144;
  float* Uf = region + 8192;        // FP32 copies [row][8] for the in-panel corrections
  float* Vf = Uf + kNumThreads * kTcNB;
  float* pivs = region + region_floats;          // (128) signed pivots
  float* rkey = pivs + 128;                      // (warps)
  int* rt = reinterpret_cast<int*>(rkey + kWarps);
  int* rlog = rt + kWarps;
  int* misc = rlog + kWarps;                     // [0] physical row of logical k, [1] abort
  uint64_t* bar = reinterpret_cast<uint64_t*>(misc + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    misc[1] = 0;
  }
  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t my_col0 = tmem + ((uint32_t)(32 * (wid & 3)) << 16) + (uint32_t)((tid >> 7) * NP);
  uint32_t phase = 0;

  const int n_work = a.count_dev ? (*a.count_dev) * a.count_mult : a.n_slots;
  const float* Ybase = static_cast<const float*>(a.Y);
  const float* Wt = static_cast<const float*>(a.Wt);
  for (int slot = blockIdx.x; slot < n_work; slot += gridDim.x) {
    const int item = a.slot_item ? a.slot_item[slot] : slot;
    if (misc[1]) {  // a wait expired earlier: mark the item instead of computing it
      if (tid == 0) {
        a.sign[item] = NAN;
        a.logabs[item] = NAN;
        if (a.flags) a.flags[item] = NH_FLAG_NONFINITE | a.flag_or;
      }
      continue;
    }
    __syncthreads();
    if (a.mode == 0) {
      const float* F = a.F + (size_t)item * n * n;
      for (int i = wid; i < n; i += kWarps) {
        const float* src = F + (size_t)i * n;
        float* dst = region + tri_off(i);
        for (int j = lane; j < i; j += 32) dst[j] = __ldg(src + j);
      }
    } else {
      gather_lower<float, D>(region, n, Ybase + (size_t)slot * n * D, a.idx + (size_t)slot * n,
                             Wt, a.Lx, a.Ly);
    }
    __syncthreads();
    // Full antisymmetric matrix into tensor memory, 32 columns per store; rows >= n are zero.
    for (int b = 0; b < NP / 32; ++b) {
      float v[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int q = 32 * b + i;
        float x = 0.0f;
        if (tid < n && q < n) x = q < tid ? region[tri_off(tid) + q] : (q > tid ? -region[tri_off(q) + tid] : 0.0f);
        v[i] = x;
      }
      tmem_st32(my_col0 + 32 * b, v);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // the staging triangle is dead from here: the operand arrays reuse it
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) misc[0] = 0;
    __syncthreads();

    int my_log = tid < n ? tid : -1;
    int flag = 0, swaps = 0;
    bool zero = false, abort = false;
    for (int k0 = 0; k0 < n - 1 && !zero && !abort; k0 += 2 * kTcNB) {
      const int steps = min(kTcNB, (n - k0) >> 1);
      float myU[kTcNB], myV[kTcNB];
#pragma unroll
      for (int j = 0; j < kTcNB; ++j) {
        myU[j] = 0.0f;
        myV[j] = 0.0f;
        if (j >= steps) {  // columns a short last panel leaves unused must be zero
          const int o = opnd_off(tid, j);
          Ub[o] = Us[o] = Vb[o] = Vs[o] = 0.0f;
        }
      }
#pragma unroll
      for (int j = 0; j < kTcNB; ++j) {
        if (j < steps && !zero) {
          const int k = k0 + 2 * j;
          const int ck = misc[0];
          float c = tmem_ld1(my_col0 + ck);
          const bool act = my_log > k;
          if (act) {
#pragma unroll
            for (int p = 0; p < kTcNB; ++p)
              if (p < j) c += myU[p] * Vf[ck * kTcNB + p] - myV[p] * Uf[ck * kTcNB + p];
          }
          const float mag = act ? (isnan(c) ? INFINITY : fabsf(c)) : -1.0f;
          float wmax = mag;
#pragma unroll
          for (int o = 16; o; o >>= 1) wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
          const unsigned hit = __ballot_sync(0xffffffffu, mag == wmax);
          if (lane == __ffs(hit) - 1) {
            rkey[wid] = wmax;
            rt[wid] = tid;
            rlog[wid] = my_log | (signbit(c) ? (int)0x80000000 : 0);
          }
          __syncthreads();  // (1) pivot candidates
          float kw[kWarps];
#pragma unroll
          for (int w = 0; w < kWarps; ++w) kw[w] = rkey[w];
          float bk = kw[0];
#pragma unroll
          for (int w = 1; w < kWarps; ++w) bk = fmaxf(bk, kw[w]);
          int w0 = kWarps - 1;
#pragma unroll
          for (int w = kWarps - 2; w >= 0; --w) w0 = kw[w] == bk ? w : w0;
          const int r = rt[w0];
          const int lw = rlog[w0];
          const int lr = lw & 0x7FFFFFFF;
          const float cr = lw < 0 ? -bk : bk;
          if (!(bk > 0.0f)) {
            zero = true;
          } else {
            if (tid == r)
              my_log = k + 1;
            else if (my_log == k + 1)
              my_log = lr;
            const float piv = -cr;
            const bool live = my_log > k + 1;
            float dv = tmem_ld1(my_col0 + r);
            float u = 0.0f, v = 0.0f;
            if (live) {
#pragma unroll
              for (int p = 0; p < kTcNB; ++p)
                if (p < j) dv += myU[p] * Vf[r * kTcNB + p] - myV[p] * Uf[r * kTcNB + p];
              u = dv;
              v = c * (1.0f / piv);
            }
            myU[j] = u;
            myV[j] = v;
            Uf[tid * kTcNB + j] = u;
            Vf[tid * kTcNB + j] = v;
            // Both parts rounded to TF32 here: the tensor cores would truncate an unrounded
            // small part, a bias that accumulates over the pivots.
            const int o = opnd_off(tid, j);
            const float ub = tf32_big(u), vb = tf32_big(v);
            Ub[o] = ub;
            Us[o] = tf32_big(u - ub);
            Vb[o] = vb;
            Vs[o] = tf32_big(v - vb);
            if (my_log == k + 2) misc[0] = tid;
            if (tid == 0) pivs[k >> 1] = lr != k + 1 ? -piv : piv;
            swaps ^= lr != k + 1 ? 1 : 0;
          }
          __syncthreads();  // (2) panel column written, next column's owner known
        }
      }
      if (zero) break;
      if (n - (k0 + 2 * steps) < 2) break;  // nothing left to update
      // Rank-16 trailing update on the tensor cores.
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // Products of the parts: big x big, big x small, small x big.
        const uint32_t u2[2] = {smem_addr(Ub), smem_addr(Us)};
        const uint32_t v2[2] = {smem_addr(Vb), smem_addr(Vs)};
        constexpr int kPa[3] = {0, 0, 1}, kPb[3] = {0, 1, 0};
        const uint32_t lbo = 4096, sbo = 128;
        const uint32_t id_pos = tf32_idesc(NP, false), id_neg = tf32_idesc(NP, true);
        for (int mt = 0; mt < n_tiles; ++mt) {
          const uint32_t d = tmem + (uint32_t)(mt * NP);
          const uint32_t ro = (uint32_t)(mt * 128 / 8 * 128);  // first row group of the tile
#pragma unroll
          for (int t = 0; t < 3; ++t) {  // + U V^T
            mma_tf32(d, tc_desc(u2[kPa[t]] + ro, lbo, sbo), tc_desc(v2[kPb[t]], lbo, sbo), id_pos);
          }
#pragma unroll
          for (int t = 0; t < 3; ++t) {  // - V U^T
            mma_tf32(d, tc_desc(v2[kPa[t]] + ro, lbo, sbo), tc_desc(u2[kPb[t]], lbo, sbo), id_neg);
          }
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_addr(bar))
            : "memory");
      }
      if (!tc_wait(bar, phase)) {
        if (tid == 0) atomicExch(err, 1);
        misc[1] = 1;
      }
      phase ^= 1u;
      __syncthreads();
      abort = misc[1] != 0;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (tid == 0) {
      float s = a.item_sign ? a.item_sign[item] : 1.0f;
      double la, pmax_all = 0.0, pmin_all = 1.0;
      if (isnan(s)) flag |= NH_FLAG_NONFINITE;
      if (abort) {
        s = NAN;
        la = NAN;
        flag |= NH_FLAG_NONFINITE;
      } else if (zero) {
        s = 0.0f;
        la = -INFINITY;
        flag |= NH_FLAG_ZERO_PIVOT;
      } else {
        double mant = 1.0;
        int expo = 0;
        double pmin = INFINITY, pmax = 0.0;
        for (int k = 0; k < n / 2; ++k) {
          const double pv = (double)pivs[k];
          if (pv < 0.0) s = -s;
          const double ap = fabs(pv);
          if (!isfinite(ap)) flag |= NH_FLAG_NONFINITE;
          pmin = fmin(pmin, ap);
          pmax = fmax(pmax, ap);
          int e;
          mant = frexp(mant * ap, &e);
          expo += e;
        }
        la = log(mant) + (double)expo * 0.6931471805599453;
        if (!isfinite(la)) flag |= NH_FLAG_NONFINITE;
        if (a.cond_tau > 0.0 && pmax > a.cond_tau * pmin) flag |= NH_FLAG_GROWTH;
        if (a.refine_tau > 0.0 && pmax > a.refine_tau * pmin) flag |= kFlagNeedRefine;
        pmax_all = pmax;
        pmin_all = pmin;
      }
      if (s == 0.0f) la = -INFINITY;
      a.sign[item] = s;
      a.logabs[item] = la;
      if (a.flags) a.flags[item] = flag | a.flag_or;
      if (a.ratio) a.ratio[item] = (zero || abort) ? INFINITY : (float)(pmax_all / pmin_all);
    }
    if (a.perm && !zero && !abort) {
      uint16_t* pr = a.perm + (size_t)item * perm_stride(n);
      if (tid < n) pr[my_log] = (uint16_t)tid;
      if (tid == 0) pr[n] = (uint16_t)swaps;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (wid == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcCols)
                 : "memory");
}

size_t pf_tc_smem(int n) {
  const size_t tri = (size_t)n * (n - 1) / 2;
  const size_t region = std::max((tri + 31) & ~(size_t)31, (size_t)kTcOpFloats);
  const size_t need = sizeof(float) * (region + 128 + kWarps) + sizeof(int) * (2 * kWarps + 4) + 32;
  // At least 120 KB, so that two CTAs never share an SM: each allocates all 512 tensor-memory
  // columns, and a second CTA would stall in tcgen05.alloc until the first one exits.
  return std::max(need, (size_t)120 * 1024);
}

template <int D>
int launch_pf_tc(const PfArgs& a, int32_t* err, cudaStream_t st) {
  const size_t smem = pf_tc_smem(a.n);
  // The limit is raised once, to the largest size any n <= 256 needs.
  static const cudaError_t attr = cudaFuncSetAttribute(
      pfaffian_tc_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)pf_tc_smem(kNumThreads));
  if (attr != cudaSuccess) return check_cuda(attr, "tensor-memory Pfaffian smem attribute");
  int grid = num_sms();
  if (grid > a.n_slots) grid = a.n_slots;
  if (grid <= 0) return NH_OK;
  ProfScope prof_scope(NH_K_PFAFFIAN_TC, st);
  pfaffian_tc_kernel<D><<<grid, kNumThreads, smem, st>>>(a, err);
  return check_launch("pfaffian_tc_kernel");
}
}  // namespace

bool pfaffian64_fits(int n) { return pf_smem<double, 2>(n) <= 227 * 1024; }

bool pfaffian_needs_scratch(int n, bool fp64) {
  if (n > kNumThreads) return true;
  return fp64 ? pf_smem<double, 2>(n) > 227 * 1024 : pf_smem<float, 4>(n) > 227 * 1024;
}

size_t pfaffian_scratch_bytes(int n) {
  const size_t tri = ((size_t)n * (n - 1) / 2 + 3) & ~(size_t)3;
  return pfaffian_needs_scratch(n, true) ? (size_t)num_sms() * tri * sizeof(double) : 0;
}

int launch_pfaffian_from_F(const float* F, int n, int batch, const int32_t* list,
                           const int32_t* count, bool fp64, double cond_tau, int flag_or,
                           float* sign, double* logabs, int32_t* flags, void* tri,
                           cudaStream_t st, uint16_t* perm, double refine_tau) {
  if (n <= 0 || n % 2 || n > kBigThreads)
    return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d must be even and <= %d", n, kBigThreads);
  PfArgs a{};
  a.n = n;
  a.mode = 0;
  a.F = F;
  a.n_slots = batch;
  a.count_dev = count;
  a.count_mult = 1;
  a.slot_item = list;
  a.sign = sign;
  a.logabs = logabs;
  a.flags = flags;
  a.cond_tau = cond_tau;
  a.flag_or = flag_or;
  a.tri = tri;
  a.perm = perm;
  a.refine_tau = refine_tau;
  return fp64 ? launch_pf_pick<double, 16>(a, st) : launch_pf_pick<float, 16>(a, st);
}

int launch_pfaffian_gather(const PfGatherArgs& g, cudaStream_t st) {
  if (g.n <= 0 || g.n % 2 || g.n > kBigThreads)
    return fail(NH_ERR_UNSUPPORTED, "amplitude: n=%d must be even and <= %d", g.n, kBigThreads);
  PfArgs a{};
  a.n = g.n;
  a.mode = 1;
  a.Y = g.Y;
  a.idx = g.idx;
  a.Wt = g.Wt;
  a.Lx = g.Lx;
  a.Ly = g.Ly;
  a.count_dev = g.count_dev;
  a.count_mult = g.count_mult;
  a.n_slots = g.n_slots;
  a.slot_item = g.slot_item;
  a.item_sign = g.item_sign;
  a.sign = g.sign;
  a.logabs = g.logabs;
  a.flags = g.flags;
  a.cond_tau = g.cond_tau;
  a.flag_or = g.flag_or;
  a.tri = g.tri;
  a.perm = g.perm;
  a.refine_tau = g.refine_tau;
  a.ratio = g.ratio;
  return g.fp64 ? launch_pf_d<double>(a, g.d, st) : launch_pf_d<float>(a, g.d, st);
}

// Fused features + FP32 Pfaffian (mode 2): shared-memory layout choice and launch.
template <int NB, int D>
int launch_fused_nb(PfArgs a, cudaStream_t st) {
  const int n = a.n, N = a.Lx * a.Ly;
  constexpr int WARPS = kWarps;
  const size_t pf = pf_smem<float, NB>(n);
  size_t cnn_end = 0, act_end = 0;  // mode 3 (rows copied from global memory): no CNN phase
  if (a.mode == 2) act_end = cnn_phase_layout(N, a.C, a.Lx, &cnn_end);
  const size_t tri_pad = ((size_t)n * (n - 1) / 2 + 3) & ~(size_t)3;
  const size_t tri_bytes = 4 * tri_pad, y_bytes = 4 * (size_t)n * D;
  const size_t two_cta = 113 * 1024;
  // A: rows after the triangle and the activation planes, modes after the rows.
  const size_t yA = (std::max(act_end, tri_bytes) + 15) & ~(size_t)15;
  const size_t totA = std::max(std::max(pf, cnn_end), yA + y_bytes + 4 * (size_t)n);
  // B: rows in the triangle's tail (rows from tail_row gathered through registers), modes in the
  // active-row list of the factorisation.
  const size_t yB = (tri_bytes - y_bytes) & ~(size_t)15;
  const size_t alist_off = 4 * (tri_pad + 2 * (size_t)n * NB + (((size_t)n / 2 + 3) & ~(size_t)3)) +
                           4 * (size_t)WARPS * 3;
  int tail = n;
  if (y_bytes < tri_bytes) {
    const size_t yf = yB / 4;
    tail = 0;
    while (tail < n && (size_t)tail * (tail - 1) / 2 + tail <= yf) ++tail;
  }
  const size_t tail_elems = (size_t)n * (n - 1) / 2 - (size_t)tail * (tail - 1) / 2;
  const size_t totB = std::max(pf, cnn_end);
  const bool okB = y_bytes < tri_bytes && yB >= act_end && alist_off >= act_end &&
                   tail_elems <= (size_t)kTailRegs * kNumThreads;
  size_t smem;
  if (totA <= two_cta || !okB || totB > two_cta) {
    smem = totA;
    a.y_off = (int)yA;
    a.idx_off = (int)(yA + y_bytes);
    a.tail_row = n;
  } else {
    smem = totB;
    a.y_off = (int)yB;
    a.idx_off = (int)alist_off;
    a.tail_row = tail;
  }
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "fused amplitude: n=%d, N=%d needs %zu B of shared memory", n,
                N, smem);
  if (int rc = raise_smem_cap(pfaffian_kernel<float, NB, D, kNumThreads>, smem)) return rc;
  const int per_sm = smem <= two_cta ? 2 : 1;
  int grid = num_sms() * per_sm;
  if (grid > a.n_slots) grid = a.n_slots;
  if (grid <= 0) return NH_OK;
  if (a.queue) {
    cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) return check_cuda(e, "fused amplitude: clear work counter");
  }
  ProfScope prof_scope(a.mode == 2 ? NH_K_FUSED : NH_K_PFAFFIAN, st);
  pfaffian_kernel<float, NB, D, kNumThreads><<<grid, kNumThreads, smem, st>>>(a);
  return check_launch("pfaffian_kernel (fused features)");
}

int launch_pfaffian_tc(const PfGatherArgs& g, int mode, const float* F, int32_t* err,
                       cudaStream_t st) {
  if (g.n <= 0 || g.n % 2 || g.n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED, "tensor-memory Pfaffian: n=%d must be even and <= %d", g.n,
                kNumThreads);
  PfArgs a{};
  a.n = g.n;
  a.mode = mode;
  a.F = F;
  a.Y = g.Y;
  a.idx = g.idx;
  a.Wt = g.Wt;
  a.Lx = g.Lx;
  a.Ly = g.Ly;
  a.count_dev = g.count_dev;
  a.count_mult = g.count_mult;
  a.n_slots = g.n_slots;
  a.slot_item = g.slot_item;
  a.item_sign = g.item_sign;
  a.sign = g.sign;
  a.logabs = g.logabs;
  a.flags = g.flags;
  a.cond_tau = g.cond_tau;
  a.flag_or = g.flag_or;
  a.perm = g.perm;
  a.refine_tau = g.refine_tau;
  a.ratio = g.ratio;
  switch (mode == 0 ? 16 : g.d) {
    case 8: return launch_pf_tc<8>(a, err, st);
    case 16: return launch_pf_tc<16>(a, err, st);
    case 32: return launch_pf_tc<32>(a, err, st);
    default: return fail(NH_ERR_UNSUPPORTED, "tensor-memory Pfaffian: d=%d", g.d);
  }
}

template <int D>
int launch_pairing_smem(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int n,
                        int batch, float* F, size_t smem, cudaStream_t st) {
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(pairing_smem_kernel<D>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "pairing smem attribute");
    configured = smem;
  }
  int grid = num_sms() * (smem <= 113 * 1024 ? 2 : 1);
  if (grid > batch) grid = batch;
  ProfScope prof_scope(NH_K_PAIRING, st);
  pairing_smem_kernel<D><<<grid, kNumThreads, smem, st>>>(Y, idx, Wt, Lx, Ly, n, batch, F);
  return check_launch("pairing_smem_kernel");
}

bool fused_supported(const nh_backflow_params& p) {
  const int n = p.n_up + p.n_dn, N = p.Lx * p.Ly, d = p.channels / 2;
  return p.net == NH_NET_CNN && n <= kNumThreads && n % 2 == 0 && N % 2 == 0 &&
         p.channels % 16 == 0 && p.channels <= 64 && (d == 8 || d == 16 || d == 32);
}

bool staged_supported(const PfGatherArgs& g) {
  return !g.fp64 && g.n <= kNumThreads && g.n % 2 == 0 && g.d % 4 == 0 && g.d <= 32 && !g.tri;
}

int launch_pfaffian_staged(const PfGatherArgs& g, cudaStream_t st) {
  PfArgs a{};
  a.n = g.n;
  a.mode = 3;
  a.Y = g.Y;
  a.idx = g.idx;
  a.Wt = g.Wt;
  a.Lx = g.Lx;
  a.Ly = g.Ly;
  a.count_dev = g.count_dev;
  a.count_mult = g.count_mult;
  a.n_slots = g.n_slots;
  a.slot_item = g.slot_item;
  a.item_sign = g.item_sign;
  a.sign = g.sign;
  a.logabs = g.logabs;
  a.flags = g.flags;
  a.cond_tau = g.cond_tau;
  a.flag_or = g.flag_or;
  a.perm = g.perm;
  a.refine_tau = g.refine_tau;
  a.ratio = g.ratio;
  const bool nb8 = pf_smem<float, 8>(a.n) <= 113 * 1024;
  switch (g.d) {
    case 8: return nb8 ? launch_fused_nb<8, 8>(a, st) : launch_fused_nb<4, 8>(a, st);
    case 16: return nb8 ? launch_fused_nb<8, 16>(a, st) : launch_fused_nb<4, 16>(a, st);
    case 32: return nb8 ? launch_fused_nb<8, 32>(a, st) : launch_fused_nb<4, 32>(a, st);
    default: return fail(NH_ERR_UNSUPPORTED, "staged Pfaffian: d=%d", g.d);
  }
}

int launch_pfaffian_fused(const FusedLaunch& f, cudaStream_t st) {
  const nh_backflow_params& p = *f.p;
  if (!fused_supported(p)) return fail(NH_ERR_UNSUPPORTED, "fused amplitude: unsupported network");
  PfArgs a{};
  a.n = p.n_up + p.n_dn;
  a.mode = 2;
  a.Wt = p.Wt;
  a.Lx = p.Lx;
  a.Ly = p.Ly;
  a.count_dev = f.cl.n_cfg_dev;
  a.count_mult = f.cl.G;
  a.n_slots = f.cl.n_cfg * f.cl.G;
  a.sign = f.sign;
  a.logabs = f.logabs;
  a.flags = f.flags;
  a.cond_tau = p.cond_tau;
  a.perm = f.perm;
  a.refine_tau = p.refine_tau;
  a.ratio = f.ratio;
  a.cl = f.cl;
  a.cnn_w = p.conv_w_packed;
  a.cnn_b = p.conv_b;
  a.C = p.channels;
  a.layers = p.layers;
  a.item_sign_out = f.item_sign;
  a.queue = f.queue;
  const bool nb8 = pf_smem<float, 8>(a.n) <= 113 * 1024;
  switch (p.channels / 2) {
    case 8: return nb8 ? launch_fused_nb<8, 8>(a, st) : launch_fused_nb<4, 8>(a, st);
    case 16: return nb8 ? launch_fused_nb<8, 16>(a, st) : launch_fused_nb<4, 16>(a, st);
    case 32: return nb8 ? launch_fused_nb<8, 32>(a, st) : launch_fused_nb<4, 32>(a, st);
    default: return fail(NH_ERR_UNSUPPORTED, "fused amplitude: d=%d", p.channels / 2);
  }
}

int launch_pairing(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  const size_t smem = pairing_smem_bytes(Lx * Ly, n, d);
  if (smem <= 227 * 1024 && Lx < 256 && Ly < 256) {
    switch (d) {
      case 8: return launch_pairing_smem<8>(Y, idx, Wt, Lx, Ly, n, batch, F, smem, st);
      case 16: return launch_pairing_smem<16>(Y, idx, Wt, Lx, Ly, n, batch, F, smem, st);
      case 32: return launch_pairing_smem<32>(Y, idx, Wt, Lx, Ly, n, batch, F, smem, st);
      default: break;
    }
  }
  int grid = num_sms() * 4;
  if (grid > batch) grid = batch;
  ProfScope prof_scope(NH_K_PAIRING, st);
  switch (d) {
    case 8: pairing_kernel<8><<<grid, kNumThreads, 0, st>>>(Y, idx, Wt, Lx, Ly, n, batch, F); break;
    case 16: pairing_kernel<16><<<grid, kNumThreads, 0, st>>>(Y, idx, Wt, Lx, Ly, n, batch, F); break;
    case 32: pairing_kernel<32><<<grid, kNumThreads, 0, st>>>(Y, idx, Wt, Lx, Ly, n, batch, F); break;
    default: return fail(NH_ERR_UNSUPPORTED, "pairing_occ: d=%d (8, 16 or 32)", d);
  }
  return check_launch("pairing_kernel");
}

int launch_combine(const float* sg, const double* la, const int32_t* fl, int G, int n_cfg,
                   const int32_t* n_cfg_dev, float* sign, double* logabs, int32_t* flags,
                   double cancel_tau, const int32_t* err, cudaStream_t st) {
  if (n_cfg <= 0) return NH_OK;
  int grid = (n_cfg + 255) / 256;
  ProfScope prof_scope(NH_K_COMBINE, st);
  combine_kernel<<<grid, 256, 0, st>>>(sg, la, fl, G, n_cfg, n_cfg_dev, sign, logabs, flags,
                                       G > 1 ? cancel_tau : 0.0, err);
  return check_launch("combine_kernel");
}

int launch_image_mark(const float* sg, const double* la, int32_t* fl, const float* ratio, int G,
                      int n_cfg, const int32_t* n_cfg_dev, double cancel_tau, double cond_tau,
                      bool weighted, cudaStream_t st) {
  weighted = weighted && ratio;
  if (n_cfg <= 0 || G <= 1 || (cancel_tau <= 0.0 && !weighted)) return NH_OK;
  int grid = (n_cfg + 255) / 256;
  ProfScope prof_scope(NH_K_COMBINE, st);
  image_mark_kernel<<<grid, 256, 0, st>>>(sg, la, fl, ratio, G, n_cfg, n_cfg_dev, cancel_tau,
                                          cond_tau, weighted);
  return check_launch("image_mark_kernel");
}

int launch_flagged(const int32_t* flags, int n_items, const int32_t* count_dev, int count_mult,
                   int32_t* list, int32_t* count, cudaStream_t st, int set_mask, int clear_mask) {
  ProfScope prof_scope(NH_K_FLAGGED, st);
  flagged_kernel<<<1, 1024, 0, st>>>(flags, n_items, count_dev, count_mult, list, count, set_mask,
                                     clear_mask);
  return check_launch("flagged_kernel");
}

}  // namespace nh

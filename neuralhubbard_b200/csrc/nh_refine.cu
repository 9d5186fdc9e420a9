// FP64 refinement of the log-Pfaffian with the pivot order of the FP32 factorisation.
//
// The FP32 kernel (nh_pfaffian.cu) does the part of Parlett-Reid that is latency-bound: the 112
// sequential pivot searches at n = 224.  It records the pivot order it chose (logical index ->
// physical row, plus the parity of the relabelling).  This kernel factorises the same matrix
// again in FP64 with that order held fixed (static pivoting): with no pivot search the
// elimination is blocked into panels of 4 steps (8 logical columns) whose trailing update is a
// rank-8 FP64 product, and it returns the FP64 pivots x_t, so log|pf| = sum_t log|x_t| and
// sign(pf) = item sign x parity x prod_t sign(x_t).  Because the FP32 pivots bound every
// multiplier by ~1, the fixed order is as stable as partial pivoting; the result carries FP64
// rounding only, against ~1e-4 for the FP32 factorisation of an ill-conditioned block.
//
// The matrix is refined against its own FP32 entries (the bits the FP32 kernel factorised, so
// the result is log|pf| of that FP32 matrix to FP64 accuracy) or against the FP64 matrix
// gathered from FP64 features (images flagged ill-conditioned or cancelling, whose FP32 features
// are not accurate enough).  The gather follows pf_kernel.py:156-166 of the reference:
// F[p, q] = sum_a (Y[p, a] Y[q, a]) Wt[2 s_p + s_q, r(p, q), a], in the same order of operations
// as the FP32 gather so that the FP32 matrix is reproduced bit for bit.
//
// One CTA (256 threads) per SM.  Phase 1 stages the Wt table and the item's features in shared
// memory and writes the permuted lower triangle to a per-CTA slice of global scratch (L2
// resident); phase 2 loads it into shared memory as FP64 (row a at roff(a), rows 16-byte
// aligned); phase 3 eliminates.  n <= kRefineMaxN (224: the FP64 triangle takes 200 KB).
#include <math.h>

#include <algorithm>

#include "nh_cnn_item.cuh"
#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kRThreads = 256;
constexpr int kRWarps = kRThreads / 32;
constexpr int kPW = 8;  // panel width: 4 elimination steps

// Row a of the padded lower triangle starts at roff(a) (even, so FP64 pairs are 16-byte aligned).
__host__ __device__ __forceinline__ int roff(int a) { return (a * (a - 1)) / 2 + a / 2; }
// Elements of a whole triangle, rounded up to a multiple of 4 so that every per-CTA slice (FP32
// or FP64) and every 16-byte vector of the copies stays aligned.
__host__ __device__ __forceinline__ int tri_elems(int n) { return (roff(n) + 3) & ~3; }
// Bytes of one CTA's slice: the FP64 triangle, or an item's FP64 rows and modes (modes 3, 4),
// whichever is larger; a multiple of 16.
__host__ __device__ __forceinline__ size_t slice_stride(int n, int d) {
  const size_t tri = 8 * (size_t)tri_elems(n), rows = 8 * (size_t)n * d + 4 * (size_t)n;
  return ((tri > rows ? tri : rows) + 15) & ~(size_t)15;
}

struct RefineArgs {
  int n;
  int mode;  // 0: dense FP32 F (items, n, n); 1: gather FP32 (Y, idx by item); 2: gather FP64
             // (Y64, idx64 by slot, Wt64); 3 / 4: FP32 / FP64 features computed in the kernel
             // from the configuration list, then gathered (Wt / Wt64)
  ConfigList cl;       // modes 3, 4
  const float* cnn_w;  // modes 3, 4: packed weights [l][ci][tap][co]
  const float* cnn_b;
  int C, layers;
  const float* F;
  const void* Y;
  const int32_t* idx;
  const void* Wt;
  int Lx, Ly, D;
  bool stage_wt;  // Wt fits in shared memory with the features
  const int32_t* list;   // slot -> item
  const int32_t* count;  // device number of slots
  const uint16_t* perm;  // per item: perm[0, n) logical -> physical, [n] relabelling parity
  int perm_stride;       // uint16 per item
  const float* item_sign;  // (items,) or null
  float* sign;
  double* logabs;
  int32_t* flags;
  void* slice;  // per CTA: slice_stride(n, D) bytes
};

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  static constexpr int k = 4;
  using V = float4;
};
template <>
struct Vec2<double> {
  static constexpr int k = 2;
  using V = double2;
};

// Phase 1: logical lower triangle A[p][q] = F[perm p][perm q] of one item into the CTA's slice
// (element type T).  Warp <-> 32 consecutive logical columns q (their features in registers
// when small), rows p > q in turn (the row's features broadcast); each element reads one Wt row.
template <typename T, int D, int kRegBytes = 64>
__device__ void gather_permuted(const RefineArgs& a, const T* Yg, const int32_t* ig,
                                const int* perm, unsigned char* smem, T* slice) {
  const int n = a.n, N = a.Lx * a.Ly;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int DP = D + (sizeof(T) == 4 ? 4 : 2);
  constexpr int VK = Vec2<T>::k;
  using V = typename Vec2<T>::V;
  const T* Wg = static_cast<const T*>(a.Wt);
  T* ys = reinterpret_cast<T*>(smem);                    // (n, DP)
  int* info = reinterpret_cast<int*>(ys + n * DP);       // (n) spin << 16 | x << 8 | y
  T* wts = reinterpret_cast<T*>(info + ((n + 3) & ~3));  // (4 N, DP) when staged
  // Row r of the source (D values, 16-byte vectors) to row r of the padded staging copy; several
  // vectors in flight per thread.  Read-only tables (nc) take the non-coherent path; the rows,
  // which modes 3 and 4 write in this kernel, plain loads.
  auto stage = [&](const T* src, T* dst, int rows, bool nc) {
    constexpr int VPR = D / VK;  // vectors per row
    const int nv = rows * VPR;
    for (int v0 = tid; v0 < nv; v0 += 4 * kRThreads) {
      V buf[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int v = v0 + u * kRThreads;
        if (v < nv) buf[u] = nc ? __ldg(reinterpret_cast<const V*>(src) + v)
                                : reinterpret_cast<const V*>(src)[v];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int v = v0 + u * kRThreads;
        if (v < nv) {
          const int r = v / VPR;
          *reinterpret_cast<V*>(dst + r * DP + (v - r * VPR) * VK) = buf[u];
        }
      }
    }
  };
  stage(Yg, ys, n, false);
  for (int p = tid; p < n; p += kRThreads) {
    const int m = ig[p];
    const int sp = m >= N ? 1 : 0, site = m - sp * N, x = site / a.Ly;
    info[p] = (sp << 16) | (x << 8) | (site - x * a.Ly);
  }
  if (a.stage_wt) stage(Wg, wts, 4 * N, true);
  __syncthreads();
  int total = 0;
  for (int qb = 0; 32 * qb + 1 < n; ++qb) total += n - 32 * qb - 1;
  int qb = 0, rem = wid, cur = -1, j = 0, infj = 0;
  // The column's features stay in registers when they are small, else they are read per element.
  constexpr bool kRegs = D * sizeof(T) <= kRegBytes;
  T yj[kRegs ? D : 1];
#pragma unroll 1
  for (int u = wid; u < total; u += kRWarps, rem += kRWarps) {
    while (rem >= n - 32 * qb - 1) {
      rem -= n - 32 * qb - 1;
      ++qb;
    }
    const int q = 32 * qb + lane;
    if (qb != cur) {
      cur = qb;
      j = perm[q < n ? q : 0];
      infj = info[j];
      if constexpr (kRegs) {
#pragma unroll
        for (int c = 0; c < D; c += VK)
          *reinterpret_cast<V*>(yj + c) = *reinterpret_cast<const V*>(ys + j * DP + c);
      }
    }
    const int p = 32 * qb + 1 + rem;
    if (q >= p) continue;
    const int i = perm[p];
    const int infi = info[i];
    const bool up = i > j;  // row i is the higher physical row
    const int ih = up ? infi : infj, il = up ? infj : infi;
    int dx = ((ih >> 8) & 0xFF) - ((il >> 8) & 0xFF), dy = (ih & 0xFF) - (il & 0xFF);
    dx += dx < 0 ? a.Lx : 0;
    dy += dy < 0 ? a.Ly : 0;
    const int r = (2 * (ih >> 16) + (il >> 16)) * N + dx * a.Ly + dy;
    // yi[c] * yj[c] equals the FP32 gather's row-times-column product bit for bit (the product
    // commutes); the accumulation order over c is the gather's.
    const T* yi = ys + i * DP;
    const T* wr = a.stage_wt ? wts + r * DP : Wg + (size_t)r * D;
    T acc = T(0);
#pragma unroll
    for (int c = 0; c < D; c += VK) {
      T vi[VK], vw[VK], vj[VK];
      *reinterpret_cast<V*>(vi) = *reinterpret_cast<const V*>(yi + c);
      if (a.stage_wt)
        *reinterpret_cast<V*>(vw) = *reinterpret_cast<const V*>(wr + c);
      else
        *reinterpret_cast<V*>(vw) = __ldg(reinterpret_cast<const V*>(wr + c));
      if constexpr (kRegs) {
#pragma unroll
        for (int k = 0; k < VK; ++k) vj[k] = yj[c + k];
      } else {
        *reinterpret_cast<V*>(vj) = *reinterpret_cast<const V*>(ys + j * DP + c);
      }
#pragma unroll
      for (int k = 0; k < VK; ++k) acc = fma(vi[k] * vj[k], vw[k], acc);
    }
    slice[roff(p) + q] = up ? acc : -acc;
  }
}

// The CTA's slice (tot = tri_elems(n) values, a multiple of 4) into the FP64 triangle, 16-byte
// vectors with four in flight per thread.
__device__ __forceinline__ void copy_slice(const float* sl, double* S, int tot) {
  const int nv = tot / 4;
  for (int v0 = threadIdx.x; v0 < nv; v0 += 4 * kRThreads) {
    float4 buf[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (v0 + u * kRThreads < nv) buf[u] = reinterpret_cast<const float4*>(sl)[v0 + u * kRThreads];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int v = v0 + u * kRThreads;
      if (v < nv) {
        reinterpret_cast<double2*>(S)[2 * v] = make_double2(buf[u].x, buf[u].y);
        reinterpret_cast<double2*>(S)[2 * v + 1] = make_double2(buf[u].z, buf[u].w);
      }
    }
  }
}
__device__ __forceinline__ void copy_slice(const double* sl, double* S, int tot) {
  const int nv = tot / 2;
  for (int v0 = threadIdx.x; v0 < nv; v0 += 4 * kRThreads) {
    double2 buf[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (v0 + u * kRThreads < nv) buf[u] = reinterpret_cast<const double2*>(sl)[v0 + u * kRThreads];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (v0 + u * kRThreads < nv) reinterpret_cast<double2*>(S)[v0 + u * kRThreads] = buf[u];
  }
}

// Modes 3 and 4: the features of the item's configuration (CNN in shared memory) written as its
// occupied rows Y (n, d) and modes to global memory (the CTA's slice, read back by the gather's
// staging before the gather overwrites it).
template <typename T>
__device__ void features_to(const RefineArgs& a, int item, unsigned char* smem, T* Ydst,
                            int32_t* idst) {
  const int N = a.Lx * a.Ly, C = a.C, M2 = 2 * N, NS = N + 1;
  const int G = a.cl.G;
  const int c = item / G, g = item - c * G;
  const int smp = a.cl.sample ? a.cl.sample[c] : c;
  const int fr = a.cl.from ? a.cl.from[c] : -1;
  const int to = a.cl.from ? a.cl.to[c] : -1;
  const int8_t* base = a.cl.spins + (int64_t)smp * M2;
  __shared__ float sign_dummy;
  int* simg = reinterpret_cast<int*>(smem);
  int* occl = simg + M2;
  int* wbuf = occl + M2;
  const size_t ints = 4 * (size_t)N + 4 * a.Lx + 32;
  T* actA = reinterpret_cast<T*>(smem + ((sizeof(int) * ints + 15) & ~(size_t)15));
  T* actB = actA + C * NS;
  T* wsm = actB + C * NS;
  wsm = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(wsm) + 15) & ~(uintptr_t)15);
  T* bsm = wsm + C * C * 9;
  __syncthreads();
  const T* in = cnn_layers<T>(a.cnn_w, a.cnn_b, a.Lx, a.Ly, C, a.layers, base, fr, to, g, actA,
                              actB, wsm, bsm, simg);
  const int d = C / 2;
  write_occupied_rows(simg, occl, wbuf, N, a.n, d, g, a.Lx, a.Ly, Ydst, idst, &sign_dummy,
                      [&](int sg, int aa, int site) { return in[(sg * d + aa) * NS + site]; });
  __syncthreads();
}

// Shared memory of the in-kernel CNN (modes 3, 4).
size_t features_smem(int N, int C, int Lx, int elt) {
  const size_t ints = 4 * (size_t)N + 4 * Lx + 32;
  const size_t act = ((sizeof(int) * ints + 15) & ~(size_t)15) + (size_t)elt * 2 * C * (N + 1);
  return ((act + 15) & ~(size_t)15) + (size_t)elt * ((size_t)C * C * 9 + C);
}

// MODE is a.mode as a template argument, so that each instance holds only its own phase-1 code
// (the register allocation of the elimination is then not shaped by the other modes).
template <int D, int MODE>
__global__ void __launch_bounds__(kRThreads, 1) refine_kernel(RefineArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int perm_s[kRefineMaxN];
  __shared__ double Lm[kPW * kPW];  // block multipliers L[r][c] of the current panel
  __shared__ double xs[kPW / 2];    // its FP64 pivots
  __shared__ double xinv[kPW / 2];  // and their reciprocals
  __shared__ double xy[2][kPW];     // pivot-block columns k, k+1 of the current step
  const int n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double* S = reinterpret_cast<double*>(smem);
  const int n_work = *a.count;
  for (int slot = blockIdx.x; slot < n_work; slot += gridDim.x) {
    const int item = a.list[slot];
    const uint16_t* pr = a.perm + (size_t)item * a.perm_stride;
    __syncthreads();
    for (int p = tid; p < n; p += kRThreads) perm_s[p] = pr[p];
    __syncthreads();
    // Phases 1 and 2: the permuted lower triangle in FP64 shared memory.
    if constexpr (MODE == 0) {
      const float* F = a.F + (size_t)item * n * n;
      for (int p = wid; p < n; p += kRWarps) {
        const int i = perm_s[p];
        for (int q = lane; q < p; q += 32) {
          const int j = perm_s[q];
          S[roff(p) + q] = i > j ? (double)__ldg(F + (size_t)i * n + j)
                                 : -(double)__ldg(F + (size_t)j * n + i);
        }
      }
    } else {
      const int tot = tri_elems(n);  // a multiple of 4
      unsigned char* slb = static_cast<unsigned char*>(a.slice) + (size_t)blockIdx.x * slice_stride(n, D);
      if constexpr (MODE == 1 || MODE == 3) {
        float* sl = reinterpret_cast<float*>(slb);
        const float* Yg = static_cast<const float*>(a.Y) + (size_t)item * n * D;
        const int32_t* ig = a.idx + (size_t)item * n;
        if constexpr (MODE == 3) {  // the item's FP32 features, rows and modes to the slice
          features_to(a, item, smem, sl, reinterpret_cast<int32_t*>(sl + n * D));
          Yg = sl;
          ig = reinterpret_cast<const int32_t*>(sl + n * D);
        }
        gather_permuted<float, D>(a, Yg, ig, perm_s, smem, sl);
        __syncthreads();  // slice written; the staging area is dead
        copy_slice(sl, S, tot);
      } else {
        double* sl = reinterpret_cast<double*>(slb);
        const double* Yg = static_cast<const double*>(a.Y) + (size_t)slot * n * D;
        const int32_t* ig = a.idx + (size_t)slot * n;
        if constexpr (MODE == 4) {
          features_to(a, item, smem, sl, reinterpret_cast<int32_t*>(sl + n * D));
          Yg = sl;
          ig = reinterpret_cast<const int32_t*>(sl + n * D);
        }
        // mode 2 keeps each column's FP64 features in registers (its instance has the room)
        gather_permuted<double, D, MODE == 2 ? 128 : 64>(a, Yg, ig, perm_s, smem, sl);
        __syncthreads();
        copy_slice(sl, S, tot);
      }
    }
    __syncthreads();

    // Phase 3: static-pivot blocked elimination.
    double mant = 1.0;  // thread 0: running product of |x_t| as mantissa and exponent
    int expo = 0, neg = 0, bad = 0;
    for (int k0 = 0; k0 < n; k0 += kPW) {
      const int w = min(kPW, n - k0), steps = w >> 1;
      if (wid == 0) {
        // (1) factorise the w x w pivot block: lane r holds row r, row[c] = B[r][c] (c < r);
        // each step's columns k, k+1 go through shared memory to every lane.
        double row[kPW];
#pragma unroll
        for (int c = 0; c < kPW; ++c)
          row[c] = (lane < w && c < lane) ? S[roff(k0 + lane) + k0 + c] : 0.0;
#pragma unroll
        for (int t = 0; t < kPW / 2; ++t) {
          if (t < steps) {
            const int k = 2 * t;
            const double xr = row[k], yr = row[k + 1];  // B[r][k], B[r][k+1] (lanes r > k+1)
            if (lane < kPW) {
              xy[0][lane] = xr;
              xy[1][lane] = yr;
            }
            __syncwarp();
            const double piv = -xy[0][k + 1];  // B[k][k+1] = -B[k+1][k]
            const double inv = 1.0 / piv;
            if (lane == 0) {
              xs[t] = piv;
              xinv[t] = inv;
            }
            if (lane >= k + 2 && lane < w) {
              Lm[lane * kPW + k] = yr * inv;
              Lm[lane * kPW + k + 1] = -xr * inv;
            }
            const double yi = yr * inv, xi = xr * inv;
#pragma unroll
            for (int c = 0; c < kPW; ++c)
              if (c >= k + 2 && c < lane && lane < w) row[c] += yi * xy[0][c] - xi * xy[1][c];
            __syncwarp();
          }
        }
      }
      __syncthreads();
      if (tid == 0) {
        for (int t = 0; t < steps; ++t) {
          const double x = xs[t];
          if (x < 0.0) neg ^= 1;
          const double ax = fabs(x);
          if (!(ax > 0.0) || !isfinite(ax)) bad |= ax == 0.0 ? NH_FLAG_ZERO_PIVOT : NH_FLAG_NONFINITE;
          int e;
          mant = frexp(mant * ax, &e);
          expo += e;
        }
      }
      const int base = k0 + w;
      const int m = n - base;
      if (m <= 0) break;
      // (2) rows c >= base: W[:, c] = L11^-1 A12[:, c] with A12[i][c] = -S[c][k0 + i]; the dead
      // slots S[c][k0, k0 + w) then hold P[c][2t] = W[2t+1][c] / x_t, P[c][2t+1] = -W[2t][c] / x_t.
      for (int c = base + tid; c < n; c += kRThreads) {
        double* sc = S + roff(c) + k0;
        double wv[kPW];
#pragma unroll
        for (int i = 0; i < kPW; i += 2) {
          if (i < w) {
            const double2 v = *reinterpret_cast<const double2*>(sc + i);
            wv[i] = -v.x;
            wv[i + 1] = -v.y;
          } else {
            wv[i] = wv[i + 1] = 0.0;
          }
        }
#pragma unroll
        for (int t = 0; t < kPW / 2; ++t) {
          const int k = 2 * t;
#pragma unroll
          for (int r = k + 2; r < kPW; ++r)
            if (r < w) wv[r] -= Lm[r * kPW + k] * wv[k] + Lm[r * kPW + k + 1] * wv[k + 1];
        }
#pragma unroll
        for (int t = 0; t < kPW / 2; ++t) {
          if (2 * t < w) {
            const double inv = xinv[t];
            *reinterpret_cast<double2*>(sc + 2 * t) =
                make_double2(wv[2 * t + 1] * inv, -wv[2 * t] * inv);
          }
        }
      }
      __syncthreads();
      // (3) trailing update S[a][b] += sum_i P[a][i] W[i][b] for base <= b < a: warp <-> a pair of
      // rows, lane <-> columns b0 = base + 64 cb + lane and b0 + 32 (their W in registers), the
      // rows' P broadcast; four elements and two partial sums each per lane keep the FP64 pipe
      // fed.  All loads of a unit precede its stores.
      if (m >= 2) {
        double xv[kPW / 2];
#pragma unroll
        for (int t = 0; t < kPW / 2; ++t) xv[t] = t < steps ? xs[t] : 0.0;
        // units: (column block cb, row pair) over rows base + 64 cb + 1 .. n - 1
        auto pairs = [&](int cb) { return (m - 64 * cb - 1 + 1) >> 1; };
        int total = 0;
        for (int cb = 0; 64 * cb + 1 < m; ++cb) total += pairs(cb);
        int cb = 0, rem = wid, cur = -1;
        double w0[kPW], w1[kPW];
        int b0 = 0, b1 = 0;
#pragma unroll 1
        for (int u = wid; u < total; u += kRWarps, rem += kRWarps) {
          while (rem >= pairs(cb)) {
            rem -= pairs(cb);
            ++cb;
          }
          if (cb != cur) {
            cur = cb;
            b0 = base + 64 * cb + lane;
            b1 = b0 + 32;
#pragma unroll
            for (int t = 0; t < kPW / 2; ++t) {
              double2 p0 = make_double2(0.0, 0.0), p1 = make_double2(0.0, 0.0);
              if (b0 < n) p0 = *reinterpret_cast<const double2*>(S + roff(b0) + k0 + 2 * t);
              if (b1 < n) p1 = *reinterpret_cast<const double2*>(S + roff(b1) + k0 + 2 * t);
              // W[2t][b] = -P[b][2t+1] x_t, W[2t+1][b] = P[b][2t] x_t
              w0[2 * t] = -p0.y * xv[t];
              w0[2 * t + 1] = p0.x * xv[t];
              w1[2 * t] = -p1.y * xv[t];
              w1[2 * t + 1] = p1.x * xv[t];
            }
          }
          const int ra = base + 64 * cb + 1 + 2 * rem;  // rows ra and ra + 1
          const int rb = ra + 1 < n ? ra + 1 : ra;
          double* rowa = S + roff(ra);
          double* rowb = S + roff(rb);
          const bool a0 = b0 < ra, a1 = b1 < ra, c0 = rb != ra && b0 < rb, c1 = rb != ra && b1 < rb;
          double acc[4][2];
          acc[0][0] = a0 ? rowa[b0] : 0.0;
          acc[1][0] = a1 ? rowa[b1] : 0.0;
          acc[2][0] = c0 ? rowb[b0] : 0.0;
          acc[3][0] = c1 ? rowb[b1] : 0.0;
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[e][1] = 0.0;
#pragma unroll
          for (int i = 0; i < kPW; i += 2) {
            const double2 pa = *reinterpret_cast<const double2*>(rowa + k0 + i);
            const double2 pb = *reinterpret_cast<const double2*>(rowb + k0 + i);
            const int h = (i >> 1) & 1;
            acc[0][h] = fma(pa.x, w0[i], acc[0][h]);
            acc[1][h] = fma(pa.x, w1[i], acc[1][h]);
            acc[2][h] = fma(pb.x, w0[i], acc[2][h]);
            acc[3][h] = fma(pb.x, w1[i], acc[3][h]);
            acc[0][h] = fma(pa.y, w0[i + 1], acc[0][h]);
            acc[1][h] = fma(pa.y, w1[i + 1], acc[1][h]);
            acc[2][h] = fma(pb.y, w0[i + 1], acc[2][h]);
            acc[3][h] = fma(pb.y, w1[i + 1], acc[3][h]);
          }
          if (a0) rowa[b0] = acc[0][0] + acc[0][1];
          if (a1) rowa[b1] = acc[1][0] + acc[1][1];
          if (c0) rowb[b0] = acc[2][0] + acc[2][1];
          if (c1) rowb[b1] = acc[3][0] + acc[3][1];
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      float s = a.item_sign ? a.item_sign[item] : 1.0f;
      if (pr[n] & 1) s = -s;
      if (neg) s = -s;
      int f = a.flags ? a.flags[item] : 0;
      f &= ~(kFlagNeedRefine | NH_FLAG_ZERO_PIVOT | NH_FLAG_NONFINITE);
      double la = log(mant) + (double)expo * 0.6931471805599453;
      if (isnan(s)) f |= NH_FLAG_NONFINITE;
      if (bad & NH_FLAG_ZERO_PIVOT) {
        s = 0.0f;
        la = -INFINITY;
      }
      if (!isfinite(la) && s != 0.0f) bad |= NH_FLAG_NONFINITE;
      f |= bad | NH_FLAG_REFINED;
      a.sign[item] = s;
      a.logabs[item] = s == 0.0f ? -INFINITY : la;
      if (a.flags) a.flags[item] = f;
    }
  }
}

size_t stage_bytes(int n, int N, int D, int elt, bool wt) {
  const int DP = D + (elt == 4 ? 4 : 2);
  return (size_t)elt * n * DP + sizeof(int) * ((n + 3) & ~3) + (wt ? (size_t)elt * 4 * N * DP : 0);
}

template <int D>
int launch_refine_d(RefineArgs a, int max_slots, cudaStream_t st) {
  const int N = a.Lx * a.Ly;
  const size_t tri = sizeof(double) * tri_elems(a.n);
  size_t smem = tri;
  if (a.mode != 0) {
    const int elt = (a.mode == 1 || a.mode == 3) ? 4 : 8;
    a.stage_wt = stage_bytes(a.n, N, D, elt, true) <= kRefineSmemLimit;
    smem = std::max(smem, stage_bytes(a.n, N, D, elt, a.stage_wt));
    if (a.mode >= 3) smem = std::max(smem, features_smem(N, a.C, a.Lx, elt));
  }
  if (smem > kRefineSmemLimit)
    return fail(NH_ERR_UNSUPPORTED, "refine: n=%d needs %zu B of shared memory", a.n, smem);
  static bool configured[5] = {false, false, false, false, false};
  auto kern = a.mode == 0 ? refine_kernel<D, 0> : a.mode == 1 ? refine_kernel<D, 1>
            : a.mode == 2 ? refine_kernel<D, 2> : a.mode == 3 ? refine_kernel<D, 3>
                                                 : refine_kernel<D, 4>;
  if (!configured[a.mode]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kRefineSmemLimit);
    if (e != cudaSuccess) return check_cuda(e, "refine smem attribute");
    configured[a.mode] = true;
  }
  int grid = num_sms();
  if (grid > max_slots) grid = max_slots;
  if (grid <= 0) return NH_OK;
  ProfScope prof_scope(NH_K_REFINE, st);
  kern<<<grid, kRThreads, smem, st>>>(a);
  return check_launch("refine_kernel");
}

}  // namespace

size_t refine_slice_bytes(int n, int d) {
  return (n > 0 && n <= kRefineMaxN) ? (size_t)num_sms() * slice_stride(n, d < 8 ? 8 : d) : 0;
}

int launch_refine(const RefineLaunch& q, cudaStream_t st) {
  if (q.n <= 0 || q.n % 2 || q.n > kRefineMaxN)
    return fail(NH_ERR_UNSUPPORTED, "refine: n=%d (even, <= %d)", q.n, kRefineMaxN);
  if (q.max_slots <= 0) return NH_OK;
  if (q.mode < 0 || q.mode > 4) return fail(NH_ERR_INVALID, "refine: mode %d", q.mode);
  if (q.mode != 0 && !q.slice) return fail(NH_ERR_INVALID, "refine: gather mode needs the slice");
  RefineArgs a{};
  a.n = q.n;
  a.mode = q.mode;
  a.F = q.F;
  a.Y = q.Y;
  a.idx = q.idx;
  a.Wt = q.Wt;
  a.Lx = q.Lx;
  a.Ly = q.Ly;
  a.D = q.d;
  a.list = q.list;
  a.count = q.count;
  a.perm = q.perm;
  a.perm_stride = q.perm_stride;
  a.item_sign = q.item_sign;
  a.sign = q.sign;
  a.logabs = q.logabs;
  a.flags = q.flags;
  a.slice = q.slice;
  a.cl = q.cl;
  a.cnn_w = q.cnn_w;
  a.cnn_b = q.cnn_b;
  a.C = q.C;
  a.layers = q.layers;
  if (q.mode >= 3 && (!q.cnn_w || !q.cnn_b || q.C % 16 || q.d * 2 != q.C))
    return fail(NH_ERR_INVALID, "refine: in-kernel features need the CNN weights");
  switch (q.mode == 0 ? 16 : q.d) {
    case 8: return launch_refine_d<8>(a, q.max_slots, st);
    case 16: return launch_refine_d<16>(a, q.max_slots, st);
    case 32: return launch_refine_d<32>(a, q.max_slots, st);
    default: return fail(NH_ERR_UNSUPPORTED, "refine: d=%d (8, 16 or 32)", q.d);
  }
}

}  // namespace nh

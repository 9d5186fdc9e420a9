// BCS-backflow amplitude: sign and log|det| of the occupied up x down pairing block
// (code/backflow/models.py:214-302, code/backflow/bcs_kernel.py:1-70),
//
//   F[p, q] = sum_a Yu[p, a] Wt_ud[site_p - site_q, a] Yd[q, a] + delta_d fd(site_p - site_q),
//   psi(s)  = det F (-1)^(n_up (n_up - 1) / 2) x the item sign of the image,
//
// with Wt_ud = block 1 (ud) of the (4, N, d) table of nh_build_wtilde and fd the
// nearest-neighbour d-wave form factor (-1 on x bonds, +1 on y bonds, code/backflow/models.py:
// 80-82).  One matrix per 512-thread CTA, held in registers: thread (warp w, lane c) owns rows
// w + 16 t and columns c + 32 u.  Each thread gathers its own elements (features staged in shared
// memory, Wt rows read through L1), then an LU elimination with implicit partial pivoting runs
// on the registers: per step each warp gathers column k of its rows onto its lanes by shuffles,
// takes its largest unused entry with two 32-bit warp reductions, stores that row as its
// candidate in shared memory and proposes it through one 64-bit shared-memory maximum; after the
// step's one barrier every thread reads the winning warp's candidate as the pivot row, and every
// unused row takes its rank-1 update.  det F = parity(pivot order) x prod of the pivots; the log-sum of the
// pivots is accumulated in FP64 as mantissa and exponent.
#include <math.h>

#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kDetThreads = 512;

struct DetArgs {
  const void* Y;       // (slots, n, d): rows [0, nh) the up modes, [nh, 2 nh) the down modes
  const int32_t* idx;  // (slots, n)
  const void* Wt;      // (4, N, d), block 1 read
  int Lx, Ly, nh;
  double delta_d;
  const int32_t* count_dev;  // device work count (times count_mult) or null
  int count_mult;
  int n_slots;
  const int32_t* slot_item;  // slot -> item, null: identity
  const float* item_sign;
  float* sign;
  double* logabs;
  int32_t* flags;
  float* ratio;  // (items,) pivot ratio, or null
  double cond_tau;
  int flag_or;
};

__device__ __forceinline__ unsigned long long det_key(float mag, int row) {
  return ((unsigned long long)__float_as_uint(mag) << 32) | (unsigned)(0x7FFFFFFF - row);
}

__device__ __forceinline__ float key_mag(float x) { return fabsf(x); }
__device__ __forceinline__ float key_mag(double x) { return __double2float_ru(fabs(x)); }

template <typename T, int TC>
__global__ void __launch_bounds__(kDetThreads, 1) det_kernel(DetArgs a) {
  constexpr int TR = 2 * TC, NP = 32 * TC;
  constexpr int D = 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nh = a.nh, n = 2 * nh, N = a.Lx * a.Ly, Lx = a.Lx, Ly = a.Ly;
  T* ys = reinterpret_cast<T*>(smem_raw);          // (n, D)
  T* colbuf = ys + (size_t)n * D;                  // [2][NP]
  T* cand = colbuf + 2 * NP;                       // [2][16][NP] each warp's best row of the step
  T* pivs = cand + 32 * NP;                        // [NP]
  int* info = reinterpret_cast<int*>(pivs + NP);   // (n) spin << 16 | x << 8 | y
  int* rho = info + n;                             // [NP] pivot row of step k
  int* mark = rho + NP;                            // [NP] parity scratch
  unsigned long long* slot = reinterpret_cast<unsigned long long*>(mark + NP);  // [3]
  int* bad_s = reinterpret_cast<int*>(slot + 3);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T* Yb = static_cast<const T*>(a.Y);
  const T* Wud = static_cast<const T*>(a.Wt) + (size_t)N * D;
  const int n_work = a.count_dev ? (*a.count_dev) * a.count_mult : a.n_slots;

  for (int slot_i = blockIdx.x; slot_i < n_work; slot_i += gridDim.x) {
    const int item = a.slot_item ? a.slot_item[slot_i] : slot_i;
    const T* Yi = Yb + (size_t)slot_i * n * D;
    const int32_t* ii = a.idx + (size_t)slot_i * n;
    __syncthreads();  // the previous item's readers are done
    for (int e = threadIdx.x; e < n * D; e += kDetThreads) ys[e] = Yi[e];
    for (int p = threadIdx.x; p < n; p += kDetThreads) {
      int m = __ldg(ii + p);
      if ((unsigned)m >= (unsigned)(2 * N)) m = 0;
      const int sp = m >= N ? 1 : 0, site = m - sp * N, x = site / Ly;
      info[p] = (sp << 16) | (x << 8) | (site - x * Ly);
    }
    if (threadIdx.x == 0) {
      slot[0] = slot[1] = 0ull;  // slot[2] is cleared after step 0's barrier
      *bad_s = 0;
    }
    __syncthreads();
    // Gather: element (I, J) = F[up row I][down row J].
    T A[TR][TC];
#pragma unroll
    for (int t = 0; t < TR; ++t) {
      const int I = warp + 16 * t;
#pragma unroll
      for (int u = 0; u < TC; ++u) {
        const int J = lane + 32 * u;
        T v = (I == J) ? T(1) : T(0);
        if (I < nh && J < nh) {
          const int ip = info[I], iq = info[nh + J];
          int dx = ((ip >> 8) & 0xFF) - ((iq >> 8) & 0xFF), dy = (ip & 0xFF) - (iq & 0xFF);
          dx += dx < 0 ? Lx : 0;
          dy += dy < 0 ? Ly : 0;
          const T* w = Wud + (size_t)(dx * Ly + dy) * D;
          const T* yp = ys + (size_t)I * D;
          const T* yq = ys + (size_t)(nh + J) * D;
          T acc = T(0);
#pragma unroll
          for (int c = 0; c < D; ++c) acc += (yp[c] * yq[c]) * __ldg(w + c);
          const int mx = min(dx, Lx - dx), my = min(dy, Ly - dy);
          const T fd = (mx == 1 && my == 0) ? T(-1) : ((mx == 0 && my == 1) ? T(1) : T(0));
          v = acc + T(a.delta_d) * fd;
        }
        A[t][u] = v;
      }
    }
    unsigned used = 0;
#pragma unroll
    for (int t = 0; t < TR; ++t)
      if (warp + 16 * t >= nh) used |= 1u << t;
    int bad = 0;
    // One barrier per step.  The key slots rotate over three (slot sl is read after the step's
    // barrier and cleared after the next step's barrier, two steps before its next use); the
    // column and candidate buffers alternate by parity (a warp writes step k + 2's copy only
    // after every warp has passed step k + 1's barrier, so after every read of step k's).
    int sl = 0;
#pragma unroll
    for (int uk = 0; uk < TC; ++uk) {
      for (int lk = 0; lk < 32; ++lk) {
        const int k = uk * 32 + lk;
        if (k >= nh || bad) break;  // uniform
        const int par = k & 1;
        {
          // Column k of this warp's rows, spread over the lanes (lane t takes row warp + 16 t)
          // so that the pivot proposal runs on TR lanes instead of the one owning the column.
          T cv = T(0);
#pragma unroll
          for (int t = 0; t < TR; ++t) {
            const T v = __shfl_sync(0xffffffffu, A[t][uk], lk);
            if (lane == t) cv = v;
          }
          unsigned long long key = 0ull;
          if (lane < TR) {
            colbuf[par * NP + warp + 16 * lane] = cv;
            if (!((used >> lane) & 1u)) key = det_key(key_mag(cv), warp + 16 * lane);
          }
          // 64-bit warp maximum as two 32-bit reductions: the magnitude bits, then the row
          // tie-break among the lanes holding that magnitude.
          const unsigned hi = (unsigned)(key >> 32);
          const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
          const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? (unsigned)key : 0u);
          key = ((unsigned long long)mh << 32) | ml;
          if (key) {  // this warp's best row goes to its candidate slot
            const int tl = (0x7FFFFFFF - (int)ml) >> 4;
            T* cw = cand + (size_t)(par * 16 + warp) * NP;
#pragma unroll
            for (int t = 0; t < TR; ++t)
              if (t == tl) {
#pragma unroll
                for (int u = 0; u < TC; ++u) cw[lane + 32 * u] = A[t][u];
              }
            if (lane == 0) atomicMax(slot + sl, key);
          }
        }
        __syncthreads();
        const unsigned long long win = slot[sl];
        const int p = 0x7FFFFFFF - (int)(unsigned)(win & 0xFFFFFFFFull);
        const float mag = __uint_as_float((unsigned)(win >> 32));
        if (win == 0ull || !(mag > 0.0f && mag <= 3.0e38f)) {
          bad = (win == 0ull || mag == 0.0f) ? NH_FLAG_ZERO_PIVOT : NH_FLAG_NONFINITE;
          __syncthreads();
          break;
        }
        if (warp == (p & 15)) used |= 1u << (p >> 4);
        if (threadIdx.x == 0) {
          slot[sl == 0 ? 2 : sl - 1] = 0ull;
          rho[k] = p;
          pivs[k] = colbuf[par * NP + p];
        }
        sl = sl == 2 ? 0 : sl + 1;
        const T* prow = cand + (size_t)(par * 16 + (p & 15)) * NP;
        const T inv = T(1) / colbuf[par * NP + p];
        T r[TC];
#pragma unroll
        for (int u = 0; u < TC; ++u) r[u] = prow[lane + 32 * u] * inv;
#pragma unroll
        for (int t = 0; t < TR; ++t) {
          if ((used >> t) & 1u) continue;  // eliminated rows keep their values (never read)
          const T f = colbuf[par * NP + warp + 16 * t];
#pragma unroll
          for (int u = 0; u < TC; ++u) A[t][u] = fma(-f, r[u], A[t][u]);
        }
      }
    }
    if (threadIdx.x == 0 && bad) *bad_s = bad;
    __syncthreads();
    if (threadIdx.x == 0) {
      bad = *bad_s;
      const float isg = a.item_sign ? a.item_sign[item] : 1.0f;
      float s = isg;
      int flag = bad;
      double la = -INFINITY, ratio = INFINITY;
      if (isnan(s)) flag |= NH_FLAG_NONFINITE;
      if (bad) {
        s = 0.0f;
      } else {
        // parity of the pivot order (cycle decomposition of k -> rho[k])
        for (int k = 0; k < nh; ++k) mark[k] = 0;
        int par = (nh * (nh - 1) / 2) & 1;  // the block's (-1)^(n_up (n_up - 1) / 2)
        for (int k = 0; k < nh; ++k) {
          if (mark[k]) continue;
          int len = 0;
          for (int j = k; !mark[j]; j = rho[j]) {
            mark[j] = 1;
            ++len;
          }
          par ^= (len - 1) & 1;
        }
        double mant = 1.0, pmin = INFINITY, pmax = 0.0;
        int expo = 0;
        for (int k = 0; k < nh; ++k) {
          const double pv = (double)pivs[k];
          if (pv < 0.0) par ^= 1;
          const double ap = fabs(pv);
          if (!isfinite(ap)) flag |= NH_FLAG_NONFINITE;
          pmin = fmin(pmin, ap);
          pmax = fmax(pmax, ap);
          int e;
          mant = frexp(mant * ap, &e);
          expo += e;
        }
        if (par) s = -s;
        la = log(mant) + (double)expo * 0.6931471805599453;
        if (!isfinite(la)) flag |= NH_FLAG_NONFINITE;
        ratio = pmax / pmin;
        if (a.cond_tau > 0.0 && pmax > a.cond_tau * pmin) flag |= NH_FLAG_GROWTH;
      }
      if (s == 0.0f) la = -INFINITY;
      a.sign[item] = s;
      a.logabs[item] = la;
      if (a.flags) a.flags[item] = flag | a.flag_or;
      if (a.ratio) a.ratio[item] = (float)ratio;
    }
  }
}

template <typename T, int TC>
size_t det_smem(int nh) {
  constexpr int NP = 32 * TC;
  const size_t n = 2 * (size_t)nh;
  return sizeof(T) * (n * 16 + 35 * NP) + sizeof(int) * (n + 2 * NP) + 24 + 16;
}

template <typename T, int TC>
int launch_det_t(const DetArgs& a, cudaStream_t st) {
  const size_t smem = det_smem<T, TC>(a.nh);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(det_kernel<T, TC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "det smem attribute");
    configured = smem;
  }
  const int slots = a.n_slots;
  if (slots <= 0) return NH_OK;
  int grid = num_sms();
  if (grid > slots) grid = slots;
  ProfScope prof_scope(sizeof(T) == 8 ? NH_K_DET64 : NH_K_DET, st);
  det_kernel<T, TC><<<grid, kDetThreads, smem, st>>>(a);
  return check_launch(sizeof(T) == 8 ? "det_kernel<double>" : "det_kernel<float>");
}

}  // namespace

bool det_supported(int nh, int d, bool fp64) {
  return d == 16 && nh >= 1 && nh <= (fp64 ? kDetMaxNh64 : kDetMaxNh);
}

int launch_det(const DetLaunch& q, cudaStream_t st) {
  if (!det_supported(q.nh, q.d, q.fp64))
    return fail(NH_ERR_UNSUPPORTED, "BCS determinant: n_up %d (<= %d FP32, %d FP64), d %d (16)",
                q.nh, kDetMaxNh, kDetMaxNh64, q.d);
  DetArgs a{q.Y, q.idx, q.Wt, q.Lx, q.Ly, q.nh, q.delta_d, q.count_dev, q.count_mult, q.n_slots,
            q.slot_item, q.item_sign, q.sign, q.logabs, q.flags, q.ratio, q.cond_tau,
            q.flag_or};
  const int tc = (q.nh + 31) / 32;
  if (q.fp64) {
    switch (tc) {
      case 1: return launch_det_t<double, 1>(a, st);
      case 2: return launch_det_t<double, 2>(a, st);
      case 3: return launch_det_t<double, 3>(a, st);
      default: return launch_det_t<double, 4>(a, st);
    }
  }
  switch (tc) {
    case 1: return launch_det_t<float, 1>(a, st);
    case 2: return launch_det_t<float, 2>(a, st);
    case 3: return launch_det_t<float, 3>(a, st);
    case 4: return launch_det_t<float, 4>(a, st);
    case 5: return launch_det_t<float, 5>(a, st);
    case 6: return launch_det_t<float, 6>(a, st);
    default: return launch_det_t<float, 7>(a, st);
  }
}

}  // namespace nh

// Batched log-Pfaffian (blocked Parlett-Reid LTL^T with partial pivoting), the pairing
// gather, and the combination of symmetry images.
//
// One CTA (256 threads) per antisymmetric n x n matrix, n even, n <= 256, two CTAs per SM at
// n = 224.  The strict lower triangle lives in shared memory in FP32 (row i at offset
// i (i - 1) / 2).  Thread t owns physical row t.  A pivot does not move data: it swaps the
// logical labels of two physical rows (my_log), so the panel needs two block barriers per
// elimination step.  Panel columns are formed lazily (stored column plus the panel's rank-2
// terms U V^T - V U^T); at the end of a panel of NB steps the active rows are compacted into a
// list and the trailing triangle receives the rank-2NB update.  The Pfaffian is the product
// of the pivots A[k, k+1] times the parity of the relabelling; the product is accumulated in
// FP64 as mantissa and exponent, logabs = log(mantissa) + exponent log 2.
//
// Replaces fermix.slogpf (code/backflow/models.py:210) and, in the gather mode, the Pallas
// pairing kernel pfsbp_pairing_fwd (code/backflow/pf_kernel.py:156-190) whose formula it
// follows: F[p, q] = sum_a (Y[p, a] Y[q, a]) Wt[2 s_p + s_q, r(p, q), a] with the product of
// the features formed first, so that F[q, p] = -F[p, q] holds bit for bit.
#include <math.h>

#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kWarps = kNumThreads / 32;
constexpr float kGrowth = 1.0e4f;  // pivot-growth flag threshold (|col max| / initial max)

struct PfArgs {
  int n;
  int mode;  // 0: F dense (batch, n, n) in global memory; 1: gather from Y / idx / Wt
  const float* F;
  const float* Y;
  const int32_t* idx;
  const float* Wt;
  int Lx, Ly, d;
  const int32_t* n_cfg_dev;  // device count of configurations (items = count * G) or null
  int G;
  int n_items;
  const float* item_sign;
  float* sign;
  double* logabs;
  int32_t* flags;
};

__device__ __forceinline__ int tri_off(int i) { return (i * (i - 1)) >> 1; }

// Element (i, j) of the antisymmetric matrix stored as a strict lower triangle.
__device__ __forceinline__ float aval(const float* Lw, int i, int j) {
  return i > j ? Lw[tri_off(i) + j] : (i < j ? -Lw[tri_off(j) + i] : 0.0f);
}

// F[p, q] of the gather for p > q (the stored lower element); the row p features are in
// registers (yp), the Wt row is gathered by displacement and spin block.
template <int D>
__device__ __forceinline__ float pair_value(const float* yp, int sp, int xp, int ypos,
                                            const float* __restrict__ Yq, int mq, int N, int Lx,
                                            int Ly, const float* __restrict__ Wt) {
  const int sq = mq >= N ? 1 : 0;
  const int siteq = mq - sq * N;
  const int xq = siteq / Ly, yq = siteq - xq * Ly;
  int dx = xp - xq, dy = ypos - yq;
  dx += dx < 0 ? Lx : 0;
  dy += dy < 0 ? Ly : 0;
  const int r = dx * Ly + dy;
  const float4* w4 = reinterpret_cast<const float4*>(Wt + ((size_t)(2 * sp + sq) * N + r) * D);
  const float4* q4 = reinterpret_cast<const float4*>(Yq);
  float acc = 0.0f;
#pragma unroll
  for (int a4 = 0; a4 < D / 4; ++a4) {
    const float4 w = __ldg(w4 + a4);
    const float4 q = __ldg(q4 + a4);
    acc = fmaf(yp[4 * a4 + 0] * q.x, w.x, acc);
    acc = fmaf(yp[4 * a4 + 1] * q.y, w.y, acc);
    acc = fmaf(yp[4 * a4 + 2] * q.z, w.z, acc);
    acc = fmaf(yp[4 * a4 + 3] * q.w, w.w, acc);
  }
  return acc;
}

template <int D>
__device__ void gather_lower(float* Lw, int n, const float* __restrict__ Y,
                             const int32_t* __restrict__ idx, const float* __restrict__ Wt,
                             int Lx, int Ly) {
  const int N = Lx * Ly;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int p = wid; p < n; p += kWarps) {
    const int mp = __ldg(idx + p);
    const int sp = mp >= N ? 1 : 0;
    const int sitep = mp - sp * N;
    const int xp = sitep / Ly, ypos = sitep - xp * Ly;
    float yp[D];
    const float4* p4 = reinterpret_cast<const float4*>(Y + (size_t)p * D);
#pragma unroll
    for (int a4 = 0; a4 < D / 4; ++a4) {
      float4 v = __ldg(p4 + a4);
      yp[4 * a4] = v.x;
      yp[4 * a4 + 1] = v.y;
      yp[4 * a4 + 2] = v.z;
      yp[4 * a4 + 3] = v.w;
    }
    float* row = Lw + tri_off(p);
    for (int q = lane; q < p; q += 32)
      row[q] = pair_value<D>(yp, sp, xp, ypos, Y + (size_t)q * D, __ldg(idx + q), N, Lx, Ly, Wt);
  }
}

template <int NB, int D>
__global__ void __launch_bounds__(kNumThreads, 2) pfaffian_kernel(PfArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int tri = tri_off(n);
  float* Lw = reinterpret_cast<float*>(smem_raw);
  float* Us = Lw + ((tri + 3) & ~3);  // (n, NB)
  float* Vs = Us + n * NB;            // (n, NB)
  int* alist = reinterpret_cast<int*>(Vs + n * NB);  // (n) active physical rows
  float* rkey = reinterpret_cast<float*>(alist + n);  // (warps) best |value|
  int* rt = reinterpret_cast<int*>(rkey + kWarps);    // (warps) its physical row
  float* rval = reinterpret_cast<float*>(rt + kWarps);  // (warps) its signed value
  int* rlog = reinterpret_cast<int*>(rval + kWarps);    // (warps) its logical label
  int* misc = rlog + kWarps;  // [0] phys of logical k, [1] phys of logical k+1, [2..] scan

  const int n_items = a.n_cfg_dev ? (*a.n_cfg_dev) * a.G : a.n_items;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    __syncthreads();
    if (a.mode == 0) {
      const float* F = a.F + (size_t)item * n * n;
      for (int i = wid; i < n; i += kWarps) {
        const float* src = F + (size_t)i * n;
        float* dst = Lw + tri_off(i);
        for (int j = lane; j < i; j += 32) dst[j] = __ldg(src + j);
      }
    } else {
      gather_lower<D>(Lw, n, a.Y + (size_t)item * n * D, a.idx + (size_t)item * n, a.Wt, a.Lx,
                      a.Ly);
    }
    // Initial max |A| for the growth flag (block reduction).
    float amax = 0.0f;
    for (int e = tid; e < tri; e += kNumThreads) amax = fmaxf(amax, fabsf(Lw[e]));
#pragma unroll
    for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if (lane == 0) rkey[wid] = amax;
    if (tid == 0) misc[0] = 0;
    __syncthreads();
    float a0max = 0.0f;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) a0max = fmaxf(a0max, rkey[w]);
    __syncthreads();

    int my_log = tid < n ? tid : -1;
    float sgn = 1.0f;
    double mant = 1.0;
    int expo = 0;
    int flag = 0;
    float colmax = 0.0f;
    bool zero = false;

    for (int k0 = 0; k0 < n - 1 && !zero; k0 += 2 * NB) {
      const int steps = min(NB, (n - k0) >> 1);
      float myU[NB], myV[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        myU[j] = 0.0f;
        myV[j] = 0.0f;
      }
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        if (j < steps && !zero) {
          const int k = k0 + 2 * j;
          const int ck = misc[0];
          float c = 0.0f;
          const bool act = my_log > k;
          if (act) {
            c = aval(Lw, tid, ck);
#pragma unroll
            for (int p = 0; p < NB; ++p)
              if (p < j) c += myU[p] * Vs[ck * NB + p] - myV[p] * Us[ck * NB + p];
          }
          float key = act ? (isnan(c) ? INFINITY : fabsf(c)) : -1.0f;
          int bt = tid;
#pragma unroll
          for (int o = 16; o; o >>= 1) {
            float ok = __shfl_xor_sync(0xffffffffu, key, o);
            int ot = __shfl_xor_sync(0xffffffffu, bt, o);
            if (ok > key || (ok == key && ot < bt)) {
              key = ok;
              bt = ot;
            }
          }
          if (tid == bt) {
            rkey[wid] = key;
            rt[wid] = bt;
            rval[wid] = c;
            rlog[wid] = my_log;
          }
          if (my_log == k + 1) misc[1] = tid;
          __syncthreads();  // (1) pivot candidates
          float bk = rkey[0];
          int r = rt[0], w0 = 0;
#pragma unroll
          for (int w = 1; w < kWarps; ++w) {
            float kw = rkey[w];
            int tw = rt[w];
            if (kw > bk || (kw == bk && tw < r)) {
              bk = kw;
              r = tw;
              w0 = w;
            }
          }
          const float cr = rval[w0];
          const int lr = rlog[w0];
          const int p1 = misc[1];
          if (!(bk > 0.0f)) {
            zero = true;  // exactly singular (or empty) column: pf = 0
          } else {
            if (tid == r)
              my_log = k + 1;
            else if (tid == p1)
              my_log = lr;
            const float piv = -cr;
            const bool live = my_log > k + 1;
            float u = 0.0f, v = 0.0f;
            if (live) {
              float dv = aval(Lw, tid, r);
#pragma unroll
              for (int p = 0; p < NB; ++p)
                if (p < j) dv += myU[p] * Vs[r * NB + p] - myV[p] * Us[r * NB + p];
              u = dv;
              v = c / piv;
            }
            myU[j] = u;
            myV[j] = v;
            if (tid < n) {
              Us[tid * NB + j] = u;
              Vs[tid * NB + j] = v;
            }
            if (my_log == k + 2) misc[0] = tid;
            if (tid == 0) {
              if (lr != k + 1) sgn = -sgn;
              if (piv < 0.0f) sgn = -sgn;
              int e;
              mant = frexp(mant * (double)fabsf(piv), &e);
              expo += e;
              colmax = fmaxf(colmax, bk);
              if (!isfinite(piv)) flag |= NH_FLAG_NONFINITE;
            }
          }
          __syncthreads();  // (2) panel column written, next column's owner known
        }
      }
      if (zero) break;
      // Trailing update over the active rows (physical order), rank 2 * steps.
      const int k_end = k0 + 2 * steps;
      const int m = n - k_end;
      if (m >= 2) {
        const bool on = tid < n && my_log >= k_end;
        unsigned bal = __ballot_sync(0xffffffffu, on);
        if (lane == 0) misc[2 + wid] = __popc(bal);
        __syncthreads();
        int before = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) before += (w < wid) ? misc[2 + w] : 0;
        if (on) alist[before + __popc(bal & ((1u << lane) - 1u))] = tid;
        __syncthreads();  // (3) active list
        const int T = (m * (m - 1)) >> 1;
        const int chunk = (T + kNumThreads - 1) / kNumThreads;
        int e = tid * chunk;
        const int e_end = min(T, e + chunk);
        if (e < e_end) {
          int ia = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)e)) * 0.5f);
          while (((ia * (ia - 1)) >> 1) > e) --ia;
          while (((ia * (ia + 1)) >> 1) <= e) ++ia;
          int ib = e - ((ia * (ia - 1)) >> 1);
          int pa = alist[ia];
          float ua[NB], va[NB];
#pragma unroll
          for (int p = 0; p < NB; ++p) {
            ua[p] = Us[pa * NB + p];
            va[p] = Vs[pa * NB + p];
          }
          float* rowp = Lw + tri_off(pa);
          for (; e < e_end; ++e) {
            const int pb = alist[ib];
            float acc = rowp[pb];
#pragma unroll
            for (int p = 0; p < NB; ++p) {
              if (p < steps) {
                acc = fmaf(ua[p], Vs[pb * NB + p], acc);
                acc = fmaf(-va[p], Us[pb * NB + p], acc);
              }
            }
            rowp[pb] = acc;
            if (++ib == ia) {
              ++ia;
              ib = 0;
              if (e + 1 < e_end) {
                pa = alist[ia];
#pragma unroll
                for (int p = 0; p < NB; ++p) {
                  ua[p] = Us[pa * NB + p];
                  va[p] = Vs[pa * NB + p];
                }
                rowp = Lw + tri_off(pa);
              }
            }
          }
        }
        __syncthreads();  // (4) trailing triangle updated
      }
    }
    if (tid == 0) {
      float s = a.item_sign ? a.item_sign[item] : 1.0f;
      double la;
      if (zero) {
        s = 0.0f;
        la = -INFINITY;
        flag |= NH_FLAG_ZERO_PIVOT;
      } else {
        s *= sgn;
        la = log(mant) + (double)expo * 0.6931471805599453;
        if (!isfinite(la)) flag |= NH_FLAG_NONFINITE;
        if (a0max > 0.0f && colmax > kGrowth * a0max) flag |= NH_FLAG_GROWTH;
      }
      if (s == 0.0f) la = -INFINITY;
      a.sign[item] = s;
      a.logabs[item] = la;
      if (a.flags) a.flags[item] = flag;
    }
  }
}

template <int NB, int D>
int launch_pf(const PfArgs& a, int items, cudaStream_t st) {
  const int n = a.n;
  size_t tri = (size_t)n * (n - 1) / 2;
  size_t smem = sizeof(float) * (((tri + 3) & ~(size_t)3) + 2 * (size_t)n * NB) +
                sizeof(int) * (size_t)n + 4 * sizeof(float) * kWarps + sizeof(int) * (2 + kWarps);
  if (smem > 227 * 1024) return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d needs %zu B smem", n, smem);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(pfaffian_kernel<NB, D>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "slogpf smem attribute");
    configured = smem;
  }
  int per_sm = smem <= 113 * 1024 ? 2 : 1;
  int grid = num_sms() * per_sm;
  if (grid > items) grid = items;
  if (grid <= 0) return NH_OK;
  pfaffian_kernel<NB, D><<<grid, kNumThreads, smem, st>>>(a);
  return check_launch("pfaffian_kernel");
}

// NB is the largest panel that keeps two CTAs per SM (<= 113 KB of shared memory).
template <int D>
int launch_pf_pick(const PfArgs& a, int items, cudaStream_t st) {
  const int n = a.n;
  size_t tri = (size_t)n * (n - 1) / 2 * 4;
  size_t base = tri + 4 * (size_t)n + 256;
  if (base + 2 * (size_t)n * 8 * 4 <= 113 * 1024) return launch_pf<8, D>(a, items, st);
  if (base + 2 * (size_t)n * 6 * 4 <= 113 * 1024) return launch_pf<6, D>(a, items, st);
  return launch_pf<4, D>(a, items, st);
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
      for (int aa = 0; aa < D; ++aa) yp[aa] = __ldg(Yi + (size_t)p * D + aa);
      for (int q = lane; q < n; q += 32) {
        float v = 0.0f;
        if (q != p)
          v = pair_value<D>(yp, sp, xp, ypos, Yi + (size_t)q * D, __ldg(ii + q), N, Lx, Ly, Wt);
        Fi[(size_t)p * n + q] = v;
      }
    }
  }
}

// ------------------------------------------------------------------ image combination
__global__ void combine_kernel(const float* __restrict__ sg, const double* __restrict__ la,
                               const int32_t* __restrict__ fl, int G, int n_cfg,
                               const int32_t* n_cfg_dev, float* sign, double* logabs,
                               int32_t* flags) {
  const int n = n_cfg_dev ? *n_cfg_dev : n_cfg;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double m = -INFINITY;
    int f = 0;
    for (int g = 0; g < G; ++g) {
      float s = sg[(size_t)c * G + g];
      double l = la[(size_t)c * G + g];
      if (s != 0.0f && l > m) m = l;
      if (fl) f |= fl[(size_t)c * G + g];
    }
    double tot = 0.0;
    if (m > -INFINITY)
      for (int g = 0; g < G; ++g) {
        float s = sg[(size_t)c * G + g];
        if (s != 0.0f) tot += (double)s * exp(la[(size_t)c * G + g] - m);
      }
    float so = tot > 0.0 ? 1.0f : (tot < 0.0 ? -1.0f : 0.0f);
    sign[c] = so;
    logabs[c] = so != 0.0f ? log(fabs(tot)) + m - log((double)G) : -INFINITY;
    if (flags) flags[c] = f;
  }
}

}  // namespace

int launch_pfaffian_from_F(const float* F, int n, int batch, float* sign, double* logabs,
                           int32_t* flags, cudaStream_t st) {
  if (n <= 0 || n % 2 || n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d must be even and <= %d", n, kNumThreads);
  PfArgs a{};
  a.n = n;
  a.mode = 0;
  a.F = F;
  a.n_items = batch;
  a.G = 1;
  a.sign = sign;
  a.logabs = logabs;
  a.flags = flags;
  return launch_pf_pick<16>(a, batch, st);
}

int launch_pfaffian_gather(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly,
                           int d, int n, int max_items, const ConfigList* cl,
                           const float* item_sign, float* sign, double* logabs, int32_t* flags,
                           cudaStream_t st) {
  if (n <= 0 || n % 2 || n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED, "amplitude: n=%d must be even and <= %d", n, kNumThreads);
  PfArgs a{};
  a.n = n;
  a.mode = 1;
  a.Y = Y;
  a.idx = idx;
  a.Wt = Wt;
  a.Lx = Lx;
  a.Ly = Ly;
  a.d = d;
  a.n_cfg_dev = cl ? cl->n_cfg_dev : nullptr;
  a.G = cl ? cl->G : 1;
  a.n_items = max_items;
  a.item_sign = item_sign;
  a.sign = sign;
  a.logabs = logabs;
  a.flags = flags;
  switch (d) {
    case 8: return launch_pf_pick<8>(a, max_items, st);
    case 16: return launch_pf_pick<16>(a, max_items, st);
    case 32: return launch_pf_pick<32>(a, max_items, st);
    default: return fail(NH_ERR_UNSUPPORTED, "amplitude: d=%d (8, 16 or 32)", d);
  }
}

int launch_pairing(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = num_sms() * 4;
  if (grid > batch) grid = batch;
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
                   cudaStream_t st) {
  if (n_cfg <= 0) return NH_OK;
  int grid = (n_cfg + 255) / 256;
  combine_kernel<<<grid, 256, 0, st>>>(sg, la, fl, G, n_cfg, n_cfg_dev, sign, logabs, flags);
  return check_launch("combine_kernel");
}

}  // namespace nh

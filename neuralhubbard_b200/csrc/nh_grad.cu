// Backward of the Pfaffian-backflow amplitude: the per-sample Jacobian
// O_k(s) = d log|psi_P(s)| / d theta_k that SR / AdamSR training consumes
// (code/train_pfaffian_16x16_tpm02.py:100-101), and its two operator-level pieces.
//
// * adjoint_kernel: the cotangent of fermix.slogpf (code/backflow/models.py:210),
//   G = d log|pf F| / dF = 1/2 F^{-T}, from an in-register Gauss-Jordan inverse of F with implicit
//   row pivoting (one matrix per 512-thread CTA; thread (warp w, lane c) holds rows w + 16 t and
//   columns c + 32 u; one barrier per pivot step, the pivot row read from the winning warp's
//   candidate row in shared memory, as in nh_det.cu).  A per-item scale multiplies G (the image weight of the projection).
// * pairing_vjp_kernel: the custom VJP of the occupied gather (pf_kernel.py:193-320,354-365):
//   dY[p, a] = sum_q (G - G^T)[p, q] Wt[blk(p, q), r(p, q), a] Y[q, a] and
//   dWt[blk, r, a] = sum over the pairs (p, q) with that block and displacement of
//   G[p, q] Y[p, a] Y[q, a].  With several images per sample their dWt are summed in registers and
//   chained through build_wtilde's backward (pf_kernel.py:107-124) into the W and theta columns.
// * cnn_vjp_kernel: the backflow CNN's backward for every image of a sample: the forward is
//   recomputed with the pre-activations kept in shared memory, the features' cotangent is the
//   image's dY scattered to its occupied modes (pf_kernel.py:395), and the convolution weight and
//   bias cotangents of all images are summed into the sample's Jacobian row.
#include <math.h>

#include <algorithm>

#include "nh_cnn_item.cuh"
#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kAdjThreads = 512;  // 16 row groups (warps) x 32 column groups (lanes)
constexpr int kVjpThreads = 512;

__device__ __forceinline__ unsigned long long pivot_key(float mag, int row) {
  // |v| >= 0 orders like its bit pattern; ties go to the smaller row.
  return ((unsigned long long)__float_as_uint(mag) << 32) | (unsigned)(0x7FFFFFFF - row);
}

// Weight of item (c, g) in d log|psi_P(c)|: sg_g exp(la_g) / sum_h sg_h exp(la_h) (sg, la: the
// item's signed log-Pfaffian with its fermionic signs folded in); 0 when the sum vanishes.
__device__ double image_weight(const float* sg, const double* la, int item, int G) {
  if (G == 1) return sg[item] != 0.0f ? 1.0 : 0.0;
  const int c = item / G;
  double m = -INFINITY;
  for (int h = 0; h < G; ++h)
    if (sg[c * G + h] != 0.0f && la[c * G + h] > m) m = la[c * G + h];
  if (!(m > -INFINITY)) return 0.0;
  double tot = 0.0;
  for (int h = 0; h < G; ++h)
    if (sg[c * G + h] != 0.0f) tot += (double)sg[c * G + h] * exp(la[c * G + h] - m);
  if (tot == 0.0 || !isfinite(tot) || sg[item] == 0.0f) return 0.0;
  return (double)sg[item] * exp(la[item] - m) / tot;
}

struct AdjArgs {
  const float* F;  // (batch, n, n)
  float* G;        // (batch, n, n), may alias F
  int n, batch;
  const float* pf_sign;     // when set: scale G by the image weight (G = n_img images per sample)
  const double* pf_logabs;
  int n_img;
  int32_t* flags;           // (batch,) or null: NH_FLAG_ZERO_PIVOT / NH_FLAG_NONFINITE
};

// Floats of the region shared by the output tile and the per-warp candidate rows.
__host__ __device__ constexpr size_t adjoint_region(int n, int np) {
  return (size_t)n * (n + 1) > (size_t)32 * np ? (size_t)n * (n + 1) : (size_t)32 * np;
}

template <int TC>
__global__ void __launch_bounds__(kAdjThreads, 1) adjoint_kernel(AdjArgs a) {
  constexpr int TR = 2 * TC, NP = 32 * TC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n, NS = n + 1;
  // tile (n, n + 1): G before the coalesced copy.  During the elimination the same region holds
  // cand [2][16][NP]: each warp's best remaining row of the step, so that the winner's row is
  // in shared memory by the step's one barrier.
  float* tile = reinterpret_cast<float*>(smem_raw);
  float* cand = tile;
  float* colbuf = tile + adjoint_region(n, NP);        // [2][NP]
  int* rho = reinterpret_cast<int*>(colbuf + 2 * NP);  // [NP] pivot row of step k
  int* rhoinv = rho + NP;                              // [NP]
  unsigned long long* slot = reinterpret_cast<unsigned long long*>(rhoinv + NP);  // [3]
  float* scale_s = reinterpret_cast<float*>(slot + 3);
  int* bad_s = reinterpret_cast<int*>(scale_s + 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  for (int item = blockIdx.x; item < a.batch; item += gridDim.x) {
    const float* F = a.F + (size_t)item * n * n;
    float A[TR][TC];
#pragma unroll
    for (int t = 0; t < TR; ++t) {
      const int i = warp + 16 * t;
#pragma unroll
      for (int u = 0; u < TC; ++u) {
        const int j = lane + 32 * u;
        A[t][u] = (i < n && j < n) ? __ldg(F + (size_t)i * n + j) : (i == j ? 1.0f : 0.0f);
      }
    }
    unsigned used = 0;  // bit t: row warp + 16 t is a pivot row already (or padding)
#pragma unroll
    for (int t = 0; t < TR; ++t)
      if (warp + 16 * t >= n) used |= 1u << t;
    if (threadIdx.x == 0) {
      slot[0] = slot[1] = 0ull;  // slot[2] is cleared after step 0's barrier
      *bad_s = 0;
      float sc = 0.5f;
      if (a.pf_sign) sc = (float)(0.5 * image_weight(a.pf_sign, a.pf_logabs, item, a.n_img));
      *scale_s = sc;
    }
    __syncthreads();
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
        if (k >= n || bad) break;  // uniform
        const int par = k & 1;
        {
          // Column k of this warp's rows, spread over the lanes (lane t takes row warp + 16 t)
          // so that the pivot proposal runs on TR lanes instead of the one owning the column.
          float cv = float(0);
#pragma unroll
          for (int t = 0; t < TR; ++t) {
            const float v = __shfl_sync(0xffffffffu, A[t][uk], lk);
            if (lane == t) cv = v;
          }
          unsigned long long key = 0ull;
          if (lane < TR) {
            colbuf[par * NP + warp + 16 * lane] = cv;
            if (!((used >> lane) & 1u)) key = pivot_key(fabsf(cv), warp + 16 * lane);
          }
          // 64-bit warp maximum as two 32-bit reductions: the magnitude bits, then the row
          // tie-break among the lanes holding that magnitude.
          const unsigned hi = (unsigned)(key >> 32);
          const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
          const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? (unsigned)key : 0u);
          key = ((unsigned long long)mh << 32) | ml;
          if (key) {  // this warp's best row goes to its candidate slot
            const int tl = (0x7FFFFFFF - (int)ml) >> 4;
            float* cw = cand + (size_t)(par * 16 + warp) * NP;
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
        if (win == 0ull || !(mag > 0.0f && mag <= 3.0e38f)) {  // zero column, or non-finite
          bad = (win == 0ull || mag == 0.0f) ? NH_FLAG_ZERO_PIVOT : NH_FLAG_NONFINITE;
          __syncthreads();
          break;
        }
        if (threadIdx.x == 0) {
          slot[sl == 0 ? 2 : sl - 1] = 0ull;
          rho[k] = p;
        }
        sl = sl == 2 ? 0 : sl + 1;
        const float* prow = cand + (size_t)(par * 16 + (p & 15)) * NP;
        const float inv = 1.0f / prow[k];
        float r[TC];
#pragma unroll
        for (int u = 0; u < TC; ++u) r[u] = prow[lane + 32 * u] * inv;
#pragma unroll
        for (int t = 0; t < TR; ++t) {
          const float f = colbuf[par * NP + warp + 16 * t];
#pragma unroll
          for (int u = 0; u < TC; ++u) A[t][u] = fmaf(-f, r[u], A[t][u]);
        }
        if (lane == lk) {
#pragma unroll
          for (int t = 0; t < TR; ++t) A[t][uk] = -colbuf[par * NP + warp + 16 * t] * inv;
        }
        if (warp == (p & 15)) {
          const int tp = p >> 4;
          used |= 1u << tp;
#pragma unroll
          for (int t = 0; t < TR; ++t)
            if (t == tp) {
#pragma unroll
              for (int u = 0; u < TC; ++u) A[t][u] = r[u];
              if (lane == lk) A[t][uk] = inv;
            }
        }
      }
    }
    // The storage holds X = (P F)^{-1} with logical row k in physical row rho[k], so
    // F^{-1}[i][j] = A[rho[i]][rhoinv[j]] and G[p][q] = 1/2 F^{-1}[q][p]: element (I, J) of the
    // storage goes to G[rho[J]][rhoinv[I]].
    if (threadIdx.x == 0 && bad) *bad_s = bad;
    __syncthreads();
    bad = *bad_s;
    if (!bad)
      for (int k = threadIdx.x; k < n; k += kAdjThreads) rhoinv[rho[k]] = k;
    __syncthreads();
    const float sc = bad ? 0.0f : *scale_s;
#pragma unroll
    for (int t = 0; t < TR; ++t) {
      const int I = warp + 16 * t;
#pragma unroll
      for (int u = 0; u < TC; ++u) {
        const int J = lane + 32 * u;
        if (I < n && J < n) {
          const int dr = bad ? J : rho[J], dc = bad ? I : rhoinv[I];
          tile[dr * NS + dc] = sc * A[t][u];
        }
      }
    }
    __syncthreads();
    float* Gi = a.G + (size_t)item * n * n;
    for (int e = threadIdx.x; e < n * n; e += kAdjThreads) {
      const int row = e / n;
      Gi[e] = tile[row * NS + (e - row * n)];
    }
    if (a.flags && threadIdx.x == 0) a.flags[item] = bad;
    __syncthreads();
  }
}

template <int TC>
size_t adjoint_smem(int n) {
  constexpr int NP = 32 * TC;
  return sizeof(float) * (adjoint_region(n, NP) + 2 * NP) + sizeof(int) * 2 * NP +
         sizeof(unsigned long long) * 3 + 16;
}

template <int TC>
int launch_adjoint_t(const AdjArgs& a, cudaStream_t st) {
  const size_t smem = adjoint_smem<TC>(a.n);
  if (smem > 227 * 1024) return fail(NH_ERR_UNSUPPORTED, "pfaffian adjoint: n = %d", a.n);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<TC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "adjoint smem attribute");
    configured = smem;
  }
  int grid = num_sms() * (smem <= 113 * 1024 ? 2 : 1);
  if (grid > a.batch) grid = a.batch;
  ProfScope prof_scope(NH_K_PF_ADJOINT, st);
  adjoint_kernel<TC><<<grid, kAdjThreads, smem, st>>>(a);
  return check_launch("adjoint_kernel");
}

// ------------------------------------------------------------------ pairing VJP
struct VjpArgs {
  const float* G;      // (items, n, n) cotangent of F
  const float* Y;      // (items, n, d)
  const int32_t* idx;  // (items, n)
  const float* Wt;     // (4, N, d)
  int Lx, Ly, n;
  int n_img;           // images per sample (items = samples * n_img)
  int samples;
  float* dY;           // (items, n, d) or null
  float* dWt;          // mode 0: (items, 4, N, d) per item
  // mode 1: the sample's W / theta cotangent (build_wtilde's backward of the images' summed dWt)
  // into jac[sample * ld + off_w ...], theta at off_w + 3 N d.
  float* jac;
  int64_t ld;
  int64_t off_w;
  float theta;
  int mode;
};

template <int D>
__global__ void __launch_bounds__(kVjpThreads, 1) pairing_vjp_kernel(VjpArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = a.n, N = a.Lx * a.Ly, Lx = a.Lx, Ly = a.Ly, NS = n + 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // Region 0: G (n, n + 1), later the summed dWt (4, N, D); then Y rows (swizzled), modes, inv.
  const size_t reg0 = ((size_t)n * NS > (size_t)4 * N * D ? (size_t)n * NS : (size_t)4 * N * D);
  float* gs = reinterpret_cast<float*>(smem_raw);
  float* ys = gs + ((reg0 + 3) & ~(size_t)3);   // (n, D), 16-byte chunks swizzled
  int* modes = reinterpret_cast<int*>(ys + (size_t)n * D);  // (spin << 16) | (x << 8) | y
  int* inv = modes + n;                                     // (2N) mode -> row or -1
  // dWt ownership: task = pass * kVjpThreads + tid -> (pair, 16-byte chunk c of a); pair ->
  // (sq, r).  A thread keeps the same chunk in every pass (kVjpThreads is a multiple of kCh)
  // and accumulates float4 partial sums per pass and spin of p.
  constexpr int kCh = D / 4;  // also the most passes: 2 N kCh <= kVjpThreads kCh
  const int c_own = tid % kCh;
  int p_base[kCh], p_rx[kCh], p_ry[kCh], p_r[kCh], p_sq[kCh];
  bool p_ok[kCh];
#pragma unroll
  for (int pi = 0; pi < kCh; ++pi) {
    const int pair = (pi * kVjpThreads + tid) / kCh;
    p_ok[pi] = pair < 2 * N;
    p_sq[pi] = p_ok[pi] ? pair / N : 0;
    p_r[pi] = p_ok[pi] ? pair - p_sq[pi] * N : 0;
    p_rx[pi] = p_r[pi] / Ly;
    p_ry[pi] = p_r[pi] - p_rx[pi] * Ly;
    p_base[pi] = p_sq[pi] * N;
  }
  float4 acc0[kCh], acc1[kCh];  // spin of p: up / down
#pragma unroll
  for (int pi = 0; pi < kCh; ++pi) acc0[pi] = acc1[pi] = make_float4(0.f, 0.f, 0.f, 0.f);

  for (int smp = blockIdx.x; smp < a.samples; smp += gridDim.x) {
    for (int g = 0; g < a.n_img; ++g) {
      const size_t item = (size_t)smp * a.n_img + g;
      const float* Gi = a.G + item * n * n;
      const float* Yi = a.Y + item * n * D;
      const int32_t* ii = a.idx + item * n;
      __syncthreads();  // previous item's readers are done
      for (int e = tid; e < n * n; e += kVjpThreads) {
        const int row = e / n;
        gs[row * NS + (e - row * n)] = __ldg(Gi + e);
      }
      for (int e = tid; e < n * D; e += kVjpThreads) {
        const int row = e / D, aa = e - row * D;
        ys[swz_index<float, D>(row, aa)] = __ldg(Yi + e);
      }
      for (int m = tid; m < 2 * N; m += kVjpThreads) inv[m] = -1;
      __syncthreads();
      for (int p = tid; p < n; p += kVjpThreads) {
        int m = __ldg(ii + p);
        if ((unsigned)m >= (unsigned)(2 * N)) m = 0;  // out-of-range mode: read as mode 0
        const int sp = m >= N ? 1 : 0, site = m - sp * N, x = site / Ly;
        modes[p] = (sp << 16) | (x << 8) | (site - x * Ly);
        inv[m] = p;
      }
      __syncthreads();
      // dY: warp per row p, lanes over q.
      if (a.dY) {
        float* dYi = a.dY + item * n * D;
        for (int p = warp; p < n; p += kVjpThreads / 32) {
          const int mp = modes[p];
          const int sp = mp >> 16, xp = (mp >> 8) & 0xFF, yp = mp & 0xFF;
          float acc[D];
#pragma unroll
          for (int j = 0; j < D; ++j) acc[j] = 0.0f;
          for (int q = lane; q < n; q += 32) {
            const float gh = gs[p * NS + q] - gs[q * NS + p];
            const int mq = modes[q];
            const int sq = mq >> 16;
            int dx = xp - ((mq >> 8) & 0xFF), dy = yp - (mq & 0xFF);
            dx += dx < 0 ? Lx : 0;
            dy += dy < 0 ? Ly : 0;
            const float4* w4 = reinterpret_cast<const float4*>(
                a.Wt + ((size_t)(2 * sp + sq) * N + dx * Ly + dy) * D);
#pragma unroll
            for (int c = 0; c < D / 4; ++c) {
              const float4 w = __ldg(w4 + c);
              const float4 y = *reinterpret_cast<const float4*>(ys + swz_index<float, D>(q, 4 * c));
              acc[4 * c + 0] = fmaf(gh * w.x, y.x, acc[4 * c + 0]);
              acc[4 * c + 1] = fmaf(gh * w.y, y.y, acc[4 * c + 1]);
              acc[4 * c + 2] = fmaf(gh * w.z, y.z, acc[4 * c + 2]);
              acc[4 * c + 3] = fmaf(gh * w.w, y.w, acc[4 * c + 3]);
            }
          }
#pragma unroll
          for (int j = 0; j < D; ++j) {
#pragma unroll
            for (int o = 16; o; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
          }
          float mine = 0.0f;
#pragma unroll
          for (int j = 0; j < D; ++j)
            if (lane == j) mine = acc[j];
          if (lane < D) dYi[(size_t)p * D + lane] = mine;
        }
      }
      // dWt: each (pair, chunk) sums over the rows p; partner q = inv[sq, site_p - r].
      for (int p = 0; p < n; ++p) {
        const int mp = modes[p];
        const int sp = mp >> 16, xp = (mp >> 8) & 0xFF, yp = mp & 0xFF;
        const float4 y1 = *reinterpret_cast<const float4*>(ys + swz_index<float, D>(p, 4 * c_own));
#pragma unroll
        for (int pi = 0; pi < kCh; ++pi) {
          if (!p_ok[pi]) continue;
          int x = xp - p_rx[pi], y = yp - p_ry[pi];
          x += x < 0 ? Lx : 0;
          y += y < 0 ? Ly : 0;
          const int q = inv[p_base[pi] + x * Ly + y];
          if (q < 0) continue;
          const float gv = gs[p * NS + q];
          const float4 y2 = *reinterpret_cast<const float4*>(ys + swz_index<float, D>(q, 4 * c_own));
          float4& acc = sp ? acc1[pi] : acc0[pi];
          acc.x = fmaf(gv * y1.x, y2.x, acc.x);
          acc.y = fmaf(gv * y1.y, y2.y, acc.y);
          acc.z = fmaf(gv * y1.z, y2.z, acc.z);
          acc.w = fmaf(gv * y1.w, y2.w, acc.w);
        }
      }
      if (a.mode == 0) {  // per-item dWt
        float* dst = a.dWt + item * 4 * N * D;
#pragma unroll
        for (int pi = 0; pi < kCh; ++pi) {
          if (!p_ok[pi]) continue;
          float* d0 = dst + ((size_t)p_sq[pi] * N + p_r[pi]) * D + 4 * c_own;
          float* d1 = dst + ((size_t)(2 + p_sq[pi]) * N + p_r[pi]) * D + 4 * c_own;
          d0[0] = acc0[pi].x, d0[1] = acc0[pi].y, d0[2] = acc0[pi].z, d0[3] = acc0[pi].w;
          d1[0] = acc1[pi].x, d1[1] = acc1[pi].y, d1[2] = acc1[pi].z, d1[3] = acc1[pi].w;
          acc0[pi] = acc1[pi] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    }
    if (a.mode != 1) continue;
    // Sample done: the summed dWt through build_wtilde's backward.
    __syncthreads();
    float* dw = gs;  // (4, N, D)
#pragma unroll
    for (int pi = 0; pi < kCh; ++pi) {
      if (!p_ok[pi]) continue;
      *reinterpret_cast<float4*>(dw + ((size_t)p_sq[pi] * N + p_r[pi]) * D + 4 * c_own) = acc0[pi];
      *reinterpret_cast<float4*>(dw + ((size_t)(2 + p_sq[pi]) * N + p_r[pi]) * D + 4 * c_own) =
          acc1[pi];
      acc0[pi] = acc1[pi] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    // Envelope pref[r] = exp(-lam D_r) / (N sum exp(-lam D)) and its mean distance, FP64.
    const double th = (double)a.theta;
    const double lam = log1p(exp(-fabs(th))) + fmax(th, 0.0);
    double se = 0.0, sde = 0.0;
    for (int r = tid; r < N; r += kVjpThreads) {
      const int rx = r / Ly, ry = r - rx * Ly;
      const double mx = (double)min(rx, Lx - rx), my = (double)min(ry, Ly - ry);
      const double dist = sqrt(mx * mx + my * my), e = exp(-lam * dist);
      se += e;
      sde += dist * e;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      se += __shfl_xor_sync(0xffffffffu, se, o);
      sde += __shfl_xor_sync(0xffffffffu, sde, o);
    }
    __shared__ double part[2][kVjpThreads / 32];
    if (lane == 0) {
      part[0][warp] = se;
      part[1][warp] = sde;
    }
    __syncthreads();
    double S = 0.0, SD = 0.0;
    for (int w = 0; w < kVjpThreads / 32; ++w) {
      S += part[0][w];
      SD += part[1][w];
    }
    const double mean_d = SD / S;
    float* row = a.jac + (size_t)smp * a.ld + a.off_w;
    double tacc = 0.0;
    for (int e = tid; e < N * D; e += kVjpThreads) {
      const int r = e / D, aa = e - r * D;
      const int rx = r / Ly, ry = r - rx * Ly;
      const int nr = (rx ? Lx - rx : 0) * Ly + (ry ? Ly - ry : 0);
      const double mx = (double)min(rx, Lx - rx), my = (double)min(ry, Ly - ry);
      const double dist = sqrt(mx * mx + my * my);
      const float pref = (float)(exp(-lam * dist) / ((double)N * S));
      const int nrx = nr / Ly, nry = nr - nrx * Ly;
      const double ndist = sqrt((double)min(nrx, Lx - nrx) * min(nrx, Lx - nrx) +
                                (double)min(nry, Ly - nry) * min(nry, Ly - nry));
      const float npref = (float)(exp(-lam * ndist) / ((double)N * S));
      const float d0 = dw[(0 * N + r) * D + aa] * pref, d0n = dw[(0 * N + nr) * D + aa] * npref;
      const float d1 = dw[(1 * N + r) * D + aa] * pref;
      const float d2n = dw[(2 * N + nr) * D + aa] * npref;
      const float d3 = dw[(3 * N + r) * D + aa] * pref, d3n = dw[(3 * N + nr) * D + aa] * npref;
      row[(0 * N + r) * D + aa] = d1 - d2n;
      row[(1 * N + r) * D + aa] = 0.5f * (d0 - d0n);
      row[(2 * N + r) * D + aa] = 0.5f * (d3 - d3n);
      double s4 = 0.0;
#pragma unroll
      for (int b = 0; b < 4; ++b)
        s4 += (double)dw[(b * N + r) * D + aa] * (double)__ldg(a.Wt + (b * N + r) * D + aa);
      tacc += s4 * (mean_d - dist);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) tacc += __shfl_xor_sync(0xffffffffu, tacc, o);
    __syncthreads();
    if (lane == 0) part[0][warp] = tacc;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < kVjpThreads / 32; ++w) t += part[0][w];
      row[3 * N * D] = (float)(t / (1.0 + exp(-th)));
    }
  }
}

template <int D>
size_t vjp_smem(int n, int N) {
  const size_t reg0 = std::max((size_t)n * (n + 1), (size_t)4 * N * D);
  return sizeof(float) * (((reg0 + 3) & ~(size_t)3) + (size_t)n * D) +
         sizeof(int) * ((size_t)n + 2 * N);
}

template <int D>
int launch_vjp_t(const VjpArgs& a, cudaStream_t st) {
  const int N = a.Lx * a.Ly;
  const size_t smem = vjp_smem<D>(a.n, N);
  if (smem > 227 * 1024 || 2 * N > kVjpThreads)
    return fail(NH_ERR_UNSUPPORTED, "pairing vjp: n = %d, N = %d", a.n, N);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(pairing_vjp_kernel<D>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "pairing vjp smem attribute");
    configured = smem;
  }
  int grid = num_sms() * (smem <= 113 * 1024 ? 2 : 1);
  if (grid > a.samples) grid = a.samples;
  ProfScope prof_scope(NH_K_PAIRING_VJP, st);
  pairing_vjp_kernel<D><<<grid, kVjpThreads, smem, st>>>(a);
  return check_launch("pairing_vjp_kernel");
}

// ------------------------------------------------------------------ CNN VJP
// One periodic 3x3 cross-correlation of cin planes (stride NS) into cout planes, weights
// [ci][tap][co] in shared memory, bias (or none), epilogue(co, site, z) stores the result.
template <typename Epi>
__device__ __forceinline__ void conv_planes(const float* in, int cin, int cout, const float* wsm,
                                            const float* bsm, int Lx, int Ly, Epi epi) {
  const int N = Lx * Ly, NS = N + 1, half = N / 2, ngroups = cout / 8;
  for (int task = threadIdx.x; task < ngroups * half; task += kNumThreads) {
    const int grp = task / half;
    const int s0 = task - grp * half, s1 = s0 + half;
    const int x0 = s0 / Ly, y0 = s0 - x0 * Ly;
    const int x1 = s1 / Ly, y1 = s1 - x1 * Ly;
    float acc0[8], acc1[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc0[j] = acc1[j] = bsm ? bsm[grp * 8 + j] : 0.0f;
    for (int ci = 0; ci < cin; ++ci) {
      const float* inc = in + ci * NS;
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        int xa = x0 + u - 1, xb = x1 + u - 1;
        xa = xa < 0 ? xa + Lx : (xa >= Lx ? xa - Lx : xa);
        xb = xb < 0 ? xb + Lx : (xb >= Lx ? xb - Lx : xb);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          int ya = y0 + v - 1, yb = y1 + v - 1;
          ya = ya < 0 ? ya + Ly : (ya >= Ly ? ya - Ly : ya);
          yb = yb < 0 ? yb + Ly : (yb >= Ly ? yb - Ly : yb);
          const float i0 = inc[xa * Ly + ya];
          const float i1 = inc[xb * Ly + yb];
          float w8[8];
          cnn_lds8(wsm + (ci * 9 + u * 3 + v) * cout + grp * 8, w8);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            acc0[j] = fmaf(i0, w8[j], acc0[j]);
            acc1[j] = fmaf(i1, w8[j], acc1[j]);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      epi(grp * 8 + j, s0, acc0[j]);
      epi(grp * 8 + j, s1, acc1[j]);
    }
  }
}

__device__ __forceinline__ float gelu_tanh_grad_dev(float x) {
  const float k0 = 0.7978845608028654f, c = 0.044715f;
  const float t = tanhf(k0 * (x + c * x * x * x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k0 * (1.0f + 3.0f * c * x * x);
}

struct CnnVjpArgs {
  const int8_t* spins;  // (samples, 2N)
  int samples, n_img;
  const float* conv_w;  // OIHW per layer, concatenated
  const float* conv_w_packed;  // [l][ci][tap][co]
  const float* conv_b;
  int Lx, Ly, C, layers, n;
  const float* dY;       // (items, n, d) cotangent of the occupied rows (image weight included)
  const int32_t* idx;    // (items, n) occupied modes of each image configuration
  float* jac;            // (samples, ld): conv weights and biases from column 0
  int64_t ld;
};

// Shared memory: z planes of layers 0 .. L-2 ((L-1) C NS), the input image (2 NS), two cotangent /
// activation buffers (2 C NS) and one layer's weights (C C 9).
__global__ void __launch_bounds__(kNumThreads) cnn_vjp_kernel(CnnVjpArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Lx = a.Lx, Ly = a.Ly, N = Lx * Ly, NS = N + 1, C = a.C, L = a.layers, d = C / 2;
  const int tid = threadIdx.x;
  float* zs = reinterpret_cast<float*>(smem_raw);        // (L-1, C, NS)
  float* img = zs + (size_t)(L - 1) * C * NS;            // (2, NS), padded to 16 bytes
  float* bufA = img + ((2 * NS + 3) & ~3);               // (C, NS)
  float* bufB = bufA + (size_t)C * NS;                   // (C, NS)
  float* wsm = bufB + (size_t)C * NS;                    // (C C 9)

  for (int smp = blockIdx.x; smp < a.samples; smp += gridDim.x) {
    float* row = a.jac + (size_t)smp * a.ld;
    const int8_t* base = a.spins + (size_t)smp * 2 * N;
    for (int g = 0; g < a.n_img; ++g) {
      const size_t item = (size_t)smp * a.n_img + g;
      const int sym = a.n_img == 1 ? 0 : g;
      __syncthreads();
      for (int m = tid; m < 2 * N; m += kNumThreads) {
        const int src = sym_map(m, sym, Lx, Ly, N);
        const int ch = m >= N ? 1 : 0;
        img[ch * NS + (m - ch * N)] = base[src] > 0 ? 1.0f : -1.0f;
      }
      // Forward, keeping the pre-activations z_l (l < L - 1); GELU(z) into bufA as next input.
      const float* in = img;
      int cin = 2;
      size_t woff = 0;
      for (int l = 0; l < L - 1; ++l) {
        __syncthreads();
        for (int i = tid; i < C * cin * 9; i += kNumThreads) wsm[i] = __ldg(a.conv_w_packed + woff + i);
        __syncthreads();
        float* z = zs + (size_t)l * C * NS;
        const float* bl = a.conv_b + l * C;
        conv_planes(in, cin, C, wsm, nullptr, Lx, Ly,
                    [&](int co, int s, float v) { z[co * NS + s] = v + __ldg(bl + co); });
        __syncthreads();
        for (int e = tid; e < C * N; e += kNumThreads) {
          const int co = e / N, s = e - co * N;
          bufA[co * NS + s] = gelu_tanh_dev(z[co * NS + s]);
        }
        in = bufA;
        woff += (size_t)C * cin * 9;
        cin = C;
      }
      // Cotangent of the last layer's output: dY scattered to the occupied modes.
      __syncthreads();
      float* dcur = bufB;
      float* dother = bufA;
      for (int e = tid; e < C * NS; e += kNumThreads) dcur[e] = 0.0f;
      __syncthreads();
      const float* dYi = a.dY + item * a.n * d;
      const int32_t* ii = a.idx + item * a.n;
      for (int e = tid; e < a.n * d; e += kNumThreads) {
        const int p = e / d, aa = e - p * d;
        const int m = __ldg(ii + p);
        const int sg = m >= N ? 1 : 0;
        dcur[(sg * d + aa) * NS + (m - sg * N)] = __ldg(dYi + e);
      }
      // Backward, last layer first.
      size_t wl_off = 0;  // OIHW offset of layer l
      int64_t col = 0;    // Jacobian column of layer l's weights
      // offsets of layer l: layer 0 has cin 2
      for (int l = L - 1; l >= 0; --l) {
        const int lcin = l == 0 ? 2 : C;
        wl_off = l == 0 ? 0 : (size_t)C * 2 * 9 + (size_t)(l - 1) * C * C * 9;
        col = l == 0 ? 0 : (int64_t)(C * 2 * 9 + C) + (int64_t)(l - 1) * (C * C * 9 + C);
        __syncthreads();
        // Layer input activation: the image for l = 0, GELU(z_{l-1}) otherwise (into dother).
        const float* ain = img;
        if (l > 0) {
          const float* z = zs + (size_t)(l - 1) * C * NS;
          for (int e = tid; e < C * N; e += kNumThreads) {
            const int ci = e / N, s = e - ci * N;
            dother[ci * NS + s] = gelu_tanh_dev(z[ci * NS + s]);
          }
          ain = dother;
        }
        __syncthreads();
        // Weight cotangent: thread owns (4 output channels, 1 input channel) x 9 taps.
        const int pairs = (C / 4) * lcin;
        for (int pr = tid; pr < pairs; pr += kNumThreads) {
          const int ci = pr % lcin, cob = pr / lcin;
          float acc[4][9];
#pragma unroll
          for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int t = 0; t < 9; ++t) acc[j][t] = 0.0f;
          const float* ap = ain + ci * NS;
          const float* dp = dcur + (size_t)(cob * 4) * NS;
          for (int x = 0; x < Lx; ++x) {
            const int xm = (x == 0 ? Lx - 1 : x - 1) * Ly, x0 = x * Ly,
                      xp = (x == Lx - 1 ? 0 : x + 1) * Ly;
            for (int y = 0; y < Ly; ++y) {
              const int ym = y == 0 ? Ly - 1 : y - 1, yp = y == Ly - 1 ? 0 : y + 1;
              const float av[9] = {ap[xm + ym], ap[xm + y], ap[xm + yp],
                                   ap[x0 + ym], ap[x0 + y], ap[x0 + yp],
                                   ap[xp + ym], ap[xp + y], ap[xp + yp]};
              const int s = x0 + y;
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const float dv = dp[j * NS + s];
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[j][t] = fmaf(dv, av[t], acc[j][t]);
              }
            }
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int co = cob * 4 + j;
            float* dst = row + col + ((int64_t)co * lcin + ci) * 9;
#pragma unroll
            for (int t = 0; t < 9; ++t) dst[t] = g == 0 ? acc[j][t] : dst[t] + acc[j][t];
          }
        }
        // Bias cotangent: warp per output channel.
        {
          const int lane = tid & 31, warp = tid >> 5;
          for (int co = warp; co < C; co += kNumThreads / 32) {
            float s = 0.0f;
            for (int e = lane; e < N; e += 32) s += dcur[co * NS + e];
#pragma unroll
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) {
              float* dst = row + col + (int64_t)C * lcin * 9 + co;
              *dst = g == 0 ? s : *dst + s;
            }
          }
        }
        if (l == 0) break;
        // Input cotangent: transposed convolution with flipped taps, times GELU'(z_{l-1}).
        __syncthreads();
        for (int i = tid; i < C * C * 9; i += kNumThreads) {
          const int cj = i % C;        // output channel of the transposed conv = layer input ci
          const int rest = i / C;      // co * 9 + tap'
          const int co = rest / 9, tp = rest - co * 9;
          wsm[i] = __ldg(a.conv_w + wl_off + ((size_t)co * C + cj) * 9 + (8 - tp));
        }
        __syncthreads();
        const float* z = zs + (size_t)(l - 1) * C * NS;
        conv_planes(dcur, C, C, wsm, nullptr, Lx, Ly, [&](int ci, int s, float v) {
          dother[ci * NS + s] = v * gelu_tanh_grad_dev(z[ci * NS + s]);
        });
        float* t = dcur;
        dcur = dother;
        dother = t;
      }
    }
  }
}

size_t cnn_vjp_smem(int N, int C, int L) {
  const size_t NS = (size_t)N + 1;
  return sizeof(float) * ((size_t)(L - 1) * C * NS + ((2 * NS + 3) & ~(size_t)3) +
                          2 * (size_t)C * NS + (size_t)C * C * 9);
}

}  // namespace

// ------------------------------------------------------------------ launchers
int launch_pf_adjoint(const float* F, float* G, int n, int batch, const float* pf_sign,
                      const double* pf_logabs, int n_img, int32_t* flags, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  AdjArgs a{F, G, n, batch, pf_sign, pf_logabs, n_img, flags};
  const int tc = (n + 31) / 32;
  switch (tc) {
    case 1: return launch_adjoint_t<1>(a, st);
    case 2: return launch_adjoint_t<2>(a, st);
    case 3: return launch_adjoint_t<3>(a, st);
    case 4: return launch_adjoint_t<4>(a, st);
    case 5: return launch_adjoint_t<5>(a, st);
    case 6: return launch_adjoint_t<6>(a, st);
    case 7: return launch_adjoint_t<7>(a, st);
    default: return fail(NH_ERR_UNSUPPORTED, "pfaffian adjoint: n = %d > %d", n, kGradMaxN);
  }
}

int launch_pairing_vjp(const float* G, const float* Y, const int32_t* idx, const float* Wt,
                       int Lx, int Ly, int d, int n, int n_img, int samples, float* dY,
                       float* dWt, float* jac, int64_t ld, int64_t off_w, float theta,
                       cudaStream_t st) {
  if (samples <= 0) return NH_OK;
  VjpArgs a{G, Y, idx, Wt, Lx, Ly, n, n_img, samples, dY, dWt, jac, ld, off_w, theta,
            jac ? 1 : 0};
  switch (d) {
    case 8: return launch_vjp_t<8>(a, st);
    case 16: return launch_vjp_t<16>(a, st);
    case 32: return launch_vjp_t<32>(a, st);
    default: return fail(NH_ERR_UNSUPPORTED, "pairing vjp: d = %d (8, 16 or 32)", d);
  }
}

int launch_cnn_vjp(const int8_t* spins, int samples, int n_img, const nh_backflow_params& p,
                   const float* dY, const int32_t* idx, float* jac, int64_t ld, cudaStream_t st) {
  if (samples <= 0) return NH_OK;
  const int N = p.Lx * p.Ly, C = p.channels;
  if (C % 8 || C < 8 || C > 64 || p.layers < 1 || N % 2)
    return fail(NH_ERR_UNSUPPORTED, "cnn vjp: channels %d, layers %d, N %d", C, p.layers, N);
  const size_t smem = cnn_vjp_smem(N, C, p.layers);
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "cnn vjp: N = %d, %d channels, %d layers need %zu B", N, C,
                p.layers, smem);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(cnn_vjp_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "cnn vjp smem attribute");
    configured = smem;
  }
  int grid = num_sms() * (smem <= 113 * 1024 ? 2 : 1);
  if (grid > samples) grid = samples;
  CnnVjpArgs a{spins, samples, n_img, p.conv_w, p.conv_w_packed, p.conv_b, p.Lx, p.Ly, C,
               p.layers, p.n_up + p.n_dn, dY, idx, jac, ld};
  ProfScope prof_scope(NH_K_CNN_VJP, st);
  cnn_vjp_kernel<<<grid, kNumThreads, smem, st>>>(a);
  return check_launch("cnn_vjp_kernel");
}

bool cnn_vjp_supported(const nh_backflow_params& p) {
  const int N = p.Lx * p.Ly, C = p.channels;
  return p.net == NH_NET_CNN && C % 8 == 0 && C >= 8 && C <= 64 && N % 2 == 0 && p.layers >= 1 &&
         cnn_vjp_smem(N, C, p.layers) <= 227 * 1024;
}

}  // namespace nh

// Learned hop proposal for the Metropolis sampler.
//
// The reference samples with quantax's uniform ParticleHop (code/states.py:397-408); the learned
// proposal has no counterpart there.  Network: periodic 3x3 CNN 2 -> 16 -> 16 -> 16 on the +-1
// occupation image (channel 0 up, 1 down), tanh-GELU after layers 1 and 2.  Output channel
// c = sigma * 8 + d at site i is the logit of hopping the spin-sigma electron at i one step in
// direction d (the hop direction order of the local energy); move index m = c * N + i.  A move is
// valid when the electron exists, d < n_dirs and the target site of the same spin is empty;
// q(m | s) is the softmax over the valid moves.
//
// Parameters: one flat vector of NH_PROPOSAL_PARAMS values, W1 (16, 2, 3, 3), b1 (16),
// W2 (16, 16, 3, 3), b2, W3 (16, 16, 3, 3), b3, held by the caller in FP32 (the training master)
// and evaluated by every kernel in BF16 (nh_proposal_pack rounds them, round-to-nearest-even).
// Activations and accumulations are FP32 on the CUDA cores: the network costs about 10 kFLOP
// per site and pass, under 2% of one projected amplitude at 16x16, so it is not worth
// tensor-core tiles.
//
// Kernels: prop_sample_kernel (one CTA per chain: forward on s, inverse-CDF draw of a move,
// forward on s' for the reverse probability), prop_logits_kernel (forward only),
// prop_backward_kernel (forward, masked softmax cross-entropy, backward; per-CTA gradient
// partials summed in a fixed order by prop_reduce_kernel) and prop_adam_kernel.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kPC = 16;  // channels of every layer (and outputs: 2 spins x 8 directions)
constexpr int kPOffB1 = 288, kPOffW2 = 304, kPOffB2 = 2608, kPOffW3 = 2624, kPOffB3 = 4928;
constexpr int kPCount = 4944;
static_assert(kPCount == NH_PROPOSAL_PARAMS, "parameter count");
constexpr int kPBwd = 2 * 2304;    // layers 2 and 3 laid out [co][tap][ci] for the transposed conv
constexpr int kPL1Scratch = 2560;  // layer-1 gradient partials: 8 site groups x 32 pairs x 10
constexpr int kPThreads = 256;
constexpr int kPWarps = kPThreads / 32;
constexpr int kPMaxParts = 1024;  // gradient partials (CTAs) of one backward call, at most
__constant__ int kOpposite[8] = {1, 0, 3, 2, 7, 6, 5, 4};

__device__ __forceinline__ float pgelu(float x) {
  return 0.5f * x * (1.0f + tanhf(0.7978845608028654f * (x + 0.044715f * x * x * x)));
}

__device__ __forceinline__ float pgelu_grad(float x) {
  const float t = tanhf(0.7978845608028654f * (x + 0.044715f * x * x * x));
  return 0.5f * (1.0f + t) +
         0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
}

// BF16 parameters -> shared FP32: forward weights [ci][tap][co] (biases at their own offsets),
// optional backward copy of W2, W3 as [co][tap][ci].
__device__ void stage_prop_weights(const __nv_bfloat16* __restrict__ g, float* wf, float* wb) {
  for (int e = threadIdx.x; e < kPCount; e += blockDim.x) {
    const float v = __bfloat162float(g[e]);
    if (e < kPOffB1) {
      const int co = e / 18, r = e - co * 18, ci = r / 9, tap = r - ci * 9;
      wf[(ci * 9 + tap) * kPC + co] = v;
    } else if (e < kPOffW2 || (e >= kPOffB2 && e < kPOffW3) || e >= kPOffB3) {
      wf[e] = v;
    } else {
      const int base = e < kPOffB2 ? kPOffW2 : kPOffW3;
      const int o = e - base, co = o / 144, r = o - co * 144, ci = r / 9, tap = r - ci * 9;
      wf[base + (ci * 9 + tap) * kPC + co] = v;
      if (wb) wb[(base == kPOffW2 ? 0 : 2304) + (co * 9 + tap) * kPC + ci] = v;
    }
  }
}

// The 3x3 periodic neighbourhood of a site, tap = u * 3 + v at offset (u - 1, v - 1).
__device__ __forceinline__ void nbr9(int site, int Lx, int Ly, int nb[9]) {
  const int x = site / Ly, y = site - x * Ly;
  const int xm = (x ? x - 1 : Lx - 1) * Ly, xc = x * Ly, xp = (x + 1 < Lx ? x + 1 : 0) * Ly;
  const int ym = y ? y - 1 : Ly - 1, yp = y + 1 < Ly ? y + 1 : 0;
  nb[0] = xm + ym;
  nb[1] = xm + y;
  nb[2] = xm + yp;
  nb[3] = xc + ym;
  nb[4] = xc + y;
  nb[5] = xc + yp;
  nb[6] = xp + ym;
  nb[7] = xp + y;
  nb[8] = xp + yp;
}

// out[co][s] = b[co] + sum_ci,tap w[ci][tap][co] in[ci][nb(s, tap)]; rows of stride NS.  With act,
// stores gelu(out) and, if gout is set, gelu'(pre-activation) into gout.  Task = (co half, site).
template <int CI>
__device__ void pconv(const float* __restrict__ in, float* __restrict__ out,
                      float* __restrict__ gout, const float* __restrict__ wt,
                      const float* __restrict__ bias, int Lx, int Ly, int NS, bool act) {
  const int N = Lx * Ly;
  for (int task = threadIdx.x; task < 2 * N; task += blockDim.x) {
    const int half = task >= N ? 1 : 0;
    const int site = task - half * N, co0 = 8 * half;
    int nb[9];
    nbr9(site, Lx, Ly, nb);
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = bias[co0 + j];
    for (int ci = 0; ci < CI; ++ci) {
      const float* ip = in + ci * NS;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const float a = ip[nb[tap]];
        const float4* wp = reinterpret_cast<const float4*>(wt + (ci * 9 + tap) * kPC + co0);
        const float4 w0 = wp[0], w1 = wp[1];
        acc[0] = fmaf(a, w0.x, acc[0]);
        acc[1] = fmaf(a, w0.y, acc[1]);
        acc[2] = fmaf(a, w0.z, acc[2]);
        acc[3] = fmaf(a, w0.w, acc[3]);
        acc[4] = fmaf(a, w1.x, acc[4]);
        acc[5] = fmaf(a, w1.y, acc[5]);
        acc[6] = fmaf(a, w1.z, acc[6]);
        acc[7] = fmaf(a, w1.w, acc[7]);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float v = acc[j];
      if (act) {
        if (gout) gout[(co0 + j) * NS + site] = pgelu_grad(v);
        v = pgelu(v);
      }
      out[(co0 + j) * NS + site] = v;
    }
  }
}

// Transposed convolution times the activation derivative, in place:
// gd[ci][s] <- gd[ci][s] * sum_co,tap W[co][ci][tap] dout[co][s - offset(tap)].
__device__ void pconv_t(const float* __restrict__ dout, float* gd, const float* __restrict__ wb,
                        int Lx, int Ly, int NS) {
  const int N = Lx * Ly;
  for (int task = threadIdx.x; task < 2 * N; task += blockDim.x) {
    const int half = task >= N ? 1 : 0;
    const int site = task - half * N, ci0 = 8 * half;
    int nb[9];
    nbr9(site, Lx, Ly, nb);
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.0f;
    for (int co = 0; co < kPC; ++co) {
      const float* dp = dout + co * NS;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const float a = dp[nb[8 - tap]];
        const float4* wp = reinterpret_cast<const float4*>(wb + (co * 9 + tap) * kPC + ci0);
        const float4 w0 = wp[0], w1 = wp[1];
        acc[0] = fmaf(a, w0.x, acc[0]);
        acc[1] = fmaf(a, w0.y, acc[1]);
        acc[2] = fmaf(a, w0.z, acc[2]);
        acc[3] = fmaf(a, w0.w, acc[3]);
        acc[4] = fmaf(a, w1.x, acc[4]);
        acc[5] = fmaf(a, w1.y, acc[5]);
        acc[6] = fmaf(a, w1.z, acc[6]);
        acc[7] = fmaf(a, w1.w, acc[7]);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int e = (ci0 + j) * NS + site;
      gd[e] = acc[j] * gd[e];
    }
  }
}

// Weight-gradient accumulation of one (co, ci) pair over the sites s_begin, s_begin + s_step, ...
__device__ __forceinline__ void pgrad_pair(const float* __restrict__ dout,
                                           const float* __restrict__ in, int co, int ci, int Lx,
                                           int Ly, int NS, int s_begin, int s_step, float acc[9],
                                           float& bacc) {
  const int N = Lx * Ly;
  for (int s = s_begin; s < N; s += s_step) {
    int nb[9];
    nbr9(s, Lx, Ly, nb);
    const float d = dout[co * NS + s];
    bacc += d;
    const float* ip = in + ci * NS;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) acc[tap] = fmaf(d, ip[nb[tap]], acc[tap]);
  }
}

__device__ __forceinline__ bool move_valid(const int8_t* s, int c, int i, int N, int Lx, int Ly,
                                           int n_dirs) {
  const int d = c & 7, sg = c >> 3;
  if (d >= n_dirs) return false;
  const int8_t* ss = s + sg * N;
  return ss[i] > 0 && ss[hop_target_site(i, d, Lx, Ly)] < 0;
}

__device__ float pblock_max(float v, float* red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = red[0];
  for (int w = 1; w < kPWarps; ++w) r = fmaxf(r, red[w]);
  __syncthreads();
  return r;
}

// Block sum in a fixed order (warp tree, then warps in ascending order): deterministic.
__device__ float pblock_sum(float v, float* red) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.0f;
  for (int w = 0; w < kPWarps; ++w) r += red[w];
  __syncthreads();
  return r;
}

// Exclusive prefix of v over the threads of the block; *total receives the sum.
__device__ float pblock_exscan(float v, float* red, float* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) red[wid] = inc;
  __syncthreads();
  float before = 0.0f, all = 0.0f;
  for (int w = 0; w < kPWarps; ++w) {
    if (w < wid) before += red[w];
    all += red[w];
  }
  __syncthreads();
  *total = all;
  return before + inc - v;
}

__device__ void load_config(const int8_t* __restrict__ src, int8_t* s_sh, float* x0, int N,
                            int NS) {
  for (int m = threadIdx.x; m < 2 * N; m += blockDim.x) {
    const int8_t v = src[m];
    s_sh[m] = v;
    const int sg = m >= N ? 1 : 0;
    x0[sg * NS + (m - sg * N)] = v > 0 ? 1.0f : -1.0f;
  }
}

// x0 (rows 0-1 of bufB) -> logits in bufA.
__device__ void prop_forward3(float* bufA, float* bufB, const float* wf, int Lx, int Ly, int NS) {
  pconv<2>(bufB, bufA, nullptr, wf, wf + kPOffB1, Lx, Ly, NS, true);
  __syncthreads();
  pconv<16>(bufA, bufB, nullptr, wf + kPOffW2, wf + kPOffB2, Lx, Ly, NS, true);
  __syncthreads();
  pconv<16>(bufB, bufA, nullptr, wf + kPOffW3, wf + kPOffB3, Lx, Ly, NS, false);
  __syncthreads();
}

size_t prop_sample_smem(int N) {
  const int NS = N + 1;
  return sizeof(float) * ((size_t)kPCount + 2 * kPC * NS + 64) + 2 * N + 16;
}

size_t prop_backward_smem(int N) {
  const int NS = N + 1;
  return sizeof(float) * ((size_t)kPCount + kPBwd + kPL1Scratch + 64 + 2 * NS + 5 * kPC * NS) +
         2 * N + 16;
}

// Shared memory of the global-plane variant (weights, scratch and the configuration).
size_t prop_backward_smem_gact(int N) {
  return sizeof(float) * ((size_t)kPCount + kPBwd + kPL1Scratch + 64) + 2 * N + 16;
}

size_t prop_plane_floats(int N) { return (size_t)(2 + 5 * kPC) * (N + 1); }

__global__ void __launch_bounds__(kPThreads) prop_sample_kernel(
    const int8_t* __restrict__ spins, int batch, const __nv_bfloat16* __restrict__ wg, int Lx,
    int Ly, int n_dirs, uint32_t k0, uint32_t k1, uint32_t step_lo, uint32_t step_hi,
    int32_t* valid, int32_t* from, int32_t* to, float* lqr) {
  extern __shared__ __align__(16) float psm[];
  const int N = Lx * Ly, NS = N + 1, M = kPC * N;
  const int tid = threadIdx.x;
  float* wf = psm;
  float* bufA = wf + kPCount;
  float* bufB = bufA + kPC * NS;
  float* red = bufB + kPC * NS;  // [0, 32) reductions, [32] selected move
  int8_t* s_sh = reinterpret_cast<int8_t*>(red + 64);
  int* sel_sh = reinterpret_cast<int*>(red + 32);
  stage_prop_weights(wg, wf, nullptr);
  const int chunk = (M + kPThreads - 1) / kPThreads;
  const int m0 = min(M, tid * chunk), m1 = min(M, m0 + chunk);
  for (int b = blockIdx.x; b < batch; b += gridDim.x) {
    __syncthreads();
    load_config(spins + (size_t)b * 2 * N, s_sh, bufB, N, NS);
    __syncthreads();
    prop_forward3(bufA, bufB, wf, Lx, Ly, NS);
    // q(. | s) over the valid moves, in ascending move order (contiguous chunk per thread)
    float mx = -INFINITY;
    for (int m = m0; m < m1; ++m) {
      const int c = m / N, i = m - c * N;
      if (move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) mx = fmaxf(mx, bufA[c * NS + i]);
    }
    mx = pblock_max(mx, red);
    if (mx == -INFINITY) {  // no electron can hop: a null move
      if (tid == 0) {
        valid[b] = 0;
        from[b] = 0;
        to[b] = 0;
        lqr[b] = 0.0f;
      }
      continue;
    }
    float part = 0.0f;
    for (int m = m0; m < m1; ++m) {
      const int c = m / N, i = m - c * N;
      if (move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) part += expf(bufA[c * NS + i] - mx);
    }
    float total;
    const float prefix = pblock_exscan(part, red, &total);
    const u32x4 r = philox4x32_10(u32x4{step_lo, (uint32_t)b, 0u, step_hi}, k0, k1);
    const float T = (float)u32_to_unit(r.x) * total;
    // Owner: the last thread with probability mass whose prefix does not exceed T.
    int cand = (part > 0.0f && prefix <= T) ? tid : -1;
#pragma unroll
    for (int o = 16; o; o >>= 1) cand = max(cand, __shfl_xor_sync(0xffffffffu, cand, o));
    if ((tid & 31) == 0) red[tid >> 5] = __int_as_float(cand);
    __syncthreads();
    int owner = -1;
    for (int w = 0; w < kPWarps; ++w) owner = max(owner, __float_as_int(red[w]));
    __syncthreads();
    if (tid == owner) {
      float acc = prefix;
      int sel = -1, last = -1;
      for (int m = m0; m < m1; ++m) {
        const int c = m / N, i = m - c * N;
        if (!move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) continue;
        last = m;
        acc += expf(bufA[c * NS + i] - mx);
        if (T < acc) {
          sel = m;
          break;
        }
      }
      *sel_sh = sel >= 0 ? sel : last;
    }
    __syncthreads();
    const int m = *sel_sh;
    const int c = m / N, i = m - c * N, sg = c >> 3, d = c & 7;
    const int j = hop_target_site(i, d, Lx, Ly);
    const float lq_fwd = bufA[c * NS + i] - mx - logf(total);
    __syncthreads();
    if (tid == 0) {
      s_sh[sg * N + i] = -1;
      s_sh[sg * N + j] = 1;
    }
    __syncthreads();
    for (int e = tid; e < 2 * N; e += blockDim.x) {
      const int s2 = e >= N ? 1 : 0;
      bufB[s2 * NS + (e - s2 * N)] = s_sh[e] > 0 ? 1.0f : -1.0f;
    }
    __syncthreads();
    prop_forward3(bufA, bufB, wf, Lx, Ly, NS);
    // log q(reverse | s')
    float mx2 = -INFINITY;
    for (int e = tid; e < M; e += blockDim.x) {
      const int c2 = e / N, i2 = e - c2 * N;
      if (move_valid(s_sh, c2, i2, N, Lx, Ly, n_dirs)) mx2 = fmaxf(mx2, bufA[c2 * NS + i2]);
    }
    mx2 = pblock_max(mx2, red);
    float se = 0.0f;
    for (int e = tid; e < M; e += blockDim.x) {
      const int c2 = e / N, i2 = e - c2 * N;
      if (move_valid(s_sh, c2, i2, N, Lx, Ly, n_dirs)) se += expf(bufA[c2 * NS + i2] - mx2);
    }
    se = pblock_sum(se, red);
    if (tid == 0) {
      const int crev = sg * 8 + kOpposite[d];
      const float lq_rev = bufA[crev * NS + j] - mx2 - logf(se);
      valid[b] = 1;
      from[b] = sg * N + i;
      to[b] = sg * N + j;
      lqr[b] = lq_rev - lq_fwd;
    }
  }
}

__global__ void __launch_bounds__(kPThreads) prop_logits_kernel(
    const int8_t* __restrict__ spins, int batch, const __nv_bfloat16* __restrict__ wg, int Lx,
    int Ly, float* __restrict__ logits) {
  extern __shared__ __align__(16) float psm[];
  const int N = Lx * Ly, NS = N + 1;
  float* wf = psm;
  float* bufA = wf + kPCount;
  float* bufB = bufA + kPC * NS;
  float* red = bufB + kPC * NS;
  int8_t* s_sh = reinterpret_cast<int8_t*>(red + 64);
  stage_prop_weights(wg, wf, nullptr);
  for (int b = blockIdx.x; b < batch; b += gridDim.x) {
    __syncthreads();
    load_config(spins + (size_t)b * 2 * N, s_sh, bufB, N, NS);
    __syncthreads();
    prop_forward3(bufA, bufB, wf, Lx, Ly, NS);
    float* out = logits + (size_t)b * kPC * N;
    for (int e = threadIdx.x; e < kPC * N; e += blockDim.x) {
      const int c = e / N, i = e - c * N;
      out[e] = bufA[c * NS + i];
    }
  }
}

// Loss -(1/B) sum_b w_b log q(m_b | s_b) and its gradient; per-CTA partials (grid, kPCount + 1).
// GACT: the activation planes (x0, a1, g1, a2, g2, z: (2 + 5 kPC) NS floats) live in a per-CTA
// slice of global memory (plane_scratch) for lattices whose planes exceed shared memory; the
// weights and the reduction scratch stay in shared memory.
template <bool GACT>
__global__ void __launch_bounds__(kPThreads, 1) prop_backward_kernel(
    const int8_t* __restrict__ spins, const int32_t* __restrict__ moves,
    const float* __restrict__ weights, int batch, const __nv_bfloat16* __restrict__ wg, int Lx,
    int Ly, int n_dirs, float inv_batch, float* __restrict__ part, float* plane_scratch) {
  extern __shared__ __align__(16) float psm[];
  const int N = Lx * Ly, NS = N + 1, M = kPC * N;
  const int tid = threadIdx.x;
  float* wf = psm;
  float* wb = wf + kPCount;
  float* l1s = wb + kPBwd;  // layer-1 partials
  float* red = l1s + kPL1Scratch;
  float* x0 = GACT ? plane_scratch + (size_t)blockIdx.x * (2 + 5 * kPC) * NS : red + 64;
  float* a1 = x0 + 2 * NS;
  float* g1 = a1 + kPC * NS;
  float* a2 = g1 + kPC * NS;
  float* g2 = a2 + kPC * NS;
  float* z = g2 + kPC * NS;
  int8_t* s_sh = reinterpret_cast<int8_t*>(GACT ? red + 64 : z + kPC * NS);
  stage_prop_weights(wg, wf, wb);
  const int co = tid >> 4, ci = tid & 15;       // pair of layers 2 and 3
  const int p1 = tid & 31, grp = tid >> 5;      // pair and site group of layer 1
  const int co1 = p1 >> 1, ci1 = p1 & 1;
  float gw3[9], gw2[9], gw1[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) gw3[t] = gw2[t] = gw1[t] = 0.0f;
  float gb3 = 0.0f, gb2 = 0.0f, gb1 = 0.0f, lsum = 0.0f;
  for (int b = blockIdx.x; b < batch; b += gridDim.x) {
    __syncthreads();
    load_config(spins + (size_t)b * 2 * N, s_sh, x0, N, NS);
    __syncthreads();
    pconv<2>(x0, a1, g1, wf, wf + kPOffB1, Lx, Ly, NS, true);
    __syncthreads();
    pconv<16>(a1, a2, g2, wf + kPOffW2, wf + kPOffB2, Lx, Ly, NS, true);
    __syncthreads();
    pconv<16>(a2, z, nullptr, wf + kPOffW3, wf + kPOffB3, Lx, Ly, NS, false);
    __syncthreads();
    const int mv = moves[b];
    const int mc = mv / N, mi = mv - mc * N;
    const bool ok = mv >= 0 && mv < M && move_valid(s_sh, mc, mi, N, Lx, Ly, n_dirs);
    if (!ok) continue;  // not a move of this configuration: the record carries no gradient
    const float w = weights[b];
    float mx = -INFINITY;
    for (int e = tid; e < M; e += blockDim.x) {
      const int c = e / N, i = e - c * N;
      if (move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) mx = fmaxf(mx, z[c * NS + i]);
    }
    mx = pblock_max(mx, red);
    float se = 0.0f;
    for (int e = tid; e < M; e += blockDim.x) {
      const int c = e / N, i = e - c * N;
      if (move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) se += expf(z[c * NS + i] - mx);
    }
    se = pblock_sum(se, red);
    if (tid == 0) lsum += w * (mx + logf(se) - z[mc * NS + mi]) * inv_batch;
    __syncthreads();
    const float sc = w * inv_batch, inv_se = 1.0f / se;
    for (int e = tid; e < M; e += blockDim.x) {
      const int c = e / N, i = e - c * N;
      float dz = 0.0f;
      if (move_valid(s_sh, c, i, N, Lx, Ly, n_dirs)) dz = sc * expf(z[c * NS + i] - mx) * inv_se;
      if (e == mv) dz -= sc;
      z[c * NS + i] = dz;
    }
    __syncthreads();
    pgrad_pair(z, a2, co, ci, Lx, Ly, NS, 0, 1, gw3, gb3);
    pconv_t(z, g2, wb + 2304, Lx, Ly, NS);  // g2 <- dL/dh2
    __syncthreads();
    pgrad_pair(g2, a1, co, ci, Lx, Ly, NS, 0, 1, gw2, gb2);
    pconv_t(g2, g1, wb, Lx, Ly, NS);  // g1 <- dL/dh1
    __syncthreads();
    pgrad_pair(g1, x0, co1, ci1, Lx, Ly, NS, grp, kPWarps, gw1, gb1);
  }
  __syncthreads();
  float* out = part + (size_t)blockIdx.x * (kPCount + 1);
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    out[kPOffW3 + (co * kPC + ci) * 9 + t] = gw3[t];
    out[kPOffW2 + (co * kPC + ci) * 9 + t] = gw2[t];
    l1s[(grp * 32 + p1) * 10 + t] = gw1[t];
  }
  l1s[(grp * 32 + p1) * 10 + 9] = gb1;
  if (ci == 0) {
    out[kPOffB3 + co] = gb3;
    out[kPOffB2 + co] = gb2;
  }
  __syncthreads();
  for (int e = tid; e < 32 * 10; e += blockDim.x) {
    const int p = e / 10, t = e - p * 10;
    float s = 0.0f;
    for (int g = 0; g < kPWarps; ++g) s += l1s[(g * 32 + p) * 10 + t];
    if (t < 9)
      out[p * 9 + t] = s;  // W1[co][ci][tap] at (co * 2 + ci) * 9 + tap, pair p = co * 2 + ci
    else if ((p & 1) == 0)
      out[kPOffB1 + (p >> 1)] = s;
  }
  if (tid == 0) out[kPCount] = lsum;
}

__global__ void prop_reduce_kernel(const float* __restrict__ part, int n_part,
                                   float* __restrict__ grad, float* __restrict__ loss) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > kPCount) return;
  float s = 0.0f;
  for (int p = 0; p < n_part; ++p) s += part[(size_t)p * (kPCount + 1) + e];
  if (e < kPCount)
    grad[e] = s;
  else if (loss)
    *loss = s;
}

__global__ void prop_adam_kernel(float* master, float* m, float* v, const float* __restrict__ g,
                                 int count, float lr, float b1, float b2, float eps, float c1,
                                 float c2, __nv_bfloat16* wbf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.0f - b1) * gi;
    const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    const float w = master[e] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    master[e] = w;
    if (wbf) wbf[e] = __float2bfloat16_rn(w);
  }
}

__global__ void prop_pack_kernel(const float* __restrict__ master, int count,
                                 __nv_bfloat16* __restrict__ wbf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x)
    wbf[e] = __float2bfloat16_rn(master[e]);
}

std::mutex g_prop_mu;

// Raise a kernel's dynamic shared-memory limit once per (kernel, size) high-water mark.
template <typename K>
int prop_smem_attr(K kernel, size_t bytes, size_t* done) {
  std::lock_guard<std::mutex> g(g_prop_mu);
  if (bytes <= *done) return NH_OK;
  cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return check_cuda(e, "proposal smem attribute");
  *done = bytes;
  return NH_OK;
}

size_t g_sample_smem = 48 * 1024, g_logits_smem = 48 * 1024, g_backward_smem = 48 * 1024;
constexpr size_t kSmemLimit = 227 * 1024;

template <typename K>
int prop_grid(K kernel, size_t smem, int work, int* grid) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPThreads, smem);
  if (e != cudaSuccess) return check_cuda(e, "proposal occupancy");
  *grid = std::max(1, std::min(work, std::max(1, per_sm) * num_sms()));
  return NH_OK;
}

}  // namespace

int check_proposal(const nh_proposal_params* q) {
  if (!q || !q->weights) return fail(NH_ERR_INVALID, "proposal: null parameters");
  if (q->Lx < 3 || q->Ly < 3 || q->Lx > 32 || q->Ly > 32)
    return fail(NH_ERR_UNSUPPORTED, "proposal: lattice %dx%d (3 <= Lx, Ly <= 32)", q->Lx, q->Ly);
  if (q->n_dirs != 4 && q->n_dirs != 8)
    return fail(NH_ERR_INVALID, "proposal: n_dirs %d", q->n_dirs);
  return NH_OK;
}

int launch_prop_sample(const int8_t* spins, int batch, const nh_proposal_params& q, uint64_t seed,
                       int64_t step, int32_t* valid, int32_t* from, int32_t* to, float* lqr,
                       cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  const size_t smem = prop_sample_smem(q.Lx * q.Ly);
  if (smem > kSmemLimit) return fail(NH_ERR_UNSUPPORTED, "proposal: lattice too large");
  int rc = prop_smem_attr(prop_sample_kernel, smem, &g_sample_smem);
  if (rc) return rc;
  int grid = 0;
  if ((rc = prop_grid(prop_sample_kernel, smem, batch, &grid))) return rc;
  ProfScope prof_scope(NH_K_PROP_SAMPLE, st);
  prop_sample_kernel<<<grid, kPThreads, smem, st>>>(
      spins, batch, static_cast<const __nv_bfloat16*>(q.weights), q.Lx, q.Ly, q.n_dirs,
      (uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)step, (uint32_t)((uint64_t)step >> 32),
      valid, from, to, lqr);
  return check_launch("prop_sample_kernel");
}

size_t proposal_backward_parts(int batch) {
  return (size_t)std::max(1, std::min(batch, kPMaxParts));
}

constexpr int kPGactPerSm = 2;  // CTAs per SM of the global-plane backward (its scratch slices)

bool prop_backward_gact(int N) { return prop_backward_smem(N) > kSmemLimit; }

}  // namespace nh

using namespace nh;

extern "C" {

int nh_proposal_pack(const float* master, int count, void* weights_bf16, void* stream) {
  if (!master || !weights_bf16 || count != kPCount)
    return fail(NH_ERR_INVALID, "proposal_pack: count %d (expected %d)", count, kPCount);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  prop_pack_kernel<<<(kPCount + 255) / 256, 256, 0, st>>>(
      master, count, static_cast<__nv_bfloat16*>(weights_bf16));
  return check_launch("prop_pack_kernel");
}

int nh_proposal_forward(const int8_t* spins, int batch, const nh_proposal_params* q,
                        float* logits, void* stream) {
  int rc = check_proposal(q);
  if (rc) return rc;
  if (!spins || !logits || batch < 0) return fail(NH_ERR_INVALID, "proposal_forward: buffers");
  if (batch == 0) return NH_OK;
  const size_t smem = prop_sample_smem(q->Lx * q->Ly);
  if (smem > kSmemLimit) return fail(NH_ERR_UNSUPPORTED, "proposal: lattice too large");
  if ((rc = prop_smem_attr(prop_logits_kernel, smem, &g_logits_smem))) return rc;
  int grid = 0;
  if ((rc = prop_grid(prop_logits_kernel, smem, batch, &grid))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ProfScope prof_scope(NH_K_PROP_FORWARD, st);
  prop_logits_kernel<<<grid, kPThreads, smem, st>>>(
      spins, batch, static_cast<const __nv_bfloat16*>(q->weights), q->Lx, q->Ly, logits);
  return check_launch("prop_logits_kernel");
}

int nh_proposal_sample(const int8_t* spins, int batch, const nh_proposal_params* q,
                       uint64_t seed, int64_t step, int32_t* from, int32_t* to, int32_t* valid,
                       float* log_q_ratio, void* stream) {
  int rc = check_proposal(q);
  if (rc) return rc;
  if (!spins || !from || !to || !valid || !log_q_ratio || batch < 0)
    return fail(NH_ERR_INVALID, "proposal_sample: buffers");
  return launch_prop_sample(spins, batch, *q, seed, step, valid, from, to, log_q_ratio,
                            static_cast<cudaStream_t>(stream));
}

size_t nh_proposal_backward_workspace_bytes(int batch, const nh_proposal_params* q) {
  size_t bytes = proposal_backward_parts(batch) * (kPCount + 1) * sizeof(float);
  if (q && prop_backward_gact(q->Lx * q->Ly)) {
    const size_t slices = std::min<size_t>(proposal_backward_parts(batch),
                                           (size_t)kPGactPerSm * num_sms());
    bytes = ((bytes + 255) & ~(size_t)255) + slices * prop_plane_floats(q->Lx * q->Ly) * 4;
  }
  return bytes;
}

int nh_proposal_backward(const int8_t* spins, const int32_t* moves, const float* weights,
                         int batch, const nh_proposal_params* q, float* loss, float* grad,
                         void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_proposal(q);
  if (rc) return rc;
  if (!spins || !moves || !weights || !grad || batch <= 0)
    return fail(NH_ERR_INVALID, "proposal_backward: buffers");
  const size_t need = nh_proposal_backward_workspace_bytes(batch, q);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "proposal_backward"))) return rc;
  const int N = q->Lx * q->Ly;
  const bool gact = prop_backward_gact(N);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float* part = static_cast<float*>(workspace);
  int grid = 0;
  if (!gact) {
    const size_t smem = prop_backward_smem(N);
    if ((rc = prop_smem_attr(prop_backward_kernel<false>, smem, &g_backward_smem))) return rc;
    if ((rc = prop_grid(prop_backward_kernel<false>, smem, batch, &grid))) return rc;
    grid = std::min<int>(grid, (int)proposal_backward_parts(batch));
    ProfScope prof_scope(NH_K_PROP_BACKWARD, st);
    prop_backward_kernel<false><<<grid, kPThreads, smem, st>>>(
        spins, moves, weights, batch, static_cast<const __nv_bfloat16*>(q->weights), q->Lx,
        q->Ly, q->n_dirs, 1.0f / (float)batch, part, nullptr);
    if ((rc = check_launch("prop_backward_kernel"))) return rc;
  } else {
    const size_t smem = prop_backward_smem_gact(N);
    static size_t g_gact_smem = 48 * 1024;
    if ((rc = prop_smem_attr(prop_backward_kernel<true>, smem, &g_gact_smem))) return rc;
    grid = (int)std::min<size_t>(proposal_backward_parts(batch),
                                 (size_t)kPGactPerSm * num_sms());
    const size_t part_bytes = proposal_backward_parts(batch) * (kPCount + 1) * sizeof(float);
    float* planes = reinterpret_cast<float*>(static_cast<char*>(workspace) +
                                             ((part_bytes + 255) & ~(size_t)255));
    ProfScope prof_scope(NH_K_PROP_BACKWARD, st);
    prop_backward_kernel<true><<<grid, kPThreads, smem, st>>>(
        spins, moves, weights, batch, static_cast<const __nv_bfloat16*>(q->weights), q->Lx,
        q->Ly, q->n_dirs, 1.0f / (float)batch, part, planes);
    if ((rc = check_launch("prop_backward_kernel<global planes>"))) return rc;
  }
  prop_reduce_kernel<<<(kPCount + 256) / 256, 256, 0, st>>>(part, grid, grad, loss);
  return check_launch("prop_reduce_kernel");
}

int nh_proposal_adam_step(float* master, float* m, float* v, const float* grad, int count,
                          int64_t t, float lr, float beta1, float beta2, float eps,
                          void* weights_bf16, void* stream) {
  if (!master || !m || !v || !grad || count != kPCount || t < 1)
    return fail(NH_ERR_INVALID, "proposal_adam_step: arguments");
  const float c1 = (float)(1.0 / (1.0 - pow((double)beta1, (double)t)));
  const float c2 = (float)(1.0 / (1.0 - pow((double)beta2, (double)t)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ProfScope prof_scope(NH_K_PROP_ADAM, st);
  prop_adam_kernel<<<(count + 255) / 256, 256, 0, st>>>(
      master, m, v, grad, count, lr, beta1, beta2, eps, c1, c2,
      static_cast<__nv_bfloat16*>(weights_bf16));
  return check_launch("prop_adam_kernel");
}

}  // extern "C"

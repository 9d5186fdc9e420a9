// Residual backflow CNN of the released Pfaffian-backflow states (quantax ResConv as built at
// code/backflow/models.py:319-329; network of data/supplement/tableS1_network/
// network_settings.json:21-56, "normal" blocks), forward on CUDA cores in FP32 (FP64 for the
// recompute of flagged items):
//
//   x_0[c, i] = E[c, occ(i)]                       occ = n_up + 2 n_dn (empty, up, down, double)
//   x_{b+1}   = x_b + Conv2(GELU(Conv1(GELU(RMSNorm(x_b)))))   b < blocks
//   y         = x_blocks / sqrt(blocks + 1)        channels [0, d) spin up, [d, 2d) spin down
//
// with 3x3 periodic cross-correlations with bias, RMSNorm over all channels and sites without
// affine parameters (eps kRmsEps inside the root) and tanh-approximated GELU.
//
// One CTA of 256 threads per item (configuration x symmetry image, grid-stride).  The three
// activation planes x, h = GELU(RMSNorm(x)) and u = GELU(Conv1(h)) are channel-major with row
// stride N + 1, in shared memory for FP32 at N <= 256 (197 KB at 64 channels), otherwise in a
// per-CTA slice of global scratch.  A convolution is a tile loop over 256 sites: thread t owns
// 16 output channels (t / 64) of 4 sites (t % 64 + 64 k) as 64 register accumulators; the
// weights stream through shared memory in chunks of 8 input channels ([ci][tap][co], 18 KB in
// FP32), the next chunk held in registers while the current one is used, so that their L2
// latency hides behind the FMAs.  Per (input channel, tap) a thread issues 4 activation loads,
// 4 broadcast 16-byte weight loads and 64 FMAs.  The output rows Y of the occupied modes, their
// indices and the item sign are written by the same epilogue as the plain CNN's.
#include <math.h>

#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kRcThreads = kNumThreads;  // 256
constexpr int kRcC = 64;                 // channels (the released states)
constexpr int kRcCoPerThread = 16;       // output channels per thread
constexpr int kRcSiteLanes = kRcThreads / (kRcC / kRcCoPerThread);                 // 64
constexpr int kRcChunk = 8;              // input channels per staged weight chunk
constexpr int kRcChunkFloats = kRcChunk * 9 * kRcC;                                // 4608
constexpr int kRcChunkVec = kRcChunkFloats / 4;                                    // float4s
constexpr int kRcPrefetch = (kRcChunkVec + kRcThreads - 1) / kRcThreads;          // 5
constexpr double kRmsEps = 1e-6;
static_assert(kRcC % kRcChunk == 0, "chunks must tile the input channels");

// Sites per thread and tile: 4 in FP32 (64 accumulators), 2 in FP64 (the same register count).
template <typename T>
struct RcSpt {
  static constexpr int value = sizeof(T) == 4 ? 4 : 2;
};

__device__ __forceinline__ float tfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double tfma(double a, double b, double c) { return ::fma(a, b, c); }
__device__ __forceinline__ float trsqrt_eps(float ms, double eps) {
  return 1.0f / sqrtf(ms + (float)eps);
}
__device__ __forceinline__ double trsqrt_eps(double ms, double eps) {
  return 1.0 / ::sqrt(ms + eps);
}

__device__ __forceinline__ float gelu_tanh(float x) {
  const float k0 = 0.7978845608028654f;  // sqrt(2 / pi)
  return 0.5f * x * (1.0f + tanhf(k0 * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ double gelu_tanh(double x) {
  const double k0 = 0.7978845608028654;
  return 0.5 * x * (1.0 + tanh(k0 * (x + 0.044715 * x * x * x)));
}

template <typename T>
struct RcArgs {
  ConfigList cl;
  const float* embed;  // packed (4, C): [occ][co]
  const float* wp;     // packed convolutions: per conv [ci][tap][co]
  const float* b;      // (2 blocks, C)
  int Lx, Ly, N, blocks, n;
  int mode;
  const int32_t* slot_item;
  const int32_t* slot_count;
  int max_slots;
  float* feat;
  T* Y;
  int32_t* idx;
  float* item_sign;
  T* act;  // GACT: per-CTA planes (3 C (N + 1))
};

// 16 weights of one (input channel, tap) row for this thread's output channels (broadcast).
__device__ __forceinline__ void ldw16(const float* p, float* w) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float4 v = reinterpret_cast<const float4*>(p)[q];
    w[4 * q] = v.x;
    w[4 * q + 1] = v.y;
    w[4 * q + 2] = v.z;
    w[4 * q + 3] = v.w;
  }
}
__device__ __forceinline__ void ldw16(const double* p, double* w) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double2 v = reinterpret_cast<const double2*>(p)[q];
    w[2 * q] = v.x;
    w[2 * q + 1] = v.y;
  }
}

// Registers holding the next weight chunk (kRcPrefetch float4 per thread).
struct ChunkRegs {
  float4 v[kRcPrefetch];
};

__device__ __forceinline__ void chunk_load(ChunkRegs& r, const float* src) {
  const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
  for (int k = 0; k < kRcPrefetch; ++k) {
    const int i = threadIdx.x + k * kRcThreads;
    if (i < kRcChunkVec) r.v[k] = __ldg(s4 + i);
  }
}

template <typename T>
__device__ __forceinline__ void chunk_store(const ChunkRegs& r, T* dst) {
#pragma unroll
  for (int k = 0; k < kRcPrefetch; ++k) {
    const int i = threadIdx.x + k * kRcThreads;
    if (i < kRcChunkVec) {
      dst[4 * i] = T(r.v[k].x);
      dst[4 * i + 1] = T(r.v[k].y);
      dst[4 * i + 2] = T(r.v[k].z);
      dst[4 * i + 3] = T(r.v[k].w);
    }
  }
}

// One 3x3 periodic convolution C -> C over all sites: dst = epi(conv(src) + bias, dst).
// Entry: pre holds chunk 0 of w; exit: pre holds chunk 0 of w_next (when not null).
// RESID: dst += result; else dst = GELU(result).
template <typename T, bool RESID>
__device__ void conv_pass(const T* src, T* dst, const float* w, const float* w_next,
                          const float* bias, T* wsm, ChunkRegs& pre, int Lx, int Ly, int N) {
  constexpr int SPT = RcSpt<T>::value;
  constexpr int kTile = kRcSiteLanes * SPT;
  const int NS = N + 1;
  const int tid = threadIdx.x;
  const int cg = tid / kRcSiteLanes;  // output-channel group (16 channels)
  const int sl = tid % kRcSiteLanes;  // site lane: sites sl + 64 k of the tile
  constexpr int kChunks = kRcC / kRcChunk;
  const int tiles = (N + kTile - 1) / kTile;
  for (int tile = 0; tile < tiles; ++tile) {
    int nb[SPT][9];
    bool live[SPT];
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
      const int site = tile * kTile + sl + k * kRcSiteLanes;
      live[k] = site < N;
      const int s = live[k] ? site : 0;
      const int x = s / Ly, y = s - x * Ly;
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        int xx = x + u - 1;
        xx = xx < 0 ? xx + Lx : (xx >= Lx ? xx - Lx : xx);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          int yy = y + v - 1;
          yy = yy < 0 ? yy + Ly : (yy >= Ly ? yy - Ly : yy);
          nb[k][u * 3 + v] = xx * Ly + yy;
        }
      }
    }
    T acc[SPT][kRcCoPerThread];
#pragma unroll
    for (int j = 0; j < kRcCoPerThread; ++j) {
      const T bj = T(__ldg(bias + cg * kRcCoPerThread + j));
#pragma unroll
      for (int k = 0; k < SPT; ++k) acc[k][j] = bj;
    }
#pragma unroll 1
    for (int ch = 0; ch < kChunks; ++ch) {
      __syncthreads();  // every thread is done with the previous chunk in wsm
      chunk_store(pre, wsm);
      __syncthreads();
      const bool last = tile == tiles - 1 && ch == kChunks - 1;
      if (!last) {
        chunk_load(pre, w + (size_t)((ch + 1) % kChunks) * kRcChunkFloats);
      } else if (w_next) {
        chunk_load(pre, w_next);
      }
#pragma unroll 1
      for (int cil = 0; cil < kRcChunk; ++cil) {
        const T* in = src + (ch * kRcChunk + cil) * NS;
        const T* wrow = wsm + cil * 9 * kRcC + cg * kRcCoPerThread;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
          T iv[SPT];
#pragma unroll
          for (int k = 0; k < SPT; ++k) iv[k] = in[nb[k][tap]];
          T wv[kRcCoPerThread];
          ldw16(wrow + tap * kRcC, wv);
#pragma unroll
          for (int k = 0; k < SPT; ++k)
#pragma unroll
            for (int j = 0; j < kRcCoPerThread; ++j) acc[k][j] = tfma(iv[k], wv[j], acc[k][j]);
        }
      }
    }
    // Epilogue: this thread's outputs are read by no other thread of this pass (dst != src).
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
      if (!live[k]) continue;
      const int site = tile * kTile + sl + k * kRcSiteLanes;
#pragma unroll
      for (int j = 0; j < kRcCoPerThread; ++j) {
        T* o = dst + (cg * kRcCoPerThread + j) * NS + site;
        if constexpr (RESID) {
          *o += acc[k][j];
        } else {
          *o = gelu_tanh(acc[k][j]);
        }
      }
    }
  }
}

template <typename T, bool GACT>
__global__ void __launch_bounds__(kRcThreads, 1) resconv_kernel(RcArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = a.N, NS = N + 1, M2 = 2 * N;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int kWarps = kRcThreads / 32;
  T* X;
  T* wsm;  // staged weight chunk [ci][tap][co]
  if constexpr (GACT) {
    X = a.act + (size_t)blockIdx.x * 3 * kRcC * NS;
    wsm = reinterpret_cast<T*>(smem_raw);
  } else {
    X = reinterpret_cast<T*>(smem_raw);
    wsm = X + 3 * kRcC * NS;
  }
  T* H = X + kRcC * NS;
  T* U = H + kRcC * NS;
  T* red = wsm + kRcChunkFloats;                       // (warps) partial sums of x^2
  int* simg = reinterpret_cast<int*>(red + kWarps);    // (2N) +-1 of the image configuration
  int* occl = simg + M2;                                // (2N) occupied modes, ascending
  int* wbuf = occl + M2;                                // 4 Lx + 32 ints of scan scratch

  const int G = a.cl.G;
  const int n_work = a.slot_item ? *a.slot_count
                                 : (a.cl.n_cfg_dev ? *a.cl.n_cfg_dev : a.cl.n_cfg) * G;
  const size_t conv_floats = (size_t)kRcC * 9 * kRcC;
  const T inv_cn = T(1) / T(kRcC * N);
  const T out_scale = trsqrt_eps(T(a.blocks + 1), 0.0);
  ChunkRegs pre;

  for (int slot = blockIdx.x; slot < n_work; slot += gridDim.x) {
    const int item = a.slot_item ? a.slot_item[slot] : slot;
    const int c = item / G, g = item - c * G;
    const int smp = a.cl.sample ? a.cl.sample[c] : c;
    const int fr = a.cl.from ? a.cl.from[c] : -1;
    const int to = a.cl.from ? a.cl.to[c] : -1;
    const int8_t* base = a.cl.spins + (int64_t)smp * M2;
    chunk_load(pre, a.wp);  // chunk 0 of the first convolution

    __syncthreads();  // the previous item's readers of simg / planes are done
    for (int m = tid; m < M2; m += kRcThreads) {
      const int src = sym_map(m, g, a.Lx, a.Ly, N);  // image[m] = s[g(m)] (g is an involution)
      int v = base[src];
      v = move_value(src, v, fr, to);
      simg[m] = v > 0 ? 1 : -1;
    }
    __syncthreads();
    for (int i = tid; i < N; i += kRcThreads) {  // occupation embedding
      const int occ = (simg[i] > 0 ? 1 : 0) + (simg[N + i] > 0 ? 2 : 0);
      const float* e = a.embed + occ * kRcC;
      for (int ch = 0; ch < kRcC; ++ch) X[ch * NS + i] = T(__ldg(e + ch));
    }

    for (int blk = 0; blk < a.blocks; ++blk) {
      __syncthreads();  // x complete
      T ss = T(0);
      for (int ch = 0; ch < kRcC; ++ch)
        for (int i = tid; i < N; i += kRcThreads) {
          const T v = X[ch * NS + i];
          ss = tfma(v, v, ss);
        }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
      if (lane == 0) red[wid] = ss;
      __syncthreads();
      T tot = T(0);
#pragma unroll
      for (int w = 0; w < kWarps; ++w) tot += red[w];
      const T r = trsqrt_eps(tot * inv_cn, kRmsEps);
      for (int ch = 0; ch < kRcC; ++ch)
        for (int i = tid; i < N; i += kRcThreads) H[ch * NS + i] = gelu_tanh(X[ch * NS + i] * r);
      // (the first chunk barrier of conv_pass orders these writes before the reads)
      const float* w1 = a.wp + (size_t)(2 * blk) * conv_floats;
      const float* w2 = w1 + conv_floats;
      conv_pass<T, false>(H, U, w1, w2, a.b + (2 * blk) * kRcC, wsm, pre, a.Lx, a.Ly, N);
      conv_pass<T, true>(U, X, w2, blk + 1 < a.blocks ? w2 + conv_floats : nullptr,
                         a.b + (2 * blk + 1) * kRcC, wsm, pre, a.Lx, a.Ly, N);
    }
    __syncthreads();
    constexpr int d = kRcC / 2;
    if (a.mode == 0) {
      float* dst = a.feat + (int64_t)item * kRcC * N;
      for (int o = tid; o < kRcC * N; o += kRcThreads) {
        const int aa = o % d;
        const int site = (o / d) % N;
        const int sg = o / (N * d);
        dst[o] = (float)(X[(sg * d + aa) * NS + site] * out_scale);
      }
      continue;
    }
    write_occupied_rows(simg, occl, wbuf, N, a.n, d, g, a.Lx, a.Ly,
                        a.Y + (int64_t)slot * a.n * d, a.idx + (int64_t)slot * a.n,
                        a.item_sign + item, [&](int sg, int aa, int site) {
                          return X[(sg * d + aa) * NS + site] * out_scale;
                        });
  }
}

// packed = [embed (4, C): [occ][co]] ++ per conv k [ci][tap][co];
// conv_w = [embed (C, 4)] ++ per conv k (C, C, 3, 3).
__global__ void resconv_pack_kernel(const float* __restrict__ w, int C, int convs,
                                    float* packed) {
  const int total = 4 * C + convs * 9 * C * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (i < 4 * C) {
      const int occ = i / C, co = i - occ * C;
      packed[i] = w[co * 4 + occ];
      continue;
    }
    const int r0 = i - 4 * C;
    const int k = r0 / (9 * C * C);
    const int r = r0 - k * 9 * C * C;  // (ci * 9 + tap) * C + co
    const int co = r % C;
    const int ct = r / C;
    packed[i] = w[4 * C + (size_t)k * 9 * C * C + co * 9 * C + ct];
  }
}

template <typename T, bool GACT>
size_t rc_smem(int N) {
  return sizeof(T) * ((GACT ? 0 : 3 * (size_t)kRcC * (N + 1)) + kRcChunkFloats + 8) +
         sizeof(int) * (4 * (size_t)N + 4 * 32 + 32);
}

constexpr int kRcBigPerSm = 2;  // CTAs per SM of the global-plane kernel (scratch bound)

template <typename T, bool GACT>
int launch_rc_t(const CnnLaunch& q, int N, cudaStream_t st) {
  const nh_backflow_params& p = *q.p;
  const size_t smem = rc_smem<T, GACT>(N);
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "resconv: N=%d needs %zu B of shared memory", N, smem);
  if (GACT && !q.act)
    return fail(NH_ERR_UNSUPPORTED, "resconv: N=%d needs the activation-plane scratch", N);
  const int slots = q.slot_item ? q.max_slots : q.cl->n_cfg * q.cl->G;
  if (slots <= 0) return NH_OK;
  int grid = num_sms() * (GACT ? kRcBigPerSm : 1);
  if (grid > slots) grid = slots;
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(resconv_kernel<T, GACT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "resconv smem attribute");
    configured = smem;
  }
  RcArgs<T> a{*q.cl, p.conv_w_packed, p.conv_w_packed + 4 * kRcC, p.conv_b, p.Lx, p.Ly, N,
              p.layers, p.n_up + p.n_dn, q.mode, q.slot_item, q.slot_count, q.max_slots,
              q.feat, static_cast<T*>(q.Y), q.idx, q.item_sign, static_cast<T*>(q.act)};
  ProfScope prof_scope(sizeof(T) == 8 ? NH_K_RESCONV64 : NH_K_RESCONV, st);
  resconv_kernel<T, GACT><<<grid, kRcThreads, smem, st>>>(a);
  return check_launch(sizeof(T) == 8 ? "resconv_kernel<double>" : "resconv_kernel<float>");
}

}  // namespace

size_t resconv_packed_floats(int channels, int blocks) {
  return 4 * (size_t)channels + 2 * (size_t)blocks * 9 * channels * channels;
}

int launch_pack_resconv(const float* conv_w, int channels, int blocks, float* packed,
                        cudaStream_t st) {
  const int total = (int)resconv_packed_floats(channels, blocks);
  ProfScope prof_scope(NH_K_PACK, st);
  resconv_pack_kernel<<<(total + 255) / 256, 256, 0, st>>>(conv_w, channels, 2 * blocks,
                                                           packed);
  return check_launch("resconv_pack_kernel");
}

// FP32 keeps its planes in shared memory up to N = 256; FP64 and larger lattices use the
// per-CTA global planes.
size_t resconv_scratch_bytes(int N) {
  return (size_t)num_sms() * kRcBigPerSm * 3 * kRcC * (N + 1) * sizeof(double);
}

int launch_resconv(const CnnLaunch& q, cudaStream_t st) {
  const nh_backflow_params& p = *q.p;
  const int N = p.Lx * p.Ly;
  if (p.channels != kRcC || p.layers < 1 || N % 2 || N > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "resconv: channels %d (64), blocks %d, N %d", p.channels,
                p.layers, N);
  if (!p.conv_w_packed || !p.conv_b)
    return fail(NH_ERR_INVALID, "resconv: conv_w_packed (nh_pack_resconv_weights) or conv_b "
                "is null");
  if (reinterpret_cast<uintptr_t>(p.conv_w_packed) % 16)
    return fail(NH_ERR_INVALID, "resconv: conv_w_packed must be 16-byte aligned");
  if (q.fp64) return launch_rc_t<double, true>(q, N, st);
  return rc_smem<float, false>(N) <= 227 * 1024 ? launch_rc_t<float, false>(q, N, st)
                                                 : launch_rc_t<float, true>(q, N, st);
}

}  // namespace nh

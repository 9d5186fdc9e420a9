// Backflow CNN forward on the 5th-generation tensor cores (tcgen05, sm_100a): the chosen form.
//
// The 3x3 periodic convolutions run as implicit GEMMs D[site, co] += A[site + tap, ci] W[tap][ci, co]
// with BF16 operands in shared memory and FP32 accumulators in tensor memory.  The activations
// of one configuration live in a padded plane: site (x, y) sits at padded position
// (x + 1, y + 1) of an (Lx + 2) x (Ly + 2) grid whose border repeats the periodic neighbours, and
// each padded site holds 8 channels in 16 bytes ("core-matrix rows"), one plane per group of 8
// channels.  An M = 128 tile is one 8-site y-block across 16 x-rows: its rows are eight
// consecutive sites (one 128-byte core matrix) per x-row, x-rows one padded row apart (the
// stride-byte offset), so every tap (dx, dy) is the same descriptor with the start address moved
// by (dx (Ly + 2) + dy) x 16 bytes, and no im2col copy is made.
//
// Precision: mode 1 uses BF16 weights and activations; mode 2 splits both into BF16 hi + lo and
// accumulates hi*hi + hi*lo + lo*hi (about 16 significant bits per product) for near-FP32
// features.  The layer-0 input (+-1 occupations) is exact in BF16.  Bias, GELU and the split run
// in FP32 in the epilogue, which reads the accumulators with tcgen05.ld (warp w % 4 owns lanes
// 32 (w % 4) .. + 31 of both tiles).
//
// Two warp groups of 128 threads run independent image streams in one CTA: each has its own
// activation planes, bookkeeping, mbarrier, 256 tensor-memory columns (four partial sums of its
// two 128 x 32 tiles, see issue_layer) and named barrier, and
// shares the resident weights; while one group's MMAs run, the other converts its accumulators
// (bias, GELU, hi/lo split) and writes its next planes.
//
// Output: the occupied rows Y (n, d) FP32 of the image configuration, the occupied-mode list and
// the item sign, like the CUDA-core kernel (mode 1 of nh_cnn.cu).
//
// The packed weight image (129 KB) is brought into shared memory once per CTA by one bulk TMA
// copy (cp.async.bulk, no multicast) that completes on an mbarrier.
//
// Supported: Lx = 16, Ly = 16, 32 channels, 4 layers (the benchmark network).  Every wait on an
// mbarrier is bounded; on expiry the kernel records an error code in *err and returns after
// releasing its tensor memory.
#include <math.h>
#include <stdint.h>

#include <cuda_bf16.h>

#include "nh_common.cuh"
#include "nh_tcgen05.cuh"

namespace nh {
namespace {

using namespace tc;

constexpr int kTcThreads = 256;
constexpr int kC = 32;          // channels
constexpr int kW0Bytes = 2 * 9 * 2 * 4 * 128;    // layer 0: q x tap x kc(2) x cg(4) x 128 B
constexpr int kW1Bytes = 2 * 9 * 4 * 4 * 128;    // layers 1..3: q x tap x kc(4) x cg(4) x 128 B
constexpr int kWBytes = kW0Bytes + 3 * kW1Bytes;
constexpr int kActBytes = 2 * 4 * kPlane;        // hi and lo, 4 planes each
constexpr int kWG = 2;                           // independent warp groups per CTA
constexpr int kWGThreads = kTcThreads / kWG;     // 128
constexpr int kIntsPerWG = 3 * 2 * kL * kL + 4 * kL + 32;  // simg, rowof, occl, scan scratch
constexpr int kParts = 4;                        // partial sums per tile: (kh, cross)
constexpr unsigned kTmemCols = 64 * kParts * kWG; // per group: 4 partials x two 128 x 32 tiles

struct TcArgs {
  ConfigList cl;
  const uint16_t* wpk;  // packed BF16 weights (kWBytes)
  const float* bias;    // (4, 32)
  int n;                // electrons per configuration
  int mode;             // 1: BF16, 2: BF16 x3
  float* Y;             // (items, n, 16)
  int32_t* idx;         // (items, n)
  float* item_sign;     // (items,)
  int32_t* err;         // error word (0 = ok)
};

// Instruction descriptor: kind::f16, BF16 x BF16 -> FP32, both K-major, M = 128, N = 32.
constexpr uint32_t kIdesc = idesc_bf16(128, 32);

// tanh-approximated GELU written as x * sigmoid(2 z), z = sqrt(2/pi) (x + 0.044715 x^3), which is
// the same function as 0.5 x (1 + tanh z); the exponential is the fast __expf intrinsic.
__device__ __forceinline__ float gelu_tanh(float x) {
  const float z2 = 1.5957691216057308f * (x + 0.044715f * x * x * x);
  return __fdividef(x, 1.0f + __expf(-z2));
}

// Issue the MMAs of one layer for both tiles (one thread).
// Partial sum p = 2 kh + cross of tile h lives at columns 64 p + 32 h of the group's 256: the
// hi*hi products of the input-channel half kh, and (cross = 1) its hi*lo + lo*hi products, so
// that every FP32 accumulation chain in the tensor core is short (9 or 18 MMAs) and the small
// cross terms are not added into the large main sum there.  The epilogue adds the partials.
__device__ void issue_layer(uint32_t tmem, uint32_t act_hi, uint32_t act_lo, uint32_t w_hi,
                            uint32_t w_lo, int kchunks, int tap_bytes, bool split_act,
                            bool split_w) {
  const uint32_t sbo_a = kP * 16;  // next x-row of the tile
  const uint32_t lbo_a = kPlane;   // next 8-channel plane
  const uint32_t lbo_b = 4 * 128;  // next 8-ci chunk of the weights
  const uint32_t sbo_b = 128;      // next 8-co group of the weights
#pragma unroll
  for (int h = 0; h < 2; ++h) {
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dx = tap / 3 - 1, dy = tap % 3 - 1;
      const uint32_t aoff = (uint32_t)pad_off(dx + 1, 8 * h + dy + 1);
#pragma unroll
      for (int kh = 0; kh < 2; ++kh) {
        if (kh >= kchunks / 2) break;
        const uint32_t d_main = tmem + 64 * (2 * kh) + 32 * h;
        const uint32_t d_cross = d_main + 64;
        const uint32_t ao = aoff + 2 * kh * kPlane;
        const uint32_t bo = tap * tap_bytes + 2 * kh * 4 * 128;
        const uint64_t ahi = make_desc(act_hi + ao, lbo_a, sbo_a);
        const uint64_t bhi = make_desc(w_hi + bo, lbo_b, sbo_b);
        mma_bf16(d_main, ahi, bhi, kIdesc, tap > 0);
        if (split_w) mma_bf16(d_cross, ahi, make_desc(w_lo + bo, lbo_b, sbo_b), kIdesc, tap > 0);
        if (split_act)
          mma_bf16(d_cross, make_desc(act_lo + ao, lbo_a, sbo_a), bhi, kIdesc,
                   tap > 0 || split_w);
      }
    }
  }
}

// Accumulators of tile h for this warp's lane quarter: the sum of the partials the layer wrote.
__device__ __forceinline__ void load_tile(uint32_t tlane, int h, int kchunks, bool cross,
                                          float* v) {
  tmem_ld32(tlane + 32 * h, v);
#pragma unroll
  for (int p = 1; p < kParts; ++p) {
    const int kh = p >> 1;
    if (kh >= kchunks / 2 || ((p & 1) && !cross)) continue;
    float w[32];
    tmem_ld32(tlane + 64 * p + 32 * h, w);
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] += w[i];
  }
}

__device__ __forceinline__ void wg_sync(int wg) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + wg), "r"(kWGThreads) : "memory");
}

struct WgSync {
  int wg;
  __device__ void operator()() const { wg_sync(wg); }
};

// Convert one 128 x 32 accumulator tile row (32 channels of one site) of layers 0-2 into the
// next layer's BF16 hi / lo 8-channel groups.
__device__ __forceinline__ void act_groups(const float* v, const float* bl, uint4* hi,
                                           uint4* lo) {
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    uint32_t ph[4], pl[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float f0 = gelu_tanh(v[8 * kc + 2 * j] + bl[8 * kc + 2 * j]);
      const float f1 = gelu_tanh(v[8 * kc + 2 * j + 1] + bl[8 * kc + 2 * j + 1]);
      const uint16_t h0 = bf16_bits(f0), h1 = bf16_bits(f1);
      ph[j] = (uint32_t)h0 | ((uint32_t)h1 << 16);
      pl[j] = (uint32_t)bf16_bits(f0 - bf16_val(h0)) |
              ((uint32_t)bf16_bits(f1 - bf16_val(h1)) << 16);
    }
    hi[kc] = make_uint4(ph[0], ph[1], ph[2], ph[3]);
    lo[kc] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
  }
}

__global__ void __launch_bounds__(kTcThreads, 1) cnn_tc_kernel(TcArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* wsm = smem;                             // packed weights (kWBytes)
  unsigned char* act_all = smem + kWBytes;               // per group: [q][kc] planes
  float* bsm = reinterpret_cast<float*>(act_all + kWG * kActBytes);  // (4, 32) biases
  int* ints_all = reinterpret_cast<int*>(bsm + 4 * kC);  // per group: kIntsPerWG
  uint64_t* bars = reinterpret_cast<uint64_t*>(ints_all + kWG * kIntsPerWG);  // per group
  uint64_t* wbar = bars + kWG;  // completion of the weight-image bulk copy
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(wbar + 1);
  int* abort_all = reinterpret_cast<int*>(tmem_slot + 1);  // per group

  const int tid = threadIdx.x;
  const int wg = tid / kWGThreads, ltid = tid - wg * kWGThreads;
  const int lane = ltid & 31, lwid = ltid >> 5;  // lwid = warp % 4: the TMEM lane quarter
  const int N = kL * kL, M2 = 2 * N;

  // Weights resident for the whole launch: one bulk TMA copy of the packed image (16-byte
  // aligned, a multiple of 16 bytes; this CTA's own shared memory, no multicast), completing on
  // wbar; the biases by plain loads.
  if (tid == 0) {
    for (int w = 0; w <= kWG; ++w) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + w)) : "memory");
      if (w < kWG) abort_all[w] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(smem_u32(wbar)),
        "r"((uint32_t)kWBytes)
        : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(wsm)),
        "l"(a.wpk), "r"((uint32_t)kWBytes), "r"(smem_u32(wbar))
        : "memory");
  }
  for (int i = tid; i < 4 * kC; i += kTcThreads) bsm[i] = __ldg(a.bias + i);
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!mbar_wait(wbar, 0)) {  // the weight copy did not complete: no item is computed
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int w = 0; w < kWG; ++w) abort_all[w] = 1;
    }
  }
  __syncthreads();

  // This warp group's state.
  const uint32_t tmem = *tmem_slot + 64u * kParts * wg;
  unsigned char* act = act_all + wg * kActBytes;
  int* simg = ints_all + wg * kIntsPerWG;  // (2N) image configuration
  int* rowof = simg + M2;                  // (2N) mode -> row of Y, or -1
  int* occl = rowof + M2;                  // (2N) ascending occupied modes
  int* wbuf = occl + M2;                   // (4 L + 32) scan scratch
  uint64_t* bar = bars + wg;
  int* abort_flag = abort_all + wg;
  const uint32_t act_hi = smem_u32(act), act_lo = act_hi + 4 * kPlane;
  const uint32_t w0 = smem_u32(wsm);
  const bool split = a.mode == 2;
  uint32_t phase = 0;

  const int G = a.cl.G;
  const int n_items = (a.cl.n_cfg_dev ? *a.cl.n_cfg_dev : a.cl.n_cfg) * G;
  for (int item = blockIdx.x * kWG + wg; item < n_items; item += gridDim.x * kWG) {
    if (*abort_flag) {  // a wait expired earlier: mark the item instead of computing it
      if (ltid == 0) a.item_sign[item] = NAN;
      continue;
    }
    const int c = item / G, g = item - c * G;
    const int smp = a.cl.sample ? a.cl.sample[c] : c;
    const int fr = a.cl.from ? a.cl.from[c] : -1;
    const int to = a.cl.from ? a.cl.to[c] : -1;
    const int8_t* base = a.cl.spins + (int64_t)smp * M2;
    wg_sync(wg);
    for (int m = ltid; m < M2; m += kWGThreads) {
      const int src = sym_map(m, g, kL, kL, N);
      int v = base[src];
      v = move_value(src, v, fr, to);
      simg[m] = v > 0 ? 1 : -1;
    }
    wg_sync(wg);
    // Layer-0 input planes: channel 0 = up, 1 = down (+-1, exact in BF16), the rest zero.
    for (int s = ltid; s < N; s += kWGThreads) {
      uint4 grp[2];
      const uint32_t up = bf16_bits((float)simg[s]), dn = bf16_bits((float)simg[N + s]);
      grp[0] = make_uint4(up | (dn << 16), 0u, 0u, 0u);
      grp[1] = make_uint4(0u, 0u, 0u, 0u);
      put_site(act, 2, s / kL, s % kL, grp);
    }
    // Occupied modes of the image configuration (ascending) and their rows in Y.
    {
      const int per = (M2 + kWGThreads - 1) / kWGThreads;
      const int m0 = ltid * per;
      int cnt = 0;
      for (int m = m0; m < m0 + per && m < M2; ++m) cnt += simg[m] > 0;
      int x = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wbuf[lwid] = x;
      wg_sync(wg);
      int before = 0, total = 0;
      for (int w = 0; w < kWGThreads / 32; ++w) {
        before += w < lwid ? wbuf[w] : 0;
        total += wbuf[w];
      }
      int pos = before + x - cnt;
      for (int m = m0; m < m0 + per && m < M2; ++m) {
        if (simg[m] > 0) {
          occl[pos] = m;
          rowof[m] = pos < a.n ? pos : -1;
          ++pos;
        } else {
          rowof[m] = -1;
        }
      }
      wg_sync(wg);
      if (ltid == 0) wbuf[0] = total;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    wg_sync(wg);
    const int total = wbuf[0];

    for (int layer = 0; layer < 4; ++layer) {
      if (ltid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (layer == 0)
          issue_layer(tmem, act_hi, act_lo, w0, w0 + kW0Bytes / 2, 2, 2 * 4 * 128, false, split);
        else {
          const uint32_t wl = w0 + kW0Bytes + (layer - 1) * kW1Bytes;
          issue_layer(tmem, act_hi, act_lo, wl, wl + kW1Bytes / 2, 4, 4 * 4 * 128, split, split);
        }
        mma_commit(bar);
      }
      if (!mbar_wait(bar, phase)) {
        if (ltid == 0) atomicExch(a.err, 1);
        *abort_flag = 1;
      }
      phase ^= 1u;
      wg_sync(wg);
      if (*abort_flag) {
        if (ltid == 0) a.item_sign[item] = NAN;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // Epilogue: warp lwid reads TMEM lanes 32 lwid .. + 31 of both tiles (rows = sites).
      const int mrow = 32 * lwid + lane;  // row of the 128 x 32 tile
      const int x = mrow >> 3;
      const float* bl = bsm + layer * kC;
      if (layer < 3) {
        uint4 hi[2][4], lo[2][4];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float v[32];
          load_tile(tmem + ((uint32_t)(32 * lwid) << 16), h, layer == 0 ? 2 : 4, split, v);
          act_groups(v, bl, hi[h], lo[h]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        wg_sync(wg);  // every tile is read before any plane is overwritten
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int y = 8 * h + (mrow & 7);
          put_site(act, 4, x, y, hi[h]);
          if (split) put_site(act + 4 * kPlane, 4, x, y, lo[h]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        wg_sync(wg);
      } else {
        // Last layer: features y_up = channels 0..15, y_down = 16..31 of occupied modes.
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float v[32];
          load_tile(tmem + ((uint32_t)(32 * lwid) << 16), h, 4, split, v);
          const int s = x * kL + 8 * h + (mrow & 7);
#pragma unroll
          for (int sg = 0; sg < 2; ++sg) {
            const int row = rowof[sg * N + s];
            if (row < 0) continue;
            float4* dst = reinterpret_cast<float4*>(a.Y + ((int64_t)item * a.n + row) * 16);
#pragma unroll
            for (int q = 0; q < 4; ++q)
              dst[q] = make_float4(v[16 * sg + 4 * q] + bl[16 * sg + 4 * q],
                                   v[16 * sg + 4 * q + 1] + bl[16 * sg + 4 * q + 1],
                                   v[16 * sg + 4 * q + 2] + bl[16 * sg + 4 * q + 2],
                                   v[16 * sg + 4 * q + 3] + bl[16 * sg + 4 * q + 3]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
    }
    if (*abort_flag) continue;
    // Occupied-mode list and item sign (eta_g times the descending-order convention).
    for (int p = ltid; p < a.n; p += kWGThreads)
      a.idx[(int64_t)item * a.n + p] = occl[p < total ? p : 0];
    const int odd = image_sign_parity_group(simg, g, kL, kL, wbuf, ltid, kWGThreads / 32,
                                            WgSync{wg});
    if (ltid == 0) {
      const long long kk = total;
      const int rev = (int)((kk * (kk - 1) / 2) & 1);
      float sgn = ((odd & 1) ^ rev) ? -1.0f : 1.0f;
      if (total != a.n) sgn = 0.0f;
      a.item_sign[item] = sgn;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (tid < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                 "r"(kTmemCols)
                 : "memory");
}

// Packed weights: per layer, q (hi, lo) x tap x kc x cg x [8 co rows x 8 ci] BF16, the K-major
// canonical layout of the B operand (N = co, K = ci); layer 0 pads ci from 2 to 16.
__global__ void pack_tc_kernel(const float* __restrict__ w, uint16_t* out) {
  const int total = kWBytes / 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    int l, r, kcs, cin, off;
    if (i < kW0Bytes / 2) {
      l = 0;
      r = i;
      kcs = 2;
      cin = 2;
      off = 0;
    } else {
      l = 1 + (i - kW0Bytes / 2) / (kW1Bytes / 2);
      r = (i - kW0Bytes / 2) % (kW1Bytes / 2);
      kcs = 4;
      cin = kC;
      off = 18 * kC + (l - 1) * 9 * kC * kC;
    }
    const int per_q = 9 * kcs * 4 * 64;
    const int q = r / per_q;
    int t = r % per_q;
    const int tap = t / (kcs * 4 * 64);
    t %= kcs * 4 * 64;
    const int kc = t / (4 * 64);
    t %= 4 * 64;
    const int cg = t / 64;
    t %= 64;
    const int row = t / 8, col = t % 8;
    const int co = cg * 8 + row, ci = kc * 8 + col;
    float val = 0.0f;
    if (ci < cin) val = w[off + (co * cin + ci) * 9 + tap];
    const float hi = __bfloat162float(__float2bfloat16_rn(val));
    out[i] = q == 0 ? bf16_bits(hi) : bf16_bits(val - hi);
  }
}

constexpr size_t kTcSmem = (size_t)kWBytes + kWG * kActBytes + 4 * kC * sizeof(float) +
                           sizeof(int) * kWG * kIntsPerWG + 64;
static_assert(kTcSmem <= 227 * 1024, "two warp groups must fit in shared memory");

}  // namespace

size_t cnn_tc_packed_bytes() { return kWBytes; }

bool cnn_tc_supported(const nh_backflow_params& p) {
  return p.Lx == kL && p.Ly == kL && p.channels == kC && p.layers == 4;
}

int launch_pack_cnn_tc(const float* conv_w, uint16_t* packed, cudaStream_t st) {
  ProfScope prof_scope(NH_K_PACK, st);
  pack_tc_kernel<<<(kWBytes / 2 + 255) / 256, 256, 0, st>>>(conv_w, packed);
  return check_launch("pack_tc_kernel");
}

int launch_cnn_tc(const ConfigList& cl, const nh_backflow_params& p, int mode, float* Y,
                  int32_t* idx, float* item_sign, int32_t* err, cudaStream_t st) {
  if (!cnn_tc_supported(p))
    return fail(NH_ERR_UNSUPPORTED, "tensor-core CNN: %dx%d lattice, %d channels, %d layers "
                "(supported: 16x16, 32, 4)", p.Lx, p.Ly, p.channels, p.layers);
  if (!p.conv_w_tc) return fail(NH_ERR_INVALID, "tensor-core CNN: conv_w_tc is null");
  if (reinterpret_cast<uintptr_t>(p.conv_w_tc) % 16)
    return fail(NH_ERR_INVALID, "tensor-core CNN: conv_w_tc must be 16-byte aligned");
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(cnn_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmem);
    if (e != cudaSuccess) return check_cuda(e, "tensor-core CNN smem attribute");
    configured = true;
  }
  const int items = cl.n_cfg * cl.G;
  if (items <= 0) return NH_OK;
  int grid = num_sms();
  if (grid > (items + kWG - 1) / kWG) grid = (items + kWG - 1) / kWG;
  TcArgs a{cl, static_cast<const uint16_t*>(p.conv_w_tc), p.conv_b, p.n_up + p.n_dn, mode, Y,
           idx, item_sign, err};
  ProfScope prof_scope(NH_K_CNN_TC, st);
  cnn_tc_kernel<<<grid, kTcThreads, kTcSmem, st>>>(a);
  return check_launch("cnn_tc_kernel");
}

}  // namespace nh

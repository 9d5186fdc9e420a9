// Residual backflow network (net = NH_NET_RESCONV) on the 5th-generation tensor cores: the
// 16 x 16, 64-channel network of the released states with BF16 x3 products (cnn_mode 2).
//
// Each 3x3 periodic convolution is an implicit GEMM D[site, co] += A[site + tap, ci] W[tap][ci, co]
// on tcgen05: M = 128 (two tiles, y-blocks 0-7 and 8-15, of 16 x-rows), N = 64 output channels,
// K = 16 input channels per MMA, FP32 accumulators in tensor memory: four partial sums per tile
// (one per group of 16 input channels, 512 columns), added in the epilogue, which keeps the
// tensor cores' FP32 accumulation chains short (one chain of 216 MMAs left a nearly constant
// offset of ~8e-4 in log|psi|; four chains, under 2e-4).  Operands are split into BF16 hi + lo
// and accumulated as hi*hi + hi*lo + lo*hi (about 16 significant bits per product).  One configuration image per CTA at a time (grid-stride), 256 threads: warp w
// owns tensor-memory lanes 32 (w % 4) .. + 31 of tile w / 4, i.e. one site per thread.
//
// Shared memory (214 KB):
//   planes  the A operand: 8 + 8 BF16 hi / lo padded planes (nh_tcgen05.cuh layout), holding
//           h = GELU(RMSNorm(x)) for the first convolution of a block and then, once those MMAs
//           have completed, u = GELU(Conv1(h) + b1) for the second;
//   x       the residual stream, FP32 [channel][tile row] (exact accumulation across blocks);
//   ring    4 slots of one tap's weights (hi + lo, 16 KB, [q][kc][cg][8 co][8 ci] BF16), filled
//           by bulk copies (no multicast) that complete on full[slot]; the MMAs that read a slot
//           commit to empty[slot], and the copy of the slice four taps ahead waits for it.
// Thread 0 issues the MMAs (all 216 of a convolution unrolled, operand descriptors formed once
// and advanced by constants); thread 32 issues the copies, so that neither waits on the other's
// instructions.  The weight stream runs ahead across convolutions: the next convolution's first
// four slices load while the epilogue of the current one runs.
// Epilogues read the accumulators with tcgen05.ld and (a) write u's planes, or (b) add the
// convolution into x, reduce sum x^2 over the CTA, and write the next h's planes.
//
// Every mbarrier wait is bounded: on expiry the kernel records an error in *err, marks the item
// NaN, waits (bounded) for its copies in flight, releases its tensor memory and returns.
#include <math.h>
#include <stdint.h>

#include "nh_common.cuh"
#include "nh_tcgen05.cuh"

namespace nh {
namespace {

using namespace tc;

constexpr int kRtThreads = 256;
constexpr int kRtC = 64;
constexpr int kRtN = kL * kL;                          // 256 sites
constexpr int kRtPlanes = kRtC / 8;                    // planes per hi / lo
constexpr int kRtActBytes = 2 * kRtPlanes * kPlane;    // 82,944
constexpr int kRtXBytes = kRtC * kRtN * 4;             // 65,536
constexpr int kRtHalfTap = kRtPlanes * 8 * 128;        // 8,192: one of hi / lo for one tap
constexpr int kRtTapBytes = 2 * kRtHalfTap;            // 16,384
constexpr int kRtConvBytes = 9 * kRtTapBytes;          // 147,456
constexpr int kRtSlots = 4;
constexpr int kRtInts = 2 * kRtN + 2 * kRtN + 4 * kL + 32;  // simg, occl, scan scratch
constexpr uint32_t kRtIdesc = idesc_bf16(128, 64);
constexpr int kRtParts = 4;           // partial accumulators per tile (one per 16-ci group)
constexpr unsigned kRtTmemCols = 128 * kRtParts;
constexpr float kRtRmsEps = 1e-6f;

constexpr size_t kOffX = kRtActBytes;
constexpr size_t kOffRing = kOffX + kRtXBytes;
constexpr size_t kOffInts = kOffRing + (size_t)kRtSlots * kRtTapBytes;
constexpr size_t kOffRed = kOffInts + sizeof(int) * kRtInts;
constexpr size_t kOffBars = (kOffRed + 8 * sizeof(float) + 7) & ~(size_t)7;
constexpr size_t kRtSmem = kOffBars + (2 * kRtSlots + 1) * 8 + 16;  // + tmem slot, flag, count
static_assert((kOffBars + (2 * kRtSlots + 1) * 8 + 8) % 8 == 0, "8-byte slot for the count");
static_assert(kOffX % 128 == 0 && kOffRing % 128 == 0, "operand regions 128-byte aligned");
static_assert(kRtSmem <= 227 * 1024, "resident set must fit in shared memory");

struct RtArgs {
  ConfigList cl;
  const unsigned char* wtc;  // packed BF16 hi / lo weights, 2 blocks x kRtConvBytes
  const float* embed;        // (4, 64): [occupation][co]
  const float* bias;         // (2 blocks, 64)
  int blocks, n;
  float* Y;                  // (items, n, 32)
  int32_t* idx;              // (items, n)
  float* item_sign;          // (items,)
  int32_t* err;
};

__device__ __forceinline__ float gelu_fast(float x) {
  const float z2 = 1.5957691216057308f * (x + 0.044715f * x * x * x);
  return __fdividef(x, 1.0f + __expf(-z2));
}

// Thread 0: the MMAs of one tap for both tiles.  dAhi / dAlo / dB are the descriptors of the hi
// planes, the lo planes and the tap's ring slot; with the tap known at compile time (the caller
// unrolls) every operand is that descriptor plus a constant (its address field counts 16-byte
// units; shared-memory offsets stay far below the field's 256 KB range).  Input-channel group kk
// accumulates into its own partial sum (columns 128 kk + 64 h), so each FP32 accumulation chain
// is a quarter as long; the epilogue adds the four.
__device__ __forceinline__ void issue_tap(uint32_t tmem, uint64_t dAhi, uint64_t dAlo,
                                          uint64_t dB, int tap) {
  const int dx = tap / 3 - 1, dy = tap % 3 - 1;
#pragma unroll
  for (int q = 0; q < 3; ++q) {  // hi*hi, hi*lo, lo*hi
#pragma unroll
    for (int kk = 0; kk < kRtParts; ++kk) {
      const uint64_t b = dB + (uint64_t)(((q == 1 ? kRtHalfTap : 0) + 2 * kk * kRtPlanes * 128) >> 4);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t ao = (uint32_t)pad_off(dx + 1, 8 * h + dy + 1) + 2 * kk * kPlane;
        const uint64_t a = (q == 2 ? dAlo : dAhi) + (uint64_t)(ao >> 4);
        mma_bf16(tmem + 128 * kk + 64 * h, a, b, kRtIdesc, tap > 0 || q > 0);
      }
    }
  }
}

// Write the 64 channels f of this thread's site (lattice x, y) as BF16 hi / lo planes.
__device__ __forceinline__ void put_channels(unsigned char* planes, int x, int y, const float* f) {
  uint4 hi[kRtPlanes], lo[kRtPlanes];
#pragma unroll
  for (int kc = 0; kc < kRtPlanes; ++kc) split8(f + 8 * kc, hi + kc, lo + kc);
  put_site(planes, kRtPlanes, x, y, hi);
  put_site(planes + kRtPlanes * kPlane, kRtPlanes, x, y, lo);
}

__global__ void __launch_bounds__(kRtThreads, 1) resconv_tc_kernel(RtArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* planes = smem;
  float* xs = reinterpret_cast<float*>(smem + kOffX);  // [c][r], r = 128 tile + row
  unsigned char* ring = smem + kOffRing;
  int* simg = reinterpret_cast<int*>(smem + kOffInts);
  int* occl = simg + 2 * kRtN;
  int* wbuf = occl + 2 * kRtN;
  float* red = reinterpret_cast<float*>(smem + kOffRed);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOffBars);
  uint64_t* empty = full + kRtSlots;
  uint64_t* accb = empty + kRtSlots;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accb + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  long long* consumed_total = reinterpret_cast<long long*>(abort_flag + 1);  // at kOffBars + 80

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int quarter = warp & 3, tile = warp >> 2;
  const int row = 32 * quarter + lane;             // row of this thread's tile
  const int r = 128 * tile + row;                  // column of x
  const int sx = row >> 3, sy = 8 * tile + (row & 7);
  const int site = sx * kL + sy;
  const int G = a.cl.G;
  const int n_items = (a.cl.n_cfg_dev ? *a.cl.n_cfg_dev : a.cl.n_cfg) * G;
  const int my_items =
      (int)blockIdx.x < n_items ? (n_items - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x
                                : 0;
  const int convs = 2 * a.blocks;
  const long long slices = (long long)my_items * convs * 9;  // weight slices this CTA uses
  constexpr int kProducer = 32;                              // thread issuing the copies
  long long loaded = 0;    // slices requested (producer thread)
  long long consumed = 0;  // slices whose MMAs are issued (thread 0)

  auto load_slice = [&](long long sidx) {  // one thread
    const int slot = (int)(sidx % kRtSlots);
    const int conv = (int)((sidx / 9) % convs), tap = (int)(sidx % 9);
    bulk_load(ring + slot * kRtTapBytes,
              a.wtc + (size_t)conv * kRtConvBytes + (size_t)tap * kRtTapBytes, kRtTapBytes,
              full + slot);
  };

  if (tid == 0) {
    for (int s = 0; s < kRtSlots; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(accb, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (long long sl = 0; sl < kRtSlots && sl < slices; ++sl) load_slice(sl);
  }
  loaded = slices < kRtSlots ? slices : kRtSlots;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kRtTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t t_lane = tmem + ((uint32_t)(32 * quarter) << 16) + 64u * tile;
  const uint32_t act_hi = smem_u32(planes), act_lo = act_hi + kRtPlanes * kPlane;
  const uint32_t ring0 = smem_u32(ring);
  const uint64_t dAhi = make_desc(act_hi, kPlane, kP * 16);
  const uint64_t dAlo = make_desc(act_lo, kPlane, kP * 16);
  const uint64_t dB0 = make_desc(ring0, kRtPlanes * 128, 128);
  const float out_scale = 1.0f / sqrtf((float)(a.blocks + 1));
  const float inv_cn = 1.0f / (float)(kRtC * kRtN);
  uint32_t acc_phase = 0;
  long long conv_seq = 0;  // convolutions processed by this CTA (all threads)

  // Writes h = GELU(RMSNorm(x)) of this thread's site into the planes (all threads call).
  auto norm_to_planes = [&]() {
    float ss = 0.0f;
#pragma unroll 8
    for (int c = 0; c < kRtC; ++c) ss = fmaf(xs[c * kRtN + r], xs[c * kRtN + r], ss);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if (lane == 0) red[warp] = ss;
    __syncthreads();
    float tot = 0.0f;
#pragma unroll
    for (int w = 0; w < kRtThreads / 32; ++w) tot += red[w];
    const float rn = 1.0f / sqrtf(tot * inv_cn + kRtRmsEps);
    float f[kRtC];
#pragma unroll
    for (int c = 0; c < kRtC; ++c) f[c] = gelu_fast(xs[c * kRtN + r] * rn);
    put_channels(planes, sx, sy, f);
  };

  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int c = item / G, g = item - c * G;
    const int smp = a.cl.sample ? a.cl.sample[c] : c;
    const int fr = a.cl.from ? a.cl.from[c] : -1;
    const int to = a.cl.from ? a.cl.to[c] : -1;
    const int8_t* base = a.cl.spins + (int64_t)smp * 2 * kRtN;
    __syncthreads();  // the previous item's readers of simg / x / red are done
    if (*abort_flag) {
      if (tid == 0) a.item_sign[item] = NAN;
      continue;
    }
    for (int m = tid; m < 2 * kRtN; m += kRtThreads) {
      const int src = sym_map(m, g, kL, kL, kRtN);
      int v = base[src];
      v = move_value(src, v, fr, to);
      simg[m] = v > 0 ? 1 : -1;
    }
    __syncthreads();
    {
      const int occ = (simg[site] > 0 ? 1 : 0) + (simg[kRtN + site] > 0 ? 2 : 0);
#pragma unroll 8
      for (int ch = 0; ch < kRtC; ++ch) xs[ch * kRtN + r] = __ldg(a.embed + occ * kRtC + ch);
    }
    norm_to_planes();

    bool failed = false;
    for (int conv = 0; conv < convs; ++conv) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();  // planes written, accumulators read
      if (tid == 0) {  // MMA issue: wait for each tap's weights, then its 72 MMAs
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) {
          const int slot = (int)(consumed % kRtSlots);
          if (!*abort_flag && !mbar_wait(full + slot, (uint32_t)((consumed / kRtSlots) & 1))) {
            atomicExch(a.err, 2);
            *abort_flag = 1;
          }
          if (*abort_flag) break;
          issue_tap(tmem, dAhi, dAlo, dB0 + (uint64_t)((slot * kRtTapBytes) >> 4), tap);
          mma_commit(empty + slot);
          ++consumed;
        }
        mma_commit(accb);  // arrives once every MMA issued so far has completed
      } else if (tid == kProducer) {
        // Copies: every slice up to the fourth of the next convolution, each into the slot of
        // the slice four back once that slice's MMAs (all of this convolution) have completed.
        const long long upto = (long long)9 * (conv_seq + 1) + kRtSlots;
        while (!*abort_flag && loaded < slices && loaded < upto) {
          const long long prev = loaded - kRtSlots;
          if (!mbar_wait(empty + (prev % kRtSlots), (uint32_t)((prev / kRtSlots) & 1))) {
            atomicExch(a.err, 3);
            *abort_flag = 1;
            break;
          }
          load_slice(loaded);
          ++loaded;
        }
      }
      ++conv_seq;
      if (!mbar_wait(accb, acc_phase)) {
        if (tid == 0) atomicExch(a.err, 4);
        *abort_flag = 1;
      }
      acc_phase ^= 1u;
      __syncthreads();
      if (*abort_flag) {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float v[kRtC];
      tmem_ld32(t_lane, v);
      tmem_ld32(t_lane + 32, v + 32);
#pragma unroll
      for (int pc = 1; pc < kRtParts; ++pc) {
        float w[32];
        tmem_ld32(t_lane + 128 * pc, w);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] += w[i];
        tmem_ld32(t_lane + 128 * pc + 32, w);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[32 + i] += w[i];
      }
      const float* b = a.bias + conv * kRtC;
      if ((conv & 1) == 0) {  // u = GELU(Conv1(h) + b1) into the planes (h is no longer read)
#pragma unroll
        for (int ch = 0; ch < kRtC; ++ch) v[ch] = gelu_fast(v[ch] + __ldg(b + ch));
        put_channels(planes, sx, sy, v);
      } else {  // x += Conv2(u) + b2, then the next block's h
#pragma unroll
        for (int ch = 0; ch < kRtC; ++ch) xs[ch * kRtN + r] += v[ch] + __ldg(b + ch);
        if (conv + 1 < convs) norm_to_planes();
      }
    }
    if (failed) {
      if (tid == 0) a.item_sign[item] = NAN;
      continue;
    }
    __syncthreads();
    constexpr int d = kRtC / 2;
    write_occupied_rows(simg, occl, wbuf, kRtN, a.n, d, g, kL, kL, a.Y + (int64_t)item * a.n * d,
                        a.idx + (int64_t)item * a.n, a.item_sign + item,
                        [&](int sg, int aa, int st) {
                          const int xx = st / kL, yy = st - xx * kL;
                          const int rr = 128 * (yy >> 3) + 8 * xx + (yy & 7);
                          return xs[(sg * d + aa) * kRtN + rr] * out_scale;
                        });
  }
  // Copies still in flight (only after an abort): wait for them, bounded, before exiting.
  if (tid == 0) *consumed_total = consumed;
  __syncthreads();
  if (tid == kProducer) {
    for (long long s = *consumed_total; s < loaded; ++s)
      mbar_wait(full + (s % kRtSlots), (uint32_t)((s / kRtSlots) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kRtTmemCols)
                 : "memory");
}

// Packed image: per convolution k and tap, [q (hi, lo)][kc][cg][co % 8][ci % 8] BF16 (the
// K-major canonical layout of the B operand, N = co, K = ci).  conv_w = [embed (64, 4)] ++
// per convolution (64, 64, 3, 3) FP32.
__global__ void pack_resconv_tc_kernel(const float* __restrict__ conv_w, int convs,
                                       uint16_t* out) {
  const long long total = (long long)convs * kRtConvBytes / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / (kRtConvBytes / 2));
    int t = (int)(i % (kRtConvBytes / 2));
    const int tap = t / (kRtTapBytes / 2);
    t %= kRtTapBytes / 2;
    const int q = t / (kRtHalfTap / 2);
    t %= kRtHalfTap / 2;
    const int kc = t / (kRtPlanes * 64);
    t %= kRtPlanes * 64;
    const int cg = t / 64;
    t %= 64;
    const int co = cg * 8 + t / 8, ci = kc * 8 + t % 8;
    const float val = conv_w[4 * kRtC + (size_t)k * 9 * kRtC * kRtC + (co * kRtC + ci) * 9 + tap];
    const float hi = __bfloat162float(__float2bfloat16_rn(val));
    out[i] = q == 0 ? bf16_bits(hi) : bf16_bits(val - hi);
  }
}

}  // namespace

size_t resconv_tc_packed_bytes(int blocks) { return (size_t)2 * blocks * kRtConvBytes; }

bool resconv_tc_supported(const nh_backflow_params& p) {
  return p.Lx == kL && p.Ly == kL && p.channels == kRtC;
}

int launch_pack_resconv_tc(const float* conv_w, int blocks, void* packed, cudaStream_t st) {
  const long long total = (long long)2 * blocks * kRtConvBytes / 2;
  ProfScope prof_scope(NH_K_PACK, st);
  pack_resconv_tc_kernel<<<(int)((total + 255) / 256), 256, 0, st>>>(
      conv_w, 2 * blocks, static_cast<uint16_t*>(packed));
  return check_launch("pack_resconv_tc_kernel");
}

int launch_resconv_tc(const ConfigList& cl, const nh_backflow_params& p, float* Y, int32_t* idx,
                      float* item_sign, int32_t* err, cudaStream_t st) {
  if (!resconv_tc_supported(p))
    return fail(NH_ERR_UNSUPPORTED, "tensor-core residual network: %dx%d lattice, %d channels "
                "(supported: 16x16, 64)", p.Lx, p.Ly, p.channels);
  if (!p.conv_w_tc || reinterpret_cast<uintptr_t>(p.conv_w_tc) % 16)
    return fail(NH_ERR_INVALID, "tensor-core residual network: conv_w_tc null or not 16-byte "
                "aligned");
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(resconv_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kRtSmem);
    if (e != cudaSuccess) return check_cuda(e, "tensor-core residual network smem attribute");
    configured = true;
  }
  const int items = cl.n_cfg * cl.G;
  if (items <= 0) return NH_OK;
  int grid = num_sms();
  if (grid > items) grid = items;
  RtArgs a{cl, static_cast<const unsigned char*>(p.conv_w_tc), p.conv_w_packed, p.conv_b,
           p.layers, p.n_up + p.n_dn, Y, idx, item_sign, err};
  ProfScope prof_scope(NH_K_RESCONV_TC, st);
  resconv_tc_kernel<<<grid, kRtThreads, kRtSmem, st>>>(a);
  return check_launch("resconv_tc_kernel");
}

}  // namespace nh

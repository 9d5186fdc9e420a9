// tcgen05 (5th-generation tensor core, sm_100a) building blocks shared by the tensor-core
// backflow networks: shared-memory matrix descriptors, BF16 MMAs with FP32 accumulators in
// tensor memory, commits and bounded mbarrier waits, tensor-memory loads, bulk copies into
// shared memory, and the padded activation planes of a 16 x 16 lattice.
//
// Padded planes: site (x, y) sits at padded position (x + 1, y + 1) of an 18 x 18 grid whose
// border repeats the periodic neighbours; each padded site holds 8 channels in 16 bytes (one
// core-matrix row), one plane per group of 8 channels.  An M = 128 tile is one 8-site y-block
// across the 16 x-rows: its rows are eight consecutive sites (one 128-byte core matrix) per
// x-row, x-rows one padded row apart, so a 3x3 tap (dx, dy) is the same descriptor with the
// start address moved by (dx * 18 + dy) * 16 bytes.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace nh {
namespace tc {

constexpr int kL = 16;                  // lattice extent of the tensor-core kernels
constexpr int kP = kL + 2;              // padded extent
constexpr int kPlane = kP * kP * 16;    // bytes of one 8-channel plane
constexpr long long kWaitLimit = 1ll << 22;  // mbarrier polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no-swizzle shared-memory matrix descriptor (tcgen05 layout, version 1).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

// Instruction descriptor of kind::f16: BF16 x BF16 -> FP32, both operands K-major, M x N.
constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t idesc, bool acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"((uint32_t)acc));
}

// Arrive on bar once every previously issued MMA of this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Wait for the phase with the given parity to complete; false after kWaitLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One thread: bulk copy of bytes (16-byte aligned, a multiple of 16) from global memory into
// this CTA's shared memory (no multicast), completing on bar with expect_tx.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 tensor-memory lanes (lane = thread).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf16_val(uint16_t b) {
  return __bfloat162float(__ushort_as_bfloat16(b));
}

// Byte offset of padded position (X, Y) inside a plane.
__device__ __forceinline__ int pad_off(int X, int Y) { return (X * kP + Y) * 16; }

// Write the 8-channel groups of lattice site (x, y), and its periodic halo copies, into
// nplanes consecutive planes.
__device__ __forceinline__ void put_site(unsigned char* planes, int nplanes, int x, int y,
                                         const uint4* grp) {
  const int xs[2] = {x + 1, x == 0 ? kL + 1 : (x == kL - 1 ? 0 : -1)};
  const int ys[2] = {y + 1, y == 0 ? kL + 1 : (y == kL - 1 ? 0 : -1)};
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      if (xs[a] < 0 || ys[b] < 0) continue;
      const int off = pad_off(xs[a], ys[b]);
      for (int kc = 0; kc < nplanes; ++kc)
        *reinterpret_cast<uint4*>(planes + kc * kPlane + off) = grp[kc];
    }
  }
}

// 8 FP32 values -> their BF16 hi parts and the BF16 of the remainders (lo), packed as 16 bytes.
__device__ __forceinline__ void split8(const float* f, uint4* hi, uint4* lo) {
  uint32_t ph[4], pl[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint16_t h0 = bf16_bits(f[2 * j]), h1 = bf16_bits(f[2 * j + 1]);
    ph[j] = (uint32_t)h0 | ((uint32_t)h1 << 16);
    pl[j] = (uint32_t)bf16_bits(f[2 * j] - bf16_val(h0)) |
            ((uint32_t)bf16_bits(f[2 * j + 1] - bf16_val(h1)) << 16);
  }
  *hi = make_uint4(ph[0], ph[1], ph[2], ph[3]);
  *lo = make_uint4(pl[0], pl[1], pl[2], pl[3]);
}

}  // namespace tc
}  // namespace nh

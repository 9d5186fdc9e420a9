// Internal declarations shared by the CUDA sources of libnh_b200.so (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nh_b200.h"

namespace nh {

constexpr int kNumThreads = 256;  // block size of every per-item kernel
constexpr int kMaxN = 1024;       // sites per lattice supported by the bookkeeping kernels

// Internal per-item flag (never returned to callers; cleared by the refinement and masked by the
// image combination): the FP32 pivot ratio exceeds refine_tau, so the item's log-Pfaffian is
// refined in FP64 with its FP32 pivot order.
constexpr int kFlagNeedRefine = 1 << 20;
constexpr int kPublicFlags = 0xFFFF;
// FP64 refinement with the FP32 pivot order (nh_refine.cu): its FP64 triangle lives in shared
// memory, so n <= kRefineMaxN; beyond, flagged items are recomputed by the pivoted FP64 kernel.
constexpr int kRefineMaxN = 224;
constexpr size_t kRefineSmemLimit = 225 * 1024;
// Backward of the amplitude (nh_grad.cu): the Gauss-Jordan inverse keeps the matrix in registers
// and its transpose in shared memory, so n <= kGradMaxN.
constexpr int kGradMaxN = 224;
// BCS determinant (nh_det.cu): the up x down block lives in registers (FP32 up to 224 rows, FP64
// up to 128).
constexpr int kDetMaxNh = 224;
constexpr int kDetMaxNh64 = 128;

// ------------------------------------------------------------------ host-side error state
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);
int check_launch(const char* what);
// Caller workspaces: NH_ERR_WORKSPACE when null or smaller than need, NH_ERR_INVALID when not
// 256-byte aligned (every carve offset is a multiple of 256 and the kernels use 16-byte vectors).
int check_workspace(const void* ws, size_t have, size_t need, const char* who);

// ------------------------------------------------------------------ lattice helpers
// Mode m = sigma * N + x * Ly + y.  Symmetry element g = fx + 2 fy + 4 si:
// Flip(axis=0) x -> -x mod Lx, Flip(axis=1) y -> -y mod Ly, SpinInverse swaps sigma.
__host__ __device__ __forceinline__ int sym_map(int m, int g, int Lx, int Ly, int N) {
  int sigma = m >= N ? 1 : 0;
  int site = m - sigma * N;
  int x = site / Ly;
  int y = site - x * Ly;
  if (g & 1) x = x ? Lx - x : 0;
  if (g & 2) y = y ? Ly - y : 0;
  if (g & 4) sigma ^= 1;
  return sigma * N + x * Ly + y;
}

// Hop directions: (1,0), (-1,0), (0,1), (0,-1), (1,1), (1,-1), (-1,1), (-1,-1).
__host__ __device__ __forceinline__ int hop_target_site(int site, int dir, int Lx, int Ly) {
  const int dxs[8] = {1, -1, 0, 0, 1, 1, -1, -1};
  const int dys[8] = {0, 0, 1, -1, 1, -1, 1, -1};
  int x = site / Ly;
  int y = site - x * Ly;
  x += dxs[dir];
  y += dys[dir];
  x = x < 0 ? x + Lx : (x >= Lx ? x - Lx : x);
  y = y < 0 ? y + Ly : (y >= Ly ? y - Ly : y);
  return x * Ly + y;
}

// Parity (0 or 1) of eta_g, the fermionic reordering sign of symmetry element g on the image
// configuration simg (+1 occupied / -1 empty per mode, ascending modes sigma N + x Ly + y).
// For the reflections x -> -x, y -> -y and the spin swap the inversion count has a closed form:
// x-flip inverts every pair of occupied sites in distinct rows x1, x2 >= 1, y-flip every pair in
// one row with y1, y2 >= 1, the spin swap every (up, down) pair.  Block-wide (all threads call
// it); scratch holds 4 Lx + 4 ints.  Lx <= 32 rows, Ly <= 32 sites per row.
// Generic form over a group of threads: local thread index ltid, nw warps, and the group's
// barrier (the block barrier below; a named warp-group barrier in the tensor-core CNN).
template <typename Sync>
__device__ __forceinline__ int image_sign_parity_group(const int* simg, int g, int Lx, int Ly,
                                                       int* scratch, int ltid, int nw, Sync sync) {
  const int lane = ltid & 31, wid = ltid >> 5;
  const int N = Lx * Ly;
  int* kx = scratch;           // (2, Lx) occupied sites per row
  int* kpx = scratch + 2 * Lx;  // (2, Lx) occupied sites with y >= 1 per row
  for (int r = wid; r < 2 * Lx; r += nw) {
    const int sg = r / Lx, x = r - sg * Lx;
    const bool occ = lane < Ly && simg[sg * N + x * Ly + lane] > 0;
    const unsigned b = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) {
      kx[r] = __popc(b);
      kpx[r] = __popc(b & ~1u);
    }
  }
  sync();
  int par = 0;
  if (ltid == 0 && g != 0) {
    int nsec[2] = {0, 0};
    for (int sg = 0; sg < 2; ++sg) {
      long long S = 0, Q = 0, Y = 0;
      for (int x = 0; x < Lx; ++x) {
        const long long k = kx[sg * Lx + x], kp = kpx[sg * Lx + x];
        nsec[sg] += (int)k;
        if (x >= 1) {
          S += k;
          Q += k * k;
        }
        Y += kp * (kp - 1) / 2;
      }
      if (g & 1) par ^= (int)(((S * S - Q) / 2) & 1);
      if (g & 2) par ^= (int)(Y & 1);
    }
    if (g & 4) par ^= (nsec[0] * nsec[1]) & 1;
  }
  return par;  // meaningful in thread 0 of the group
}

struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ int image_sign_parity(const int* simg, int g, int Lx, int Ly,
                                                 int* scratch) {
  return image_sign_parity_group(simg, g, Lx, Ly, scratch, (int)threadIdx.x,
                                 (int)(blockDim.x >> 5), BlockSync{});
}

// Exclusive scan of one int per thread over a TH-thread block (TH <= 1024); returns the exclusive
// prefix, *total the sum.  warp_buf: TH / 32 ints.
template <int TH = kNumThreads>
__device__ __forceinline__ int block_scan(int v, int* warp_buf, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_buf[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < (TH / 32) ? warp_buf[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (TH / 32)) warp_buf[lane] = w;
  }
  __syncthreads();
  int base = wid ? warp_buf[wid - 1] : 0;
  *total = warp_buf[TH / 32 - 1];
  __syncthreads();
  return base + x - v;
}

// Shared-memory rows of W values whose 16-byte chunks are XOR-swizzled by a row key, so that
// eight consecutive rows reading the same chunk (one quarter-warp of 16-byte loads) hit eight
// different groups of four banks: element a of row r sits at swz_index(r, a).  K = W * size / 16
// chunks per row (1, 2, 4 or 8); the key is ((r K) >> 3) & (K - 1), zero for one-chunk rows.
__host__ __device__ __forceinline__ int swz_key(int r, int K) {
  return K > 1 ? ((r * K) >> 3) & (K - 1) : 0;
}
template <typename T, int W>
__host__ __device__ __forceinline__ int swz_index(int r, int a) {
  constexpr int E = 16 / sizeof(T), K = W / E;
  return r * W + (((a / E) ^ swz_key(r, K)) * E) + (a % E);
}

// Mode-1 output of the backflow networks for one item, by a TH-thread block: the ascending
// occupied modes of the image configuration simg (+-1, 2N), the rows Y[p, a] = feat(spin, a,
// site) of those modes (p < n), their mode indices, and the item sign eta_g(s) (-1)^(k(k-1)/2)
// (0 for a wrong particle number k != n).  occl: 2N ints; wbuf: 4 Lx + 32 ints.
// swizzle: rows in the chunk-swizzled layout of swz_index (shared-memory destinations).
template <typename T, typename Feat, int TH = kNumThreads>
__device__ void write_occupied_rows(const int* simg, int* occl, int* wbuf, int N, int n, int d,
                                    int g, int Lx, int Ly, T* Ydst, int32_t* idst,
                                    float* sign_dst, Feat feat, bool swizzle = false) {
  const int tid = threadIdx.x, M2 = 2 * N;
  const int per = (M2 + TH - 1) / TH;
  const int m0 = tid * per;
  int cnt = 0;
  for (int m = m0; m < m0 + per && m < M2; ++m) cnt += simg[m] > 0;
  int total;
  int pos = block_scan<TH>(cnt, wbuf, &total);
  for (int m = m0; m < m0 + per && m < M2; ++m)
    if (simg[m] > 0) occl[pos++] = m;
  __syncthreads();
  const int E = 16 / (int)sizeof(T), K = d / E;  // swizzled rows: K 16-byte chunks of E values
  for (int o = tid; o < n * d; o += TH) {
    const int p = o / d, aa = o - p * d;
    const int m = occl[p < total ? p : 0];
    const int sg = m >= N ? 1 : 0;
    const int dst = swizzle ? p * d + ((aa / E) ^ swz_key(p, K)) * E + aa % E : o;
    Ydst[dst] = feat(sg, aa, m - sg * N);
  }
  for (int p = tid; p < n; p += TH) idst[p] = occl[p < total ? p : 0];
  // eta_g from per-row occupation counts (closed form of the inversion parity).
  const int odd = image_sign_parity(simg, g, Lx, Ly, wbuf);
  if (tid == 0) {
    const long long kk = total;
    const int rev = (int)((kk * (kk - 1) / 2) & 1);
    float s = ((odd & 1) ^ rev) ? -1.0f : 1.0f;
    if (total != n) s = 0.0f;  // wrong particle number: amplitude 0
    *sign_dst = s;
  }
}

// ------------------------------------------------------------------ moves
// A move is one or two electron hops packed into (from, to): bits [0, 16) hold the first hop's
// source and target modes, bits [16, 32) the second hop's modes plus one (0: no second hop).
// A site exchange of an up and a down electron is two hops; every other move is one.  from = -1
// (all bits set) matches no mode.
__host__ __device__ __forceinline__ int pack_move(int m1, int m2) {
  return (m1 & 0xFFFF) | (m2 >= 0 ? (m2 + 1) << 16 : 0);
}
__host__ __device__ __forceinline__ int move_first(int x) { return x & 0xFFFF; }
__host__ __device__ __forceinline__ int move_second(int x) { return ((x >> 16) & 0xFFFF) - 1; }

// Occupation of mode src after the move (from, to), v its value before.
__host__ __device__ __forceinline__ int move_value(int src, int v, int from, int to) {
  if (src == move_first(from) || src == move_second(from)) return -1;
  if (src == move_first(to) || src == move_second(to)) return 1;
  return v;
}

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
struct u32x4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// u = (x >> 8) * 2^-24, exact in FP32 and FP64.
__host__ __device__ __forceinline__ double u32_to_unit(uint32_t x) {
  return (double)(x >> 8) * (1.0 / 16777216.0);
}

// ------------------------------------------------------------------ amplitude pipeline
// A "configuration" c is spins[sample(c)] with an optional hop from(c) -> to(c) applied;
// an "item" is (configuration c, symmetry image g), item = c * G + g.
struct ConfigList {
  const int8_t* spins;       // (n_samples, 2N)
  const int32_t* sample;     // (n_cfg,) sample of each configuration, null: c itself
  const int32_t* from;       // (n_cfg,) packed move sources (pack_move) or -1, null: no move
  const int32_t* to;         // (n_cfg,) packed move targets
  const int32_t* n_cfg_dev;  // device count (overrides n_cfg when not null)
  int n_cfg;                 // host count (upper bound when n_cfg_dev is set)
  int G;                     // images per configuration: 1 or 8
};

struct PipelineBuffers {
  float* Y;           // (items, n, d)
  int32_t* idx;       // (items, n)
  float* item_sign;   // (items,)
  float* pf_sign;     // (items,)
  double* pf_logabs;  // (items,)
  int32_t* pf_flags;  // (items,)
  int32_t* list;      // (items,) items recomputed in FP64
  int32_t* count;     // (1,) their number
  double* Y64;        // (items, n, d)
  int32_t* idx64;     // (items, n)
  int32_t* err;       // (1,) device error word of the tensor-core CNN
  void* pf_tri;       // large lattices: per-CTA Pfaffian triangles (pfaffian_scratch_bytes)
  void* cnn_act;      // large lattices: per-CTA CNN activation planes (cnn_scratch_bytes)
  float* pf_ratio;    // (items,) pivot ratio of the FP32 factorisation
  uint16_t* perm;     // (items, perm_stride) FP32 pivot order of every item (n <= kRefineMaxN)
  int32_t* list32;    // (items,) items refined against their FP32 matrix
  int32_t* count32;   // (1,) their number
  void* slice;        // refinement: per-CTA permuted triangles (refine_slice_bytes)
};

// uint16 words per item of the pivot-order record: perm[0, n) then the relabelling parity.
__host__ __device__ __forceinline__ int perm_stride(int n) { return (n + 1 + 7) & ~7; }

// FP64 refinement of items listed in list[0, *count) (nh_refine.cu).
struct RefineLaunch {
  int n, d;
  int mode;  // 0: dense FP32 F (items, n, n); 1: gather FP32 Y / idx (indexed by item);
             // 2: gather FP64 Y64 / idx64 (indexed by slot) with Wt64; 3 / 4: the item's FP32 /
             // FP64 features computed in the kernel from cl (backflow CNN), gathered with Wt / Wt64
  const float* F;
  const void* Y;
  const int32_t* idx;
  const void* Wt;
  int Lx, Ly;
  const int32_t* list;
  const int32_t* count;
  int max_slots;  // host upper bound of *count
  const uint16_t* perm;
  int perm_stride;
  const float* item_sign;
  float* sign;
  double* logabs;
  int32_t* flags;
  void* slice;  // refine_slice_bytes(n), required by the gather modes
  ConfigList cl{};         // modes 3, 4
  const float* cnn_w = nullptr;
  const float* cnn_b = nullptr;
  int C = 0, layers = 0;
};
int launch_refine(const RefineLaunch& q, cudaStream_t st);
size_t refine_slice_bytes(int n, int d);

size_t pipeline_bytes(int max_items, const nh_backflow_params& p);
PipelineBuffers carve_pipeline(void* ws, int max_items, const nh_backflow_params& p);

// CNN launch: all items of a configuration list (slot = item), or the items of a device list.
struct CnnLaunch {
  const ConfigList* cl;
  const nh_backflow_params* p;
  int mode;                   // 0: features (items, 2, N, d) FP32; 1: occupied Y + idx + sign
  bool fp64;                  // FP64 activations and outputs (mode 1 only)
  const int32_t* slot_item;   // slot -> item, null: identity
  const int32_t* slot_count;  // device number of slots when slot_item is set
  int max_slots;
  float* feat;
  void* Y;                    // float or double (fp64)
  int32_t* idx;
  float* item_sign;
  void* act;                  // per-CTA activation planes when they exceed shared memory, or null
};

struct PfGatherArgs {
  const void* Y;       // (slots, n, d) float or double
  const int32_t* idx;  // (slots, n)
  const void* Wt;      // (4, N, d) float or double
  int Lx, Ly, d, n;
  const int32_t* count_dev;  // device work count (times count_mult) or null
  int count_mult;
  int n_slots;
  const int32_t* slot_item;  // slot -> item, null: identity
  const float* item_sign;
  float* sign;
  double* logabs;
  int32_t* flags;
  double cond_tau;
  int flag_or;
  bool fp64;
  void* tri;  // per-CTA triangles for n beyond shared memory (pfaffian_scratch_bytes), or null
  uint16_t* perm = nullptr;  // when set: the pivot order of every item (perm_stride(n) words)
  double refine_tau = 0.0;   // pivot ratio above which kFlagNeedRefine is set (0: never)
  float* ratio = nullptr;    // when set: every item's pivot ratio
};

// Launchers (return NH_OK or an error code).
int launch_cnn(const CnnLaunch& q, cudaStream_t st);
int launch_pack_cnn(const float* conv_w, int channels, int layers, float* packed, cudaStream_t st);
// tri: pfaffian_scratch_bytes(n) of per-CTA triangles, required when pfaffian_needs_scratch(n,
// fp64) (n up to 1024), else unused and may be null.
int launch_pfaffian_from_F(const float* F, int n, int batch, const int32_t* list,
                           const int32_t* count, bool fp64, double cond_tau, int flag_or,
                           float* sign, double* logabs, int32_t* flags, void* tri,
                           cudaStream_t st, uint16_t* perm = nullptr, double refine_tau = 0.0);
int launch_pfaffian_gather(const PfGatherArgs& g, cudaStream_t st);
// Features and FP32 Pfaffian of every item of a configuration list in one launch (the CNN of
// each item runs in the block that factorises its pairing block; no feature workspace); items
// come off the work counter queue (zeroed by the launch).  Writes per item: sign, logabs, flags,
// pivot ratio, item sign and the pivot order.  fused_supported: the backflow CNN (not the
// residual network), n <= 256.
struct FusedLaunch {
  ConfigList cl;
  const nh_backflow_params* p;
  float* sign;
  double* logabs;
  int32_t* flags;
  float* ratio;
  float* item_sign;
  uint16_t* perm;
  int32_t* queue;
};
bool fused_supported(const nh_backflow_params& p);
// The FP32 gather + Pfaffian with the item's rows copied into shared memory first (the gather
// reads them there instead of from global memory per element); FP32, n <= 256, d % 4 == 0.
bool staged_supported(const PfGatherArgs& g);
int launch_pfaffian_staged(const PfGatherArgs& g, cudaStream_t st);
int launch_pfaffian_fused(const FusedLaunch& f, cudaStream_t st);
// Tensor-memory Pfaffian (one matrix per SM, trailing updates on tcgen05): mode 1 gathers from
// g.Y / g.idx / g.Wt (FP32), mode 0 reads dense F (items, n, n) FP32.
int launch_pfaffian_tc(const PfGatherArgs& g, int mode, const float* F, int32_t* err,
                       cudaStream_t st);
int launch_pairing(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, cudaStream_t st);
// err (or null): the device error word of the tensor-core kernels; when it is set every
// output flag carries NH_FLAG_TIMEOUT.
int launch_combine(const float* sg, const double* la, const int32_t* fl, int G, int n_cfg,
                   const int32_t* n_cfg_dev, float* sign, double* logabs, int32_t* flags,
                   double cancel_tau, const int32_t* err, cudaStream_t st);
// Projected amplitudes (G > 1): marks every image of a configuration whose images cancel
// (sum |.| > cancel_tau |sum|) with NH_FLAG_GROWTH | NH_FLAG_CANCEL and, with weighted, marks
// exactly the other images whose share of psi_P times pivot ratio exceeds cond_tau, before the
// FP64 recompute list is built.
int launch_image_mark(const float* sg, const double* la, int32_t* fl, const float* ratio, int G,
                      int n_cfg, const int32_t* n_cfg_dev, double cancel_tau, double cond_tau,
                      bool weighted, cudaStream_t st);
// Ordered list of the items whose flags have a bit of set_mask and none of clear_mask.
int launch_flagged(const int32_t* flags, int n_items, const int32_t* count_dev, int count_mult,
                   int32_t* list, int32_t* count, cudaStream_t st, int set_mask = NH_FLAG_GROWTH,
                   int clear_mask = 0);
int launch_wtilde(const float* W, float theta, int Lx, int Ly, int d, float* Wt, double* Wt64,
                  cudaStream_t st);
// Tensor-core CNN (nh_cnn_tc.cu).
size_t cnn_tc_packed_bytes();
bool cnn_tc_supported(const nh_backflow_params& p);
int launch_pack_cnn_tc(const float* conv_w, uint16_t* packed, cudaStream_t st);
int launch_cnn_tc(const ConfigList& cl, const nh_backflow_params& p, int mode, float* Y,
                  int32_t* idx, float* item_sign, int32_t* err, cudaStream_t st);
// Whether the FP64 Pfaffian of an n x n matrix fits in shared memory.
bool pfaffian64_fits(int n);
// Large lattices: bytes of global scratch the Pfaffian (FP32 and FP64) and the CNN need when
// their working set exceeds shared memory (0 when it does not).
bool pfaffian_needs_scratch(int n, bool fp64);
size_t pfaffian_scratch_bytes(int n);
size_t cnn_scratch_bytes(int N, int C);
// Residual network (nh_resconv.cu): packed weight size, packing, forward (same CnnLaunch
// contract as launch_cnn) and its per-CTA activation-plane scratch.
size_t resconv_packed_floats(int channels, int blocks);
int launch_pack_resconv(const float* conv_w, int channels, int blocks, float* packed,
                        cudaStream_t st);
int launch_resconv(const CnnLaunch& q, cudaStream_t st);
size_t resconv_scratch_bytes(int N);
// Residual network on the tensor cores (nh_resconv_tc.cu): 16x16, 64 channels, BF16 x3.
size_t resconv_tc_packed_bytes(int blocks);
bool resconv_tc_supported(const nh_backflow_params& p);
int launch_pack_resconv_tc(const float* conv_w, int blocks, void* packed, cudaStream_t st);
int launch_resconv_tc(const ConfigList& cl, const nh_backflow_params& p, float* Y, int32_t* idx,
                      float* item_sign, int32_t* err, cudaStream_t st);

// Full amplitude of a configuration list: CNN -> gather + Pfaffian -> image combination.
int run_pipeline(const ConfigList& cl, const nh_backflow_params& p, const PipelineBuffers& b,
                 float* sign, double* logabs, int32_t* flags, cudaStream_t st);

// Hops / local energy / sampler.
int launch_hop_count(const int8_t* spins, int batch, int Lx, int Ly, int n_dirs,
                     int32_t* counts, cudaStream_t st);
int launch_scan_counts(const int32_t* counts, int batch, int64_t* offsets, cudaStream_t st);
int launch_chunk_counts(const int64_t* total, int n_chunks, int chunk, int32_t* out,
                        cudaStream_t st);
// Writes at most cap records (connections beyond cap, only possible for configurations with
// more electrons than the buffers were sized for, are dropped; callers check the total).
int launch_hop_emit(const int8_t* spins, int batch, int Lx, int Ly, const nh_hubbard_params& h,
                    const int64_t* offsets, int64_t cap, int32_t* rec, double* hval,
                    int32_t* owner, int32_t* from, int32_t* to, cudaStream_t st);
int launch_eloc_reduce(const int8_t* spins, const float* sign, const double* logabs, int batch,
                       int N, double U, const int64_t* offsets, const double* hval,
                       const float* csign, const double* clogabs, double* eloc,
                       cudaStream_t st);
// Chains b < first_exchange propose a uniform hop, chains b >= first_exchange a uniform site
// exchange (a site and one of its n_dirs neighbours swap their occupations).
int launch_mh_propose(const int8_t* spins, int batch, int Lx, int Ly, int n_dirs,
                      uint64_t seed, int64_t step, int32_t* valid, int32_t* from, int32_t* to,
                      cudaStream_t st, int first_exchange = INT32_MAX);
int launch_compact(const int32_t* valid, const int32_t* from, const int32_t* to, int batch,
                   int32_t* c_sample, int32_t* c_from, int32_t* c_to, int32_t* c_count,
                   cudaStream_t st);
// Learned proposal (nh_proposal.cu).
int check_proposal(const nh_proposal_params* q);
int launch_prop_sample(const int8_t* spins, int batch, const nh_proposal_params& q, uint64_t seed,
                       int64_t step, int32_t* valid, int32_t* from, int32_t* to, float* lqr,
                       cudaStream_t st);
int launch_mh_accept(int8_t* spins, float* sign, double* logabs, int batch, int N,
                     const int32_t* c_sample, const int32_t* c_from, const int32_t* c_to,
                     const int32_t* c_count, const float* psign, const double* plogabs,
                     const float* lqr, uint64_t seed, int64_t step, int32_t* accepted,
                     cudaStream_t st);

// Backward of the amplitude (nh_grad.cu).
// G = scale 1/2 F^{-T} per matrix (in place allowed); with pf_sign set the scale is the image
// weight of item i in its configuration (n_img images per configuration), else 1.
int launch_pf_adjoint(const float* F, float* G, int n, int batch, const float* pf_sign,
                      const double* pf_logabs, int n_img, int32_t* flags, cudaStream_t st);
// Per item dY (may be null) and, with jac null, per item dWt (items, 4, N, d); with jac set the
// images' dWt of each sample are summed and chained through build_wtilde's backward into
// jac[sample * ld + off_w + (3 N d W values, theta)].
int launch_pairing_vjp(const float* G, const float* Y, const int32_t* idx, const float* Wt,
                       int Lx, int Ly, int d, int n, int n_img, int samples, float* dY,
                       float* dWt, float* jac, int64_t ld, int64_t off_w, float theta,
                       cudaStream_t st);
// Convolution weight and bias cotangents of every sample's images, summed into jac[sample * ld].
int launch_cnn_vjp(const int8_t* spins, int samples, int n_img, const nh_backflow_params& p,
                   const float* dY, const int32_t* idx, float* jac, int64_t ld, cudaStream_t st);
bool cnn_vjp_supported(const nh_backflow_params& p);

// BCS determinant of every item (or of the items of a device list) from its occupied rows.
struct DetLaunch {
  const void* Y;       // (slots, n, d) float or double
  const int32_t* idx;  // (slots, n)
  const void* Wt;      // (4, N, d) float or double
  int Lx, Ly, nh, d;
  double delta_d;
  const int32_t* count_dev;  // device work count (times count_mult) or null
  int count_mult;
  int n_slots;               // host upper bound of the slots
  const int32_t* slot_item;  // slot -> item, null: identity
  const float* item_sign;
  float* sign;
  double* logabs;
  int32_t* flags;
  float* ratio;
  double cond_tau;
  int flag_or;
  bool fp64;
};
bool det_supported(int nh, int d, bool fp64);
int launch_det(const DetLaunch& q, cudaStream_t st);

// Packed observables (nh_obs.cu): terms per sample of a family, the connection list (counts,
// scan, emit in term order), and the binned reduction of the local values.
int obs_terms(int kind, int N);
int launch_obs_list(const int8_t* spins, int batch, int Lx, int Ly, int kind, int a0, int a1,
                    int32_t* counts, int64_t* offsets, int32_t* owner, int32_t* from,
                    int32_t* to, double* hval, int32_t* bin, cudaStream_t st);
int launch_obs_reduce(const int8_t* spins, const float* sign, const double* logabs, int batch,
                      int N, int kind, int a0, int a1, int diag_bin, const int64_t* total,
                      const int32_t* owner, const int32_t* bin, const double* hval,
                      const float* csign, const double* clogabs, double* V, double* out,
                      cudaStream_t st);

int num_sms();

// Per-kernel CUDA-event timing (enabled by nh_profile_enable).  Construct before the launch,
// destroy after it: records an event pair on the launching stream when profiling is on.
class ProfScope {
 public:
  ProfScope(int id, cudaStream_t st);
  ~ProfScope();

 private:
  int id_;
  cudaStream_t st_;
  cudaEvent_t a_ = nullptr;
};

}  // namespace nh

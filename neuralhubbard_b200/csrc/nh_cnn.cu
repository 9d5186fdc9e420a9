// Backflow CNN forward on CUDA cores, FP32 (the plain form) or FP64 (recompute of items flagged
// ill-conditioned), and the weight packing it reads.
//
// One CTA per item (configuration x symmetry image, grid-stride).  The item's configuration
// is built in shared memory from the int8 sample, its optional hop and the image map, then the
// periodic 3x3 layers run with both activation buffers resident in shared memory
// (channel-major, row stride N + 1) and each layer's weights staged there in the packed
// [ci][tap][co] layout.  Output mode 0 writes the features (2, N, d) of
// code/backflow/models.py:163-167; mode 1 writes only the occupied rows Y (n, d) of the image
// configuration in ascending mode order (the gather y.reshape(2N, d)[idx] of
// code/backflow/pf_kernel.py:395), the occupied mode list idx (n,) and the item sign
// eta_g(s) * (-1)^(n(n-1)/2) (fermionic reordering sign of the image times the
// descending-order convention).
#include <math.h>

#include "nh_cnn_item.cuh"
#include "nh_common.cuh"

namespace nh {
namespace {

template <typename T>
struct CnnArgs {
  ConfigList cl;
  const float* wp;  // packed weights, per layer [ci][tap][co]
  const float* b;
  int Lx, Ly, N, C, layers, n;
  int mode;
  const int32_t* slot_item;   // slot -> item, null: identity over all items
  const int32_t* slot_count;  // device number of slots when slot_item is set
  int max_slots;
  float* feat;
  T* Y;
  int32_t* idx;
  float* item_sign;
  T* act;  // GACT: per-CTA activation planes (2 C (N + 1)) in global memory
};

// GACT: the two activation planes live in a per-CTA slice of global memory (large lattices,
// where they exceed shared memory); shared memory then holds the weights and scratch only.
// TH: threads per CTA; the FP64 instance with resident planes runs 512 (one CTA per SM: its
// planes and weights take ~210 KB), so that twice the warps hide the FP64 latency.
template <typename T, bool GACT = false, int TH = kNumThreads>
__global__ void __launch_bounds__(TH) cnn_kernel(CnnArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = a.N, C = a.C, NS = N + 1, M2 = 2 * N;
  const int tid = threadIdx.x;
  T* actA;
  T* wsm;  // [ci][tap][co]
  if constexpr (GACT) {
    actA = a.act + (size_t)blockIdx.x * 2 * C * NS;
    wsm = reinterpret_cast<T*>(smem_raw);
  } else {
    actA = reinterpret_cast<T*>(smem_raw);
    wsm = actA + 2 * C * NS;
  }
  T* actB = actA + C * NS;
  T* bsm = wsm + C * C * 9;    // [co]
  int* simg = reinterpret_cast<int*>(bsm + C);  // (2N) +-1 of the image configuration
  int* occl = simg + M2;       // (2N) ascending occupied modes of the image configuration
  int* wbuf = occl + M2;       // 4 Lx + 32 ints of scan scratch

  const int G = a.cl.G;
  const int n_work = a.slot_item ? *a.slot_count
                                 : (a.cl.n_cfg_dev ? *a.cl.n_cfg_dev : a.cl.n_cfg) * G;
  for (int slot = blockIdx.x; slot < n_work; slot += gridDim.x) {
    const int item = a.slot_item ? a.slot_item[slot] : slot;
    const int c = item / G, g = item - c * G;
    const int smp = a.cl.sample ? a.cl.sample[c] : c;
    const int fr = a.cl.from ? a.cl.from[c] : -1;
    const int to = a.cl.from ? a.cl.to[c] : -1;
    const int8_t* base = a.cl.spins + (int64_t)smp * M2;

    __syncthreads();  // previous item's readers of simg/act are done
    const T* in = cnn_layers<T, TH>(a.wp, a.b, a.Lx, a.Ly, C, a.layers, base, fr, to, g, actA,
                                    actB, wsm, bsm, simg);
    const int d = C / 2;
    if (a.mode == 0) {
      float* dst = a.feat + (int64_t)item * C * N;
      for (int o = tid; o < C * N; o += TH) {
        const int aa = o % d;
        const int site = (o / d) % N;
        const int sg = o / (N * d);
        dst[o] = (float)in[(sg * d + aa) * NS + site];
      }
      continue;
    }
    auto feat_of = [&](int sg, int aa, int site) { return in[(sg * d + aa) * NS + site]; };
    write_occupied_rows<T, decltype(feat_of), TH>(simg, occl, wbuf, N, a.n, d, g, a.Lx, a.Ly,
                                                  a.Y + (int64_t)slot * a.n * d,
                                                  a.idx + (int64_t)slot * a.n,
                                                  a.item_sign + item, feat_of);
  }
}

// packed[l][ci][tap][co] = conv_w[l][co][ci][tap]
__global__ void pack_kernel(const float* __restrict__ w, int C, int layers, float* packed) {
  const int total = 18 * C + (layers - 1) * 9 * C * C;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    int l = 0, off = 0, cin = 2;
    if (i >= 18 * C) {
      l = 1 + (i - 18 * C) / (9 * C * C);
      off = 18 * C + (l - 1) * 9 * C * C;
      cin = C;
    }
    const int r = i - off;  // (ci * 9 + tap) * C + co
    const int co = r % C;
    const int ct = r / C;  // ci * 9 + tap
    packed[i] = w[off + co * cin * 9 + ct];
  }
}

template <typename T, bool GACT = false>
size_t cnn_smem(int N, int C) {
  return sizeof(T) * ((GACT ? 0 : 2 * (size_t)C * (N + 1)) + (size_t)C * C * 9 + C) +
         sizeof(int) * (4 * (size_t)N + 4 * 32 + 32);
}

constexpr int kCnnBigPerSm = 4;  // CTAs per SM of the global-activation kernel (grid bound)

}  // namespace

int launch_pack_cnn(const float* conv_w, int channels, int layers, float* packed, cudaStream_t st) {
  const int total = 18 * channels + (layers - 1) * 9 * channels * channels;
  ProfScope prof_scope(NH_K_PACK, st);
  pack_kernel<<<(total + 255) / 256, 256, 0, st>>>(conv_w, channels, layers, packed);
  return check_launch("pack_kernel");
}

template <typename T, bool GACT, int TH = kNumThreads>
int launch_cnn_t(const CnnLaunch& q, int N, int C, cudaStream_t st) {
  const nh_backflow_params& p = *q.p;
  const size_t smem = cnn_smem<T, GACT>(N, C);
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "cnn: lattice N=%d with %d channels needs %zu B of smem",
                N, C, smem);
  if (GACT && !q.act)
    return fail(NH_ERR_UNSUPPORTED, "cnn: N=%d needs the large-lattice activation scratch", N);
  const int slots = q.slot_item ? q.max_slots : q.cl->n_cfg * q.cl->G;
  if (slots <= 0) return NH_OK;
  int grid = GACT ? num_sms() * kCnnBigPerSm
                  : num_sms() * (smem > 113 * 1024 || TH > kNumThreads ? 1 : 2) * 4;
  if (grid > slots) grid = slots;
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(cnn_kernel<T, GACT, TH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "cnn smem attribute");
    configured = smem;
  }
  CnnArgs<T> a{*q.cl, p.conv_w_packed, p.conv_b, p.Lx, p.Ly, N, C, p.layers,
               p.n_up + p.n_dn, q.mode, q.slot_item, q.slot_count, q.max_slots,
               q.feat, static_cast<T*>(q.Y), q.idx, q.item_sign, static_cast<T*>(q.act)};
  ProfScope prof_scope(sizeof(T) == 8 ? NH_K_CNN64 : NH_K_CNN, st);
  cnn_kernel<T, GACT, TH><<<grid, TH, smem, st>>>(a);
  return check_launch(sizeof(T) == 8 ? "cnn_kernel<double>" : "cnn_kernel<float>");
}

size_t cnn_scratch_bytes(int N, int C) {
  if (cnn_smem<double>(N, C) <= 227 * 1024) return 0;
  return (size_t)num_sms() * kCnnBigPerSm * 2 * C * (N + 1) * sizeof(double);
}

int launch_cnn(const CnnLaunch& q, cudaStream_t st) {
  const nh_backflow_params& p = *q.p;
  if (p.net == NH_NET_RESCONV) return launch_resconv(q, st);
  const int N = p.Lx * p.Ly, C = p.channels;
  if (C % 16 || C < 16 || C > 64 || p.layers < 1 || N % 2 || N > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "cnn: channels %d (multiple of 16, <= 64), layers %d, N %d",
                C, p.layers, N);
  if (!p.conv_w_packed)
    return fail(NH_ERR_INVALID, "cnn: conv_w_packed is null (call nh_pack_cnn_weights)");
  if (q.fp64)
    return cnn_smem<double>(N, C) <= 227 * 1024 ? launch_cnn_t<double, false, 512>(q, N, C, st)
                                                 : launch_cnn_t<double, true>(q, N, C, st);
  return cnn_smem<float>(N, C) <= 227 * 1024 ? launch_cnn_t<float, false>(q, N, C, st)
                                              : launch_cnn_t<float, true>(q, N, C, st);
}

}  // namespace nh

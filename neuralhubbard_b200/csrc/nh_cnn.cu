// Backflow CNN forward, FP32 on CUDA cores (the plain form).
//
// One CTA per item (configuration x symmetry image, grid-stride).  The item's configuration
// is built in shared memory from the int8 sample, its optional hop and the image map, then the
// 4 periodic 3x3 layers run with both activation buffers resident in shared memory
// (channel-major, row stride N + 1).  Output mode 0 writes the features (2, N, d) of
// code/backflow/models.py:163-167; mode 1 writes only the occupied rows Y (n, d) of the image
// configuration in ascending mode order (the gather y.reshape(2N, d)[idx] of
// code/backflow/pf_kernel.py:395), the occupied mode list idx (n,) and the item sign
// eta_g(s) * (-1)^(n(n-1)/2) (fermionic reordering sign of the image times the
// descending-order convention).
#include <math.h>

#include "nh_common.cuh"

namespace nh {
namespace {

struct CnnArgs {
  ConfigList cl;
  const float* w;
  const float* b;
  int Lx, Ly, N, C, layers, n;
  int mode;
  float* feat;
  float* Y;
  int32_t* idx;
  float* item_sign;
};

__device__ __forceinline__ float gelu_tanh(float x) {
  const float k0 = 0.7978845608028654f;  // sqrt(2 / pi)
  return 0.5f * x * (1.0f + tanhf(k0 * (x + 0.044715f * x * x * x)));
}

// Exclusive block scan of one int per thread; returns the exclusive prefix, *total the sum.
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
    int w = lane < (kNumThreads / 32) ? warp_buf[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (kNumThreads / 32)) warp_buf[lane] = w;
  }
  __syncthreads();
  int base = wid ? warp_buf[wid - 1] : 0;
  *total = warp_buf[kNumThreads / 32 - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void __launch_bounds__(kNumThreads) cnn_fp32_kernel(CnnArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = a.N, C = a.C, NS = N + 1, M2 = 2 * N;
  const int tid = threadIdx.x;
  float* actA = reinterpret_cast<float*>(smem_raw);
  float* actB = actA + C * NS;
  float* wsm = actB + C * NS;      // [ci][tap][co]
  float* bsm = wsm + C * C * 9;    // [co]
  int* simg = reinterpret_cast<int*>(bsm + C);  // (2N) +-1 of the image configuration
  int* occl = simg + M2;           // (2N) ascending occupied modes of the image configuration
  int* wbuf = occl + M2;           // 32 ints of scan scratch

  const int n_cfg = a.cl.n_cfg_dev ? *a.cl.n_cfg_dev : a.cl.n_cfg;
  const int G = a.cl.G;
  const int n_items = n_cfg * G;
  const int half = N / 2;
  const int ngroups = C / 8;

  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int c = item / G, g = item - c * G;
    const int smp = a.cl.sample ? a.cl.sample[c] : c;
    const int fr = a.cl.from ? a.cl.from[c] : -1;
    const int to = a.cl.from ? a.cl.to[c] : -1;
    const int8_t* base = a.cl.spins + (int64_t)smp * M2;

    __syncthreads();  // previous item's readers of simg/act are done
    for (int m = tid; m < M2; m += kNumThreads) {
      int src = sym_map(m, g, a.Lx, a.Ly, N);  // image[m] = s[g(m)] (g is an involution)
      int v = base[src];
      v = (src == fr) ? -1 : ((src == to) ? 1 : v);
      simg[m] = v > 0 ? 1 : -1;
      int ch = m >= N ? 1 : 0;
      actA[ch * NS + (m - ch * N)] = v > 0 ? 1.0f : -1.0f;
    }

    float* in = actA;
    float* out = actB;
    int cin = 2;
    const float* wl = a.w;
    for (int l = 0; l < a.layers; ++l) {
      __syncthreads();
      const int cnt = C * cin * 9;
      for (int i = tid; i < cnt; i += kNumThreads) {
        int co = i / (cin * 9);
        int rem = i - co * cin * 9;  // ci * 9 + tap
        wsm[rem * C + co] = wl[i];
      }
      for (int i = tid; i < C; i += kNumThreads) bsm[i] = a.b[l * C + i];
      __syncthreads();
      const bool act_fn = l < a.layers - 1;
      for (int task = tid; task < ngroups * half; task += kNumThreads) {
        const int grp = task / half;
        const int s0 = task - grp * half, s1 = s0 + half;
        const int x0 = s0 / a.Ly, y0 = s0 - x0 * a.Ly;
        const int x1 = s1 / a.Ly, y1 = s1 - x1 * a.Ly;
        float acc0[8], acc1[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) acc0[j] = acc1[j] = bsm[grp * 8 + j];
        for (int ci = 0; ci < cin; ++ci) {
          const float* inc = in + ci * NS;
#pragma unroll
          for (int u = 0; u < 3; ++u) {
            int xa = x0 + u - 1, xb = x1 + u - 1;
            xa = xa < 0 ? xa + a.Lx : (xa >= a.Lx ? xa - a.Lx : xa);
            xb = xb < 0 ? xb + a.Lx : (xb >= a.Lx ? xb - a.Lx : xb);
#pragma unroll
            for (int v = 0; v < 3; ++v) {
              int ya = y0 + v - 1, yb = y1 + v - 1;
              ya = ya < 0 ? ya + a.Ly : (ya >= a.Ly ? ya - a.Ly : ya);
              yb = yb < 0 ? yb + a.Ly : (yb >= a.Ly ? yb - a.Ly : yb);
              const float i0 = inc[xa * a.Ly + ya];
              const float i1 = inc[xb * a.Ly + yb];
              const float4* wp =
                  reinterpret_cast<const float4*>(wsm + (ci * 9 + u * 3 + v) * C + grp * 8);
              const float4 wa = wp[0], wb = wp[1];
              const float w8[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
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
          float r0 = act_fn ? gelu_tanh(acc0[j]) : acc0[j];
          float r1 = act_fn ? gelu_tanh(acc1[j]) : acc1[j];
          out[(grp * 8 + j) * NS + s0] = r0;
          out[(grp * 8 + j) * NS + s1] = r1;
        }
      }
      wl += C * cin * 9;
      cin = C;
      float* t = in;
      in = out;
      out = t;
    }
    __syncthreads();
    const int d = C / 2;
    if (a.mode == 0) {
      float* dst = a.feat + (int64_t)item * C * N;
      for (int o = tid; o < C * N; o += kNumThreads) {
        int aa = o % d;
        int site = (o / d) % N;
        int sg = o / (N * d);
        dst[o] = in[(sg * d + aa) * NS + site];
      }
      continue;
    }
    // Occupied list of the image configuration, ascending (block scan over mode chunks).
    const int per = (M2 + kNumThreads - 1) / kNumThreads;
    const int m0 = tid * per;
    int cnt = 0;
    for (int m = m0; m < m0 + per && m < M2; ++m) cnt += simg[m] > 0;
    int total;
    int pos = block_scan(cnt, wbuf, &total);
    for (int m = m0; m < m0 + per && m < M2; ++m)
      if (simg[m] > 0) occl[pos++] = m;
    __syncthreads();
    const int n = a.n;
    float* Ydst = a.Y + (int64_t)item * n * d;
    for (int o = tid; o < n * d; o += kNumThreads) {
      int p = o / d, aa = o - p * d;
      int m = occl[p < total ? p : 0];
      int sg = m >= N ? 1 : 0;
      Ydst[o] = in[(sg * d + aa) * NS + (m - sg * N)];
    }
    int32_t* idst = a.idx + (int64_t)item * n;
    for (int p = tid; p < n; p += kNumThreads) idst[p] = occl[p < total ? p : 0];
    // eta_g: parity of the inversions of (g(a_1), ..., g(a_n)).
    int par = 0;
    if (g != 0) {
      for (int i = tid; i < total; i += kNumThreads) {
        int gi = sym_map(occl[i], g, a.Lx, a.Ly, N);
        int inv = 0;
        for (int j = i + 1; j < total; ++j) inv += sym_map(occl[j], g, a.Lx, a.Ly, N) < gi;
        par ^= inv & 1;
      }
    }
    int odd = __syncthreads_count(par);
    if (tid == 0) {
      long long kk = total;
      int rev = (int)((kk * (kk - 1) / 2) & 1);
      float s = ((odd & 1) ^ rev) ? -1.0f : 1.0f;
      if (total != n) s = 0.0f;  // wrong particle number: amplitude 0
      a.item_sign[item] = s;
    }
  }
}

}  // namespace

int launch_cnn(const ConfigList& cl, const nh_backflow_params& p, int out_mode, float* feat,
               float* Y, int32_t* idx, float* item_sign, cudaStream_t st) {
  CnnArgs a;
  a.cl = cl;
  a.w = p.conv_w;
  a.b = p.conv_b;
  a.Lx = p.Lx;
  a.Ly = p.Ly;
  a.N = p.Lx * p.Ly;
  a.C = p.channels;
  a.layers = p.layers;
  a.n = p.n_up + p.n_dn;
  a.mode = out_mode;
  a.feat = feat;
  a.Y = Y;
  a.idx = idx;
  a.item_sign = item_sign;
  if (a.C % 16 || a.C < 16 || a.C > 64 || a.layers < 1 || a.N % 2 || a.N > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "cnn: channels %d (multiple of 16, <= 64), layers %d, N %d",
                a.C, a.layers, a.N);
  const int N = a.N, C = a.C;
  size_t smem = sizeof(float) * (2 * (size_t)C * (N + 1) + (size_t)C * C * 9 + C) +
                sizeof(int) * (4 * (size_t)N + 32);
  if (smem > 227 * 1024)
    return fail(NH_ERR_UNSUPPORTED, "cnn: lattice N=%d with %d channels needs %zu B of smem", N,
                C, smem);
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    cudaError_t e = cudaFuncSetAttribute(cnn_fp32_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return check_cuda(e, "cnn smem attribute");
    configured = smem;
  }
  int items = cl.n_cfg * cl.G;
  if (items <= 0) return NH_OK;
  int per_sm = smem > 113 * 1024 ? 1 : 2;
  int grid = num_sms() * per_sm * 4;
  if (grid > items) grid = items;
  cnn_fp32_kernel<<<grid, kNumThreads, smem, st>>>(a);
  return check_launch("cnn_fp32_kernel");
}

}  // namespace nh

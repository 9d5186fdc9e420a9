// The backflow CNN of one item (configuration x symmetry image) by one 256-thread block: the
// device function behind cnn_kernel (nh_cnn.cu) and the fused kernels that compute an item's
// features and consume them in the same block (the amplitude/Pfaffian kernel of the persistent
// local energy, nh_pfaffian.cu, and the FP64 refinement, nh_refine.cu).
//
// Periodic 3x3 convolutions (cross-correlation, code/backflow/models.py:163-167), tanh-GELU
// between layers, on the 2-channel +-1 occupation image of the item's configuration (sample s,
// optional move, image map g: image[m] = s'[g(m)], g an involution).  Activations are
// channel-major with row stride N + 1; each layer's weights are staged in the packed
// [ci][tap][co] layout.
#pragma once

#include "nh_common.cuh"

namespace nh {

__device__ __forceinline__ float gelu_tanh_dev(float x) {
  const float k0 = 0.7978845608028654f;  // sqrt(2 / pi)
  return 0.5f * x * (1.0f + tanhf(k0 * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ double gelu_tanh_dev(double x) {
  const double k0 = 0.7978845608028654;
  return 0.5 * x * (1.0 + tanh(k0 * (x + 0.044715 * x * x * x)));
}

__device__ __forceinline__ void cnn_lds8(const float* p, float* o) {
  const float4 a = reinterpret_cast<const float4*>(p)[0];
  const float4 b = reinterpret_cast<const float4*>(p)[1];
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
  o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
}
__device__ __forceinline__ void cnn_lds8(const double* p, double* o) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double2 v = reinterpret_cast<const double2*>(p)[k];
    o[2 * k] = v.x;
    o[2 * k + 1] = v.y;
  }
}

// Builds the item's image configuration in simg (2N ints, +-1) and runs the layers; returns the
// activation buffer (actA or actB) that holds the last layer's output, C planes of stride N + 1.
// wsm: C * C * 9 values, bsm: C values (shared memory); actA, actB: C (N + 1) values each
// (shared or per-block global memory).  Block-wide: every thread of the TH-thread block calls it.
template <typename T, int TH = kNumThreads>
__device__ T* cnn_layers(const float* __restrict__ wp, const float* __restrict__ bias, int Lx,
                         int Ly, int C, int layers, const int8_t* __restrict__ base, int fr,
                         int to, int g, T* actA, T* actB, T* wsm, T* bsm, int* simg) {
  const int tid = threadIdx.x;
  const int N = Lx * Ly, NS = N + 1, M2 = 2 * N;
  const int half = N / 2, ngroups = C / 8;
  for (int m = tid; m < M2; m += TH) {
    const int src = sym_map(m, g, Lx, Ly, N);  // image[m] = s[g(m)] (g is an involution)
    const int v = move_value(src, base[src], fr, to);
    simg[m] = v > 0 ? 1 : -1;
    const int ch = m >= N ? 1 : 0;
    actA[ch * NS + (m - ch * N)] = v > 0 ? T(1) : T(-1);
  }
  T* in = actA;
  T* out = actB;
  int cin = 2;
  const float* wl = wp;
  for (int l = 0; l < layers; ++l) {
    __syncthreads();
    const int cnt = C * cin * 9;
    for (int i = tid; i < cnt; i += TH) wsm[i] = T(__ldg(wl + i));
    for (int i = tid; i < C; i += TH) bsm[i] = T(__ldg(bias + l * C + i));
    __syncthreads();
    const bool act_fn = l < layers - 1;
    for (int task = tid; task < ngroups * half; task += TH) {
      const int grp = task / half;
      const int s0 = task - grp * half, s1 = s0 + half;
      const int x0 = s0 / Ly, y0 = s0 - x0 * Ly;
      const int x1 = s1 / Ly, y1 = s1 - x1 * Ly;
      T acc0[8], acc1[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) acc0[j] = acc1[j] = bsm[grp * 8 + j];
      for (int ci = 0; ci < cin; ++ci) {
        const T* inc = in + ci * NS;
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
            const T i0 = inc[xa * Ly + ya];
            const T i1 = inc[xb * Ly + yb];
            T w8[8];
            cnn_lds8(wsm + (ci * 9 + u * 3 + v) * C + grp * 8, w8);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              acc0[j] = fma(i0, w8[j], acc0[j]);
              acc1[j] = fma(i1, w8[j], acc1[j]);
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        out[(grp * 8 + j) * NS + s0] = act_fn ? gelu_tanh_dev(acc0[j]) : acc0[j];
        out[(grp * 8 + j) * NS + s1] = act_fn ? gelu_tanh_dev(acc1[j]) : acc1[j];
      }
    }
    wl += C * cin * 9;
    cin = C;
    T* t = in;
    in = out;
    out = t;
  }
  __syncthreads();
  return in;
}

// Shared-memory footprint of cnn_layers' staging (wsm + bsm) plus simg, occl (2N ints each) and
// the scan scratch of write_occupied_rows (4 Lx + 32 ints), without the activation planes.
template <typename T>
__host__ __device__ constexpr size_t cnn_item_scratch_bytes(int N, int C, int Lx) {
  return sizeof(T) * ((size_t)C * C * 9 + C) + sizeof(int) * (4 * (size_t)N + 4 * Lx + 32);
}

}  // namespace nh

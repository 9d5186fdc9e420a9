// Hubbard hop enumeration, local-energy reduction, Metropolis hop sampler and the small
// bookkeeping kernels they need (scan, compaction, Wt table).
//
// Connections of a configuration s: every occupied mode m (ascending) and hop direction d
// whose target mode m' (same spin) is empty; <s|H|s'> = -t_d (-1)^(occupied modes strictly
// between m and m'), the Jordan-Wigner sign of |s> = c+_{m1} ... c+_{mk} |0> with ascending
// modes (Hubbard(U=8, t=[1, t'], n_neighbor=[1, 2]) of code/states.py:244-247; the packed
// connected-configuration evaluation of H.Oloc, code/measure/transverse_spin.py:44-80).
#include <math.h>

#include "nh_common.cuh"

namespace nh {
namespace {

__device__ __forceinline__ int warp_incl_scan(int x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Exclusive block scan (blockDim.x == kNumThreads); *total = block sum.
__device__ __forceinline__ int block_excl_scan(int v, int* buf, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = warp_incl_scan(v);
  if (lane == 31) buf[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < kNumThreads / 32 ? buf[lane] : 0;
    w = warp_incl_scan(w);
    if (lane < kNumThreads / 32) buf[lane] = w;
  }
  __syncthreads();
  int r = (wid ? buf[wid - 1] : 0) + x - v;
  *total = buf[kNumThreads / 32 - 1];
  __syncthreads();
  return r;
}

// One CTA per configuration: occupancy prefix P[m] = #occupied modes < m in shared memory,
// then per-thread contiguous mode chunks (ascending), block scan of their connection counts.
template <bool EMIT>
__global__ void __launch_bounds__(kNumThreads) hop_kernel(const int8_t* __restrict__ spins,
                                                          int batch, int Lx, int Ly, int n_dirs,
                                                          double t, double tp,
                                                          int32_t* counts,
                                                          const int64_t* offsets, int64_t cap,
                                                          int32_t* rec, double* hval,
                                                          int32_t* owner, int32_t* cfrom,
                                                          int32_t* cto) {
  __shared__ int occ[2 * kMaxN];
  __shared__ int pre[2 * kMaxN + 1];
  __shared__ int buf[32];
  const int N = Lx * Ly, M2 = 2 * N;
  const int tid = threadIdx.x;
  const int per = (M2 + kNumThreads - 1) / kNumThreads;
  const int m0 = tid * per, m1 = min(M2, m0 + per);
  for (int b = blockIdx.x; b < batch; b += gridDim.x) {
    const int8_t* s = spins + (size_t)b * M2;
    __syncthreads();
    int cnt = 0;
    for (int m = m0; m < m1; ++m) {
      int o = s[m] > 0;
      occ[m] = o;
      cnt += o;
    }
    int tot;
    int run = block_excl_scan(cnt, buf, &tot);
    for (int m = m0; m < m1; ++m) {
      pre[m] = run;
      run += occ[m];
    }
    if (tid == 0) pre[M2] = tot;
    __syncthreads();
    int nc = 0;
    for (int m = m0; m < m1; ++m) {
      if (!occ[m]) continue;
      const int sg = m >= N ? 1 : 0;
      const int site = m - sg * N;
      for (int d = 0; d < n_dirs; ++d) nc += !occ[sg * N + hop_target_site(site, d, Lx, Ly)];
    }
    int total;
    int pos = block_excl_scan(nc, buf, &total);
    if (!EMIT) {
      if (tid == 0) counts[b] = total;
      continue;
    }
    int64_t o = offsets[b] + pos;
    for (int m = m0; m < m1; ++m) {
      if (!occ[m]) continue;
      const int sg = m >= N ? 1 : 0;
      const int site = m - sg * N;
      for (int d = 0; d < n_dirs; ++d) {
        const int mj = sg * N + hop_target_site(site, d, Lx, Ly);
        if (occ[mj]) continue;
        const int lo = m < mj ? m : mj, hi = m < mj ? mj : m;
        const int between = pre[hi] - pre[lo + 1];
        const double amp = d < 4 ? t : tp;
        if (o >= cap) break;  // more electrons than the buffers were sized for
        if (rec) {
          rec[2 * o] = m;
          rec[2 * o + 1] = mj;
        }
        if (hval) hval[o] = (between & 1) ? amp : -amp;
        if (owner) owner[o] = b;
        if (cfrom) cfrom[o] = m;
        if (cto) cto[o] = mj;
        ++o;
      }
    }
  }
}

// Single-CTA exclusive scan of int32 counts into int64 offsets (offsets[batch] = total).
__global__ void __launch_bounds__(1024) scan_kernel(const int32_t* counts, int batch,
                                                    int64_t* offsets) {
  __shared__ long long wsum[32];
  __shared__ long long carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < batch; base += 1024) {
    const int i = base + threadIdx.x;
    long long v = i < batch ? counts[i] : 0;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      long long w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const long long excl = carry + (wid ? wsum[wid - 1] : 0) + x - v;
    if (i < batch) offsets[i] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) offsets[batch] = carry;
}

// E_loc[b] = U * docc + sum_c hval_c * (sign_c sign_b) exp(logabs_c - logabs_b), FP64.
__global__ void eloc_reduce_kernel(const int8_t* __restrict__ spins, const float* sign,
                                   const double* logabs, int batch, int N, double U,
                                   const int64_t* offsets, const double* hval,
                                   const float* csign, const double* clogabs, double* eloc) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int b = warp; b < batch; b += nwarps) {
    const int8_t* s = spins + (size_t)b * 2 * N;
    int docc = 0;
    for (int i = lane; i < N; i += 32) docc += (s[i] > 0) & (s[N + i] > 0);
    double acc = 0.0;
    const double l0 = logabs[b];
    const float s0 = sign[b];
    const int64_t c1 = offsets[b + 1];
    int64_t c = offsets[b] + lane;
    // Four connections per lane per pass, all loads issued before any is used.
    for (; c + 96 < c1; c += 128) {
      float sc[4];
      double hv[4], la[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        sc[u] = csign[c + 32 * u];
        hv[u] = hval[c + 32 * u];
        la[u] = clogabs[c + 32 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (sc[u] != 0.0f) acc += hv[u] * (double)(sc[u] * s0) * exp(la[u] - l0);
    }
    for (; c < c1; c += 32) {
      const float sc = csign[c];
      const double hv = hval[c], la = clogabs[c];
      if (sc != 0.0f) acc += hv * (double)(sc * s0) * exp(la - l0);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      acc += __shfl_xor_sync(0xffffffffu, acc, o);
      docc += __shfl_xor_sync(0xffffffffu, docc, o);
    }
    if (lane == 0) eloc[b] = U * (double)docc + (s0 != 0.0f ? acc : NAN);
  }
}

// One warp per chain: Philox draws (step, chain, 0, 0), electron of rank e = (r0 k) >> 32
// among the k occupied modes (ascending), direction (r1 n_dirs) >> 32.
// Site exchange (SiteExchange of code/states.py:397-408): a uniform site i and a uniform one of
// its n_dirs neighbours j swap their occupations (up and down); equal occupations are a null
// move.  Word 0 of the chain's draw picks the site, word 1 the direction (the reverse move picks
// j and the opposite direction with the same probability: the proposal is symmetric).
__device__ __forceinline__ void propose_exchange(const int8_t* s, int N, int Lx, int Ly,
                                                 int n_dirs, u32x4 r, int32_t* valid,
                                                 int32_t* from, int32_t* to) {
  const int i = (int)(((uint64_t)r.x * (uint64_t)N) >> 32);
  const int dir = (int)(((uint64_t)r.y * (uint64_t)n_dirs) >> 32);
  const int j = hop_target_site(i, dir, Lx, Ly);
  int src[2] = {-1, -1}, dst[2] = {-1, -1}, h = 0;
  for (int sg = 0; sg < 2; ++sg) {
    const bool oi = s[sg * N + i] > 0, oj = s[sg * N + j] > 0;
    if (oi != oj) {
      src[h] = sg * N + (oi ? i : j);
      dst[h] = sg * N + (oi ? j : i);
      ++h;
    }
  }
  *valid = h > 0 ? 1 : 0;
  *from = h > 0 ? pack_move(src[0], src[1]) : -1;
  *to = h > 0 ? pack_move(dst[0], dst[1]) : -1;
}

__global__ void mh_propose_kernel(const int8_t* __restrict__ spins, int batch, int Lx, int Ly,
                                  int n_dirs, uint32_t k0, uint32_t k1, uint32_t step_lo,
                                  uint32_t step_hi, int32_t* valid, int32_t* from, int32_t* to,
                                  int first_exchange) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int N = Lx * Ly, M2 = 2 * N;
  for (int b = warp; b < batch; b += nwarps) {
    const int8_t* s = spins + (size_t)b * M2;
    if (b >= first_exchange) {
      if (lane == 0) {
        const u32x4 r = philox4x32_10(u32x4{step_lo, (uint32_t)b, 0u, step_hi}, k0, k1);
        propose_exchange(s, N, Lx, Ly, n_dirs, r, valid + b, from + b, to + b);
      }
      continue;
    }
    int k = 0;
    for (int m = lane; m < M2; m += 32) k += s[m] > 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    u32x4 r = philox4x32_10(u32x4{step_lo, (uint32_t)b, 0u, step_hi}, k0, k1);
    const int e = (int)(((uint64_t)r.x * (uint64_t)k) >> 32);
    const int dir = (int)(((uint64_t)r.y * (uint64_t)n_dirs) >> 32);
    int seen = 0, mode = -1;
    for (int base = 0; base < M2 && mode < 0; base += 32) {
      const int m = base + lane;
      const bool o = m < M2 && s[m] > 0;
      const unsigned bal = __ballot_sync(0xffffffffu, o);
      const int c = __popc(bal);
      if (e < seen + c) {
        // the (e - seen)-th set bit of bal
        int want = e - seen;
        unsigned x = bal;
        for (int i = 0; i < want; ++i) x &= x - 1;
        mode = base + __ffs(x) - 1;
      }
      seen += c;
    }
    if (lane == 0) {
      const int sg = mode >= N ? 1 : 0;
      const int mj = sg * N + hop_target_site(mode - sg * N, dir, Lx, Ly);
      from[b] = mode;
      to[b] = mj;
      valid[b] = (k > 0 && mode >= 0 && s[mj] < 0) ? 1 : 0;
    }
  }
}

// Ordered compaction of the valid proposals (single CTA, 1024 threads).
__global__ void __launch_bounds__(1024) compact_kernel(const int32_t* valid, const int32_t* from,
                                                       const int32_t* to, int batch,
                                                       int32_t* c_sample, int32_t* c_from,
                                                       int32_t* c_to, int32_t* c_count) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < batch; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < batch ? valid[i] : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, v);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    if (wid == 0) {
      int w = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    if (v) {
      const int pos = carry + (wid ? wsum[wid - 1] : 0) + __popc(bal & ((1u << lane) - 1u));
      c_sample[pos] = i;
      c_from[pos] = from[i];
      c_to[pos] = to[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *c_count = carry;
}

// Accept when u < |psi'/psi|^2 q(s|s')/q(s'|s), compared as
// log(u) < 2 (logabs' - logabs) + lqr[b] in FP64 (lqr null: symmetric proposal).
__global__ void mh_accept_kernel(int8_t* spins, float* sign, double* logabs, int N,
                                 const int32_t* c_sample, const int32_t* c_from,
                                 const int32_t* c_to, const int32_t* c_count,
                                 const float* psign, const double* plogabs,
                                 const float* __restrict__ lqr, uint32_t k0,
                                 uint32_t k1, uint32_t step_lo, uint32_t step_hi,
                                 int32_t* accepted) {
  const int cnt = *c_count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int b = c_sample[i];
    u32x4 r = philox4x32_10(u32x4{step_lo, (uint32_t)b, 0u, step_hi}, k0, k1);
    const double u = u32_to_unit(r.z);
    const float sp = psign[i];
    const double lr2 = 2.0 * (plogabs[i] - logabs[b]) + (lqr ? (double)lqr[b] : 0.0);
    const bool acc = sp != 0.0f && (u == 0.0 || log(u) < lr2);
    if (acc) {
      int8_t* s = spins + (size_t)b * 2 * N;
      const int f = c_from[i], t = c_to[i];
      s[move_first(f)] = -1;
      s[move_first(t)] = 1;
      if (move_second(f) >= 0) {
        s[move_second(f)] = -1;
        s[move_second(t)] = 1;
      }
      sign[b] = sp;
      logabs[b] = plogabs[i];
      if (accepted) accepted[b] += 1;
    }
  }
}

// Wt (4, N, d) = [uu, ud, du, dd] blocks times exp(-lam D_r) / (N sum_r exp(-lam D_r)),
// lam = softplus(theta) (code/backflow/pf_kernel.py:107-124).  Single CTA.
__global__ void __launch_bounds__(1024) wtilde_kernel(const float* __restrict__ W, float theta,
                                                      int Lx, int Ly, int d, float* Wt,
                                                      double* Wt64) {
  __shared__ double part[32];
  __shared__ double total;
  const int N = Lx * Ly;
  const double th = (double)theta;
  const double lam = log1p(exp(-fabs(th))) + fmax(th, 0.0);
  double acc = 0.0;
  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    const int rx = r / Ly, ry = r - rx * Ly;
    const double mx = (double)min(rx, Lx - rx), my = (double)min(ry, Ly - ry);
    acc += exp(-lam * sqrt(mx * mx + my * my));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += part[w];
    total = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 4 * N * d; e += blockDim.x) {
    const int blk = e / (N * d);
    const int r = (e / d) % N;
    const int a = e % d;
    const int rx = r / Ly, ry = r - rx * Ly;
    const int nr = (rx ? Lx - rx : 0) * Ly + (ry ? Ly - ry : 0);
    const double mx = (double)min(rx, Lx - rx), my = (double)min(ry, Ly - ry);
    const double pref64 = exp(-lam * sqrt(mx * mx + my * my)) / ((double)N * total);
    const float pref = (float)pref64;
    float w;
    double w64;
    if (blk == 0) {
      w = (W[(size_t)(1 * N + r) * d + a] - W[(size_t)(1 * N + nr) * d + a]) / 2.0f;
      w64 = ((double)W[(size_t)(1 * N + r) * d + a] - (double)W[(size_t)(1 * N + nr) * d + a]) / 2.0;
    } else if (blk == 1) {
      w = W[(size_t)r * d + a];
      w64 = w;
    } else if (blk == 2) {
      w = -W[(size_t)nr * d + a];
      w64 = w;
    } else {
      w = (W[(size_t)(2 * N + r) * d + a] - W[(size_t)(2 * N + nr) * d + a]) / 2.0f;
      w64 = ((double)W[(size_t)(2 * N + r) * d + a] - (double)W[(size_t)(2 * N + nr) * d + a]) / 2.0;
    }
    Wt[e] = w * pref;
    if (Wt64) Wt64[e] = w64 * pref64;
  }
}

}  // namespace

int launch_hop_count(const int8_t* spins, int batch, int Lx, int Ly, int n_dirs,
                     int32_t* counts, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = min(batch, num_sms() * 8);
  ProfScope prof_scope(NH_K_HOP_COUNT, st);
  hop_kernel<false><<<grid, kNumThreads, 0, st>>>(spins, batch, Lx, Ly, n_dirs, 0.0, 0.0, counts,
                                                  nullptr, 0, nullptr, nullptr, nullptr, nullptr,
                                                  nullptr);
  return check_launch("hop_kernel<count>");
}

// Work count of every chunk of the connection list: clamp(total - i * chunk, 0, chunk), with
// total = offsets[batch] read on the device (no host round trip).
__global__ void chunk_counts_kernel(const int64_t* __restrict__ total, int n_chunks, int chunk,
                                    int32_t* __restrict__ out) {
  const int64_t t = *total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_chunks; i += gridDim.x * blockDim.x) {
    const int64_t left = t - (int64_t)i * chunk;
    out[i] = (int32_t)(left <= 0 ? 0 : (left < chunk ? left : chunk));
  }
}

int launch_chunk_counts(const int64_t* total, int n_chunks, int chunk, int32_t* out,
                        cudaStream_t st) {
  if (n_chunks <= 0) return NH_OK;
  ProfScope prof_scope(NH_K_SCAN, st);
  chunk_counts_kernel<<<(n_chunks + 255) / 256, 256, 0, st>>>(total, n_chunks, chunk, out);
  return check_launch("chunk_counts_kernel");
}

int launch_scan_counts(const int32_t* counts, int batch, int64_t* offsets, cudaStream_t st) {
  ProfScope prof_scope(NH_K_SCAN, st);
  scan_kernel<<<1, 1024, 0, st>>>(counts, batch, offsets);
  return check_launch("scan_kernel");
}

int launch_hop_emit(const int8_t* spins, int batch, int Lx, int Ly, const nh_hubbard_params& h,
                    const int64_t* offsets, int64_t cap, int32_t* rec, double* hval,
                    int32_t* owner, int32_t* from, int32_t* to, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = min(batch, num_sms() * 8);
  ProfScope prof_scope(NH_K_HOP_EMIT, st);
  hop_kernel<true><<<grid, kNumThreads, 0, st>>>(spins, batch, Lx, Ly, h.n_dirs, h.t, h.tp,
                                                 nullptr, offsets, cap, rec, hval, owner, from,
                                                 to);
  return check_launch("hop_kernel<emit>");
}

int launch_eloc_reduce(const int8_t* spins, const float* sign, const double* logabs, int batch,
                       int N, double U, const int64_t* offsets, const double* hval,
                       const float* csign, const double* clogabs, double* eloc,
                       cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = min((batch + 7) / 8, num_sms() * 16);
  ProfScope prof_scope(NH_K_ELOC_REDUCE, st);
  eloc_reduce_kernel<<<grid, 256, 0, st>>>(spins, sign, logabs, batch, N, U, offsets, hval,
                                           csign, clogabs, eloc);
  return check_launch("eloc_reduce_kernel");
}

int launch_mh_propose(const int8_t* spins, int batch, int Lx, int Ly, int n_dirs,
                      uint64_t seed, int64_t step, int32_t* valid, int32_t* from, int32_t* to,
                      cudaStream_t st, int first_exchange) {
  if (batch <= 0) return NH_OK;
  int grid = min((batch + 7) / 8, num_sms() * 16);
  ProfScope prof_scope(NH_K_MH_PROPOSE, st);
  mh_propose_kernel<<<grid, 256, 0, st>>>(spins, batch, Lx, Ly, n_dirs, (uint32_t)seed,
                                          (uint32_t)(seed >> 32), (uint32_t)step,
                                          (uint32_t)((uint64_t)step >> 32), valid, from, to,
                                          first_exchange);
  return check_launch("mh_propose_kernel");
}

int launch_compact(const int32_t* valid, const int32_t* from, const int32_t* to, int batch,
                   int32_t* c_sample, int32_t* c_from, int32_t* c_to, int32_t* c_count,
                   cudaStream_t st) {
  ProfScope prof_scope(NH_K_COMPACT, st);
  compact_kernel<<<1, 1024, 0, st>>>(valid, from, to, batch, c_sample, c_from, c_to, c_count);
  return check_launch("compact_kernel");
}

int launch_mh_accept(int8_t* spins, float* sign, double* logabs, int batch, int N,
                     const int32_t* c_sample, const int32_t* c_from, const int32_t* c_to,
                     const int32_t* c_count, const float* psign, const double* plogabs,
                     const float* lqr, uint64_t seed, int64_t step, int32_t* accepted,
                     cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = min((batch + 255) / 256, num_sms() * 4);
  ProfScope prof_scope(NH_K_MH_ACCEPT, st);
  mh_accept_kernel<<<grid, 256, 0, st>>>(spins, sign, logabs, N, c_sample, c_from, c_to, c_count,
                                         psign, plogabs, lqr, (uint32_t)seed, (uint32_t)(seed >> 32),
                                         (uint32_t)step, (uint32_t)((uint64_t)step >> 32),
                                         accepted);
  return check_launch("mh_accept_kernel");
}

int launch_wtilde(const float* W, float theta, int Lx, int Ly, int d, float* Wt, double* Wt64,
                  cudaStream_t st) {
  ProfScope prof_scope(NH_K_WTILDE, st);
  wtilde_kernel<<<1, 1024, 0, st>>>(W, theta, Lx, Ly, d, Wt, Wt64);
  return check_launch("wtilde_kernel");
}

}  // namespace nh

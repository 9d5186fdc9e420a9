// Packed observables on the connected-configuration engine (code/measure/transverse_spin.py,
// code/measure/dwave_packed.py).  The terms of one operator family O = sum_t O_t are enumerated
// for every sample as connections s -> s' (each term moves at most one up and one down
// electron), their amplitudes psi(s') run through the same pipeline as the local energy, and
// every local value <s|O_t|s'> psi(s') / psi(s) is binned by its term t:
//
//   NH_OBS_TRANSVERSE_SPIN  T[c, r] = <S+_a S-_{a+r}> (c = 0), <S-_a S+_{a+r}> (c = 1)
//   NH_OBS_PAIR             F[t]    = <A+(a, b) A(c_t, d_t)>, A+(a, b) = c+_{a up} c+_{b dn},
//                                     t over the nearest-neighbour bonds (site, axis) and their
//                                     two orientations (up end, down end)
//   NH_OBS_HOP              G[j]    = <c+_{i s} c_{j s}>
//
// The diagonal term of each family (r = 0; (c, d) = (a, b); j = i) is taken from the
// occupations, as the reference does.  <s|O_t|s'> is the coefficient of O_t^dag |s>, evaluated by
// applying the operators one by one with the Jordan-Wigner sign (occupied modes below each
// mode) from a per-sample bit mask and its word prefix counts.
#include "nh_common.cuh"

namespace nh {
namespace {

constexpr int kObsWarps = 8;
constexpr int kObsMaxWords = 64;  // 2N <= 2048 modes

struct ObsSample {
  const uint32_t* bits;  // 2N bits
  const int* pre;        // occupied modes in the words below
  __device__ int occ(int m) const { return (bits[m >> 5] >> (m & 31)) & 1; }
  __device__ int below(int m) const {
    return pre[m >> 5] + __popc(bits[m >> 5] & ((1u << (m & 31)) - 1u));
  }
};

// Applies ops[0], ops[1], ... (mode, create) to the sample's state; returns false when an
// operator annihilates the state, else the parity of the Jordan-Wigner sign in *par.
template <int K>
__device__ bool apply_ops(const ObsSample& S, const int (&mode)[K], const bool (&create)[K],
                          int* par) {
  int tm[K], tc[K];
  int nt = 0, p = 0;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int m = mode[k];
    int cur = S.occ(m), below = S.below(m);
    for (int u = 0; u < nt; ++u) {
      if (tm[u] == m) cur = tc[u];
      else if (tm[u] < m) below += tc[u] - S.occ(tm[u]);
    }
    if (create[k] ? cur : !cur) return false;
    p ^= below & 1;
    int u = 0;
    while (u < nt && tm[u] != m) ++u;
    if (u == nt) tm[nt++] = m;
    tc[u] = create[k] ? 1 : 0;
  }
  *par = p;
  return true;
}

struct ObsTerm {
  bool valid;
  int from, to, bin;
  double h;
};

__device__ ObsTerm obs_term(const ObsSample& S, int kind, int t, int a0, int a1, int Lx,
                            int Ly) {
  const int N = Lx * Ly;
  ObsTerm r{false, -1, -1, 0, 0.0};
  int par = 0;
  if (kind == NH_OBS_TRANSVERSE_SPIN) {
    const int chan = t / N, j = t - chan * N, a = a0;
    if (j == a) return r;
    const int au = a, ad = N + a, ju = j, jd = N + j;
    // O^dag |s> with O = S+_a S-_j: c(a up), c+(a dn), c(j dn), c+(j up); O = S-_a S+_j: the
    // spins swapped.
    const int m0[4] = {chan ? ad : au, chan ? au : ad, chan ? ju : jd, chan ? jd : ju};
    const bool cr[4] = {false, true, false, true};
    if (!apply_ops<4>(S, m0, cr, &par)) return r;
    r.from = chan ? pack_move(ju, ad) : pack_move(au, jd);
    r.to = chan ? pack_move(au, jd) : pack_move(ju, ad);
    const int xa = a / Ly, ya = a - xa * Ly, xj = j / Ly, yj = j - xj * Ly;
    int dx = xj - xa, dy = yj - ya;
    dx += dx < 0 ? Lx : 0;
    dy += dy < 0 ? Ly : 0;
    r.bin = chan * N + dx * Ly + dy;
  } else if (kind == NH_OBS_PAIR) {
    const int site = t >> 2, axis = (t >> 1) & 1, o = t & 1;
    const int x = site / Ly, y = site - x * Ly;
    const int hi = axis == 0 ? ((x + 1) % Lx) * Ly + y : x * Ly + (y + 1) % Ly;
    const int c = o == 0 ? site : hi, d = o == 0 ? hi : site;
    const int a = a0, b = a1;
    if (c == a && d == b) return r;  // the diagonal term n_{a up} n_{b dn}
    // O = c+(a up) c+(b dn) c(d dn) c(c up); O^dag |s>: c(a up), c(b dn), c+(d dn), c+(c up).
    const int m0[4] = {a, N + b, N + d, c};
    const bool cr[4] = {false, false, true, true};
    if (!apply_ops<4>(S, m0, cr, &par)) return r;
    if (c != a && d != b) {
      r.from = pack_move(a, N + b);
      r.to = pack_move(c, N + d);
    } else if (c == a) {
      r.from = pack_move(N + b, -1);
      r.to = pack_move(N + d, -1);
    } else {
      r.from = pack_move(a, -1);
      r.to = pack_move(c, -1);
    }
    r.bin = t;
  } else {  // NH_OBS_HOP: O = c+(i s) c(j s); O^dag |s>: c(i s), c+(j s)
    const int j = t, i = a0, sg = a1;
    if (j == i) return r;
    const int m0[2] = {sg * N + i, sg * N + j};
    const bool cr[2] = {false, true};
    if (!apply_ops<2>(S, m0, cr, &par)) return r;
    r.from = pack_move(sg * N + i, -1);
    r.to = pack_move(sg * N + j, -1);
    r.bin = j;
  }
  r.valid = true;
  r.h = par ? -1.0 : 1.0;
  return r;
}

// One warp per sample: EMIT = false counts the sample's connections, EMIT = true writes them at
// offsets[sample] in term order.
template <bool EMIT>
__global__ void __launch_bounds__(32 * kObsWarps) obs_kernel(
    const int8_t* __restrict__ spins, int batch, int Lx, int Ly, int kind, int a0, int a1,
    int32_t* counts, const int64_t* __restrict__ offsets, int32_t* owner, int32_t* from,
    int32_t* to, double* hval, int32_t* bin) {
  __shared__ uint32_t bits_s[kObsWarps][kObsMaxWords];
  __shared__ int pre_s[kObsWarps][kObsMaxWords + 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int N = Lx * Ly, M2 = 2 * N, words = (M2 + 31) >> 5;
  const int nterms = kind == NH_OBS_TRANSVERSE_SPIN ? 2 * N : (kind == NH_OBS_PAIR ? 4 * N : N);
  for (int b = blockIdx.x * kObsWarps + w; b < batch; b += gridDim.x * kObsWarps) {
    const int8_t* s = spins + (size_t)b * M2;
    for (int k = 0; k < words; ++k) {
      const int m = 32 * k + lane;
      const unsigned v = __ballot_sync(0xffffffffu, m < M2 && s[m] > 0);
      if (lane == 0) bits_s[w][k] = v;
    }
    __syncwarp();
    if (lane == 0) {
      int acc = 0;
      for (int k = 0; k < words; ++k) {
        pre_s[w][k] = acc;
        acc += __popc(bits_s[w][k]);
      }
    }
    __syncwarp();
    const ObsSample S{bits_s[w], pre_s[w]};
    int cnt = 0;
    const int64_t base = EMIT ? offsets[b] : 0;
    for (int t0 = 0; t0 < nterms; t0 += 32) {
      const int t = t0 + lane;
      ObsTerm r{false, -1, -1, 0, 0.0};
      if (t < nterms) r = obs_term(S, kind, t, a0, a1, Lx, Ly);
      const unsigned m = __ballot_sync(0xffffffffu, r.valid);
      if (EMIT && r.valid) {
        const int64_t pos = base + cnt + __popc(m & ((1u << lane) - 1u));
        owner[pos] = b;
        from[pos] = r.from;
        to[pos] = r.to;
        hval[pos] = r.h;
        bin[pos] = r.bin;
      }
      cnt += __popc(m);
    }
    if (!EMIT && lane == 0) counts[b] = cnt;
    __syncwarp();
  }
}

// V[owner, bin] = <s|O_t|s'> psi(s') / psi(s) for every connection (one per sample and bin).
__global__ void obs_scatter_kernel(const int64_t* __restrict__ total, const int32_t* owner,
                                   const int32_t* bin, const double* hval, const float* csign,
                                   const double* clogabs, const float* sign, const double* logabs,
                                   int nbins, double* V) {
  const int64_t n = *total;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int o = owner[c];
    const double ratio = (double)(csign[c] * sign[o]) * exp(clogabs[c] - logabs[o]);
    V[(size_t)o * nbins + bin[c]] = hval[c] * ratio;
  }
}

// out[bin] = (sum over the samples in order of V[., bin], plus the diagonal term from the
// occupations at diag_bin) / batch.
__global__ void obs_reduce_kernel(const double* __restrict__ V, const int8_t* __restrict__ spins,
                                  int batch, int N, int nbins, int kind, int a0, int a1,
                                  int diag_bin, double* out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nbins; k += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < batch; ++b) acc += V[(size_t)b * nbins + k];
    int diag = 0;
    const bool d0 = k == diag_bin, d1 = kind == NH_OBS_TRANSVERSE_SPIN && k == N;
    if (d0 || d1) {
      for (int b = 0; b < batch; ++b) {
        const int8_t* s = spins + (size_t)b * 2 * N;
        if (kind == NH_OBS_TRANSVERSE_SPIN) {
          const bool up = s[a0] > 0, dn = s[N + a0] > 0;
          diag += d0 ? (up && !dn) : (dn && !up);
        } else if (kind == NH_OBS_PAIR) {
          diag += s[a0] > 0 && s[N + a1] > 0;
        } else {
          diag += s[a1 * N + a0] > 0;
        }
      }
    }
    out[k] = (acc + (double)diag) / (double)batch;
  }
}

}  // namespace

int obs_terms(int kind, int N) {
  return kind == NH_OBS_TRANSVERSE_SPIN ? 2 * N : (kind == NH_OBS_PAIR ? 4 * N : N);
}

int launch_obs_list(const int8_t* spins, int batch, int Lx, int Ly, int kind, int a0, int a1,
                    int32_t* counts, int64_t* offsets, int32_t* owner, int32_t* from,
                    int32_t* to, double* hval, int32_t* bin, cudaStream_t st) {
  if (batch <= 0) return NH_OK;
  int grid = (batch + kObsWarps - 1) / kObsWarps;
  if (grid > num_sms() * 16) grid = num_sms() * 16;
  {
    ProfScope prof_scope(NH_K_OBS, st);
    obs_kernel<false><<<grid, 32 * kObsWarps, 0, st>>>(spins, batch, Lx, Ly, kind, a0, a1,
                                                       counts, nullptr, nullptr, nullptr,
                                                       nullptr, nullptr, nullptr);
  }
  int rc = check_launch("obs_kernel<count>");
  if (rc) return rc;
  if ((rc = launch_scan_counts(counts, batch, offsets, st))) return rc;
  ProfScope prof_scope(NH_K_OBS, st);
  obs_kernel<true><<<grid, 32 * kObsWarps, 0, st>>>(spins, batch, Lx, Ly, kind, a0, a1, counts,
                                                    offsets, owner, from, to, hval, bin);
  return check_launch("obs_kernel<emit>");
}

int launch_obs_reduce(const int8_t* spins, const float* sign, const double* logabs, int batch,
                      int N, int kind, int a0, int a1, int diag_bin, const int64_t* total,
                      const int32_t* owner, const int32_t* bin, const double* hval,
                      const float* csign, const double* clogabs, double* V, double* out,
                      cudaStream_t st) {
  const int nbins = obs_terms(kind, N);
  int rc = check_cuda(cudaMemsetAsync(V, 0, (size_t)batch * nbins * sizeof(double), st),
                      "observable: clear bins");
  if (rc) return rc;
  ProfScope prof_scope(NH_K_OBS, st);
  obs_scatter_kernel<<<num_sms() * 8, 256, 0, st>>>(total, owner, bin, hval, csign, clogabs,
                                                    sign, logabs, nbins, V);
  if ((rc = check_launch("obs_scatter_kernel"))) return rc;
  obs_reduce_kernel<<<(nbins + 255) / 256, 256, 0, st>>>(V, spins, batch, N, nbins, kind, a0, a1,
                                                        diag_bin, out);
  return check_launch("obs_reduce_kernel");
}

}  // namespace nh

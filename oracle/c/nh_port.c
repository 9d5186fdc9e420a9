/* Compiled CPU restatement of the projected Pfaffian-backflow amplitude (test infrastructure and
 * the timed CPU baseline; nothing in the library links it).
 *
 * Same algorithm and FP64 arithmetic as the numpy oracle (oracle/backflow.py,
 * oracle/projection.py, oracle/pfaffian.py), written for speed on the host's cores:
 *
 *   psi_P(s) = 1/G sum_g eta_g(s) psi(g s),   psi(s) = pf(F(s)) (-1)^(k(k-1)/2)
 *
 * with the backflow CNN of the graded configuration (periodic 3x3 convolutions, tanh-GELU
 * between layers; code/backflow/models.py:163-167), the occupied pairing block
 * F[p, q] = sum_a Y[p, a] Wt[2 s_p + s_q, r(p, q), a] Y[q, a] made exactly antisymmetric
 * (code/backflow/pf_kernel.py:156-166, 371-382), and the Parlett-Reid LTL^T log-Pfaffian with
 * partial pivoting (M. Wimmer, ACM TOMS 38, 30 (2012)), the stand-in for fermix.slogpf
 * (code/backflow/models.py:210).  Images g s are given by mode maps, s_g[map_g[m]] = s[m], and
 * eta_g is the parity of the permutation that sorts the mapped occupied modes
 * (code/states.py:274-279).  One configuration per OpenMP thread at a time.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Arithmetic type: double by default; the FP32 build (-DNHP_FP32) computes the CNN, the gather
 * and the Parlett-Reid updates in float, the precision of the reference's own JAX path
 * (FP32 with TF32 convolutions), and exports nhp_amplitudes_f32.  The log-sum of the pivots and
 * of the images stays in double in both builds. */
#ifdef NHP_FP32
typedef float real;
#define RTANH tanhf
#define RFABS fabsf
#define NHP_ENTRY nhp_amplitudes_f32
#else
typedef double real;
#define RTANH tanh
#define RFABS fabs
#define NHP_ENTRY nhp_amplitudes
#endif

typedef struct {
  int Lx, Ly, N, C, layers, d, n, G;
  const real* conv_w; /* layers concatenated: (C_out, C_in, 3, 3), C_in = 2 for layer 0 */
  const real* conv_b; /* (layers, C) */
  const real* Wt;     /* (4, N, d) */
  const int64_t* maps;  /* (G, 2N) */
} Net;

typedef struct {
  real* act[2]; /* padded planes (C, Lx + 2, Ly + 2) */
  real* Y;      /* (n, d) */
  real* A;      /* (n, n) */
  real* tmp;    /* (2n) Pfaffian row buffers */
  int* xyz;       /* (3n) x, y, spin of each occupied mode */
  int* occ;       /* (n) occupied modes of the image */
  int8_t* img;    /* (2N) */
} Work;

static real gelu_tanh(real x) {
  const real k0 = (real)0.7978845608028654; /* sqrt(2 / pi) */
  return (real)0.5 * x * ((real)1 + RTANH(k0 * (x + (real)0.044715 * x * x * x)));
}

/* Periodic halo of one padded plane. */
static void fill_halo(real* p, int Lx, int Ly) {
  const int P = Ly + 2;
  for (int x = 1; x <= Lx; ++x) {
    p[x * P] = p[x * P + Ly];
    p[x * P + Ly + 1] = p[x * P + 1];
  }
  memcpy(p, p + Lx * P, sizeof(real) * P);
  memcpy(p + (Lx + 1) * P, p + P, sizeof(real) * P);
}

/* Features of the image configuration: the last layer's channels, act[out] (C planes). */
static int cnn(const Net* net, Work* w, const int8_t* s) {
  const int Lx = net->Lx, Ly = net->Ly, N = net->N, C = net->C, P = Ly + 2;
  const int plane = (Lx + 2) * P;
  real* in = w->act[0];
  real* out = w->act[1];
  for (int ch = 0; ch < 2; ++ch) {
    real* p = in + ch * plane;
    for (int x = 0; x < Lx; ++x)
      for (int y = 0; y < Ly; ++y) p[(x + 1) * P + y + 1] = s[ch * N + x * Ly + y] > 0 ? (real)1 : (real)-1;
    fill_halo(p, Lx, Ly);
  }
  const real* wl = net->conv_w;
  int cin = 2;
  for (int l = 0; l < net->layers; ++l) {
    const real* bl = net->conv_b + (size_t)l * C;
    /* Four output channels at a time: each input row is loaded once for four FMA streams. */
    for (int o0 = 0; o0 < C; o0 += 4) {
      const int no = C - o0 < 4 ? C - o0 : 4;
      for (int x = 0; x < Lx; ++x) {
        real acc[4][64];
        for (int j = 0; j < no; ++j)
          for (int y = 0; y < Ly; ++y) acc[j][y] = bl[o0 + j];
        for (int i = 0; i < cin; ++i) {
          const real* pi = in + i * plane;
          for (int u = 0; u < 3; ++u) {
            const real* srow = pi + (x + u) * P;
            for (int v = 0; v < 3; ++v) {
              const real* src = srow + v;
              real wv[4];
              for (int j = 0; j < 4; ++j)
                wv[j] = j < no ? wl[((size_t)(o0 + j) * cin + i) * 9 + u * 3 + v] : (real)0;
              for (int y = 0; y < Ly; ++y) {
                const real sv = src[y];
                acc[0][y] += wv[0] * sv;
                acc[1][y] += wv[1] * sv;
                acc[2][y] += wv[2] * sv;
                acc[3][y] += wv[3] * sv;
              }
            }
          }
        }
        for (int j = 0; j < no; ++j) {
          real* dst = out + (o0 + j) * plane + (x + 1) * P + 1;
          if (l < net->layers - 1)
            for (int y = 0; y < Ly; ++y) dst[y] = gelu_tanh(acc[j][y]);
          else
            for (int y = 0; y < Ly; ++y) dst[y] = acc[j][y];
        }
      }
    }
    for (int o = 0; o < C; ++o) fill_halo(out + o * plane, Lx, Ly);
    wl += (size_t)C * cin * 9;
    cin = C;
    real* t = in;
    in = out;
    out = t;
  }
  return in == w->act[0] ? 0 : 1;
}

/* (sign, log|pf|) of the antisymmetric n x n matrix A (destroyed); tmp holds 2n values. */
static void slogpf(real* A, int n, real* tmp, double* sign, double* logabs) {
  double sg = 1.0, la = 0.0;
  for (int k = 0; k + 1 < n; k += 2) {
    int kp = k + 1;
    real best = RFABS(A[(size_t)(k + 1) * n + k]);
    for (int i = k + 2; i < n; ++i) {
      const real v = RFABS(A[(size_t)i * n + k]);
      if (v > best) {
        best = v;
        kp = i;
      }
    }
    if (kp != k + 1) { /* swap rows and columns k + 1 and kp */
      for (int j = 0; j < n; ++j) {
        const real t = A[(size_t)(k + 1) * n + j];
        A[(size_t)(k + 1) * n + j] = A[(size_t)kp * n + j];
        A[(size_t)kp * n + j] = t;
      }
      for (int i = 0; i < n; ++i) {
        const real t = A[(size_t)i * n + k + 1];
        A[(size_t)i * n + k + 1] = A[(size_t)i * n + kp];
        A[(size_t)i * n + kp] = t;
      }
      sg = -sg;
    }
    const real piv = A[(size_t)k * n + k + 1];
    if (piv == (real)0) {
      *sign = 0.0;
      *logabs = -INFINITY;
      return;
    }
    sg *= piv > 0 ? 1.0 : -1.0;
    la += log(fabs((double)piv));
    /* A[k+2:, k+2:] += tau a^T - a tau^T, tau = A[k, k+2:] / piv, a = A[k+2:, k+1], with tau
     * and a copied into contiguous buffers so that the row updates vectorise. */
    real* tau = tmp;
    real* acol = tmp + n;
    for (int j = k + 2; j < n; ++j) {
      tau[j] = A[(size_t)k * n + j] / piv;
      acol[j] = A[(size_t)j * n + k + 1];
    }
    for (int i = k + 2; i < n; ++i) {
      const real ti = tau[i], ai = acol[i];
      real* row = A + (size_t)i * n;
      for (int j = k + 2; j < n; ++j) row[j] += ti * acol[j] - ai * tau[j];
    }
  }
  *sign = sg;
  *logabs = la;
}

/* psi of one image configuration: (sign, log|psi|) including (-1)^(k(k-1)/2). */
static void amplitude(const Net* net, Work* w, const int8_t* img, double* sign, double* logabs) {
  const int N = net->N, n = net->n, d = net->d, Lx = net->Lx, Ly = net->Ly, P = Ly + 2;
  const int plane = (Lx + 2) * P;
  int k = 0;
  for (int m = 0; m < 2 * N; ++m)
    if (img[m] > 0) {
      if (k < n) w->occ[k] = m;
      ++k;
    }
  if (k != n) {
    *sign = 0.0;
    *logabs = -INFINITY;
    return;
  }
  const real* feat = w->act[cnn(net, w, img)];
  for (int p = 0; p < n; ++p) {
    const int m = w->occ[p], sp = m >= N, site = m - sp * N;
    const int x = site / Ly, y = site - x * Ly;
    for (int a = 0; a < d; ++a) w->Y[p * d + a] = feat[(sp * d + a) * plane + (x + 1) * P + y + 1];
  }
  int* X = w->xyz;
  int* Yc = X + n;
  int* S = Yc + n;
  for (int p = 0; p < n; ++p) {
    const int m = w->occ[p];
    S[p] = m >= N;
    X[p] = (m - S[p] * N) / Ly;
    Yc[p] = (m - S[p] * N) % Ly;
  }
  for (int p = 0; p < n; ++p) {
    const int sp = S[p], xp = X[p], yp = Yc[p];
    w->A[(size_t)p * n + p] = 0;
    for (int q = 0; q < p; ++q) {
      const int sq = S[q];
      int dx = xp - X[q], dy = yp - Yc[q];
      dx += dx < 0 ? Lx : 0;
      dy += dy < 0 ? Ly : 0;
      const int r = dx * Ly + dy;
      const int rn = (dx ? Lx - dx : 0) * Ly + (dy ? Ly - dy : 0);
      const real* wpq = net->Wt + ((size_t)(2 * sp + sq) * N + r) * d;
      const real* wqp = net->Wt + ((size_t)(2 * sq + sp) * N + rn) * d;
      real fpq = 0, fqp = 0;
      for (int a = 0; a < d; ++a) {
        const real yy = w->Y[p * d + a] * w->Y[q * d + a];
        fpq += yy * wpq[a];
        fqp += yy * wqp[a];
      }
      const real f = (real)0.5 * (fpq - fqp);
      w->A[(size_t)p * n + q] = f;
      w->A[(size_t)q * n + p] = -f;
    }
  }
  slogpf(w->A, n, w->tmp, sign, logabs);
  if (((long long)k * (k - 1) / 2) & 1) *sign = -*sign;
}

/* Projected (G = 8) or plain (G = 1, identity map) amplitudes of B configurations. */
int NHP_ENTRY(const int8_t* spins, int B, int Lx, int Ly, int C, int layers,
              const double* conv_w, const double* conv_b, const double* Wt, int n,
              const int64_t* maps, int G, double* sign, double* logabs, int nthreads) {
  if (!spins || !conv_w || !conv_b || !Wt || !maps || !sign || !logabs || B < 0 || G < 1 ||
      C < 2 || C % 2 || layers < 1 || n < 2 || Ly > 64 || G > 64)
    return -1; /* (the row accumulators hold 64 sites, the image sums 64 images) */
  /* Parameters in the arithmetic type (a copy in the FP32 build). */
  size_t n_w = 0;
  for (int l = 0, cin = 2; l < layers; ++l, cin = C) n_w += (size_t)C * cin * 9;
  const size_t n_b = (size_t)layers * C, n_t = (size_t)4 * Lx * Ly * (C / 2);
#ifdef NHP_FP32
  real* pw = malloc(sizeof(real) * (n_w + n_b + n_t));
  if (!pw) return -2;
  for (size_t i = 0; i < n_w; ++i) pw[i] = (real)conv_w[i];
  for (size_t i = 0; i < n_b; ++i) pw[n_w + i] = (real)conv_b[i];
  for (size_t i = 0; i < n_t; ++i) pw[n_w + n_b + i] = (real)Wt[i];
  Net net = {Lx, Ly, Lx * Ly, C, layers, C / 2, n, G, pw, pw + n_w, pw + n_w + n_b, maps};
#else
  (void)n_t;
  (void)n_b;
  Net net = {Lx, Ly, Lx * Ly, C, layers, C / 2, n, G, conv_w, conv_b, Wt, maps};
#endif
  const int N = net.N;
  int err = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel
  {
    Work w;
    const size_t plane = (size_t)(Lx + 2) * (Ly + 2);
    w.act[0] = malloc(sizeof(real) * plane * (C > 2 ? C : 2));
    w.act[1] = malloc(sizeof(real) * plane * (C > 2 ? C : 2));
    w.Y = malloc(sizeof(real) * (size_t)n * net.d);
    w.A = malloc(sizeof(real) * (size_t)n * n);
    w.tmp = malloc(sizeof(real) * (size_t)2 * n);
    w.xyz = malloc(sizeof(int) * (size_t)3 * n);
    w.occ = malloc(sizeof(int) * (size_t)n);
    w.img = malloc((size_t)2 * N);
    int* occs = malloc(sizeof(int) * (size_t)2 * N);
    const int ok = w.act[0] && w.act[1] && w.Y && w.A && w.tmp && w.xyz && w.occ && w.img && occs;
    if (!ok) {
#pragma omp atomic write
      err = -2;
    }
    /* Every thread meets the worksharing loop (an OpenMP requirement); a thread whose buffers
       are missing takes its share of iterations without computing them (err is set). */
#pragma omp for schedule(dynamic, 1)
    for (int b = 0; b < B; ++b) {
      if (!ok) continue;
      const int8_t* s = spins + (size_t)b * 2 * N;
      int k = 0;
      for (int m = 0; m < 2 * N; ++m)
        if (s[m] > 0) occs[k++] = m;
      double mx = -INFINITY, sg[64], la[64];
      for (int g = 0; g < G && g < 64; ++g) {
        const int64_t* mp = maps + (size_t)g * 2 * N;
        for (int m = 0; m < 2 * N; ++m) w.img[mp[m]] = s[m];
        int inv = 0; /* eta_g: parity of sorting the mapped occupied modes */
        for (int i = 0; i < k; ++i)
          for (int j = i + 1; j < k; ++j) inv += mp[occs[i]] > mp[occs[j]];
        amplitude(&net, &w, w.img, &sg[g], &la[g]);
        if (inv & 1) sg[g] = -sg[g];
        if (sg[g] != 0.0 && la[g] > mx) mx = la[g];
      }
      if (!isfinite(mx)) mx = 0.0;
      double tot = 0.0;
      for (int g = 0; g < G && g < 64; ++g) tot += sg[g] * exp(la[g] - mx);
      sign[b] = tot > 0 ? 1.0 : (tot < 0 ? -1.0 : 0.0);
      logabs[b] = log(fabs(tot)) + mx - log((double)G);
    }
    free(w.act[0]);
    free(w.act[1]);
    free(w.Y);
    free(w.A);
    free(w.tmp);
    free(w.xyz);
    free(w.occ);
    free(w.img);
    free(occs);
  }
#ifdef NHP_FP32
  free(pw);
#endif
  return err;
}

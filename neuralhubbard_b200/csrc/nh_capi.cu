// extern "C" entry points of libnh_b200.so (declared in include/nh_b200.h) and the host-side
// orchestration of the amplitude pipeline.  No entry point allocates device memory: scratch
// comes from the caller's workspace.
#include <stdarg.h>
#include <stdio.h>

#include "nh_common.cuh"

namespace nh {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return NH_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return NH_ERR_CUDA;
}

int check_launch(const char* what) { return check_cuda(cudaGetLastError(), what); }

int num_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t pipeline_bytes(int max_items, int n, int d) {
  size_t it = (size_t)(max_items > 0 ? max_items : 1);
  return align256(it * n * d * sizeof(float)) + align256(it * n * sizeof(int32_t)) +
         align256(it * sizeof(float)) * 2 + align256(it * sizeof(double)) +
         align256(it * sizeof(int32_t));
}

PipelineBuffers carve_pipeline(void* ws, int max_items, int n, int d) {
  size_t it = (size_t)(max_items > 0 ? max_items : 1);
  char* p = static_cast<char*>(ws);
  PipelineBuffers b;
  b.Y = reinterpret_cast<float*>(p);
  p += align256(it * n * d * sizeof(float));
  b.idx = reinterpret_cast<int32_t*>(p);
  p += align256(it * n * sizeof(int32_t));
  b.item_sign = reinterpret_cast<float*>(p);
  p += align256(it * sizeof(float));
  b.pf_sign = reinterpret_cast<float*>(p);
  p += align256(it * sizeof(float));
  b.pf_logabs = reinterpret_cast<double*>(p);
  p += align256(it * sizeof(double));
  b.pf_flags = reinterpret_cast<int32_t*>(p);
  return b;
}

int run_pipeline(const ConfigList& cl, const nh_backflow_params& p, const PipelineBuffers& b,
                 float* sign, double* logabs, int32_t* flags, cudaStream_t st) {
  const int n = p.n_up + p.n_dn, d = p.channels / 2;
  const int max_items = cl.n_cfg * cl.G;
  if (max_items <= 0) return NH_OK;
  int rc = launch_cnn(cl, p, 1, nullptr, b.Y, b.idx, b.item_sign, st);
  if (rc) return rc;
  if (cl.G == 1)
    return launch_pfaffian_gather(b.Y, b.idx, p.Wt, p.Lx, p.Ly, d, n, max_items, &cl,
                                  b.item_sign, sign, logabs, flags, st);
  rc = launch_pfaffian_gather(b.Y, b.idx, p.Wt, p.Lx, p.Ly, d, n, max_items, &cl, b.item_sign,
                              b.pf_sign, b.pf_logabs, b.pf_flags, st);
  if (rc) return rc;
  return launch_combine(b.pf_sign, b.pf_logabs, b.pf_flags, cl.G, cl.n_cfg, cl.n_cfg_dev, sign,
                        logabs, flags, st);
}

static int check_params(const nh_backflow_params* p) {
  if (!p || !p->conv_w || !p->conv_b || !p->Wt) return fail(NH_ERR_INVALID, "null parameter pointer");
  if (p->Lx < 3 || p->Ly < 3 || p->Lx * p->Ly > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "lattice %dx%d (3 <= L, N <= %d)", p->Lx, p->Ly, kMaxN);
  const int n = p->n_up + p->n_dn;
  if (p->n_up < 0 || p->n_dn < 0 || n < 2 || n % 2 || n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED, "electrons %d + %d (even total <= %d)", p->n_up, p->n_dn,
                kNumThreads);
  const int d = p->channels / 2;
  if (p->channels % 2 || (d != 8 && d != 16 && d != 32))
    return fail(NH_ERR_UNSUPPORTED, "channels %d (16, 32 or 64)", p->channels);
  if (p->layers < 1 || p->layers > 16) return fail(NH_ERR_UNSUPPORTED, "layers %d", p->layers);
  return NH_OK;
}

}  // namespace nh

using namespace nh;

extern "C" {

int nh_abi_version(void) { return NH_ABI_VERSION; }

const char* nh_last_error(void) { return g_err; }

int nh_build_wtilde(const float* W, float theta, int Lx, int Ly, int d, float* Wt, void* stream) {
  if (!W || !Wt) return fail(NH_ERR_INVALID, "build_wtilde: null pointer");
  if (Lx < 1 || Ly < 1 || Lx * Ly > kMaxN || d < 1)
    return fail(NH_ERR_UNSUPPORTED, "build_wtilde: %dx%d, d=%d", Lx, Ly, d);
  return launch_wtilde(W, theta, Lx, Ly, d, Wt, static_cast<cudaStream_t>(stream));
}

int nh_cnn_forward(const int8_t* spins, int batch, const nh_backflow_params* p, float* features,
                   void* stream) {
  if (!p || !p->conv_w || !p->conv_b) return fail(NH_ERR_INVALID, "cnn_forward: null parameters");
  if (!spins || !features || batch < 0) return fail(NH_ERR_INVALID, "cnn_forward: bad buffers");
  if (p->Lx < 3 || p->Ly < 3 || p->Lx * p->Ly > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "cnn_forward: lattice %dx%d", p->Lx, p->Ly);
  ConfigList cl{spins, nullptr, nullptr, nullptr, nullptr, batch, 1};
  return launch_cnn(cl, *p, 0, features, nullptr, nullptr, nullptr,
                    static_cast<cudaStream_t>(stream));
}

int nh_pairing_occ(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, void* stream) {
  if (!Y || !idx || !Wt || !F || batch < 0 || n < 1)
    return fail(NH_ERR_INVALID, "pairing_occ: bad arguments");
  if (Lx < 1 || Ly < 1 || Lx * Ly > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "pairing_occ: lattice %dx%d", Lx, Ly);
  return launch_pairing(Y, idx, Wt, Lx, Ly, d, n, batch, F, static_cast<cudaStream_t>(stream));
}

int nh_slogpf(const float* F, int n, int batch, float* sign, double* logabs, int32_t* flags,
              void* stream) {
  if (!F || !sign || !logabs || batch < 0) return fail(NH_ERR_INVALID, "slogpf: bad arguments");
  if (batch == 0) return NH_OK;
  return launch_pfaffian_from_F(F, n, batch, sign, logabs, flags,
                                static_cast<cudaStream_t>(stream));
}

size_t nh_amplitude_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p) {
  if (!p) return 0;
  return pipeline_bytes(batch * n_symm, p->n_up + p->n_dn, p->channels / 2);
}

int nh_amplitude(const int8_t* spins, int batch, int n_symm, const nh_backflow_params* p,
                 float* sign, double* logabs, int32_t* flags, void* workspace,
                 size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (!spins || !sign || !logabs || batch < 0) return fail(NH_ERR_INVALID, "amplitude: bad buffers");
  if (n_symm != 1 && n_symm != 8) return fail(NH_ERR_INVALID, "amplitude: n_symm %d (1 or 8)", n_symm);
  if (batch == 0) return NH_OK;
  const size_t need = nh_amplitude_workspace_bytes(batch, n_symm, p);
  if (!workspace || workspace_bytes < need)
    return fail(NH_ERR_WORKSPACE, "amplitude: workspace %zu < %zu bytes", workspace_bytes, need);
  const int n = p->n_up + p->n_dn, d = p->channels / 2;
  PipelineBuffers b = carve_pipeline(workspace, batch * n_symm, n, d);
  ConfigList cl{spins, nullptr, nullptr, nullptr, nullptr, batch, n_symm};
  return run_pipeline(cl, *p, b, sign, logabs, flags, static_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------------ local energy

static const int kDefaultChunk = 8192;

struct ElocLayout {
  int32_t* counts;
  int64_t* offsets;
  double* hval;
  int32_t* owner;
  int32_t* from;
  int32_t* to;
  float* csign;
  double* clogabs;
  void* pipe;
  size_t bytes;
};

static ElocLayout eloc_layout(void* ws, int batch, int n_symm, int chunk,
                              const nh_backflow_params* p, int n_dirs) {
  const int n = p->n_up + p->n_dn, d = p->channels / 2;
  const size_t cmax = (size_t)batch * n * n_dirs;
  char* q = static_cast<char*>(ws);
  ElocLayout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* r = q ? q + off : nullptr;
    off += align256(bytes);
    return r;
  };
  L.counts = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.offsets = reinterpret_cast<int64_t*>(take((size_t)(batch + 1) * 8));
  L.hval = reinterpret_cast<double*>(take(cmax * 8));
  L.owner = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.from = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.to = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.csign = reinterpret_cast<float*>(take(cmax * 4));
  L.clogabs = reinterpret_cast<double*>(take(cmax * 8));
  L.pipe = take(pipeline_bytes(chunk * n_symm, n, d));
  L.bytes = off;
  return L;
}

size_t nh_local_energy_workspace_bytes(int batch, int n_symm, int chunk_configs,
                                       const nh_backflow_params* p) {
  if (!p) return 0;
  int chunk = chunk_configs > 0 ? chunk_configs : kDefaultChunk;
  return eloc_layout(nullptr, batch, n_symm, chunk, p, 8).bytes;
}

int nh_local_energy(const int8_t* spins, const float* sign, const double* logabs, int batch,
                    int n_symm, const nh_backflow_params* p, const nh_hubbard_params* h,
                    int chunk_configs, double* eloc, int64_t* n_conn_out, void* workspace,
                    size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (!h || (h->n_dirs != 4 && h->n_dirs != 8)) return fail(NH_ERR_INVALID, "local_energy: n_dirs");
  if (!spins || !sign || !logabs || !eloc || batch < 0)
    return fail(NH_ERR_INVALID, "local_energy: bad buffers");
  if (n_symm != 1 && n_symm != 8) return fail(NH_ERR_INVALID, "local_energy: n_symm %d", n_symm);
  if (batch == 0) return NH_OK;
  const int chunk = chunk_configs > 0 ? chunk_configs : kDefaultChunk;
  const size_t need = nh_local_energy_workspace_bytes(batch, n_symm, chunk, p);
  if (!workspace || workspace_bytes < need)
    return fail(NH_ERR_WORKSPACE, "local_energy: workspace %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ElocLayout L = eloc_layout(workspace, batch, n_symm, chunk, p, 8);
  const int N = p->Lx * p->Ly, n = p->n_up + p->n_dn, d = p->channels / 2;
  if ((rc = launch_hop_count(spins, batch, p->Lx, p->Ly, h->n_dirs, L.counts, st))) return rc;
  if ((rc = launch_scan_counts(L.counts, batch, L.offsets, st))) return rc;
  if ((rc = launch_hop_emit(spins, batch, p->Lx, p->Ly, *h, L.offsets, nullptr, L.hval, L.owner,
                            L.from, L.to, st)))
    return rc;
  int64_t total = 0;
  if ((rc = check_cuda(cudaMemcpyAsync(&total, L.offsets + batch, sizeof(int64_t),
                                       cudaMemcpyDeviceToHost, st),
                       "local_energy: read connection count")))
    return rc;
  if ((rc = check_cuda(cudaStreamSynchronize(st), "local_energy: sync"))) return rc;
  if (n_conn_out) *n_conn_out = total;
  PipelineBuffers b = carve_pipeline(L.pipe, chunk * n_symm, n, d);
  for (int64_t c0 = 0; c0 < total; c0 += chunk) {
    const int nc = (int)((total - c0) < chunk ? (total - c0) : chunk);
    ConfigList cl{spins, L.owner + c0, L.from + c0, L.to + c0, nullptr, nc, n_symm};
    if ((rc = run_pipeline(cl, *p, b, L.csign + c0, L.clogabs + c0, nullptr, st))) return rc;
  }
  return launch_eloc_reduce(spins, sign, logabs, batch, N, h->U, L.offsets, L.hval, L.csign,
                            L.clogabs, eloc, st);
}

int nh_hop_list(const int8_t* spins, int batch, int Lx, int Ly, const nh_hubbard_params* h,
                int32_t* counts, int64_t* offsets, int32_t* rec, double* hval, void* stream) {
  if (!spins || !counts || !offsets || !h || batch < 0)
    return fail(NH_ERR_INVALID, "hop_list: bad arguments");
  if (h->n_dirs != 4 && h->n_dirs != 8) return fail(NH_ERR_INVALID, "hop_list: n_dirs");
  if (Lx < 3 || Ly < 3 || Lx * Ly > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "hop_list: lattice %dx%d", Lx, Ly);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if ((rc = launch_hop_count(spins, batch, Lx, Ly, h->n_dirs, counts, st))) return rc;
  if ((rc = launch_scan_counts(counts, batch, offsets, st))) return rc;
  if (!rec && !hval) return NH_OK;
  return launch_hop_emit(spins, batch, Lx, Ly, *h, offsets, rec, hval, nullptr, nullptr, nullptr,
                         st);
}

// ------------------------------------------------------------------ Metropolis sampler

struct MhLayout {
  int32_t *valid, *from, *to, *c_sample, *c_from, *c_to, *c_count;
  float* psign;
  double* plogabs;
  void* pipe;
  size_t bytes;
};

static MhLayout mh_layout(void* ws, int batch, int n_symm, const nh_backflow_params* p) {
  const int n = p->n_up + p->n_dn, d = p->channels / 2;
  char* q = static_cast<char*>(ws);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* r = q ? q + off : nullptr;
    off += align256(bytes);
    return r;
  };
  MhLayout L;
  L.valid = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.from = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.to = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.c_sample = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.c_from = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.c_to = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.c_count = reinterpret_cast<int32_t*>(take(4));
  L.psign = reinterpret_cast<float*>(take((size_t)batch * 4));
  L.plogabs = reinterpret_cast<double*>(take((size_t)batch * 8));
  L.pipe = take(pipeline_bytes(batch * n_symm, n, d));
  L.bytes = off;
  return L;
}

size_t nh_metropolis_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p) {
  if (!p) return 0;
  return mh_layout(nullptr, batch, n_symm, p).bytes;
}

int nh_metropolis_steps(int8_t* spins, float* sign, double* logabs, int batch, int n_symm,
                        const nh_backflow_params* p, int n_dirs, uint64_t seed, int64_t step0,
                        int nsteps, int32_t* accepted, void* workspace, size_t workspace_bytes,
                        void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (n_dirs != 4 && n_dirs != 8) return fail(NH_ERR_INVALID, "metropolis: n_dirs %d", n_dirs);
  if (!spins || !sign || !logabs || batch < 0 || nsteps < 0)
    return fail(NH_ERR_INVALID, "metropolis: bad buffers");
  if (n_symm != 1 && n_symm != 8) return fail(NH_ERR_INVALID, "metropolis: n_symm %d", n_symm);
  if (batch == 0 || nsteps == 0) return NH_OK;
  const size_t need = nh_metropolis_workspace_bytes(batch, n_symm, p);
  if (!workspace || workspace_bytes < need)
    return fail(NH_ERR_WORKSPACE, "metropolis: workspace %zu < %zu bytes", workspace_bytes, need);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  MhLayout L = mh_layout(workspace, batch, n_symm, p);
  const int n = p->n_up + p->n_dn, d = p->channels / 2, N = p->Lx * p->Ly;
  PipelineBuffers b = carve_pipeline(L.pipe, batch * n_symm, n, d);
  for (int t = 0; t < nsteps; ++t) {
    const int64_t step = step0 + t;
    if ((rc = launch_mh_propose(spins, batch, p->Lx, p->Ly, n_dirs, seed, step, L.valid, L.from,
                                L.to, st)))
      return rc;
    if ((rc = launch_compact(L.valid, L.from, L.to, batch, L.c_sample, L.c_from, L.c_to,
                             L.c_count, st)))
      return rc;
    ConfigList cl{spins, L.c_sample, L.c_from, L.c_to, L.c_count, batch, n_symm};
    if ((rc = run_pipeline(cl, *p, b, L.psign, L.plogabs, nullptr, st))) return rc;
    if ((rc = launch_mh_accept(spins, sign, logabs, batch, N, L.c_sample, L.c_from, L.c_to,
                               L.c_count, L.psign, L.plogabs, seed, step, accepted, st)))
      return rc;
  }
  return NH_OK;
}

}  // extern "C"

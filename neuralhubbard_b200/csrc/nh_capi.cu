// extern "C" entry points of libnh_b200.so (declared in include/nh_b200.h) and the host-side
// orchestration of the amplitude pipeline.  No entry point allocates device memory: scratch
// comes from the caller's workspace.
#include <stdarg.h>
#include <stdio.h>

#include <mutex>
#include <vector>

#include "nh_common.cuh"

namespace nh {

// ------------------------------------------------------------------ per-kernel timing
namespace {
struct ProfRecord {
  int id;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRecord> g_prof_pending;
std::vector<cudaEvent_t> g_prof_free;
double g_prof_ms[NH_K_COUNT];
int64_t g_prof_n[NH_K_COUNT];

cudaEvent_t prof_event() {
  if (!g_prof_free.empty()) {
    cudaEvent_t e = g_prof_free.back();
    g_prof_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

ProfScope::ProfScope(int id, cudaStream_t st) : id_(id), st_(st) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  if (!g_prof_on) return;
  a_ = prof_event();
  cudaEventRecord(a_, st_);
}

ProfScope::~ProfScope() {
  if (!a_) return;
  std::lock_guard<std::mutex> g(g_prof_mu);
  cudaEvent_t b = prof_event();
  cudaEventRecord(b, st_);
  g_prof_pending.push_back(ProfRecord{id_, a_, b});
}

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

int check_workspace(const void* ws, size_t have, size_t need, const char* who) {
  if (!ws || have < need)
    return fail(NH_ERR_WORKSPACE, "%s: workspace %zu < %zu bytes", who, ws ? have : 0, need);
  if (reinterpret_cast<uintptr_t>(ws) % 256)
    return fail(NH_ERR_INVALID, "%s: workspace %p is not 256-byte aligned", who, ws);
  return NH_OK;
}

int num_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Activation-plane scratch of the backflow network (0 when its planes fit in shared memory).
static size_t act_scratch_bytes(const nh_backflow_params& p) {
  const int N = p.Lx * p.Ly;
  return p.net == NH_NET_RESCONV ? resconv_scratch_bytes(N) : cnn_scratch_bytes(N, p.channels);
}

// Pivot-order records and refinement scratch: only where the FP64 refinement applies.
static size_t refine_bytes(size_t items, int n, int d) {
  if (n > kRefineMaxN) return 0;
  return align256(items * perm_stride(n) * sizeof(uint16_t)) + align256(items * sizeof(int32_t)) +
         align256(sizeof(int32_t)) + align256(refine_slice_bytes(n, d));
}

size_t pipeline_bytes(int max_items, const nh_backflow_params& p) {
  const size_t it = (size_t)(max_items > 0 ? max_items : 1);
  const size_t n = (size_t)(p.n_up + p.n_dn), d = (size_t)(p.channels / 2);
  return align256(it * n * d * sizeof(float)) + align256(it * n * sizeof(int32_t)) +
         align256(it * sizeof(float)) * 2 + align256(it * sizeof(double)) +
         align256(it * sizeof(int32_t)) * 2 + align256(sizeof(int32_t)) +
         align256(it * n * d * sizeof(double)) + align256(it * n * sizeof(int32_t)) +
         align256(sizeof(int32_t)) + align256(pfaffian_scratch_bytes((int)n)) +
         align256(act_scratch_bytes(p)) + align256(it * sizeof(float)) + refine_bytes(it, (int)n, (int)d);
}

PipelineBuffers carve_pipeline(void* ws, int max_items, const nh_backflow_params& prm) {
  const size_t it = (size_t)(max_items > 0 ? max_items : 1);
  const size_t n = (size_t)(prm.n_up + prm.n_dn), d = (size_t)(prm.channels / 2);
  char* p = static_cast<char*>(ws);
  auto take = [&](size_t bytes) {
    char* r = p;
    p += align256(bytes);
    return r;
  };
  PipelineBuffers b;
  b.Y = reinterpret_cast<float*>(take(it * n * d * sizeof(float)));
  b.idx = reinterpret_cast<int32_t*>(take(it * n * sizeof(int32_t)));
  b.item_sign = reinterpret_cast<float*>(take(it * sizeof(float)));
  b.pf_sign = reinterpret_cast<float*>(take(it * sizeof(float)));
  b.pf_logabs = reinterpret_cast<double*>(take(it * sizeof(double)));
  b.pf_flags = reinterpret_cast<int32_t*>(take(it * sizeof(int32_t)));
  b.list = reinterpret_cast<int32_t*>(take(it * sizeof(int32_t)));
  b.count = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  b.Y64 = reinterpret_cast<double*>(take(it * n * d * sizeof(double)));
  b.idx64 = reinterpret_cast<int32_t*>(take(it * n * sizeof(int32_t)));
  b.err = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  const size_t tri_bytes = pfaffian_scratch_bytes((int)n), act_bytes = act_scratch_bytes(prm);
  b.pf_tri = tri_bytes ? take(tri_bytes) : nullptr;
  b.cnn_act = act_bytes ? take(act_bytes) : nullptr;
  b.pf_ratio = reinterpret_cast<float*>(take(it * sizeof(float)));
  b.perm = nullptr;
  b.list32 = b.count32 = nullptr;
  b.slice = nullptr;
  if ((int)n <= kRefineMaxN) {
    b.perm = reinterpret_cast<uint16_t*>(take(it * perm_stride((int)n) * sizeof(uint16_t)));
    b.list32 = reinterpret_cast<int32_t*>(take(it * sizeof(int32_t)));
    b.count32 = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
    b.slice = take(refine_slice_bytes((int)n, prm.channels / 2));
  }
  return b;
}

// CNN -> gather + Pfaffian (FP32, recording each item's pivot order) -> FP64 features for the
// items flagged ill-conditioned or cancelling -> FP64 refinement of the log-Pfaffian with the
// FP32 pivot order (against the FP64 pairing block for those items, against the item's own FP32
// block for the others above refine_tau) -> combination of the symmetry images (or a copy for
// G = 1).  Beyond n = kRefineMaxN the flagged items are recomputed by the pivoted FP64 kernel.
int run_pipeline(const ConfigList& cl, const nh_backflow_params& p, const PipelineBuffers& b,
                 float* sign, double* logabs, int32_t* flags, cudaStream_t st) {
  const int n = p.n_up + p.n_dn, d = p.channels / 2;
  const int max_items = cl.n_cfg * cl.G;
  if (max_items <= 0) return NH_OK;
  int rc;
  const bool tc = p.cnn_mode == 1 || p.cnn_mode == 2 || p.pf_mode == 1;
  if (tc && (rc = check_cuda(cudaMemsetAsync(b.err, 0, sizeof(int32_t), st), "clear error word")))
    return rc;
  if (p.net == NH_NET_RESCONV && p.cnn_mode == 2) {
    rc = launch_resconv_tc(cl, p, b.Y, b.idx, b.item_sign, b.err, st);
  } else if (p.cnn_mode == 1 || p.cnn_mode == 2) {
    rc = launch_cnn_tc(cl, p, p.cnn_mode, b.Y, b.idx, b.item_sign, b.err, st);
  } else {
    CnnLaunch c{&cl, &p, 1, false, nullptr, nullptr, 0, nullptr, b.Y, b.idx, b.item_sign,
                b.cnn_act};
    rc = launch_cnn(c, st);
  }
  if (rc) return rc;
  if (p.ansatz == NH_ANSATZ_BCS) {
    // Determinant of the up x down block, FP32; flagged images again from FP64 features.
    DetLaunch dq{b.Y, b.idx, p.Wt, p.Lx, p.Ly, p.n_up, d, p.delta_d, cl.n_cfg_dev, cl.G,
                 max_items, nullptr, b.item_sign, b.pf_sign, b.pf_logabs, b.pf_flags,
                 b.pf_ratio, p.cond_tau, 0, false};
    if ((rc = launch_det(dq, st))) return rc;
    const bool fp64 = p.Wt64 && det_supported(p.n_up, d, true) &&
                      (p.cond_tau > 0.0 || (p.cancel_tau > 0.0 && cl.G > 1));
    if (fp64) {
      if ((rc = launch_image_mark(b.pf_sign, b.pf_logabs, b.pf_flags, b.pf_ratio, cl.G, cl.n_cfg,
                                  cl.n_cfg_dev, p.cancel_tau, p.cond_tau, p.cond_tau > 1.0, st)))
        return rc;
      if ((rc = launch_flagged(b.pf_flags, max_items, cl.n_cfg_dev, cl.G, b.list, b.count, st)))
        return rc;
      CnnLaunch c64{&cl, &p, 1, true, b.list, b.count, max_items, nullptr, b.Y64, b.idx64,
                    b.item_sign, b.cnn_act};
      if ((rc = launch_cnn(c64, st))) return rc;
      DetLaunch d64{b.Y64, b.idx64, p.Wt64, p.Lx, p.Ly, p.n_up, d, p.delta_d, b.count, 1,
                    max_items, b.list, b.item_sign, b.pf_sign, b.pf_logabs, b.pf_flags, nullptr,
                    0.0, NH_FLAG_GROWTH | NH_FLAG_REFINED, true};
      if ((rc = launch_det(d64, st))) return rc;
    }
    return launch_combine(b.pf_sign, b.pf_logabs, b.pf_flags, cl.G, cl.n_cfg, cl.n_cfg_dev, sign,
                          logabs, flags, p.cancel_tau, tc ? b.err : nullptr, st);
  }
  const bool refine = b.perm != nullptr;  // n <= kRefineMaxN
  PfGatherArgs g{b.Y, b.idx, p.Wt, p.Lx, p.Ly, d, n, cl.n_cfg_dev, cl.G, max_items, nullptr,
                 b.item_sign, b.pf_sign, b.pf_logabs, b.pf_flags, p.cond_tau, 0, false, b.pf_tri};
  g.ratio = b.pf_ratio;
  if (refine) {
    g.perm = b.perm;
    g.refine_tau = p.refine_tau;
  }
  if (p.pf_mode == 1)
    rc = launch_pfaffian_tc(g, 1, nullptr, b.err, st);
  else if (staged_supported(g))
    rc = launch_pfaffian_staged(g, st);
  else
    rc = launch_pfaffian_gather(g, st);
  if (rc) return rc;
  const bool fp64 = p.Wt64 && (p.cond_tau > 0.0 || (p.cancel_tau > 0.0 && cl.G > 1));
  if (fp64) {
    // cond_tau <= 1 flags every image (the all-FP64 form): no weighting then.
    if ((rc = launch_image_mark(b.pf_sign, b.pf_logabs, b.pf_flags, b.pf_ratio, cl.G, cl.n_cfg,
                                cl.n_cfg_dev, p.cancel_tau, p.cond_tau, p.cond_tau > 1.0, st)))
      return rc;
    if ((rc = launch_flagged(b.pf_flags, max_items, cl.n_cfg_dev, cl.G, b.list, b.count, st)))
      return rc;
    CnnLaunch c64{&cl, &p, 1, true, b.list, b.count, max_items, nullptr, b.Y64, b.idx64,
                  b.item_sign, b.cnn_act};
    if ((rc = launch_cnn(c64, st))) return rc;
    if (refine) {
      RefineLaunch r{n, d, 2, nullptr, b.Y64, b.idx64, p.Wt64, p.Lx, p.Ly, b.list, b.count,
                     max_items, b.perm, perm_stride(n), b.item_sign, b.pf_sign, b.pf_logabs,
                     b.pf_flags, b.slice};
      if ((rc = launch_refine(r, st))) return rc;
    } else {
      PfGatherArgs g64{b.Y64, b.idx64, p.Wt64, p.Lx, p.Ly, d, n, b.count, 1, max_items, b.list,
                       b.item_sign, b.pf_sign, b.pf_logabs, b.pf_flags, 0.0,
                       NH_FLAG_GROWTH | NH_FLAG_REFINED, true, b.pf_tri};
      if ((rc = launch_pfaffian_gather(g64, st))) return rc;
    }
  }
  if (refine && p.refine_tau > 0.0) {
    // Items above refine_tau that did not get FP64 features: refined against their FP32 block.
    const int skip = NH_FLAG_ZERO_PIVOT | NH_FLAG_REFINED;
    if ((rc = launch_flagged(b.pf_flags, max_items, cl.n_cfg_dev, cl.G, b.list32, b.count32, st,
                             kFlagNeedRefine, skip)))
      return rc;
    RefineLaunch r{n, d, 1, nullptr, b.Y, b.idx, p.Wt, p.Lx, p.Ly, b.list32, b.count32, max_items,
                   b.perm, perm_stride(n), b.item_sign, b.pf_sign, b.pf_logabs, b.pf_flags,
                   b.slice};
    if ((rc = launch_refine(r, st))) return rc;
  }
  return launch_combine(b.pf_sign, b.pf_logabs, b.pf_flags, cl.G, cl.n_cfg, cl.n_cfg_dev, sign,
                        logabs, flags, p.cancel_tau, tc ? b.err : nullptr, st);
}

// ------------------------------------------------------------------ persistent (fused) pipeline
// One fused launch computes every item's features and FP32 Pfaffian (items off a device work
// counter), then the FP64 refinement runs over device lists with in-kernel features: no
// per-item feature workspace, a launch sequence independent of the number of items.
struct FusedBuffers {
  float* pf_sign;
  double* pf_logabs;
  int32_t* pf_flags;
  float* pf_ratio;
  float* item_sign;
  uint16_t* perm;
  int32_t *list, *count, *list32, *count32, *queue;
  void* slice;
};

static bool fused_ok(const nh_backflow_params& p) {
  return p.ansatz == NH_ANSATZ_PFAFFIAN && fused_supported(p) && p.n_up + p.n_dn <= kRefineMaxN;
}

static size_t fused_bytes(size_t items, const nh_backflow_params& p) {
  const int n = p.n_up + p.n_dn;
  return align256(items * sizeof(float)) * 3 + align256(items * sizeof(double)) +
         align256(items * sizeof(int32_t)) * 3 + align256(items * perm_stride(n) * 2) +
         align256(sizeof(int32_t)) * 3 + align256(refine_slice_bytes(n, p.channels / 2));
}

static FusedBuffers carve_fused(void* ws, size_t items, const nh_backflow_params& p) {
  const int n = p.n_up + p.n_dn;
  char* q = static_cast<char*>(ws);
  auto take = [&](size_t bytes) {
    char* r = q;
    q += align256(bytes);
    return r;
  };
  FusedBuffers b;
  b.pf_sign = reinterpret_cast<float*>(take(items * sizeof(float)));
  b.pf_ratio = reinterpret_cast<float*>(take(items * sizeof(float)));
  b.item_sign = reinterpret_cast<float*>(take(items * sizeof(float)));
  b.pf_logabs = reinterpret_cast<double*>(take(items * sizeof(double)));
  b.pf_flags = reinterpret_cast<int32_t*>(take(items * sizeof(int32_t)));
  b.list = reinterpret_cast<int32_t*>(take(items * sizeof(int32_t)));
  b.list32 = reinterpret_cast<int32_t*>(take(items * sizeof(int32_t)));
  b.perm = reinterpret_cast<uint16_t*>(take(items * perm_stride(n) * 2));
  b.count = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  b.count32 = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  b.queue = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  b.slice = take(refine_slice_bytes(n, p.channels / 2));
  return b;
}

static int run_pipeline_fused(const ConfigList& cl, const nh_backflow_params& p,
                              const FusedBuffers& b, float* sign, double* logabs, int32_t* flags,
                              cudaStream_t st) {
  const int n = p.n_up + p.n_dn, d = p.channels / 2;
  const int max_items = cl.n_cfg * cl.G;
  if (max_items <= 0) return NH_OK;
  int rc;
  FusedLaunch f{cl, &p, b.pf_sign, b.pf_logabs, b.pf_flags, b.pf_ratio, b.item_sign, b.perm,
                b.queue};
  if ((rc = launch_pfaffian_fused(f, st))) return rc;
  const bool fp64 = p.Wt64 && (p.cond_tau > 0.0 || (p.cancel_tau > 0.0 && cl.G > 1));
  if (fp64) {
    if ((rc = launch_image_mark(b.pf_sign, b.pf_logabs, b.pf_flags, b.pf_ratio, cl.G, cl.n_cfg,
                                cl.n_cfg_dev, p.cancel_tau, p.cond_tau, p.cond_tau > 1.0, st)))
      return rc;
    if ((rc = launch_flagged(b.pf_flags, max_items, cl.n_cfg_dev, cl.G, b.list, b.count, st)))
      return rc;
    RefineLaunch r{n, d, 4, nullptr, nullptr, nullptr, p.Wt64, p.Lx, p.Ly, b.list, b.count,
                   max_items, b.perm, perm_stride(n), b.item_sign, b.pf_sign, b.pf_logabs,
                   b.pf_flags, b.slice};
    r.cl = cl;
    r.cnn_w = p.conv_w_packed;
    r.cnn_b = p.conv_b;
    r.C = p.channels;
    r.layers = p.layers;
    if ((rc = launch_refine(r, st))) return rc;
  }
  if (p.refine_tau > 0.0) {
    if ((rc = launch_flagged(b.pf_flags, max_items, cl.n_cfg_dev, cl.G, b.list32, b.count32, st,
                             kFlagNeedRefine, NH_FLAG_ZERO_PIVOT | NH_FLAG_REFINED)))
      return rc;
    RefineLaunch r{n, d, 3, nullptr, nullptr, nullptr, p.Wt, p.Lx, p.Ly, b.list32, b.count32,
                   max_items, b.perm, perm_stride(n), b.item_sign, b.pf_sign, b.pf_logabs,
                   b.pf_flags, b.slice};
    r.cl = cl;
    r.cnn_w = p.conv_w_packed;
    r.cnn_b = p.conv_b;
    r.C = p.channels;
    r.layers = p.layers;
    if ((rc = launch_refine(r, st))) return rc;
  }
  return launch_combine(b.pf_sign, b.pf_logabs, b.pf_flags, cl.G, cl.n_cfg, cl.n_cfg_dev, sign,
                        logabs, flags, p.cancel_tau, nullptr, st);
}

// The plain form (FP32 CNN on CUDA cores, CUDA-core Pfaffian) runs the fused pipeline wherever it
// applies; the other forms the unfused one.
static bool use_fused(const nh_backflow_params& p) {
  return p.cnn_mode == 0 && p.pf_mode == 0 && fused_ok(p);
}

static size_t amp_bytes(int items, const nh_backflow_params& p) {
  return use_fused(p) ? fused_bytes((size_t)(items > 0 ? items : 1), p) : pipeline_bytes(items, p);
}

static int run_amplitudes(const ConfigList& cl, const nh_backflow_params& p, void* ws, int items,
                          float* sign, double* logabs, int32_t* flags, cudaStream_t st) {
  if (use_fused(p))
    return run_pipeline_fused(cl, p, carve_fused(ws, (size_t)items, p), sign, logabs, flags, st);
  return run_pipeline(cl, p, carve_pipeline(ws, items, p), sign, logabs, flags, st);
}

static int check_params(const nh_backflow_params* p) {
  if (!p || !p->conv_w || !p->conv_b || !p->Wt || !p->conv_w_packed)
    return fail(NH_ERR_INVALID, "null parameter pointer (conv_w, conv_b, conv_w_packed, Wt)");
  if (p->Lx < 3 || p->Ly < 3 || p->Lx > 32 || p->Ly > 32)
    return fail(NH_ERR_UNSUPPORTED, "lattice %dx%d (3 <= Lx, Ly <= 32)", p->Lx, p->Ly);
  const int n = p->n_up + p->n_dn;
  if (p->n_up < 0 || p->n_dn < 0 || n < 2 || n % 2 || n > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "electrons %d + %d (even total <= %d)", p->n_up, p->n_dn,
                kMaxN);
  const int d = p->channels / 2;
  if (p->channels % 2 || (d != 8 && d != 16 && d != 32))
    return fail(NH_ERR_UNSUPPORTED, "channels %d (16, 32 or 64)", p->channels);
  if (p->layers < 1 || p->layers > 16) return fail(NH_ERR_UNSUPPORTED, "layers %d", p->layers);
  if (p->net != NH_NET_CNN && p->net != NH_NET_RESCONV)
    return fail(NH_ERR_INVALID, "net %d (NH_NET_CNN or NH_NET_RESCONV)", p->net);
  if (p->cnn_mode < 0 || p->cnn_mode > 2) return fail(NH_ERR_INVALID, "cnn_mode %d", p->cnn_mode);
  if (p->net == NH_NET_RESCONV) {
    if (p->channels != 64 || p->cnn_mode == 1 || (p->cnn_mode == 2 && !resconv_tc_supported(*p)))
      return fail(NH_ERR_UNSUPPORTED, "the residual network needs 64 channels and cnn_mode 0, "
                  "or cnn_mode 2 on a 16x16 lattice");
  } else if (p->cnn_mode && !cnn_tc_supported(*p)) {
    return fail(NH_ERR_UNSUPPORTED, "cnn_mode %d needs a 16x16 lattice, 32 channels, 4 layers",
                p->cnn_mode);
  }
  if (p->cnn_mode && !p->conv_w_tc) return fail(NH_ERR_INVALID, "cnn_mode %d: conv_w_tc is null",
                                                p->cnn_mode);
  if (p->pf_mode < 0 || p->pf_mode > 1) return fail(NH_ERR_INVALID, "pf_mode %d", p->pf_mode);
  if (p->pf_mode == 1 && n > kNumThreads)
    return fail(NH_ERR_UNSUPPORTED, "pf_mode 1 needs n <= %d", kNumThreads);
  if (p->ansatz != NH_ANSATZ_PFAFFIAN && p->ansatz != NH_ANSATZ_BCS)
    return fail(NH_ERR_INVALID, "ansatz %d (NH_ANSATZ_PFAFFIAN or NH_ANSATZ_BCS)", p->ansatz);
  if (p->ansatz == NH_ANSATZ_BCS &&
      (p->n_up != p->n_dn || !det_supported(p->n_up, d, false) || p->pf_mode != 0))
    return fail(NH_ERR_UNSUPPORTED, "BCS ansatz: n_up == n_dn <= %d, d = 16, pf_mode 0 "
                "(got %d, %d, d %d, pf_mode %d)", kDetMaxNh, p->n_up, p->n_dn, d, p->pf_mode);
  return NH_OK;
}

}  // namespace nh

using namespace nh;

extern "C" {

int nh_abi_version(void) { return NH_ABI_VERSION; }

int nh_profile_enable(int on) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_prof_on = on != 0;
  return NH_OK;
}

int nh_profile_read(double* ms, int64_t* launches, int n_ids) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  int rc = NH_OK;
  for (const ProfRecord& r : g_prof_pending) {
    float t = 0.0f;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess && rc == NH_OK) rc = check_cuda(e, "profile_read");
    if (r.id >= 0 && r.id < NH_K_COUNT) {
      g_prof_ms[r.id] += t;
      g_prof_n[r.id] += 1;
    }
    g_prof_free.push_back(r.a);
    g_prof_free.push_back(r.b);
  }
  g_prof_pending.clear();
  for (int i = 0; i < n_ids && i < NH_K_COUNT; ++i) {
    if (ms) ms[i] = g_prof_ms[i];
    if (launches) launches[i] = g_prof_n[i];
  }
  for (int i = 0; i < NH_K_COUNT; ++i) {
    g_prof_ms[i] = 0.0;
    g_prof_n[i] = 0;
  }
  return rc;
}

const char* nh_last_error(void) { return g_err; }

int nh_build_wtilde(const float* W, float theta, int Lx, int Ly, int d, float* Wt, double* Wt64,
                    void* stream) {
  if (!W || !Wt) return fail(NH_ERR_INVALID, "build_wtilde: null pointer");
  if (Lx < 1 || Ly < 1 || Lx * Ly > kMaxN || d < 1)
    return fail(NH_ERR_UNSUPPORTED, "build_wtilde: %dx%d, d=%d", Lx, Ly, d);
  return launch_wtilde(W, theta, Lx, Ly, d, Wt, Wt64, static_cast<cudaStream_t>(stream));
}

int nh_pack_cnn_weights(const float* conv_w, int channels, int layers, float* packed,
                        void* stream) {
  if (!conv_w || !packed || channels < 1 || layers < 1)
    return fail(NH_ERR_INVALID, "pack_cnn_weights: bad arguments");
  return launch_pack_cnn(conv_w, channels, layers, packed, static_cast<cudaStream_t>(stream));
}

size_t nh_pack_resconv_weights_floats(int channels, int blocks) {
  return channels > 0 && blocks > 0 ? resconv_packed_floats(channels, blocks) : 0;
}

int nh_pack_resconv_weights(const float* conv_w, int channels, int blocks, float* packed,
                            void* stream) {
  if (!conv_w || !packed || blocks < 1) return fail(NH_ERR_INVALID, "pack_resconv_weights: "
                                                     "bad arguments");
  if (channels != 64)
    return fail(NH_ERR_UNSUPPORTED, "pack_resconv_weights: %d channels (64)", channels);
  return launch_pack_resconv(conv_w, channels, blocks, packed, static_cast<cudaStream_t>(stream));
}

size_t nh_pack_resconv_weights_tc_bytes(int blocks) {
  return blocks > 0 ? resconv_tc_packed_bytes(blocks) : 0;
}

int nh_pack_resconv_weights_tc(const float* conv_w, int channels, int blocks, void* packed,
                               void* stream) {
  if (!conv_w || !packed || blocks < 1)
    return fail(NH_ERR_INVALID, "pack_resconv_weights_tc: bad arguments");
  if (channels != 64)
    return fail(NH_ERR_UNSUPPORTED, "pack_resconv_weights_tc: %d channels (64)", channels);
  return launch_pack_resconv_tc(conv_w, blocks, packed, static_cast<cudaStream_t>(stream));
}

size_t nh_pack_cnn_weights_tc_bytes(void) { return cnn_tc_packed_bytes(); }

int nh_pack_cnn_weights_tc(const float* conv_w, int channels, int layers, void* packed,
                           void* stream) {
  if (!conv_w || !packed) return fail(NH_ERR_INVALID, "pack_cnn_weights_tc: null pointer");
  if (channels != 32 || layers != 4)
    return fail(NH_ERR_UNSUPPORTED, "pack_cnn_weights_tc: %d channels, %d layers (32, 4)",
                channels, layers);
  return launch_pack_cnn_tc(conv_w, static_cast<uint16_t*>(packed),
                            static_cast<cudaStream_t>(stream));
}

int nh_cnn_forward(const int8_t* spins, int batch, const nh_backflow_params* p, float* features,
                   void* stream) {
  if (!p || !p->conv_w_packed || !p->conv_b)
    return fail(NH_ERR_INVALID, "cnn_forward: null parameters");
  if (!spins || !features || batch < 0) return fail(NH_ERR_INVALID, "cnn_forward: bad buffers");
  if (p->Lx < 3 || p->Ly < 3 || p->Lx > 32 || p->Ly > 32)
    return fail(NH_ERR_UNSUPPORTED, "cnn_forward: lattice %dx%d", p->Lx, p->Ly);
  ConfigList cl{spins, nullptr, nullptr, nullptr, nullptr, batch, 1};
  CnnLaunch c{&cl, p, 0, false, nullptr, nullptr, 0, features, nullptr, nullptr, nullptr,
              nullptr};
  return launch_cnn(c, static_cast<cudaStream_t>(stream));
}

int nh_pairing_occ(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, void* stream) {
  if (!Y || !idx || !Wt || !F || batch < 0 || n < 1)
    return fail(NH_ERR_INVALID, "pairing_occ: bad arguments");
  if (Lx < 1 || Ly < 1 || Lx * Ly > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "pairing_occ: lattice %dx%d", Lx, Ly);
  return launch_pairing(Y, idx, Wt, Lx, Ly, d, n, batch, F, static_cast<cudaStream_t>(stream));
}

// Layout: [per-CTA triangles when n exceeds shared memory][refinement list (batch)][count]
// [pivot orders (batch) and the refinement's per-CTA slice, n <= kRefineMaxN].
size_t nh_slogpf_workspace_bytes(int n, int batch) {
  const bool ok = n > 0 && n % 2 == 0 && n <= kMaxN;
  const size_t tri = ok ? align256(pfaffian_scratch_bytes(n)) : 0;
  const size_t b = (size_t)(batch > 0 ? batch : 1);
  const size_t ref = (ok && n <= kRefineMaxN)
                         ? align256(b * perm_stride(n) * sizeof(uint16_t)) +
                               align256(refine_slice_bytes(n, 16))
                         : 0;
  return tri + align256(b * sizeof(int32_t)) + align256(sizeof(int32_t)) + ref;
}

int nh_slogpf(const float* F, int n, int batch, double cond_tau, float* sign, double* logabs,
              int32_t* flags, void* workspace, size_t workspace_bytes, void* stream) {
  if (!F || !sign || !logabs || batch < 0) return fail(NH_ERR_INVALID, "slogpf: bad arguments");
  if (n <= 0 || n % 2 || n > kMaxN)
    return fail(NH_ERR_UNSUPPORTED, "slogpf: n=%d must be even and <= %d", n, kMaxN);
  const bool refine = cond_tau > 0.0;
  if (refine && !flags) return fail(NH_ERR_INVALID, "slogpf: refinement needs flags");
  if (batch == 0) return NH_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Scratch: the refinement list (and, n <= kRefineMaxN, the pivot orders) when refining, the
  // FP32 triangles beyond n = 256, the FP64 ones beyond 236.
  const bool scratch = pfaffian_needs_scratch(n, refine);
  int rc;
  if ((refine || scratch) &&
      (rc = check_workspace(workspace, workspace_bytes, nh_slogpf_workspace_bytes(n, batch),
                            "slogpf")))
    return rc;
  const size_t tri_bytes = align256(pfaffian_scratch_bytes(n));
  void* tri = tri_bytes ? workspace : nullptr;
  char* w = static_cast<char*>(workspace) + tri_bytes;
  int32_t* list = refine ? reinterpret_cast<int32_t*>(w) : nullptr;
  w += align256((size_t)batch * sizeof(int32_t));
  int32_t* count = refine ? reinterpret_cast<int32_t*>(w) : nullptr;
  w += align256(sizeof(int32_t));
  const bool static_pivot = refine && n <= kRefineMaxN;
  uint16_t* perm = static_pivot ? reinterpret_cast<uint16_t*>(w) : nullptr;
  void* slice = static_pivot ? w + align256((size_t)batch * perm_stride(n) * sizeof(uint16_t))
                             : nullptr;
  rc = launch_pfaffian_from_F(F, n, batch, nullptr, nullptr, false, cond_tau, 0, sign, logabs,
                              flags, tri, st, perm, 0.0);
  if (rc || !refine) return rc;
  if ((rc = launch_flagged(flags, batch, nullptr, 1, list, count, st))) return rc;
  if (static_pivot) {
    RefineLaunch r{n, 16, 0, F, nullptr, nullptr, nullptr, 0, 0, list, count, batch, perm,
                   perm_stride(n), nullptr, sign, logabs, flags, slice};
    return launch_refine(r, st);
  }
  return launch_pfaffian_from_F(F, n, batch, list, count, true, 0.0,
                                NH_FLAG_GROWTH | NH_FLAG_REFINED, sign, logabs, flags, tri, st);
}

size_t nh_amplitude_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p) {
  if (!p) return 0;
  return amp_bytes(batch * n_symm, *p);
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
  if ((rc = check_workspace(workspace, workspace_bytes, need, "amplitude"))) return rc;
  ConfigList cl{spins, nullptr, nullptr, nullptr, nullptr, batch, n_symm};
  return run_amplitudes(cl, *p, workspace, batch * n_symm, sign, logabs, flags,
                        static_cast<cudaStream_t>(stream));
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
  int32_t* chunk_cnt;  // device work count of every chunk of the connection list
  int n_chunks;
  void* pipe;
  size_t bytes;
};

static ElocLayout eloc_layout(void* ws, int batch, int n_symm, int chunk,
                              const nh_backflow_params* p, int n_dirs) {
  const int n = p->n_up + p->n_dn;
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
  // chunk 0: the persistent path, one pass over the whole connection list
  const size_t ch = chunk > 0 ? (size_t)chunk : cmax;
  L.n_chunks = (int)((cmax + ch - 1) / ch);
  L.chunk_cnt = reinterpret_cast<int32_t*>(take((size_t)(L.n_chunks > 0 ? L.n_chunks : 1) * 4));
  L.pipe = take(chunk > 0 ? pipeline_bytes(chunk * n_symm, *p) : fused_bytes(cmax * n_symm, *p));
  L.bytes = off;
  return L;
}

// chunk_configs <= 0 selects the persistent path where the form runs the fused pipeline (plain
// FP32 CNN and CUDA-core Pfaffian); the tensor-core forms keep their own kernels, chunked.
static int eloc_chunk(int chunk_configs, const nh_backflow_params* p) {
  if (chunk_configs > 0) return chunk_configs;
  return use_fused(*p) ? 0 : kDefaultChunk;
}

size_t nh_local_energy_workspace_bytes(int batch, int n_symm, int chunk_configs,
                                       const nh_backflow_params* p) {
  if (!p) return 0;
  return eloc_layout(nullptr, batch, n_symm, eloc_chunk(chunk_configs, p), p, 8).bytes;
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
  const int chunk = eloc_chunk(chunk_configs, p);
  const size_t need = nh_local_energy_workspace_bytes(batch, n_symm, chunk, p);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "local_energy"))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ElocLayout L = eloc_layout(workspace, batch, n_symm, chunk, p, 8);
  const int N = p->Lx * p->Ly, n = p->n_up + p->n_dn;
  if ((rc = launch_hop_count(spins, batch, p->Lx, p->Ly, h->n_dirs, L.counts, st))) return rc;
  if ((rc = launch_scan_counts(L.counts, batch, L.offsets, st))) return rc;
  // At most n_dirs hops per electron: the emitted list never exceeds cmax (the emit kernel
  // also stops at cmax).
  const int64_t cmax = (int64_t)batch * n * 8;
  if ((rc = launch_hop_emit(spins, batch, p->Lx, p->Ly, *h, L.offsets, cmax, nullptr, L.hval,
                            L.owner, L.from, L.to, st)))
    return rc;
  // The ragged connection list is processed in one persistent pass (chunk 0: items off a device
  // work counter) or in chunks; either way the work counts live on the device, so the launch
  // sequence does not depend on the data.  Without n_conn_out the call never waits for the GPU
  // (chunked: all ceil(cmax / chunk) chunks run, the empty ones exit at once); with it, the count
  // is read back first and only the chunks that hold connections are launched.
  if ((rc = launch_chunk_counts(L.offsets + batch, L.n_chunks, chunk > 0 ? chunk : (int)cmax,
                                L.chunk_cnt, st)))
    return rc;
  int used = L.n_chunks;
  if (n_conn_out) {
    int64_t total = 0;
    if ((rc = check_cuda(cudaMemcpyAsync(&total, L.offsets + batch, sizeof(int64_t),
                                         cudaMemcpyDeviceToHost, st),
                         "local_energy: read connection count")))
      return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(st), "local_energy: sync"))) return rc;
    *n_conn_out = total;
    used = chunk > 0 ? (int)((total + chunk - 1) / chunk) : (total > 0 ? 1 : 0);
  }
  if (chunk == 0) {  // persistent: one fused pass over every connection
    if (used > 0) {
      ConfigList cl{spins, L.owner, L.from, L.to, L.chunk_cnt, (int)cmax, n_symm};
      FusedBuffers fb = carve_fused(L.pipe, (size_t)cmax * n_symm, *p);
      if ((rc = run_pipeline_fused(cl, *p, fb, L.csign, L.clogabs, nullptr, st))) return rc;
    }
    return launch_eloc_reduce(spins, sign, logabs, batch, N, h->U, L.offsets, L.hval, L.csign,
                              L.clogabs, eloc, st);
  }
  PipelineBuffers b = carve_pipeline(L.pipe, chunk * n_symm, *p);
  for (int i = 0; i < used; ++i) {
    const int64_t c0 = (int64_t)i * chunk;
    ConfigList cl{spins, L.owner + c0, L.from + c0, L.to + c0, L.chunk_cnt + i, chunk, n_symm};
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
  // rec / hval must hold batch * (electrons per configuration) * n_dirs records.
  return launch_hop_emit(spins, batch, Lx, Ly, *h, offsets, INT64_MAX, rec, hval, nullptr,
                         nullptr, nullptr, st);
}

// ------------------------------------------------------------------ Metropolis sampler

struct MhLayout {
  int32_t *valid, *from, *to, *c_sample, *c_from, *c_to, *c_count;
  float* psign;
  double* plogabs;
  float* lqr;  // learned proposal: log q(reverse) - log q(move) per chain
  void* pipe;
  size_t bytes;
};

static MhLayout mh_layout(void* ws, int batch, int n_symm, const nh_backflow_params* p) {
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
  L.lqr = reinterpret_cast<float*>(take((size_t)batch * 4));
  L.pipe = take(amp_bytes(batch * n_symm, *p));
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
  return nh_metropolis_steps_mixed(spins, sign, logabs, batch, n_symm, p, n_dirs, batch, seed,
                                   step0, nsteps, accepted, workspace, workspace_bytes, stream);
}

int nh_metropolis_steps_mixed(int8_t* spins, float* sign, double* logabs, int batch, int n_symm,
                              const nh_backflow_params* p, int n_dirs, int first_exchange,
                              uint64_t seed, int64_t step0, int nsteps, int32_t* accepted,
                              void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (n_dirs != 4 && n_dirs != 8) return fail(NH_ERR_INVALID, "metropolis: n_dirs %d", n_dirs);
  if (!spins || !sign || !logabs || batch < 0 || nsteps < 0)
    return fail(NH_ERR_INVALID, "metropolis: bad buffers");
  if (first_exchange < 0 || first_exchange > batch)
    return fail(NH_ERR_INVALID, "metropolis: first_exchange %d outside [0, %d]", first_exchange,
                batch);
  if (n_symm != 1 && n_symm != 8) return fail(NH_ERR_INVALID, "metropolis: n_symm %d", n_symm);
  if (batch == 0 || nsteps == 0) return NH_OK;
  const size_t need = nh_metropolis_workspace_bytes(batch, n_symm, p);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "metropolis"))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  MhLayout L = mh_layout(workspace, batch, n_symm, p);
  const int N = p->Lx * p->Ly;
  for (int t = 0; t < nsteps; ++t) {
    const int64_t step = step0 + t;
    if ((rc = launch_mh_propose(spins, batch, p->Lx, p->Ly, n_dirs, seed, step, L.valid, L.from,
                                L.to, st, first_exchange)))
      return rc;
    if ((rc = launch_compact(L.valid, L.from, L.to, batch, L.c_sample, L.c_from, L.c_to,
                             L.c_count, st)))
      return rc;
    ConfigList cl{spins, L.c_sample, L.c_from, L.c_to, L.c_count, batch, n_symm};
    if ((rc = run_amplitudes(cl, *p, L.pipe, batch * n_symm, L.psign, L.plogabs, nullptr, st)))
      return rc;
    if ((rc = launch_mh_accept(spins, sign, logabs, batch, N, L.c_sample, L.c_from, L.c_to,
                               L.c_count, L.psign, L.plogabs, nullptr, seed, step, accepted,
                               st)))
      return rc;
  }
  return NH_OK;
}

size_t nh_metropolis_learned_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p) {
  return nh_metropolis_workspace_bytes(batch, n_symm, p);
}

int nh_metropolis_steps_learned(int8_t* spins, float* sign, double* logabs, int batch,
                                int n_symm, const nh_backflow_params* p,
                                const nh_proposal_params* q, uint64_t seed, int64_t step0,
                                int nsteps, int32_t* accepted, void* workspace,
                                size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if ((rc = check_proposal(q))) return rc;
  if (q->Lx != p->Lx || q->Ly != p->Ly)
    return fail(NH_ERR_INVALID, "metropolis_learned: proposal lattice %dx%d != %dx%d", q->Lx,
                q->Ly, p->Lx, p->Ly);
  if (!spins || !sign || !logabs || batch < 0 || nsteps < 0)
    return fail(NH_ERR_INVALID, "metropolis_learned: bad buffers");
  if (n_symm != 1 && n_symm != 8)
    return fail(NH_ERR_INVALID, "metropolis_learned: n_symm %d", n_symm);
  if (batch == 0 || nsteps == 0) return NH_OK;
  const size_t need = nh_metropolis_learned_workspace_bytes(batch, n_symm, p);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "metropolis_learned"))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  MhLayout L = mh_layout(workspace, batch, n_symm, p);
  const int N = p->Lx * p->Ly;
  for (int t = 0; t < nsteps; ++t) {
    const int64_t step = step0 + t;
    if ((rc = launch_prop_sample(spins, batch, *q, seed, step, L.valid, L.from, L.to, L.lqr, st)))
      return rc;
    if ((rc = launch_compact(L.valid, L.from, L.to, batch, L.c_sample, L.c_from, L.c_to,
                             L.c_count, st)))
      return rc;
    ConfigList cl{spins, L.c_sample, L.c_from, L.c_to, L.c_count, batch, n_symm};
    if ((rc = run_amplitudes(cl, *p, L.pipe, batch * n_symm, L.psign, L.plogabs, nullptr, st)))
      return rc;
    if ((rc = launch_mh_accept(spins, sign, logabs, batch, N, L.c_sample, L.c_from, L.c_to,
                               L.c_count, L.psign, L.plogabs, L.lqr, seed, step, accepted, st)))
      return rc;
  }
  return NH_OK;
}

// ------------------------------------------------------------------ backward (Jacobian)

int nh_pfaffian_adjoint(const float* F, int n, int batch, float* G, int32_t* flags,
                        void* stream) {
  if (!F || !G || batch < 0) return fail(NH_ERR_INVALID, "pfaffian_adjoint: bad arguments");
  if (n <= 0 || n % 2 || n > kGradMaxN)
    return fail(NH_ERR_UNSUPPORTED, "pfaffian_adjoint: n = %d (even, <= %d)", n, kGradMaxN);
  return launch_pf_adjoint(F, G, n, batch, nullptr, nullptr, 1, flags,
                           static_cast<cudaStream_t>(stream));
}

int nh_pairing_occ_vjp(const float* Y, const int32_t* idx, const float* Wt, const float* G,
                       int Lx, int Ly, int d, int n, int batch, float* dY, float* dWt,
                       void* stream) {
  if (!Y || !idx || !Wt || !G || !dY || !dWt || batch < 0 || n < 1)
    return fail(NH_ERR_INVALID, "pairing_occ_vjp: bad arguments");
  if (Lx < 1 || Ly < 1 || 2 * Lx * Ly > 512 || n > kGradMaxN)
    return fail(NH_ERR_UNSUPPORTED, "pairing_occ_vjp: lattice %dx%d, n = %d", Lx, Ly, n);
  return launch_pairing_vjp(G, Y, idx, Wt, Lx, Ly, d, n, 1, batch, dY, dWt, nullptr, 0, 0, 0.0f,
                            static_cast<cudaStream_t>(stream));
}

int64_t nh_param_count(const nh_backflow_params* p) {
  if (!p || p->net != NH_NET_CNN || p->layers < 1 || p->channels < 1) return 0;
  const int64_t C = p->channels, N = (int64_t)p->Lx * p->Ly;
  return (C * 2 * 9 + C) + (int64_t)(p->layers - 1) * (C * C * 9 + C) + 3 * N * (C / 2) + 1;
}

static const int kJacChunkItems = 4096;

static int jac_chunk_samples(int batch, int n_symm) {
  const int cs = kJacChunkItems / n_symm;
  return batch < cs ? (batch > 0 ? batch : 1) : cs;
}

size_t nh_log_jacobian_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p) {
  if (!p || (n_symm != 1 && n_symm != 8)) return 0;
  const size_t items = (size_t)jac_chunk_samples(batch, n_symm) * n_symm;
  const size_t n = (size_t)(p->n_up + p->n_dn), d = (size_t)(p->channels / 2);
  return pipeline_bytes((int)items, *p) + align256(items * n * n * sizeof(float)) +
         align256(items * n * d * sizeof(float));
}

int nh_log_jacobian(const int8_t* spins, int batch, int n_symm, const nh_backflow_params* p,
                    const float* W, float theta, float* jac, float* sign, double* logabs,
                    int32_t* flags, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (!spins || !W || !jac || !sign || !logabs || batch < 0)
    return fail(NH_ERR_INVALID, "log_jacobian: bad buffers");
  if (n_symm != 1 && n_symm != 8)
    return fail(NH_ERR_INVALID, "log_jacobian: n_symm %d (1 or 8)", n_symm);
  const int n = p->n_up + p->n_dn, d = p->channels / 2, N = p->Lx * p->Ly;
  if (p->net != NH_NET_CNN || p->ansatz != NH_ANSATZ_PFAFFIAN || !cnn_vjp_supported(*p) ||
      n > kGradMaxN || 2 * N > 512 ||
      (d != 8 && d != 16 && d != 32))
    return fail(NH_ERR_UNSUPPORTED,
                "log_jacobian: the backflow CNN with n <= %d, 2N <= 512, d in {8, 16, 32} "
                "(got net %d, n %d, N %d, d %d)", kGradMaxN, p->net, n, N, d);
  if (batch == 0) return NH_OK;
  const size_t need = nh_log_jacobian_workspace_bytes(batch, n_symm, p);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "log_jacobian"))) return rc;
  nh_backflow_params q = *p;  // the backward is FP32 on CUDA cores: so is its forward
  q.cnn_mode = 0;
  q.pf_mode = 0;
  const int cs = jac_chunk_samples(batch, n_symm);
  const int items = cs * n_symm;
  PipelineBuffers b = carve_pipeline(workspace, items, q);
  char* extra = static_cast<char*>(workspace) + pipeline_bytes(items, q);
  float* Fbuf = reinterpret_cast<float*>(extra);
  float* dYbuf = reinterpret_cast<float*>(extra + align256((size_t)items * n * n * sizeof(float)));
  const int64_t P = nh_param_count(p);
  const int64_t off_w = P - 1 - 3 * (int64_t)N * d;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int c0 = 0; c0 < batch; c0 += cs) {
    const int m = batch - c0 < cs ? batch - c0 : cs;
    const int8_t* sp = spins + (size_t)c0 * 2 * N;
    ConfigList cl{sp, nullptr, nullptr, nullptr, nullptr, m, n_symm};
    if ((rc = run_pipeline(cl, q, b, sign + c0, logabs + c0, flags ? flags + c0 : nullptr, st)))
      return rc;
    if ((rc = launch_pairing(b.Y, b.idx, q.Wt, q.Lx, q.Ly, d, n, m * n_symm, Fbuf, st))) return rc;
    if ((rc = launch_pf_adjoint(Fbuf, Fbuf, n, m * n_symm, b.pf_sign, b.pf_logabs, n_symm,
                                nullptr, st)))
      return rc;
    float* jrow = jac + (size_t)c0 * P;
    if ((rc = launch_pairing_vjp(Fbuf, b.Y, b.idx, q.Wt, q.Lx, q.Ly, d, n, n_symm, m, dYbuf,
                                 nullptr, jrow, P, off_w, theta, st)))
      return rc;
    if ((rc = launch_cnn_vjp(sp, m, n_symm, q, dYbuf, b.idx, jrow, P, st))) return rc;
  }
  return NH_OK;
}

// ------------------------------------------------------------------ packed observables

struct ObsLayout {
  int32_t *counts, *owner, *from, *to, *bin, *chunk_cnt;
  int64_t* offsets;
  double *hval, *clogabs, *V;
  float* csign;
  int n_chunks;
  void* pipe;
  size_t bytes;
};

static ObsLayout obs_layout(void* ws, int batch, int n_symm, int kind, int chunk,
                            const nh_backflow_params* p) {
  const size_t T = (size_t)obs_terms(kind, p->Lx * p->Ly);
  const size_t cmax = (size_t)batch * T;
  char* q = static_cast<char*>(ws);
  ObsLayout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* r = q ? q + off : nullptr;
    off += align256(bytes);
    return r;
  };
  L.counts = reinterpret_cast<int32_t*>(take((size_t)batch * 4));
  L.offsets = reinterpret_cast<int64_t*>(take((size_t)(batch + 1) * 8));
  L.owner = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.from = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.to = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.bin = reinterpret_cast<int32_t*>(take(cmax * 4));
  L.hval = reinterpret_cast<double*>(take(cmax * 8));
  L.csign = reinterpret_cast<float*>(take(cmax * 4));
  L.clogabs = reinterpret_cast<double*>(take(cmax * 8));
  L.V = reinterpret_cast<double*>(take((size_t)batch * T * 8));
  const size_t ch = chunk > 0 ? (size_t)chunk : (cmax > 0 ? cmax : 1);
  L.n_chunks = (int)((cmax + ch - 1) / ch);
  L.chunk_cnt = reinterpret_cast<int32_t*>(take((size_t)(L.n_chunks > 0 ? L.n_chunks : 1) * 4));
  L.pipe = take(chunk > 0 ? pipeline_bytes(chunk * n_symm, *p) : fused_bytes(cmax * n_symm, *p));
  L.bytes = off;
  return L;
}

size_t nh_observable_workspace_bytes(int batch, int n_symm, int kind, const nh_backflow_params* p) {
  if (!p || batch <= 0 || kind < NH_OBS_TRANSVERSE_SPIN || kind > NH_OBS_HOP) return 0;
  return obs_layout(nullptr, batch, n_symm, kind, eloc_chunk(0, p), p).bytes;
}

int nh_observable(const int8_t* spins, const float* sign, const double* logabs, int batch,
                  int n_symm, const nh_backflow_params* p, int kind, int arg0, int arg1,
                  double* out, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_params(p);
  if (rc) return rc;
  if (!spins || !sign || !logabs || !out || batch < 0)
    return fail(NH_ERR_INVALID, "observable: bad buffers");
  if (n_symm != 1 && n_symm != 8) return fail(NH_ERR_INVALID, "observable: n_symm %d", n_symm);
  const int Lx = p->Lx, Ly = p->Ly, N = Lx * Ly;
  if (kind < NH_OBS_TRANSVERSE_SPIN || kind > NH_OBS_HOP)
    return fail(NH_ERR_INVALID, "observable: kind %d", kind);
  if (2 * N > 32 * 64) return fail(NH_ERR_UNSUPPORTED, "observable: N = %d (<= 1024)", N);
  if (arg0 < 0 || arg0 >= N || (kind == NH_OBS_PAIR && (arg1 < 0 || arg1 >= N)) ||
      (kind == NH_OBS_HOP && arg1 != 0 && arg1 != 1))
    return fail(NH_ERR_INVALID, "observable: arguments %d, %d", arg0, arg1);
  if (batch == 0) return NH_OK;
  const int chunk = eloc_chunk(0, p);
  const size_t need = nh_observable_workspace_bytes(batch, n_symm, kind, p);
  if ((rc = check_workspace(workspace, workspace_bytes, need, "observable"))) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ObsLayout L = obs_layout(workspace, batch, n_symm, kind, chunk, p);
  // Diagonal term's bin: r = 0 (and N), (c, d) = (a, b) when that pair is a bond, j = i.
  int diag_bin = kind == NH_OBS_HOP ? arg0 : (kind == NH_OBS_TRANSVERSE_SPIN ? 0 : -1);
  if (kind == NH_OBS_PAIR) {
    for (int t = 0; t < 4 * N && diag_bin < 0; ++t) {
      const int site = t >> 2, axis = (t >> 1) & 1, o = t & 1, x = site / Ly, y = site % Ly;
      const int hi = axis == 0 ? ((x + 1) % Lx) * Ly + y : x * Ly + (y + 1) % Ly;
      if ((o == 0 ? site : hi) == arg0 && (o == 0 ? hi : site) == arg1) diag_bin = t;
    }
  }
  if ((rc = launch_obs_list(spins, batch, Lx, Ly, kind, arg0, arg1, L.counts, L.offsets, L.owner,
                            L.from, L.to, L.hval, L.bin, st)))
    return rc;
  int64_t total = 0;
  if ((rc = check_cuda(cudaMemcpyAsync(&total, L.offsets + batch, sizeof(int64_t),
                                       cudaMemcpyDeviceToHost, st),
                       "observable: read connection count")))
    return rc;
  if ((rc = check_cuda(cudaStreamSynchronize(st), "observable: sync"))) return rc;
  if (total > 0) {
    const int64_t cmax = (int64_t)batch * obs_terms(kind, N);
    if ((rc = launch_chunk_counts(L.offsets + batch, L.n_chunks, chunk > 0 ? chunk : (int)cmax,
                                  L.chunk_cnt, st)))
      return rc;
    if (chunk == 0) {
      ConfigList cl{spins, L.owner, L.from, L.to, L.chunk_cnt, (int)cmax, n_symm};
      FusedBuffers fb = carve_fused(L.pipe, (size_t)cmax * n_symm, *p);
      if ((rc = run_pipeline_fused(cl, *p, fb, L.csign, L.clogabs, nullptr, st))) return rc;
    } else {
      PipelineBuffers b = carve_pipeline(L.pipe, chunk * n_symm, *p);
      const int used = (int)((total + chunk - 1) / chunk);
      for (int i = 0; i < used; ++i) {
        const int64_t c0 = (int64_t)i * chunk;
        ConfigList cl{spins, L.owner + c0, L.from + c0, L.to + c0, L.chunk_cnt + i, chunk,
                      n_symm};
        if ((rc = run_pipeline(cl, *p, b, L.csign + c0, L.clogabs + c0, nullptr, st))) return rc;
      }
    }
  }
  return launch_obs_reduce(spins, sign, logabs, batch, N, kind, arg0, arg1, diag_bin,
                           L.offsets + batch, L.owner, L.bin, L.hval, L.csign, L.clogabs, L.V, out,
                           st);
}

}  // extern "C"

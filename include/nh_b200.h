/* C ABI of the B200 Pfaffian-backflow VMC hot path (libnh_b200.so).
 *
 * Every entry point takes raw device pointers, sizes and a CUDA stream (as void*), returns an
 * int status (NH_OK = 0, negative on error; nh_last_error() gives the message of the calling
 * thread) and never synchronises the host unless its comment says so.  The caller owns every
 * buffer.  Entry points that need scratch memory take (workspace, workspace_bytes) and have a
 * *_workspace_bytes() query; a workspace must be 256-byte aligned, as cudaMalloc returns it
 * (NH_ERR_INVALID otherwise).  Configurations are int8 +-1 arrays of length 2N (spin-up sites
 * first, site index x * Ly + y), as in the reference's quantax convention.
 *
 * Reference interfaces replaced (paths inside the ChenAo-Phys/NeuralHubbard tree):
 *   nh_build_wtilde      <- code/backflow/pf_kernel.py:107-124   build_wtilde(W, theta, geom)
 *   nh_pairing_occ       <- code/backflow/pf_kernel.py:335-351   pairing_occ(Y, idx, Wt, geom)
 *   nh_slogpf            <- code/backflow/models.py:210          fermix.slogpf(F)
 *   nh_cnn_forward       <- code/backflow/models.py:163-167      PfaffianBackflow.features(s)
 *   nh_amplitude         <- code/backflow/models.py:208-211 and code/states.py:318-320
 *                           quantax Variational.__call__(spins) -> LogArray (sign, logabs)
 *   nh_local_energy      <- code/quick_start.py:33               H.Oloc(state, Samples(spins, psi))
 *   nh_metropolis_steps  <- code/states.py:397-408               ParticleHop ... sweep()
 *   nh_metropolis_steps_mixed <- code/states.py:397-408          MixSampler([ParticleHop,
 *                                                                 SiteExchange]) ... sweep()
 *   nh_metropolis_steps_learned, nh_proposal_*: the learned hop proposal, new (the reference
 *                           samples with the uniform ParticleHop only); they extend the same
 *                           sampler call (code/states.py:397-408).
 */
#ifndef NH_B200_H
#define NH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NH_ABI_VERSION 10

enum {
  NH_OK = 0,
  NH_ERR_INVALID = -1,     /* bad shape, null pointer or inconsistent argument */
  NH_ERR_UNSUPPORTED = -2, /* size outside what the kernels support */
  NH_ERR_CUDA = -3,        /* launch or runtime error */
  NH_ERR_WORKSPACE = -4    /* workspace too small */
};

/* Per-amplitude status flags (int32 output arrays). */
enum {
  NH_FLAG_ZERO_PIVOT = 1,  /* exactly singular pairing block: sign 0, logabs -inf */
  NH_FLAG_NONFINITE = 2,   /* a non-finite value met during the factorisation */
  NH_FLAG_GROWTH = 4,      /* pivot ratio above cond_tau (near-nodal, ill-conditioned block) */
  NH_FLAG_REFINED = 8,     /* log-Pfaffian refined in FP64 (see refine_tau and cond_tau) */
  NH_FLAG_CANCEL = 16,     /* projected amplitude: sum_g |psi_g| > cancel_tau |sum_g eta_g psi_g| */
  NH_FLAG_TIMEOUT = 32     /* a bounded wait of a tensor-core kernel expired during this call:
                              the amplitudes it aborted are NaN; treat the whole call as failed */
};

/* Backflow networks (nh_backflow_params.net). */
#define NH_NET_CNN 0     /* periodic 3x3 CNN on the +-1 occupation image (layers conv layers) */
#define NH_NET_RESCONV 1 /* residual CNN of the released states (layers residual blocks) */

/* Ansatz (nh_backflow_params.ansatz). */
#define NH_ANSATZ_PFAFFIAN 0 /* psi = pf(F[idx, idx]) (code/backflow/models.py:121-211) */
#define NH_ANSATZ_BCS 1      /* psi = det(F_ud) (code/backflow/models.py:214-302) */

/* Parameters of the backflow network (device pointers).
 * net:           NH_NET_CNN or NH_NET_RESCONV.
 * conv_w:        NH_NET_CNN: FP32, layers concatenated, layer l of shape (C_out, C_in, 3, 3)
 *                (C_in = 2 for l = 0, else channels); conv_b: FP32, (channels,) per layer.
 *                NH_NET_RESCONV (channels 64, cnn_mode 0): the occupation embedding (C, 4)
 *                (occupation index n_up + 2 n_dn: empty, up, down, double) followed by the
 *                2 * layers convolutions (C, C, 3, 3) of the residual blocks
 *                x + Conv2(GELU(Conv1(GELU(RMSNorm(x))))) in order; conv_b: (2 * layers, C).
 *                RMSNorm is over all channels and sites without affine parameters; the
 *                features are the last block's output divided by sqrt(layers + 1)
 *                (code/backflow/models.py:319-329, quantax ResConv).
 *                Either way the features are the last channels [0, d) spin up, [d, 2d) spin
 *                down, d = channels / 2.
 * conv_w_packed: the same weights repacked by nh_pack_cnn_weights (NH_NET_CNN) or
 *                nh_pack_resconv_weights (NH_NET_RESCONV, 16-byte aligned); read by the kernels.
 * cnn_mode:      0 = FP32 CUDA cores; 1 = tcgen05 BF16; 2 = tcgen05 BF16 x3 (hi*hi + hi*lo +
 *                lo*hi, near-FP32).  NH_NET_CNN: modes 1 and 2 need a 16x16 lattice, 32 channels,
 *                4 layers.  NH_NET_RESCONV: modes 0 and 2, mode 2 on a 16x16 lattice.
 * conv_w_tc:     BF16 hi/lo tensor-core image from nh_pack_cnn_weights_tc (NH_NET_CNN) or
 *                nh_pack_resconv_weights_tc (NH_NET_RESCONV); 16-byte aligned.
 * pf_mode:       0 = Pfaffian on CUDA cores (two matrices per SM in shared memory); 1 = matrix
 *                resident in tensor memory, rank-16 trailing updates as 3xTF32 tcgen05 MMAs
 *                (one matrix per SM).  The FP64 recompute always uses the CUDA-core kernel.
 * Wt:            FP32 (4, N, d) spin-block table from nh_build_wtilde, blocks [uu, ud, du, dd].
 * Wt64:          the same table in FP64 (nh_build_wtilde), or null to disable the FP64
 *                recompute of ill-conditioned items.
 * refine_tau:    an item whose largest / smallest FP32 pivot magnitude exceeds refine_tau has its
 *                log-Pfaffian refined: the same matrix is factorised again in FP64 with the
 *                pivot order of the FP32 factorisation held fixed (no pivot search; a blocked
 *                rank-8 FP64 elimination), which removes the FP32 factorisation error
 *                (NH_FLAG_REFINED).  <= 0: off; 1: every item.  Needs n <= 224; for larger n the
 *                refinement is the pivoted FP64 recompute of cond_tau below.
 * cond_tau:      an item whose pivot ratio exceeds cond_tau is flagged NH_FLAG_GROWTH and, when
 *                Wt64 is set, its features are recomputed in FP64 (CNN) and its log-Pfaffian is
 *                refined against the FP64 pairing block (NH_FLAG_REFINED; n > 224: a pivoted
 *                FP64 Pfaffian); <= 0 disables both.  For projected amplitudes with
 *                cond_tau > 1 an image whose |psi(g s)| is below 1e-3 of |psi_P(s)| is not
 *                recomputed in FP64 (its error cannot move log|psi_P| by more than ~1e-5);
 *                cond_tau <= 1 recomputes every image (the all-FP64 form).
 * cancel_tau:    projected amplitudes only: a configuration whose 8 images cancel, i.e.
 *                sum_g |psi(g s)| > cancel_tau |sum_g eta_g psi(g s)|, amplifies the FP32
 *                error of its images by that factor; with cancel_tau > 0 (and Wt64 set) all its
 *                images are recomputed in FP64 and the output carries NH_FLAG_CANCEL.  <= 0:
 *                off (the flag is then never set).
 * ansatz:        NH_ANSATZ_PFAFFIAN, or NH_ANSATZ_BCS: psi(s) = det F (-1)^(n_up (n_up - 1) / 2)
 *                x fermion_inverse_sign(s) with the occupied up x down block
 *                F[p, q] = sum_a y_up[p, a] Wt[1, site_p - site_q, a] y_dn[q, a]
 *                + delta_d fd(site_p - site_q), fd = -1 on x bonds and +1 on y bonds
 *                (code/backflow/models.py:214-302, bcs_kernel.py:1-70).  Wt is the table of
 *                nh_build_wtilde for W = [W_ud, 0, 0] (block 1 is read).  Needs n_up == n_dn
 *                <= 224, d = 16 and pf_mode 0; the FP64 recompute of flagged images (cond_tau,
 *                cancel_tau) covers n_up <= 128.
 * delta_d:       the BCS d-wave amplitude (ignored by the Pfaffian ansatz). */
typedef struct {
  const float* conv_w;
  const float* conv_b;
  const float* conv_w_packed;
  const void* conv_w_tc;
  const float* Wt;
  const double* Wt64;
  int32_t Lx, Ly;
  int32_t n_up, n_dn;
  int32_t channels;
  int32_t layers;
  int32_t cnn_mode;
  int32_t pf_mode;
  int32_t net;
  int32_t ansatz;
  double cond_tau;
  double cancel_tau;
  double refine_tau;
  double delta_d;
} nh_backflow_params;

/* Hubbard model H = -sum t_ij c+_i c_j + U sum n_up n_dn; n_dirs = 4 (nearest) or 8
 * (nearest and next-nearest). */
typedef struct {
  double t, tp, U;
  int32_t n_dirs;
} nh_hubbard_params;

int nh_abi_version(void);
const char* nh_last_error(void);

/* Per-kernel timing (no counterpart in the reference, whose timing is wall clock around calls,
 * code/train_pfaffian_16x16_tpm02.py:107,124).  While enabled, every kernel launch of the library
 * is bracketed by CUDA events on its launching stream.  nh_profile_read waits for the pending
 * events, writes the accumulated milliseconds and launch counts of each kernel id (< n_ids,
 * ids NH_K_*), and resets the totals. */
enum {
  NH_K_CNN = 0,
  NH_K_PFAFFIAN = 1,
  NH_K_PAIRING = 2,
  NH_K_COMBINE = 3,
  NH_K_HOP_COUNT = 4,
  NH_K_SCAN = 5,
  NH_K_HOP_EMIT = 6,
  NH_K_ELOC_REDUCE = 7,
  NH_K_MH_PROPOSE = 8,
  NH_K_COMPACT = 9,
  NH_K_MH_ACCEPT = 10,
  NH_K_WTILDE = 11,
  NH_K_PFAFFIAN64 = 12,
  NH_K_CNN64 = 13,
  NH_K_FLAGGED = 14,
  NH_K_PACK = 15,
  NH_K_CNN_TC = 16,
  NH_K_PFAFFIAN_TC = 17,
  NH_K_PROP_SAMPLE = 18,
  NH_K_PROP_FORWARD = 19,
  NH_K_PROP_BACKWARD = 20,
  NH_K_PROP_ADAM = 21,
  NH_K_RESCONV = 22,
  NH_K_RESCONV64 = 23,
  NH_K_RESCONV_TC = 24,
  NH_K_REFINE = 25,
  NH_K_FUSED = 26,
  NH_K_PF_ADJOINT = 27,
  NH_K_PAIRING_VJP = 28,
  NH_K_CNN_VJP = 29,
  NH_K_DET = 30,
  NH_K_DET64 = 31,
  NH_K_OBS = 32,
  NH_K_COUNT = 40
};
int nh_profile_enable(int on);
int nh_profile_read(double* ms, int64_t* launches, int n_ids);

/* Wt (4, N, d) FP32 and, when Wt64 is not null, the same table in FP64, from
 * W (3, N, d) = [W_ud, V_uu, V_dd] and theta. */
int nh_build_wtilde(const float* W, float theta, int Lx, int Ly, int d, float* Wt, double* Wt64,
                    void* stream);

/* packed (18 C + 9 C^2 (layers - 1),) = conv_w rearranged per layer as [ci][tap][co]. */
int nh_pack_cnn_weights(const float* conv_w, int channels, int layers, float* packed,
                        void* stream);

/* Residual network: packed (nh_pack_resconv_weights_floats(channels, blocks) floats) =
 * embedding as [occupation][co], then every convolution as [ci][tap][co]. */
size_t nh_pack_resconv_weights_floats(int channels, int blocks);
int nh_pack_resconv_weights(const float* conv_w, int channels, int blocks, float* packed,
                            void* stream);
/* Residual network, tensor-core image (nh_pack_resconv_weights_tc_bytes(blocks) bytes): per
 * convolution and tap the BF16 hi and lo weights in the K-major core-matrix layout; 64 channels. */
size_t nh_pack_resconv_weights_tc_bytes(int blocks);
int nh_pack_resconv_weights_tc(const float* conv_w, int channels, int blocks, void* packed,
                               void* stream);

/* Tensor-core weight image (nh_pack_cnn_weights_tc_bytes() bytes): BF16 hi and lo parts in the
 * K-major core-matrix layout; 32 channels, 4 layers. */
size_t nh_pack_cnn_weights_tc_bytes(void);
int nh_pack_cnn_weights_tc(const float* conv_w, int channels, int layers, void* packed,
                           void* stream);

/* Features y (batch, 2, N, d) of batch configurations (no symmetry image).  The residual network
 * runs here up to N = 256 (beyond, its activation planes need nh_amplitude's workspace). */
int nh_cnn_forward(const int8_t* spins, int batch, const nh_backflow_params* p, float* features,
                   void* stream);

/* Occupied pairing block F (batch, n, n), exactly antisymmetric:
 * F[p, q] = sum_a Y[p, a] Wt[2 s_p + s_q, r(p, q), a] Y[q, a], idx the ascending occupied modes. */
int nh_pairing_occ(const float* Y, const int32_t* idx, const float* Wt, int Lx, int Ly, int d,
                   int n, int batch, float* F, void* stream);

/* sign and log|pf| of batch antisymmetric n x n FP32 matrices (n even, n <= 1024); only the
 * strict lower triangle is read.  With cond_tau > 0 the matrices whose pivot ratio exceeds it
 * are flagged NH_FLAG_GROWTH and factorised again in FP64 (NH_FLAG_REFINED): for n <= 224 with
 * the pivot order of the FP32 factorisation held fixed, beyond with FP64 partial pivoting.  The
 * workspace (nh_slogpf_workspace_bytes(n, batch) bytes) holds the list of those matrices, their
 * FP32 pivot orders and, where a triangle exceeds shared memory (FP32 n > 256, FP64 n > 236), one
 * triangle per SM; it may be null when cond_tau <= 0 and n <= 256. */
size_t nh_slogpf_workspace_bytes(int n, int batch);
int nh_slogpf(const float* F, int n, int batch, double cond_tau, float* sign, double* logabs,
              int32_t* flags, void* workspace, size_t workspace_bytes, void* stream);

/* nh_slogpf without a workspace (no counterpart in the reference): for callers that hold only
 * their input and output buffers and cannot allocate device memory (for example a plugin whose
 * host runtime owns all device memory, or a path where cudaMalloc's possible device
 * synchronisation is not acceptable).  The FP64 refinement list lives in a static device array of
 * NH_SLOGPF_NOALLOC_MAX_BATCH + 64 int32 words held by every GPU that loads the library; batch
 * beyond that limit returns NH_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * address (make it before any stream capture); all calls share the array, so calls that overlap
 * on the GPU race.  Allocates nothing.  n <= 256; same results as nh_slogpf for n <= 236, while
 * for 236 < n <= 256 flagged matrices keep their FP32 result (the FP64 triangle would need
 * workspace). */
#define NH_SLOGPF_NOALLOC_MAX_BATCH 65536
int nh_slogpf_noalloc(const float* F, int n, int batch, double cond_tau, float* sign,
                      double* logabs, int32_t* flags, void* stream);

/* Amplitudes of batch configurations.  n_symm = 1: psi(s); n_symm = 8: the projection onto the
 * trivial representation of Flip(0) Flip(1) SpinInverse, psi_P(s) = 1/8 sum_g eta_g psi(g s).
 * Lattices up to 32 x 32 and n = n_up + n_dn <= 1024: beyond n = 256 (FP32) / 236 (FP64) the
 * Pfaffian keeps its triangles, and beyond shared memory the CNN its activation planes, in a
 * per-CTA scratch that the workspace query includes (e.g. ~0.4 GB at 32 x 32). */
size_t nh_amplitude_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p);
int nh_amplitude(const int8_t* spins, int batch, int n_symm, const nh_backflow_params* p,
                 float* sign, double* logabs, int32_t* flags, void* workspace,
                 size_t workspace_bytes, void* stream);

/* Local energies E_loc (batch,) FP64 of configurations with amplitudes (sign, logabs).  The
 * ragged list of connected configurations (configuration x image x connection items) is
 * evaluated, with chunk_configs <= 0, in one persistent pass: a fused kernel takes items off a
 * device work counter and computes each item's features and FP32 Pfaffian in one block, the FP64
 * refinement runs over device-built lists, and the launch sequence is the same whatever the
 * number of connections (the backflow CNN with n <= 224; other networks fall back to chunks of
 * 8192 configurations).  chunk_configs > 0 evaluates chunks of that many configurations with
 * the unfused pipeline.  Work counts stay on the device either way.  With n_conn_out null the
 * call never synchronises, so a caller may record it into a CUDA graph and replay it.  With
 * n_conn_out set it synchronises the stream once, writes the number of connections and launches
 * only the chunks that hold connections. */
size_t nh_local_energy_workspace_bytes(int batch, int n_symm, int chunk_configs,
                                       const nh_backflow_params* p);
int nh_local_energy(const int8_t* spins, const float* sign, const double* logabs, int batch,
                    int n_symm, const nh_backflow_params* p, const nh_hubbard_params* h,
                    int chunk_configs, double* eloc, int64_t* n_conn_out, void* workspace,
                    size_t workspace_bytes, void* stream);

/* Connection list of batch configurations: counts (batch,) int32 and, when rec is not null,
 * records (total,) of (from_mode, to_mode) int32 pairs and matrix elements hval (total,) in
 * enumeration order (ascending occupied mode, then hop direction). offsets (batch + 1,) int64
 * are written by the call.  A pure bookkeeping entry point, used by tests. */
int nh_hop_list(const int8_t* spins, int batch, int Lx, int Ly, const nh_hubbard_params* h,
                int32_t* counts, int64_t* offsets, int32_t* rec, double* hval, void* stream);

/* nsteps plain Metropolis hop steps (uniform electron, uniform direction, null move when
 * the target is occupied) on every chain, updating spins, sign and logabs in place.
 * Random numbers: Philox4x32-10, key (seed_lo, seed_hi), counter (step_lo, chain, 0, step_hi)
 * for step = step0 + t; draws: x -> electron rank, y -> direction, z -> acceptance uniform.
 * accepted (batch,) int32 is incremented per accepted move. */
size_t nh_metropolis_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p);
int nh_metropolis_steps(int8_t* spins, float* sign, double* logabs, int batch, int n_symm,
                        const nh_backflow_params* p, int n_dirs, uint64_t seed, int64_t step0,
                        int nsteps, int32_t* accepted, void* workspace, size_t workspace_bytes,
                        void* stream);

/* Mixed hop / site-exchange Metropolis (the reference's MixSampler of a ParticleHop and a
 * SiteExchange sampler, code/states.py:397-408): chains b < first_exchange make the plain hop
 * steps of nh_metropolis_steps; chains b >= first_exchange make site-exchange steps, in which a
 * uniform site i and a uniform one of its n_dirs neighbours j swap their occupations (both spin
 * species; equal occupations are a null move), so one step can move an up and a down electron.
 * The proposal is symmetric and accepted with min(1, |psi(s')/psi(s)|^2).  Same random-number
 * streams and buffers as nh_metropolis_steps (draw x -> site, y -> direction, z -> acceptance);
 * nh_metropolis_steps is this call with first_exchange = batch. */
int nh_metropolis_steps_mixed(int8_t* spins, float* sign, double* logabs, int batch, int n_symm,
                              const nh_backflow_params* p, int n_dirs, int first_exchange,
                              uint64_t seed, int64_t step0, int nsteps, int32_t* accepted,
                              void* workspace, size_t workspace_bytes, void* stream);

/* ---- Backward of the amplitude (the per-sample Jacobian that SR / AdamSR training consumes,
 * code/train_pfaffian_16x16_tpm02.py:100-101).  FP32 throughout; n <= 224, 2 N <= 512,
 * d in {8, 16, 32}. */

/* Cotangent of the log-Pfaffian (the derivative of fermix.slogpf, code/backflow/models.py:210):
 * G = d log|pf F| / dF = 1/2 F^{-T} for batch antisymmetric n x n FP32 matrices, from a
 * Gauss-Jordan inverse with partial pivoting.  flags (batch,) or null: NH_FLAG_ZERO_PIVOT
 * (singular) or NH_FLAG_NONFINITE; G is zero for such matrices. */
int nh_pfaffian_adjoint(const float* F, int n, int batch, float* G, int32_t* flags, void* stream);

/* The custom VJP of the occupied gather (code/backflow/pf_kernel.py:193-320, 354-365, per
 * matrix): for the cotangent G (batch, n, n) of F = nh_pairing_occ(Y, idx, Wt),
 * dY (batch, n, d) = sum_q (G - G^T)[p, q] Wt[blk(p, q), r(p, q), a] Y[q, a] and
 * dWt (batch, 4, N, d) = sum over the pairs (p, q) of each block and displacement of
 * G[p, q] Y[p, a] Y[q, a] (one table per matrix; a batched caller sums them). */
int nh_pairing_occ_vjp(const float* Y, const int32_t* idx, const float* Wt, const float* G,
                       int Lx, int Ly, int d, int n, int batch, float* dY, float* dWt,
                       void* stream);

/* Number of parameters P of the backflow CNN state: sum over layers of C_out C_in 9 + C_out,
 * plus 3 N d (W) + 1 (theta).  0 for NH_NET_RESCONV. */
int64_t nh_param_count(const nh_backflow_params* p);

/* Per-sample Jacobian jac (batch, P) FP32 of log|psi_P(s)| (n_symm = 8) or log|psi(s)|
 * (n_symm = 1) with respect to the parameters, in the order conv_w[0] (OIHW), conv_b[0], ...,
 * conv_w[L-1], conv_b[L-1], W (3, N, d), theta; W and theta are the raw pairing parameters that
 * p->Wt was built from (nh_build_wtilde).  The amplitude (sign, logabs, flags) is computed on the
 * way with p's recompute policy; the backward runs on the FP32 CUDA-core path whatever p's
 * cnn_mode / pf_mode.  Images are weighted by eta_g psi(g s) / sum_h eta_h psi(h s); a
 * configuration whose projected amplitude is zero gets a zero row.  NH_NET_CNN only. */
size_t nh_log_jacobian_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p);
int nh_log_jacobian(const int8_t* spins, int batch, int n_symm, const nh_backflow_params* p,
                    const float* W, float theta, float* jac, float* sign, double* logabs,
                    int32_t* flags, void* workspace, size_t workspace_bytes, void* stream);

/* ---- Packed observables (code/measure/transverse_spin.py:44-119, dwave_packed.py:24-103):
 * one operator family O = sum_t O_t per call.  Every sample's connections s -> s' of the terms
 * go through the amplitude pipeline (as for the local energy; the call synchronises the stream
 * once to read the number of connections), and the local values
 * <s|O_t|s'> psi(s') / psi(s) are summed per term t over the batch in a fixed order and divided
 * by batch; the diagonal term of the family comes from the occupations.  out (device, FP64):
 *   NH_OBS_TRANSVERSE_SPIN  arg0 = reference site a: out (2, N), [0, r] = <S+_a S-_{a+r}>,
 *                           [1, r] = <S-_a S+_{a+r}> (r = x Ly + y, periodic), r = 0 holding
 *                           n_up (1 - n_dn) and n_dn (1 - n_up) at a;
 *   NH_OBS_PAIR             arg0, arg1 = sites a, b of A+ = c+_{a up} c+_{b dn}: out (4 N),
 *                           [t] = <A+(a, b) A(c_t, d_t)> over the bonds t = 4 site + 2 axis + o
 *                           (axis 0: +x, 1: +y; (c, d) = (site, site + axis) for o = 0 and
 *                           swapped for o = 1); the term (c, d) = (a, b) is n_{a up} n_{b dn};
 *   NH_OBS_HOP              arg0 = site i, arg1 = spin (0 up, 1 down): out (N),
 *                           [j] = <c+_{i s} c_{j s}>, [i] = n_{i s}. */
#define NH_OBS_TRANSVERSE_SPIN 0
#define NH_OBS_PAIR 1
#define NH_OBS_HOP 2
size_t nh_observable_workspace_bytes(int batch, int n_symm, int kind, const nh_backflow_params* p);
int nh_observable(const int8_t* spins, const float* sign, const double* logabs, int batch,
                  int n_symm, const nh_backflow_params* p, int kind, int arg0, int arg1,
                  double* out, void* workspace, size_t workspace_bytes, void* stream);

/* ---- Learned hop proposal ----
 * A periodic 3x3 CNN 2 -> 16 -> 16 -> 16 (tanh-GELU after layers 1 and 2) on the +-1 occupation
 * image; output channel c = sigma * 8 + d at site i is the logit of hopping the spin-sigma
 * electron at site i one step in hop direction d (the direction order of nh_hop_list).  Move
 * index m = c * N + i.  A move is valid when the electron exists, d < n_dirs and the target site
 * of the same spin is empty; q(m | s) = softmax over the valid moves.  Parameters: a flat FP32
 * vector of NH_PROPOSAL_PARAMS values, W1 (16, 2, 3, 3), b1 (16), W2 (16, 16, 3, 3), b2 (16),
 * W3 (16, 16, 3, 3), b3 (16); the kernels evaluate the BF16 image from nh_proposal_pack. */
#define NH_PROPOSAL_PARAMS 4944
typedef struct {
  const void* weights; /* BF16 (NH_PROPOSAL_PARAMS,) */
  int32_t Lx, Ly;
  int32_t n_dirs; /* 4 or 8 */
  int32_t reserved;
} nh_proposal_params;

/* BF16 (round to nearest even) image of the FP32 parameters; count = NH_PROPOSAL_PARAMS. */
int nh_proposal_pack(const float* master, int count, void* weights_bf16, void* stream);
/* Raw logits (batch, 16, N) FP32 (invalid moves are not masked). */
int nh_proposal_forward(const int8_t* spins, int batch, const nh_proposal_params* q,
                        float* logits, void* stream);
/* One proposal per configuration with the Philox draw of (seed, step, chain) word 0: from/to
 * modes, valid (0 when no electron can hop) and log q(reverse | s') - log q(move | s). */
int nh_proposal_sample(const int8_t* spins, int batch, const nh_proposal_params* q,
                       uint64_t seed, int64_t step, int32_t* from, int32_t* to, int32_t* valid,
                       float* log_q_ratio, void* stream);
/* Training: loss = -(1/batch) sum_b weights[b] log q(moves[b] | spins[b]) (records whose move
 * is not valid contribute nothing) into loss (1,) and its gradient (NH_PROPOSAL_PARAMS,) into
 * grad, both FP32, summed in a fixed order (deterministic).  The workspace holds per-CTA
 * gradient partials and, for lattices whose activation planes exceed shared memory (more than 559
 * sites, e.g. 24x24 and 32x32), per-CTA planes (about 100 MB at 32x32). */
size_t nh_proposal_backward_workspace_bytes(int batch, const nh_proposal_params* q);
int nh_proposal_backward(const int8_t* spins, const int32_t* moves, const float* weights,
                         int batch, const nh_proposal_params* q, float* loss, float* grad,
                         void* workspace, size_t workspace_bytes, void* stream);
/* Adam (bias-corrected, step t >= 1) on the FP32 master; refreshes the BF16 image when
 * weights_bf16 is not null.  The optimiser step of the training loop. */
int nh_proposal_adam_step(float* master, float* m, float* v, const float* grad, int count,
                          int64_t t, float lr, float beta1, float beta2, float eps,
                          void* weights_bf16, void* stream);
/* Metropolis steps with the learned proposal and the exact Hastings correction: accept when
 * log u < 2 (log|psi(s')| - log|psi(s)|) + log q(reverse | s') - log q(move | s), u from word 2
 * of the chain's Philox draw.  Same buffers as nh_metropolis_steps; q's lattice must equal p's. */
size_t nh_metropolis_learned_workspace_bytes(int batch, int n_symm, const nh_backflow_params* p);
int nh_metropolis_steps_learned(int8_t* spins, float* sign, double* logabs, int batch,
                                int n_symm, const nh_backflow_params* p,
                                const nh_proposal_params* q, uint64_t seed, int64_t step0,
                                int nsteps, int32_t* accepted, void* workspace,
                                size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NH_B200_H */

/*
 * gfmc_b200.h -- C ABI of the B200 Green's-function Monte Carlo engine.
 *
 * The drop-in boundary behind pygfmc_b200.run(...), which mirrors PyGFMC's
 * pygfmc.run (engine/multi_gpu.py:822-868 -> engine/driver.py:1148).  Plain C
 * types only: host descriptors for the model and the guide, raw device
 * pointers for walker state (e.g. torch.Tensor.data_ptr()), and a CUDA stream
 * handle (e.g. torch.cuda.current_stream().cuda_stream).  Every function
 * returns GFMC_OK (0) or a negative error code; gfmc_last_error() gives the
 * message of the calling thread's last failure.
 *
 * Ownership: the caller owns every buffer it passes; the engine owns only
 * its handle, the device copies of the tables and its scratch.  A handle is
 * not thread-safe: use one handle per host thread / stream.
 *
 * Random numbers are the JAX Threefry-2x32 stream PyGFMC draws from, with
 * its key semantics (split(key)[i] = fold_in(key, i)); fed the same keys and
 * walkers, the float64 engine reproduces PyGFMC's trajectories.
 */
#ifndef GFMC_B200_H
#define GFMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GFMC_OK 0
#define GFMC_ERR_INVALID (-1)     /* bad argument (ValueError in the Python layer) */
#define GFMC_ERR_CUDA (-2)        /* a CUDA call failed */
#define GFMC_ERR_UNSUPPORTED (-3) /* model/guide/method combination not built */
#define GFMC_ERR_DEVICE (-4)      /* a kernel raised a status bit (see gfmc_read_status) */

#define GFMC_MODEL_SPIN_HALF 0
#define GFMC_MODEL_BOSE_HUBBARD 1

#define GFMC_GUIDE_NONE 0
#define GFMC_GUIDE_JASTROW_SPIN_HALF 1
#define GFMC_GUIDE_JASTROW_BOSE_HUBBARD 2
#define GFMC_GUIDE_RBM_SPIN_HALF 3        /* no counterpart in PyGFMC */
#define GFMC_GUIDE_MLP_BOSE_HUBBARD 4     /* no counterpart in PyGFMC */
#define GFMC_GUIDE_EXACT_SPIN_HALF 5      /* ExactGroundState on a SpinHalf model */

#define GFMC_METHOD_CONT_TIME 0
#define GFMC_METHOD_SINGLE_STEP 1
#define GFMC_METHOD_MULTI_STEP 2

#define GFMC_PRECISION_FP64 0  /* every step quantity in float64 */
#define GFMC_PRECISION_MIXED 1 /* rates, ratios, local energies in float32; weight
                                  accumulators, resampling sums, energies in float64 */

/* Device status bits (gfmc_read_status). */
#define GFMC_STATUS_HOP_CAP 1     /* a walker hit the per-step iteration cap */
#define GFMC_STATUS_BAD_CONFIG 2  /* a configuration value outside the model's basis */
#define GFMC_STATUS_NONFINITE 4   /* non-finite mean branch weight (extinct population) */
#define GFMC_STATUS_TIMEOUT 8     /* a bounded wait on the tensor-core pipeline ran out */

/* Model description (host arrays, float64, read during gfmc_create only).
 * SpinHalf: the stored-sign fields of hamiltonian/SpinHalf.py:101-117
 *   (jpm = (J_x+J_y)/4, jpmpm = (J_x-J_y)/4 per edge; jz one value when
 *   uniform_jz, else per edge; hz = -h_z per site; hx_half = -h_x/2 per site;
 *   n_hx in {0, N}, n_jpm in {0, n_edges}).
 * BoseHubbard: hamiltonian/bose_hubbard.py:67-103 (t, eta per edge; U, mu per
 *   site; hpm = -h_pm per site; n_hop, n_eta in {0, 2 n_edges}; n_hpm in {0, N}). */
typedef struct {
  int kind;
  int n_sites, n_edges;
  const int32_t *edge_i, *edge_j;
  int n_hx, n_jpm, has_jz, uniform_jz, has_hz;
  const double *jz, *jpm, *jpmpm, *hz, *hx_half;
  int n_max, n_hop, n_eta, n_hpm, has_U, has_mu;
  const double *t, *eta, *U, *mu, *hpm;
} gfmc_model_desc;

/* Guide description.
 * JastrowSpinHalf (wavefunction/jastrow_spin_half.py:79-157): pair list with
 *   pair_w = J = -beta per pair, h per site (NULL: zero).
 * JastrowBoseHubbard (wavefunction/jastrow_bose_hubbard.py:97-125): pair list
 *   with pair_w = the neighbour-sum weight (-beta per pair, or 1 for a tied
 *   beta with beta_tied = 1, beta0 = beta); h_mode/d_mode 0 none, 1 tied
 *   (h0/d0), 2 per site (h/d). */
typedef struct {
  int kind;
  int n_pairs;
  const int32_t *pair_i, *pair_j;
  const double *pair_w;
  const double *h;
  int beta_tied;
  double beta0;
  int h_mode;
  double h0;
  int d_mode;
  double d0;
  const double *d;
  /* RBM (GFMC_GUIDE_RBM_SPIN_HALF; no PyGFMC counterpart): log psi(s) =
   * sum_h log cosh(b_h + sum_i W_hi s_i) + a.s over spins s = +-1; rbm_W
   * (n_hidden, n_sites) row-major, rounded to bfloat16 on the device;
   * rbm_b (n_hidden), rbm_a (n_sites); n_hidden <= 1024. */
  int n_hidden;
  const float *rbm_W, *rbm_b, *rbm_a;
  /* MLP (GFMC_GUIDE_MLP_BOSE_HUBBARD; no PyGFMC counterpart; float32 build
   * only, methods cont_time and the local energy): over the one-hot
   * occupations x (input k (n_max + 1) + n_k), h1 = tanh(W1 x + b1) rounded
   * to bfloat16, log psi = w3 . tanh(W2 h1 + b2) + b3.  mlp_W1 (mlp_H1,
   * n_sites (n_max + 1)) and mlp_W2 (mlp_H2, mlp_H1) row-major, rounded to
   * bfloat16 on the device, as are mlp_w3 (mlp_H2); mlp_b1, mlp_b2 float32.
   * mlp_H1 in {64, 128, 192, 256}; mlp_H2 a multiple of 16 in [16, 256]. */
  int mlp_H1, mlp_H2;
  const float *mlp_W1, *mlp_b1, *mlp_W2, *mlp_b2, *mlp_w3;
  double mlp_b3;
  /* ExactGroundState (GFMC_GUIDE_EXACT_SPIN_HALF; wavefunction/
   * exact_ground_state.py:43-190): psi_T(x) = exp(exact_log_amp[idx(x)]) with
   * idx(x) = sum_i b_i 2^(N-1-i), b_i = 1 for x_i = -1 (site 0 most
   * significant; the positional index over SpinHalf.local_hilbert_space
   * (1, -1)); exact_log_amp has 2^exact_n_sites entries, exact_n_sites = the
   * model's N <= 26.  Nodes carry a large negative log amplitude, not -inf. */
  int exact_n_sites;
  const double *exact_log_amp;
} gfmc_guide_desc;

typedef struct gfmc_handle gfmc_handle;

/* Builds the device tables of (model, guide) once -- the analogue of
 * guide.build_cache(hamiltonian) (engine/evolution.py guide_cache:192) -- on
 * the current CUDA device.  precision: GFMC_PRECISION_*. */
int gfmc_create(const gfmc_model_desc *model, const gfmc_guide_desc *guide, int precision,
                gfmc_handle **out);
int gfmc_destroy(gfmc_handle *h);

/* Bytes of one packed walker configuration: ceil(N/64) uint64 words for a
 * spin-1/2 model (bit 1 = +1), ceil(N/16)*16 uint8 occupations for bosons. */
int gfmc_config_bytes(const gfmc_handle *h);
int gfmc_n_transitions(const gfmc_handle *h); /* M_total */

/* Walker.config (float64, row-major (n, N), +-1 or occupations; device) <->
 * packed device configurations. */
int gfmc_pack(gfmc_handle *h, int n_walkers, const double *cfg, void *packed, void *stream);
int gfmc_unpack(gfmc_handle *h, int n_walkers, const void *packed, double *cfg, void *stream);

/* n_steps branching steps of the production/warm-up scan
 * (engine/driver.py _make_prod_step_fn:194-342 main chain): per step s,
 * evolve_walkers with key keys[4s..4s+1] (engine/evolution.py
 * evolve_walkers:761, per-walker split) then reconfiguration with key
 * keys[4s+2..4s+3] (walkers/reconfiguration.py:27).  keys is host memory.
 * State: the packed configurations cfg (device) and the parent map of the
 * last reconfiguration (device, n_walkers int32); the population is
 * cfg[parents[i]].  parents_valid = 0 means identity (a fresh population).
 * cfg_tmp is a second packed buffer of the same size.  log_w/e_loc (device,
 * float64, n_walkers) receive the pre-resampling weights and local energies
 * of the last step.  logG_out/E_out (device, float64, n_steps) receive
 * log G_n = logsumexp(log_w) - log N and E_n = sum w e_L / sum w; hops_out
 * (device, uint64, n_steps, nullable) the moves made per step.
 * method: GFMC_METHOD_*; step = beta (cont_time) or the integer n_bra;
 * lam is used by the discrete methods; alw = avg_log_weight. */
int gfmc_run_steps(gfmc_handle *h, int method, double step, double lam, double alw, int n_steps,
                   const uint32_t *keys, int n_walkers, void *cfg, void *cfg_tmp, int32_t *parents,
                   int parents_valid, double *log_w, double *e_loc, double *logG_out,
                   double *E_out, uint64_t *hops_out, void *stream);

/* Local energies e_L(x) = sum of the guide-transformed rates
 * (engine/estimators.py estimate_average_log_branch_weight:722-751 input) of
 * cfg[parents[i]] (parents nullable). */
int gfmc_local_energy(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                      double *e_loc, void *stream);
/* The same with the diagonal element H_xx of each configuration (device,
 * float64, n_walkers): the sampler-health probes of engine/estimators.py
 * statistics:1139 (escape rate diag - e_L, stay probability). */
int gfmc_local_energy_parts(gfmc_handle *h, int n_walkers, const void *cfg,
                            const int32_t *parents, double *e_loc, double *diag, void *stream);

/* Applies a parent map: cfg_out[i] = cfg_in[parents[i]], e_out[i] = e_in[parents[i]],
 * log_w[i] = 0 (any output nullable except cfg_out). */
int gfmc_gather(gfmc_handle *h, int n_walkers, const int32_t *parents, const void *cfg_in,
                void *cfg_out, const double *e_in, double *e_out, double *log_w, void *stream);

/* Windowed mixed estimator of the energy (engine/estimators.py
 * _energy_and_diagonal_estimates:268-305) on the device in float64; p (host,
 * n_p windows, each < n_steps), out (host, n_p).  Synchronises the stream. */
int gfmc_windowed_energy(int n_steps, const double *logG, const double *E, int n_p, const int *p,
                         double *out, void *stream);

/* Per-walker, per-step cap on the propagator's iterations (default 2^22).
 * A walker reaching it stops its step and raises GFMC_STATUS_HOP_CAP; the
 * loop never runs unbounded.  No counterpart in PyGFMC (its while_loop is
 * unbounded). */
int gfmc_set_max_iters(gfmc_handle *h, int max_iters);

/* Carried guide state of sparse Jastrow guides (degree < 16; the float64
 * build carries it by default, the float32 build rebuilds).  mode 1 (the
 * default): carry each walker's guide fields and last rate evaluation
 * through the parent map, while their buffers fit in half of the device
 * memory free at the call that sizes them; mode 0: rebuild them per walker
 * every step; mode < 0: leave the mode as it is.  Carried and rebuilt runs
 * agree to the last bits in float64 (identical moves on every tested case).
 * Dense guides and the learned guides always carry.  *carrying_out (host,
 * may be NULL): 1 when the handle carries guide state (as decided by the
 * last gfmc_run_steps call, or the mode just set).  No counterpart in
 * PyGFMC; its JastrowBoseHubbard(incremental=True) neighbour sums
 * (wavefunction/jastrow_bose_hubbard.py:87-92) are the nearest analogue. */
int gfmc_carry_mode(gfmc_handle *h, int mode, int *carrying_out);

/* ---- diagonal observables with forward walking ------------------------- */
#define GFMC_DIAG_SPIN_HALF 0   /* SpinHalf.diagonal_weight (J_z edges, h_z)     */
#define GFMC_DIAG_BOSE_HUBBARD 1 /* BoseHubbard.diagonal_weight (U, mu)          */
#define GFMC_DIAG_SZSZ 2        /* SzSzStructureFactor: n_k values per walker    */

/* A diagonal operator (host arrays, float64, read by gfmc_set_diag_operators).
 * SpinHalf / BoseHubbard fields as in gfmc_model_desc; SZSZ: (n_k, N) cos/sin
 * tables of k.r and the dropped i == j constant (hamiltonian/observables.py:68). */
typedef struct {
  int kind;
  int n_sites, n_edges;
  const int32_t *edge_i, *edge_j;
  int has_jz, uniform_jz, has_hz;
  const double *jz, *hz;
  int has_U, has_mu;
  const double *U, *mu;
  int n_k;
  const double *cos_kr, *sin_kr;
  double offset;
} gfmc_diag_desc;

/* Diagonal operators measured by the ancestry-traced (forward-walking) pure
 * estimator of engine/driver.py:228-288 at the windows m_array (sorted, p//2),
 * at most 16.  Replaces any previous set. */
int gfmc_set_diag_operators(gfmc_handle *h, int n_ops, const gfmc_diag_desc *ops, int n_p,
                            const int *m_array);
/* Values per walker of the operator set (the sum of their widths). */
int gfmc_diag_width(const gfmc_handle *h);
/* Resets the ancestry and value ring buffers (identity maps, zeros) for a
 * population of n_walkers (engine/driver.py _diag_ring_buffers:810-838). */
int gfmc_reset_diag(gfmc_handle *h, int n_walkers, void *stream);
/* Device output of the next gfmc_run_steps call: (n_steps, width, n_p)
 * float64, the mean over walkers of each value traced m steps back; NULL
 * stops the measurement. */
int gfmc_set_diag_output(gfmc_handle *h, double *out);

/* ---- RBM guide ---------------------------------------------------------- */
/* Hidden pre-activations theta = b + W s (float32, row-major (n_walkers, Hp))
 * of the configurations cfg[parents[i]] (parents read when parents_valid)
 * on the tensor cores (bf16 inputs, float32 accumulation); Hp is
 * gfmc_rbm_hidden_padded(h) >= n_hidden (padding rows are zero).  No
 * counterpart in PyGFMC. */
int gfmc_rbm_theta(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                   int parents_valid, float *theta_out, void *stream);
int gfmc_rbm_hidden_padded(const gfmc_handle *h);

/* Local-energy variance loss of the RBM guide over the walkers cfg[parents[i]]
 * with weights omega (device float64, NULL: all 1):
 *   L = sum omega (e_L - E)^2 / sum omega,  E = sum omega e_L / sum omega.
 * gfmc_rbm_gradient writes dL/dW (n_hidden, n_sites), dL/db, dL/da (device
 * float32, each nullable) and stats = (E, L) (host); the dW contraction over
 * every walker's connected configurations runs on the tensor cores (bf16
 * inputs, float32 accumulation).  gfmc_rbm_train_step takes one Adam step
 * (beta1 0.9, beta2 0.999, eps 1e-8) of rate lr on float32 master parameters
 * and writes them back to the guide rounded to bf16; stats are those before
 * the step.  Float32 (mixed) handles, at most 448 sites.  No counterpart in
 * PyGFMC (it trains guides by NetKet VMC). */
int gfmc_rbm_gradient(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                      int parents_valid, const double *omega, float *grad_W, float *grad_b,
                      float *grad_a, double stats[2], void *stream);
int gfmc_rbm_train_step(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                        int parents_valid, const double *omega, double lr, double stats[2],
                        void *stream);
/* The guide's current parameters (host float32: W (n_hidden, n_sites) as
 * used, i.e. bf16 values; b; a). */
int gfmc_rbm_get_params(gfmc_handle *h, float *W, float *b, float *a);

/* ---- MLP guide trainer ---------------------------------------------------- */
/* The same variance loss for the MLP guide (float32 handles; mlp_H2 a
 * multiple of 64; at most 800 one-hot inputs n_sites (n_max + 1); at
 * least 9 moves per configuration).  The
 * parameters, and the gradient, are one float32 array of
 * gfmc_mlp_param_count(h) values: W1 (mlp_H1, n_sites (n_max + 1)), b1
 * (mlp_H1), W2 (mlp_H2, mlp_H1), b2 (mlp_H2), w3 (mlp_H2) (b3 cancels in
 * every ratio and is not trained).  gfmc_mlp_gradient writes dL/dp (device,
 * nullable) and stats = (E, L) (host); the second layer forward, its
 * backward into the first layer and dL/dW2 run on the tensor cores (bf16
 * inputs, float32 accumulation), dL/dW1 by one-hot accumulation.
 * gfmc_mlp_train_step takes one Adam step (beta1 0.9, beta2 0.999, eps 1e-8)
 * of rate lr on float32 master parameters and writes them back to the guide
 * (weights rounded to bf16).  gfmc_mlp_get_params copies the guide's
 * parameters as used (bf16 values) to host memory.  No counterpart in
 * PyGFMC. */
long long gfmc_mlp_param_count(const gfmc_handle *h);
int gfmc_mlp_gradient(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                      int parents_valid, const double *omega, float *grad, double stats[2],
                      void *stream);
int gfmc_mlp_train_step(gfmc_handle *h, int n_walkers, const void *cfg, const int32_t *parents,
                        int parents_valid, const double *omega, double lr, double stats[2],
                        void *stream);
int gfmc_mlp_get_params(gfmc_handle *h, float *params);

/* ---- off-diagonal observables with forward walking ---------------------- */
/* At most this many windows per forward walk. */
#define GFMC_FW_MAX_P 16

/* Applies the measurement operator of handle `op` (a model handle built from
 * the operator and the run's guide) to the population cfg (read through
 * parents when parents_valid): each walker moves to a successor drawn in
 * proportion to the operator's guide-transformed rates, slot 0 (the diagonal)
 * meaning stay, with the uniform of Threefry key fold_in(key, walker); its
 * value is the sum of the rates, 0 when that is not positive.  A purely
 * diagonal operator keeps the walker and returns its diagonal element.
 * Replaces engine/evolution.py apply_operator_one:849-888 (vmapped in
 * forward_walk_operator:1008-1012).  Outputs (device): cfg_out (packed,
 * n_walkers), vals (float64, n_walkers). */
int gfmc_apply_operator(gfmc_handle *op, const uint32_t key[2], int n_walkers, const void *cfg,
                        const int32_t *parents, int parents_valid, void *cfg_out, double *vals,
                        void *stream);

/* Forward-walking pure estimator of one operator at one measured step
 * (engine/evolution.py forward_walk_operator:891-1101): gfmc_apply_operator
 * with op and apply_key, then a shadow chain of m_max = m_array[n_m - 1]
 * branching steps of the model of handle `shadow` (the run's model and guide)
 * started from the operator-applied walkers with zero log weights, keyed by
 * shadow_keys (host, (m_max, 4): the (k1, k2) pairs of the main chain's next
 * m_max steps, so the shadow replays the main chain's future draws).  After
 * every shadow reconfiguration the values follow the parent map.  Outputs
 * (device, n_m each): val_out[j] = mean of the values after m_array[j] shadow
 * steps, norm_out[j] = sum of the shadow's log G over those steps (row m = 0:
 * the plain mean, norm 0).  m_array: host, sorted, non-negative, at most
 * GFMC_FW_MAX_P entries.  The shadow population lives in s_cfg, s_cfg_tmp,
 * s_parents, s_log_w, s_e_loc (device, n_walkers each) and vals, vals_tmp
 * (float64 device scratch, n_walkers); the main population is only read.
 * `shadow` may be the main chain's handle: its carried guide state is then
 * rebuilt on the main chain's next step, and its diagonal measurement pauses
 * during the shadow steps. */
int gfmc_forward_walk(gfmc_handle *shadow, gfmc_handle *op, int method, double step, double lam,
                      double alw, const uint32_t apply_key[2], const uint32_t *shadow_keys,
                      int n_walkers, const void *cfg, const int32_t *parents, int parents_valid,
                      void *s_cfg, void *s_cfg_tmp, int32_t *s_parents, double *s_log_w,
                      double *s_e_loc, double *vals, double *vals_tmp, int n_m,
                      const int *m_array, double *val_out, double *norm_out, void *stream);

/* Smallest guide-transformed rate of the operator of handle `op` over all its
 * M_total slots, per walker of cfg (read through parents when parents_valid);
 * NaN where a rate is not finite.  The positivity check of engine/
 * estimators.py check_off_diag_operator_positivity:631-681 reads it.
 * Output (device): min_out (float64, n_walkers). */
int gfmc_operator_min_rate(gfmc_handle *op, int n_walkers, const void *cfg, const int32_t *parents,
                           int parents_valid, double *min_out, void *stream);

/* ---- walkers sharded over GPUs ---------------------------------------- */
/* The evolve half of a branching step alone (no resampling): walkers
 * cfg[parents[i]] (parents read when parents_valid) propagated with key
 * into cfg_out, with their log weights and local energies.  Walker i draws
 * from fold_in(key, walker_offset + i): a rank holding global walkers
 * [offset, offset + n) of a sharded population reproduces the streams of the
 * unsharded one.  Carried guide state is rebuilt. */
int gfmc_evolve(gfmc_handle *h, int method, double step, double lam, double alw,
                const uint32_t key[2], long long walker_offset, int n_walkers, const void *cfg,
                const int32_t *parents, int parents_valid, void *cfg_out, double *log_w,
                double *e_loc, uint64_t *hops, void *stream);
/* One evolution of a population with its own log weights, no resampling:
 * replaces PyGFMC's evolve_walkers (engine/evolution.py:761-843).  Walker i
 * (packed row i of cfg) draws from fold_in(key, i) = split(key, n)[i],
 * propagates into row i of cfg_out (cfg_out != cfg), and its log weight
 * accumulates onto log_w[i] in place (the step's terms added to the incoming
 * value in PyGFMC's order); e_loc[i] is the local energy of its final
 * configuration.  The guide state is built from cfg. */
int gfmc_evolve_walkers(gfmc_handle *h, int method, double step, double lam, double alw,
                        const uint32_t key[2], int n_walkers, const void *cfg, void *cfg_out,
                        double *log_w, double *e_loc, uint64_t *hops, void *stream);
/* Systematic resampling of a population sharded over ranks in contiguous
 * blocks (walkers/reconfiguration.py:9-62 applied to the concatenated
 * population):
 * 1. gfmc_dist_local_max: the rank's max log weight (host); the caller takes
 *    the max over ranks as the common shift.
 * 2. gfmc_dist_local_sums: (S_r, sum_r w e_loc, last positive index) of the
 *    rank's weights w = exp(log_w - shift) (host).  Over ranks: S = sum S_r,
 *    E_n = sum (sum w e) / S, log G_n = log S + shift - log N.
 * 3. gfmc_dist_parents: the rank's local parents of the global output slots
 *    [slot_lo, slot_lo + count), the slots whose point U_i = (i + psi) / N S
 *    lies in [offset, offset + S_r) (offset = the earlier ranks' S sum);
 *    psi = uniform(reconfiguration key), N = N_total.  The caller sends each
 *    slot's walker to the rank that owns the slot (contiguous blocks).
 * PyGFMC's multi-device path all-gathers every configuration instead
 * (engine/multi_gpu.py:91-155). */
int gfmc_dist_local_max(gfmc_handle *h, int n_walkers, const double *log_w, double *max_out,
                        void *stream);
int gfmc_dist_local_sums(gfmc_handle *h, int n_walkers, const double *log_w,
                         const double *e_loc, double shift, double out[3], void *stream);
int gfmc_dist_parents(gfmc_handle *h, int n_walkers, const double *log_w, double shift,
                      double offset, double S_total, double psi, long long N_total,
                      long long slot_lo, int count, int last_pos, int32_t *parents_out,
                      void *stream);
/* Steps 1 and 2 with their results left in device memory and no wait on the
 * stream, for callers whose collectives run on device buffers (NCCL):
 * gfmc_dist_local_max_dev writes the rank's max log weight to max_out
 * (device, 1 double); after the caller's max-reduction over ranks into
 * shift (device, 1 double), gfmc_dist_local_sums_dev writes out (device, 4
 * doubles) = (the shift used -- 0 when the max is not finite --, S_r,
 * sum_r w e_loc, last positive index).  One gather of the 4-double rows
 * then gives every rank the slot partition and log G_n, E_n. */
int gfmc_dist_local_max_dev(gfmc_handle *h, int n_walkers, const double *log_w, double *max_out,
                            void *stream);
int gfmc_dist_local_sums_dev(gfmc_handle *h, int n_walkers, const double *log_w,
                             const double *e_loc, const double *shift, double *out, void *stream);

/* Largest population gfmc_reconfigure_noalloc accepts. */
#define GFMC_NOALLOC_MAX_WALKERS 131072

/* Systematic resampling of a population (the reconfiguration step of
 * gfmc_run_steps, on its own) that allocates no device memory, for callers
 * that must not allocate inside a call: a host framework that owns the device
 * through its own pool allocator, or a latency-critical loop that cannot
 * take the device synchronisation cudaMalloc/cudaFree imply.  No counterpart
 * in PyGFMC.  Inputs (device): log_w, e_loc (float64, n_walkers); key (host):
 * the reconfiguration key.  Outputs (device): parents_out (int32, n_walkers),
 * logG_out = logsumexp(log_w) - log N, E_out = sum w e_loc / sum w (scalars).
 * Scratch is a fixed ~2 MB file-scope device array that every GPU loading the
 * library holds until exit: at most GFMC_NOALLOC_MAX_WALKERS walkers (larger
 * counts return GFMC_ERR_INVALID); all calls on a device share it, so calls
 * that overlap on the GPU race.  The first call on a device looks up the
 * array's address on that (current) device; make it before any stream
 * capture.  The return code covers the arguments and the launches only:
 * the call does not wait for the GPU and reports no status word.  A
 * population whose weights sum to zero or overflow is signalled by a
 * non-finite *logG_out (and *E_out) alone -- check that it is finite; the
 * parents are then in range but meaningless. */
int gfmc_reconfigure_noalloc(int n_walkers, const double *log_w, const double *e_loc,
                             const uint32_t key[2], int32_t *parents_out, double *logG_out,
                             double *E_out, void *stream);

/* Reads and clears the device status word (GFMC_STATUS_* bits); synchronises. */
int gfmc_read_status(gfmc_handle *h, int *status_out, void *stream);

/* Host-side key schedule of the production chain (engine/driver.py:218-221):
 * key, rng = split(key); k1, k2 = fold_in(rng, 0), fold_in(rng, 1).  Writes
 * keys_out[4 s .. 4 s + 3] = (k1, k2) for n_steps steps and the final key. */
int gfmc_key_schedule(const uint32_t key[2], int n_steps, uint32_t *keys_out,
                      uint32_t key_next[2]);
/* The same recurrence with n_sub sub-keys per step: keys_out[2 (s n_sub + j)
 * .. + 1] = fold_in(rng_s, j), j < n_sub (folds
 * 0 = evolve, 1 = reconfigure, 2 = off-diagonal measurement; driver.py:218-221). */
int gfmc_key_schedule_ex(const uint32_t key[2], int n_steps, int n_sub, uint32_t *keys_out,
                         uint32_t key_next[2]);
/* Threefry-2x32 and fold_in on the host (jax key semantics). */
int gfmc_threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t out[2]);

/* Message of the calling thread's last error (empty when none). */
int gfmc_last_error(char *buf, size_t len);
/* Library version string. */
const char *gfmc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GFMC_B200_H */

// Internal interfaces of the GFMC engine: device-resident model and guide
// tables, kernel parameter blocks and the launchers the C ABI calls.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gfmc_device.cuh"

namespace gfmc {

enum Family { SPIN_HALF = 0, BOSE_HUBBARD = 1 };
enum Method { CONT_TIME = 0, SINGLE_STEP = 1, MULTI_STEP = 2, EVALUATE = 3, APPLY = 4, MIN_RATE = 5 };
enum GuideKind {
  GUIDE_NONE = 0, GUIDE_JASTROW_SPIN = 1, GUIDE_JASTROW_BOSE = 2, GUIDE_RBM_SPIN = 3,
  GUIDE_EXACT_SPIN = 5
};

// Status bits the kernels raise (atomicOr into a device word).
enum StatusBits {
  ST_HOP_CAP = 1,        // a walker hit the per-step iteration cap
  ST_BAD_CONFIG = 2,     // an occupation outside [0, n_max] (Bose-Hubbard)
  ST_NONFINITE = 4,      // non-finite population weight in reconfiguration
  ST_TIMEOUT = 8,        // a bounded wait on the tensor-core pipeline ran out
};

// Model tables (device pointers).  Couplings follow the stored-sign
// conventions of hamiltonian/SpinHalf.py:101-117 and
// hamiltonian/bose_hubbard.py:67-103.
template <typename T> struct DevModel {
  int family;
  int N, E, M;            // sites, edges, M_total
  int n_off;              // M - 1
  const uint32_t *edge;   // (E,) packed ei | ej << 16
  // SpinHalf
  int n_hx, n_jpm, has_jz, uniform_jz, has_hz;
  const T *jz, *jpm, *jpmpm, *hz, *hx_half;
  int uniform_pm;         // every edge has the same (J_pm, J_pmpm)
  T jpm0, jpmpm0;
  // Fast spin layout: no site-flip moves, uniform couplings (and uniform
  // guide edge constants), no h_z.  Edge rate = k_anti |s_i s_j| for
  // anti-parallel spins, k_par |s_i s_j| for parallel ones, where
  // s_k = x_k A_k are the signed ratio factors (A = 1 without a guide).
  int fast;               // 0 general; 1 fast with k_par = 0 (float32 only); 2 other fast
  T k_anti, k_par;
  // BoseHubbard
  int n_max, n_hop, n_eta, n_hpm, has_U, has_mu;
  const T *sqrt_tab;      // sqrt(k), k = 0 .. (n_max + 1)^2: the elements' square roots
  const T *t, *eta, *U, *mu, *hpm;
};

// Guide tables.  Per-site partner lists (deduplicated; each partner at most
// once per site) carry the coupling the incremental field update needs:
//   spin-1/2 Jastrow: W_k = sum_p J_kp x_p, J = -beta
//   Bose-Hubbard Jastrow: S_k = sum_p w_kp n_p, w = -beta (1 for tied beta)
template <typename T> struct DevGuide {
  int kind;
  int deg;                // row stride of the partner tables
  const uint32_t *nbr;    // (N, deg) partner sites
  const T *nbr_w;         // (N, deg) couplings
  const int *nbr_cnt;     // (N,) partners per site
  const T *h;             // (N,) one-body field (spin: JastrowSpinHalf.h)
  const T *trans_pw;      // (M,) bose: summed pair weight joining each transition's sites
  // Bose: the guide ratio as a product, exp(out) = Gs_a(da) Gs_b(db) slot_q[o + 1]
  // site_t[a][n_a][da] site_t[b][n_b][db], with the walker's carried factors
  // Gs_k(+-1) = exp(+-beta_scale F_k) (per-warp shared memory, beside F),
  // slot_q = exp(beta_scale da db pw) per transition (index o + 1 like
  // trans_pw) and site_t[(k (n_max + 1) + n) 2 + (s > 0)] =
  // exp(-d_k ((n + s)^2 - n^2) + h_k s) for s = -1, +1
  const T *slot_q;
  const T *site_t;
  T beta_scale;           // bose: -beta for a tied beta, else 1
  int h_mode;             // bose: 0 none, 1 tied (h0), 2 array (h)
  T h0;
  int d_mode;             // bose: 0 none, 1 tied (d0), 2 array (d)
  T d0;
  const T *d;
  int has_h;              // spin: any nonzero one-body field
  // spin-1/2 Jastrow ratio of an edge flip, factored as A_i A_j c_e with the
  // per-site A_k = exp(-2 x_k (W_k + h_k)) and the per-edge constant
  // c_e = exp(4 Jsum_e x_i x_j): c_anti = exp(-4 Jsum_e), c_par = exp(4 Jsum_e)
  const T *c_anti, *c_par;
  int uniform_c;
  T c_anti0, c_par0;
  // multiplicative factor updates after a flip of site s (x_s before the
  // flip): A_k *= exp(4 x_k x_s J_sk), i.e. Ep = exp(4 J), Em = exp(-4 J)
  const T *Ep, *Em;       // dense: (N, N)
  const T *nbr_ep, *nbr_em;   // sparse: (N, deg), aligned with nbr
  // Translation-invariant dense couplings on an Lx x Ly torus (site
  // x + Lx y): J_ak = J_0[d(a, k)], d the displacement ((x_k - x_a) mod Lx) +
  // Lx ((y_k - y_a) mod Ly).  The factor of site k after a flip of a is then
  // tE[tq[k] - tq[a] + tE_off + (x_k != x_a)], tq[k] = 2 (x_k + 2 Lx y_k),
  // tE_off = 2 (Lx + 2 Lx Ly): tE runs over the unwrapped displacements
  // (dx + Lx) + 2 Lx (dy + Ly), two entries each, exp(4 J_0[d]) for parallel
  // spins and exp(-4 J_0[d]) for anti-parallel ones (8 N entries, staged in
  // shared memory with tq).
  int ti, Lx, Ly, tE_off;
  const T *tE;
  const int *tq;
  // exact amplitudes (GUIDE_EXACT_SPIN): log |psi_0| over the 2^N basis
  // states, indexed by the configuration's bits with site 0 most
  // significant; the walker's factors are then the plain spins x_k
  const T *lamp;
  int dense;              // couplings as a dense symmetric (N, N) matrix Jd
  const T *Jd;            // (N, N) row-major, zero diagonal (dense == 1)
  // Jd as jdig_d balanced base-128 int8 digits for the population product
  // (fields.cu): jdig[(t 256 + d (256 / jdig_d) + j) jdig_kp + p] is digit d of
  // Jd[p, 256 t / jdig_d + j], Jd = 128 jdig_scale sum_d digit_d 128^-(d+1);
  // jdig_kp = N rounded up to 128 (zero padding); nullptr when absent
  const int8_t *jdig;
  double jdig_scale;
  int jdig_kp, jdig_d;
};

// Digits of the couplings in the population product: 8 (56 bits) for the
// float64 build, 4 (28 bits) for the float32 build.
template <typename T> __host__ __device__ constexpr int fields_digits() {
  return sizeof(T) == 8 ? 8 : 4;
}

struct EvolveArgs {
  int method;
  double step;            // beta (cont_time) or n_bra (discrete)
  double lam;
  double alw;
  Key key;                // the step's evolve key (split over walkers)
  int n_walkers;
  const int *parents;     // gather map applied on load (nullptr: identity)
  const void *cfg_in;
  void *cfg_out;
  double *log_w;
  double *e_loc;
  unsigned long long *hops;   // per-step hop counter (nullable)
  int *work_ctr;          // zeroed work counter of this launch
  double *partial_max;    // (grid,) block max of log_w
  int *status;
  int max_iters;          // per-walker hop cap
  const void *field_in;   // carried guide fields (N per walker), read at parents[w]; nullable
  void *field_out;        // guide fields after the step (N per walker); nullable
  float *rates_out;       // EVALUATE, learned guides: (n_walkers, M - 1) guided rates; nullable
  float *rsum_out;        // EVALUATE, learned guides: (n_walkers,) sum of those rates; nullable
  double *diag_out;       // EVALUATE: (n_walkers,) diagonal element H_xx; nullable
  long long walker_offset;  // global index of walker 0 (streams fold_in(key, offset + i))
  // cont_time, Jastrow and plain kernels: the rate evaluation of each
  // walker's final configuration (EVAL_REC values of T: the 32 lanes' scan
  // prefixes, their chunk ends, H_xx, the total, a valid flag), written at
  // the end of the step and read through the parent map by the next step,
  // whose first evaluation is then that record; nullable
  const void *eval_in;
  void *eval_out;
  // incoming log weights, read at parents[w] (nullable: every walker starts
  // from 0, its state after resampling); the step's log weight accumulates
  // onto it as PyGFMC's evolve_walkers does (engine/evolution.py:356-400)
  const double *lw_in;
};
constexpr int EVAL_REC = 68;

struct LaunchPlan {
  int grid, block, wpb;   // blocks, threads per block, warps per block
  size_t smem;            // dynamic shared memory bytes
};

// Launchers (evolve.cu).
template <typename T>
cudaError_t launch_evolve(const DevModel<T> &m, const DevGuide<T> &g, const LaunchPlan &plan,
                          const EvolveArgs &a, cudaStream_t s);
template <typename T>
cudaError_t plan_evolve(const DevModel<T> &m, const DevGuide<T> &g, int n_slots_max,
                        LaunchPlan *plan);
// Number of per-warp partial maxima an evolve launch over n_walkers writes.
int evolve_partials(const LaunchPlan &plan, int n_walkers);

// Guide state of n configurations at once for a dense coupling matrix
// (fields.cu, int8 tensor cores on the coupling digits): spin-1/2 the signed
// ratio factors, Bose-Hubbard the fields, (n, N) values of T.  Needs g.jdig;
// a bounded wait that runs out sets ST_TIMEOUT in *status.
template <typename T>
cudaError_t launch_fields(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg, T *out,
                          int *status, cudaStream_t s);

// Sharded reconfiguration pieces (recon_dist.cu), float64.  out: (max, S,
// sum w e, last positive index).
int dist_tiles(int n);
cudaError_t launch_dist_max(int n, const double *lw, double *tmax, double *out, cudaStream_t s);
// shift_dev (nullable): the shift in device memory, used instead of shift
cudaError_t launch_dist_sums(int n, const double *lw, const double *e, double shift,
                             const double *shift_dev, double *tS, double *tE, int *tlp,
                             double *out, cudaStream_t s);
cudaError_t launch_dist_parents(int n, const double *lw, double shift, double offset,
                                const double *tS, double *cdf, double *wbuf, double psi,
                                double S_total, long long N_total, long long i_lo, int count,
                                int last_pos, int *parents, cudaStream_t s);

// Reconfiguration (reconfig.cu), always float64.
struct ReconArgs {
  int n;                  // walkers
  const double *log_w;
  const double *e_loc;
  const double *partial_max;
  int n_partial_max;
  Key key;                // the step's reconfiguration key
  double *psum;           // (nb,)
  double *pE;             // (nb,) per-step partial weighted energies
  int *plp;               // (nb,) last positive index per tile
  double *cdf;            // (n,)
  double *wbuf;           // (n,)
  int *parents;           // (n,) output
  double *logG_out;       // scalar slot of this step
  int *status;
  double *E_step;         // the one-launch resampling only: the step's E_n (sum of
                          // pE in tile order), or nullptr
};
int recon_tiles(int n);
cudaError_t launch_reconfigure(const ReconArgs &a, cudaStream_t s);
// The same resampling as one cooperative launch of recon_tiles(a.n) blocks
// with two grid barriers on *ctr (a counter only this launch family touches,
// zero when allocated; bar_base = its value before the launch, which then
// adds 2 recon_tiles(a.n)).  Needs recon_tiles(a.n) <= recon_fused_max_tiles().
cudaError_t launch_reconfigure_fused(const ReconArgs &a, unsigned *ctr, unsigned bar_base,
                                     cudaStream_t s);
int recon_fused_max_tiles();
cudaError_t launch_series_reduce(const double *pE, int nb, int n_steps, double *E_out,
                                 cudaStream_t s);
cudaError_t launch_gather(int n, int cfg_bytes, const int *parents, const void *cfg_in,
                          void *cfg_out, const double *e_in, double *e_out, double *log_w,
                          cudaStream_t s);
cudaError_t launch_windowed(const double *logG, const double *E, int n_steps, const int *p,
                            int n_p, double *out, cudaStream_t s);
cudaError_t launch_pack(int family, int n, int N, int cfg_bytes, const double *cfg,
                        void *packed, int n_max, int *status, cudaStream_t s);
cudaError_t launch_unpack(int family, int n, int N, int cfg_bytes, const void *packed,
                          double *cfg, cudaStream_t s);

}  // namespace gfmc

// RBM guide on the device: tables and launchers (rbm.cu, rbm_gemm.cu).
//
// log psi(s) = sum_h log cosh(theta_h) + a . s,  theta = b + W s,
// s in {+-1}^N, W (H, N) with bfloat16 values.  The hidden axis is padded to
// Hp, a multiple of 256, with zero weights and biases (a padded unit adds a
// constant log cosh(0) that cancels in every ratio).
#pragma once
#include <cuda_bf16.h>

#include <vector>

#include "engine.cuh"

namespace gfmc {

struct RbmTables {
  const __nv_bfloat16 *WT;   // (N, Hp) site-major: row i = W[:, i]
  const __nv_bfloat16 *W;    // (Hp, Np) hidden-major, Np = N rounded up to 64 (the GEMM's
                             // K-major operand; padding zero)
  const float *b;            // (Hp,)
  const float *a;            // (N,)
  int H, Hp, Np;
  // The float32 step kernel's tables (rbm_f32.cu), derived from WT:
  // RT row i (RS = Hp + 32 floats) = tanh(2 W[h, i]) for every h, then per
  // lane l the log2 of prod_{h in lane l} cosh(2 W[h, i]).
  float *RT;
  int RS;
  // Slots in chunks whose flipped sites' RT rows are staged together:
  // chunk c covers slots [ch_start[c], ch_start[c + 1]) and stages the rows
  // ch_sites[c U .. c U + ch_n[c]).  Slot o's record is ch_rec[2 o],
  // ch_rec[2 o + 1]: (i | row_i << 16, j | row_j << 16 (j = 0xFFFF and
  // row_j = row_i for a site flip), the couplings for anti-parallel and
  // parallel spins (float bits; a site flip's h_x / 2 twice)) and
  // (2 log2(e) a_i, 2 log2(e) a_j (0 for a site flip), 0, 0).
  const int *ch_start, *ch_sites, *ch_n;
  int4 *ch_rec;
  int n_chunks, ch_U, n_rec;
};

// Hidden units per lane of the step kernel's warp (Hp / 32).
inline int rbm_hpl(int Hp) { return Hp / 32; }

// One launch of the RBM step kernel (methods CONT_TIME, SINGLE_STEP,
// MULTI_STEP, EVALUATE); a.field_in / a.field_out carry theta (Hp values of T
// per walker) through the parent map.
template <typename T>
cudaError_t launch_rbm_evolve(const DevModel<T> &m, const RbmTables &r, const EvolveArgs &a,
                              int grid, cudaStream_t s);
// Grid (blocks) that keeps every SM busy for this model.
template <typename T> int rbm_grid(const DevModel<T> &m, const RbmTables &r);
// Per-warp partial maxima of log_w a launch over n walkers writes (f32: the
// float32 kernel's blocks of 8 warps, else the float64 kernel's blocks of 4).
int rbm_partials(int grid, int n_walkers, bool f32);

// The float32 step kernel (rbm_f32.cu): the walkers of a block evaluate their
// rates in lockstep over staged chunks of the derived tables.
cudaError_t launch_rbm_evolve_f32(const DevModel<float> &m, const RbmTables &r,
                                  const EvolveArgs &a, int grid, cudaStream_t s);
int rbm_grid_f32(const DevModel<float> &m, const RbmTables &r);
constexpr int RBF_WARPS = 8;   // warps (walkers) per block of the float32 kernel
// Sites staged per chunk (at most 16) for the model's slot count, so that
// two blocks fit on an SM; 0 when not even two sites fit.
int rbm_chunk_sites(int Hp, int N, int M);
// Host: greedy chunks of the off-diagonal slots (site flips first, then the
// edges edge_i / edge_j), at most U sites each.
void rbm_build_chunks(int N, int n_hx, int n_edges, const int *edge_i, const int *edge_j, int U,
                      std::vector<int> &start, std::vector<int> &sites, std::vector<int> &nsites,
                      std::vector<uint16_t> &pos);
// RT from WT (after the guide's weights are written).
cudaError_t launch_rbm_derive(const RbmTables &r, int N, cudaStream_t s);

// theta (float32, (n, Hp)) of the packed spin configurations cfg[parents[w]]
// (parents nullable) on the tensor cores (rbm_gemm.cu); status bit 8 when a
// bounded wait ran out.
cudaError_t launch_rbm_theta(const RbmTables &r, int n, const void *cfg, const int *parents,
                             int NW, float *theta, int *status, cudaStream_t s);

// Arguments of the gradient kernel of the variance loss (rbm_train.cu); the
// population is gathered (cfg row w is walker w), theta / rates / rsum come
// from the tensor-core GEMM and the EVALUATE pass, gw from launch_train_coeff.
struct GradArgs {
  const uint64_t *cfg;       // (n, NW) population (already gathered)
  int NW, n, N, Np, Hp, n_off, n_hx;
  const uint32_t *edge;      // (E,) packed sites
  const __nv_bfloat16 *WT;   // (N, Hp)
  const float *theta;        // (n, Hp)
  const float *rates;        // (n, n_off)
  const float *rsum;         // (n,)
  const float *gw;           // (n,)
  float *grad_W;             // (Hp, Np)
  float *grad_b;             // (Hp,)
  float *grad_a;             // (Np,)
  int walkers_per_cta;
  int *status;
};

// Gradient of the variance loss into grad_W (Hp, Np), grad_b (Hp), grad_a
// (Np) (accumulated: zero them first).  Np <= 256.  recs: scratch of
// n (n_off + 1) x 16 bytes for the row records.
cudaError_t launch_rbm_grad(const GradArgs &a, void *recs, int sms, cudaStream_t s);
// gw[w] = 2 omega_w (e_w - E) / sum omega; stats = (E, variance) (device).
cudaError_t launch_train_coeff(int n, const double *e, const double *omega, float *gw,
                               double *stats, cudaStream_t s);
// One Adam step (bias corrections of step `step`) on the float32 master
// parameters, writing the guide's bf16 / float tables.
cudaError_t launch_adam(int H, int N, int Hp, int Np, float *W, float *b, float *a, const float *gW,
                        const float *gb, const float *ga, float *m, float *v, float lr, float b1,
                        float b2, float eps, int step, __nv_bfloat16 *WT_t, __nv_bfloat16 *W_t,
                        float *b_t, float *a_t, cudaStream_t s);
// Float32 master parameters (W (H, N), b, a) from the guide's tables.
cudaError_t launch_rbm_master_init(const RbmTables &r, int N, float *W, float *b, float *a,
                                   cudaStream_t s);

}  // namespace gfmc

// RBM guide on the device: tables and launchers (rbm.cu, rbm_gemm.cu).
//
// log psi(s) = sum_h log cosh(theta_h) + a . s,  theta = b + W s,
// s in {+-1}^N, W (H, N) with bfloat16 values.  The hidden axis is padded to
// Hp, a multiple of 256, with zero weights and biases (a padded unit adds a
// constant log cosh(0) that cancels in every ratio).
#pragma once
#include <cuda_bf16.h>

#include "engine.cuh"

namespace gfmc {

struct RbmTables {
  const __nv_bfloat16 *WT;   // (N, Hp) site-major: row i = W[:, i]
  const __nv_bfloat16 *W;    // (Hp, Np) hidden-major, Np = N rounded up to 64 (the GEMM's
                             // K-major operand; padding zero)
  const float *b;            // (Hp,)
  const float *a;            // (N,)
  int H, Hp, Np;
};

// Hidden units per lane of the step kernel's warp (Hp / 32).
inline int rbm_hpl(int Hp) { return Hp / 32; }

// One launch of the RBM step kernel (methods CONT_TIME, SINGLE_STEP,
// MULTI_STEP, EVALUATE); a.field_in / a.field_out carry theta (Hp values of T
// per walker) through the parent map.
template <typename T>
cudaError_t launch_rbm_evolve(const DevModel<T> &m, const RbmTables &r, const EvolveArgs &a,
                              int grid, cudaStream_t s);
// Grid (blocks of 128 threads) that keeps every SM busy for this model.
template <typename T> int rbm_grid(const DevModel<T> &m, const RbmTables &r);
// Per-warp partial maxima of log_w a launch over n_walkers writes.
int rbm_partials(int grid, int n_walkers);

// theta (float32, (n, Hp)) of the packed spin configurations cfg[parents[w]]
// (parents nullable) on the tensor cores (rbm_gemm.cu); status bit 8 when a
// bounded wait ran out.
cudaError_t launch_rbm_theta(const RbmTables &r, int n, const void *cfg, const int *parents,
                             int NW, float *theta, int *status, cudaStream_t s);

}  // namespace gfmc

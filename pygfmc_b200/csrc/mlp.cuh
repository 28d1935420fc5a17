// Dense MLP guide for Bose-Hubbard occupations on the device (mlp.cu).
//
//   x = one-hot occupations (input index k (n_max + 1) + n_k),
//   h1 = bf16(tanh(W1 x + b1)), h2 = tanh(W2 h1 + b2), log psi = w3 . h2 + b3
//
// W1 is stored input-major (W1T[c] = the column of input c) and W2 (H2, H1)
// row-major, both bfloat16; the biases and the readout are float32.
#pragma once
#include <cuda_bf16.h>

#include "engine.cuh"

namespace gfmc {

struct MlpTables {
  const __nv_bfloat16 *W1T;  // (N (n_max + 1), H1)
  const float *b1;           // (H1,)
  const __nv_bfloat16 *W2;   // (H2, H1)
  const float *b2;           // (H2,)
  const float *w3;           // (H2,)
  float b3;
  int H1, H2;                // H1 in {64, 128, 192, 256}; H2 a multiple of 16 in [16, 256]
  int np1;                   // n_max + 1
};

// Dynamic shared memory of the step kernel (bytes) for these sizes.
size_t mlp_smem_bytes(int H1, int H2, int n_off, int N);
// Persistent grid: one CTA per SM.
int mlp_grid();
// Partial maxima of log_w a launch over n_walkers writes (one per pipeline).
int mlp_partials(int grid, int n_walkers);
// One launch of the MLP step kernel (methods CONT_TIME and EVALUATE, float).
cudaError_t launch_mlp_evolve(const DevModel<float> &m, const MlpTables &t, const EvolveArgs &a,
                              int grid, cudaStream_t s);

}  // namespace gfmc

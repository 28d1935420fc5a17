// Diagonal observables with forward walking (diag.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "engine.cuh"

#define GFMC_DIAG_MAX_P 16

namespace gfmc {

enum DiagKind { DIAG_SPIN = 0, DIAG_BOSE = 1, DIAG_SZSZ = 2 };

// One diagonal operator (device pointers, float64).
struct DiagOp {
  int kind;
  int col;          // first column of its values in a walker's value row
  int N, E;
  const int *ei, *ej;
  int has_jz, uniform_jz, has_hz;
  const double *jz, *hz;
  int has_U, has_mu;
  const double *U, *mu;
  int n_k;
  const double *cos_kr, *sin_kr;   // (n_k, N)
  double offset;
};

struct DiagSet {
  int n_ops;
  const DiagOp *ops;    // device array
  int width;            // total values per walker
  int n_p;
  int m[GFMC_DIAG_MAX_P];
  int m_max;
  int *ring_parents;    // (m_max + 1, n)
  double *ring_vals;    // (m_max + 1, n, width)
};

int diag_walk_blocks(int n);
cudaError_t launch_diag_step(const DiagSet &D, int family, int n, int NW, int CB, const void *cfg,
                             const int *parents, int slot, double *partial, double *out,
                             cudaStream_t s);
cudaError_t launch_diag_reset(const DiagSet &D, int n, cudaStream_t s);

}  // namespace gfmc

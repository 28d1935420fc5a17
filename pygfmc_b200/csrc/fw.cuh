// Off-diagonal forward walking: value remap and estimate kernels (fw.cu).
#pragma once
#include <cuda_runtime.h>

#include "../../include/gfmc_b200.h"

namespace gfmc {

// The windows of one forward walk: shadow depths m (sorted, non-negative).
struct FwRows {
  int n_m;
  int m[GFMC_FW_MAX_P];
};

// Per-walker value bookkeeping of the shadow chain, installed on the shadow
// handle for the length of one forward walk.
struct FwHook {
  double *v[2];         // values of the walkers before / after a remap
  int cur;              // which of v holds the current values
  const char *rec;      // host, per shadow depth t (0..m_max): 1 if recorded
  double *partial;      // (m_max + 1, nb) block sums of the recorded depths
  int nb;
};

int fw_blocks(int n);
// v_out[i] = v_in[parents[i]] (parents nullable: identity; v_out nullable:
// sums only); block sums of the result into partial (nullable).
cudaError_t launch_fw_remap(int n, const int *parents, const double *v_in, double *v_out,
                            double *partial, cudaStream_t s);
// val_out[j] = sum(partial[m_j]) / n, norm_out[j] = sum_{t < m_j} logG[t].
cudaError_t launch_fw_finish(const double *partial, int nb, int n, const double *logG,
                             const FwRows &rows, double *val_out, double *norm_out,
                             cudaStream_t s);

}  // namespace gfmc

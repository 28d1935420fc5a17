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
  const __nv_bfloat16 *W2T;  // (H1, H2): W2 transposed (the trainer's backward operand)
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

// ---- trainer (mlp_train.cu) ----
// Training rows: r = w (n_off + 1) + s (s < n_off the moves of walker w,
// s = n_off the walker itself), padded with zero rows to Mpad (a multiple of
// 128).  Master parameters and gradients are one float32 array in the order
// W1 (H1, D), b1 (H1), W2 (H2, H1), b2 (H2), w3 (H2), D = N (n_max + 1).
long long mlp_param_count(int H1, int H2, int D);
// Row coefficients (g_w r_ws for a move, -g_w R_w for the walker itself, 0
// for rows without an element), the W1 columns each move row exchanges
// (rowcols: old a, new a, old b, new b; x < 0 for none), first-layer
// activations h1 (Mpad, H1), their bf16 rounding residuals h1lo (Mpad, H1)
// and h1 transposed (H1, Mpad), bf16.  At least 10 rows per walker.
cudaError_t launch_mlp_rows(const DevModel<float> &m, const MlpTables &t, const void *cfg, int CB,
                            int n, long long Mpad, const float *rates, const float *rsum,
                            const float *gw, float *coef, int4 *rowcols, __nv_bfloat16 *h1,
                            __nv_bfloat16 *h1lo, __nv_bfloat16 *h1T, cudaStream_t s);

enum MlpEpilogue { MLP_EPI_FWD = 0, MLP_EPI_BWD = 1, MLP_EPI_ACC = 2 };

// C (M x N) = A (M x K) B (N x K)^T on the tensor cores, A and B bf16 with K
// contiguous (row strides lda, ldb elements), N a multiple of 32 up to 256, K
// a multiple of 64; the epilogue consumes C:
//   MLP_EPI_FWD (C = W2 h1 per row): d2 = coef w3 (1 - h2^2), h2 = tanh(C +
//     b2), as a bf16 pair hi + lo (hi = bf16(d2), lo = bf16(d2 - hi)); writes
//     d2 (M, 2N) = [hi | lo] per row and d2T (N, 2M) = [hi^T | lo^T] per
//     column (ldT = 2M), adds sum coef h2 to g_w3 and sum d2 to g_b2;
//   MLP_EPI_BWD (C = W2^T d2 per row): d1 = C (1 - t1^2), t1 = h1 + h1lo
//     (the unrounded activation; both (M, N) bf16); writes d1 (M, N)
//     float32, adds sum d1 to g_b1;
//   MLP_EPI_ACC: C is added into the float32 matrix C_out (ldc); K is split
//     over the grid.
struct MlpGemmArgs {
  const __nv_bfloat16 *A;
  long long lda;
  const __nv_bfloat16 *B;
  long long ldb;
  int M, N, K;
  int kb;                    // B's K extent (0: K); A's K index k pairs with B's k mod kb
  int kchunks_per_cta;
  int mode;
  const float *coef, *b2, *w3;
  __nv_bfloat16 *d2, *d2T;
  long long ldT;
  float *g_w3, *g_b2;
  const __nv_bfloat16 *h1, *h1lo;
  float *d1, *g_b1;
  float *C;
  long long ldc;
  int *status;
};
cudaError_t launch_mlp_gemm(const MlpGemmArgs &g, cudaStream_t s);
// dW1 (H1, D) += sum over rows of d1 x^T (x one-hot), d1 (rows, H1) float32,
// the move rows' columns from launch_mlp_rows.
cudaError_t launch_mlp_dw1(const DevModel<float> &m, const MlpTables &t, const void *cfg, int CB,
                           int n, const float *d1, const int4 *rowcols, float *gW1, cudaStream_t s);
// Adam (beta 0.9 / 0.999, eps 1e-8, bias corrections of step `step`).
cudaError_t launch_mlp_adam(long long np, float *p, const float *g, float *m1, float *m2, float lr,
                            int step, cudaStream_t s);
// Master parameters -> the guide's tables; the tables -> master parameters.
cudaError_t launch_mlp_tables(const MlpTables &t, int D, const float *p, __nv_bfloat16 *W1T, float *b1,
                              __nv_bfloat16 *W2, __nv_bfloat16 *W2T, float *b2, float *w3,
                              cudaStream_t s);
cudaError_t launch_mlp_master_init(const MlpTables &t, int D, float *p, cudaStream_t s);

}  // namespace gfmc

// Diagonal observables with forward walking (ancestry tracing), float64.
//
// engine/driver.py:228-288 and _diag_ring_buffers:810-838: after every
// reconfiguration the parent map and the diagonal operator values of the
// resampled walkers enter ring buffers of depth m_max + 1; the estimate at
// window p (m = p / 2) is the mean over walkers of the value their ancestor
// had m steps earlier, found by walking m parent maps back.  Unwritten slots
// hold identity maps and zeros, as in the reference.
//
// diag_values: one warp per walker, the population read through the parent
//   map, every operator's values (SpinHalf.diagonal_weight:291-314,
//   BoseHubbard.diagonal_weight:271-281, SzSzStructureFactor.diagonal_weight
//   (hamiltonian/observables.py:68-176)) into the value ring.
// diag_walk: one thread per walker, the ancestry walk for every window and
//   per-block sums of the traced values; diag_finish sums the blocks in a
//   fixed order and divides by N.
#include <cfloat>

#include "diag.cuh"

namespace gfmc {
namespace {

constexpr int WT = 256;

__device__ __forceinline__ double spin_val(const uint64_t *w, int k) {
  return ((w[k >> 6] >> (k & 63)) & 1ull) ? 1.0 : -1.0;
}

__global__ void diag_values_kernel(DiagSet D, int family, int n, int NW, int CB,
                                   const void *cfg, const int *parents, int slot) {
  const int lane = threadIdx.x & 31;
  const int walker = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (walker >= n) return;
  const int src = parents ? parents[walker] : walker;
  const uint64_t *bits = family == SPIN_HALF
                             ? reinterpret_cast<const uint64_t *>(cfg) + (size_t)src * NW
                             : nullptr;
  const uint8_t *occ = family == SPIN_HALF
                           ? nullptr
                           : reinterpret_cast<const uint8_t *>(cfg) + (size_t)src * CB;
  double *vals = D.ring_vals + ((size_t)slot * n + walker) * D.width;
  for (int o = 0; o < D.n_ops; ++o) {
    const DiagOp &op = D.ops[o];
    if (op.kind == DIAG_SPIN) {
      int na = 0;
      double jzs = 0.0, hzs = 0.0;
      if (op.has_jz) {
        for (int e = lane; e < op.E; e += 32) {
          const bool anti = spin_val(bits, op.ei[e]) != spin_val(bits, op.ej[e]);
          if (op.uniform_jz) na += anti;
          else jzs += anti ? -op.jz[e] / 4.0 : op.jz[e] / 4.0;
        }
      }
      if (op.has_hz)
        for (int k = lane; k < op.N; k += 32) hzs += op.hz[k] * spin_val(bits, k);
      double d = 0.0;
      if (op.has_jz) {
        if (op.uniform_jz) d = (op.jz[0] / 4.0) * (double)(op.E - 2 * warp_sum(na));
        else d = warp_sum(jzs);
      }
      if (op.has_hz) d = d + warp_sum(hzs) / 2.0;
      if (lane == 0) vals[op.col] = d;
    } else if (op.kind == DIAG_BOSE) {
      double su = 0.0, sm = 0.0;
      for (int k = lane; k < op.N; k += 32) {
        const double nk = (double)occ[k];
        if (op.has_U) su += op.U[k] * nk * (nk - 1.0);
        if (op.has_mu) sm += op.mu[k] * nk;
      }
      double d = 0.0;
      if (op.has_U) d = d + 0.5 * warp_sum(su);
      if (op.has_mu) d = d - warp_sum(sm);
      if (lane == 0) vals[op.col] = d;
    } else {  // DIAG_SZSZ: 0.25 (|sum x cos|^2 + |sum x sin|^2) - offset, per k
      for (int q = 0; q < op.n_k; ++q) {
        double c = 0.0, s = 0.0;
        const double *cr = op.cos_kr + (size_t)q * op.N, *sr = op.sin_kr + (size_t)q * op.N;
        for (int k = lane; k < op.N; k += 32) {
          const double x = family == SPIN_HALF ? spin_val(bits, k) : (double)occ[k];
          c += x * cr[k];
          s += x * sr[k];
        }
        c = warp_sum(c);
        s = warp_sum(s);
        if (lane == 0) vals[op.col + q] = 0.25 * (c * c + s * s) - op.offset;
      }
    }
  }
  if (lane == 0) D.ring_parents[(size_t)slot * n + walker] = parents ? parents[walker] : walker;
}

// partial layout: [block][col][j]
__global__ void diag_walk_kernel(DiagSet D, int n, int slot, double *partial) {
  extern __shared__ double sh[];   // [WT/32] per reduction
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const int size = D.m_max + 1;
  int anc[GFMC_DIAG_MAX_P];
  int a = w < n ? w : 0;
  int back = 0;
  for (int j = 0; j < D.n_p; ++j) {
    const int m = D.m[j];
    for (; back < m; ++back) {
      const int idx = ((slot - back) % size + size) % size;
      a = D.ring_parents[(size_t)idx * n + a];
    }
    anc[j] = a;
  }
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (int j = 0; j < D.n_p; ++j) {
    const int old = ((slot - D.m[j]) % size + size) % size;
    for (int c = 0; c < D.width; ++c) {
      double v = w < n ? D.ring_vals[((size_t)old * n + anc[j]) * D.width + c] : 0.0;
      v = warp_sum(v);
      if (lane == 0) sh[wi] = v;
      __syncthreads();
      if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
        partial[((size_t)blockIdx.x * D.width + c) * D.n_p + j] = s;
      }
      __syncthreads();
    }
  }
}

__global__ void diag_finish_kernel(const double *partial, int nblocks, int cols, int n,
                                   double *out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cols) return;
  double s = 0.0;
  for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * cols + t];
  out[t] = s / (double)n;
}

__global__ void diag_reset_kernel(DiagSet D, int n) {
  const size_t total = (size_t)(D.m_max + 1) * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    D.ring_parents[i] = (int)(i % n);
    for (int c = 0; c < D.width; ++c) D.ring_vals[i * D.width + c] = 0.0;
  }
}

}  // namespace

int diag_walk_blocks(int n) { return (n + WT - 1) / WT; }

cudaError_t launch_diag_step(const DiagSet &D, int family, int n, int NW, int CB, const void *cfg,
                             const int *parents, int slot, double *partial, double *out,
                             cudaStream_t s) {
  diag_values_kernel<<<(n + 7) / 8, 256, 0, s>>>(D, family, n, NW, CB, cfg, parents, slot);
  const int nb = diag_walk_blocks(n);
  diag_walk_kernel<<<nb, WT, (WT / 32) * sizeof(double), s>>>(D, n, slot, partial);
  const int cols = D.width * D.n_p;
  diag_finish_kernel<<<(cols + 127) / 128, 128, 0, s>>>(partial, nb, cols, n, out);
  return cudaGetLastError();
}

cudaError_t launch_diag_reset(const DiagSet &D, int n, cudaStream_t s) {
  diag_reset_kernel<<<256, 256, 0, s>>>(D, n);
  return cudaGetLastError();
}

}  // namespace gfmc

// The per-rank pieces of a systematic resampling over walkers sharded across
// GPUs (contiguous walker blocks per rank), float64.
//
// Weights are exp(log_w - shift) with one global shift (the max over ranks),
// so the ranks' weight sums S_r add up to the global sum S.  Output slot i of
// the global population (i < N) takes U_i = (i + psi) / N * S and the walker
// whose cumulative weight interval contains it; rank r owns the slots whose
// U_i falls in [O_r, O_r + S_r), O_r = sum_{k<r} S_k, a contiguous slot range
// every rank computes identically from the gathered sums.  Each rank finds
// the parents of its own slots in its local cdf and sends the walkers to the
// ranks that own the slots (the data moves once, in contiguous blocks).
//
// Per-tile partials are combined in a fixed sequential order (the canonical
// order of reconfig.cu).
#include <cfloat>

#include "engine.cuh"

namespace gfmc {
namespace {

constexpr int DT = 256;
constexpr int DPT = 4;
constexpr int DTILE = DT * DPT;

__global__ void dist_tile_max(int n, const double *lw, double *tmax) {
  __shared__ double sh[DT / 32];
  double v = -DBL_MAX;
  for (int j = 0; j < DPT; ++j) {
    const int k = blockIdx.x * DTILE + j * DT + threadIdx.x;
    if (k < n) v = lw[k] > v ? lw[k] : v;
  }
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = -DBL_MAX;
    for (int i = 0; i < DT / 32; ++i) r = sh[i] > r ? sh[i] : r;
    tmax[blockIdx.x] = r;
  }
}

// the common shift: the host value, or the one in device memory when given
// (the max over ranks reduced there); a non-finite max (no live walker) is 0
__device__ __forceinline__ double dist_shift(double shift, const double *shift_p) {
  const double v = shift_p ? *shift_p : shift;
  return (v > -DBL_MAX && v < DBL_MAX) ? v : 0.0;
}

// per tile: sum w, sum w e, last positive index (w = exp(lw - shift))
__global__ void dist_tile_sums(int n, const double *lw, const double *e, double shift_h,
                               const double *shift_p, double *tS, double *tE, int *tlp) {
  __shared__ double s1[DT / 32], s2[DT / 32];
  __shared__ int s3[DT / 32];
  const double shift = dist_shift(shift_h, shift_p);
  double a = 0.0, b = 0.0;
  int lp = -1;
  const int base = blockIdx.x * DTILE + threadIdx.x * DPT;
  for (int j = 0; j < DPT; ++j) {
    const int k = base + j;
    if (k < n) {
      const double w = exp(lw[k] - shift);
      a += w;
      b += w * e[k];
      if (w > 0.0) lp = k;
    }
  }
  a = warp_sum(a);
  b = warp_sum(b);
  lp = warp_max(lp);
  if ((threadIdx.x & 31) == 0) {
    s1[threadIdx.x >> 5] = a;
    s2[threadIdx.x >> 5] = b;
    s3[threadIdx.x >> 5] = lp;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    int l = -1;
    for (int i = 0; i < DT / 32; ++i) {
      x += s1[i];
      y += s2[i];
      l = s3[i] > l ? s3[i] : l;
    }
    tS[blockIdx.x] = x;
    tE[blockIdx.x] = y;
    tlp[blockIdx.x] = l;
  }
}

// over the tiles: out[0] = max (tmax given) or the shift the sums used;
// out[1..3] = (S, sum w e, last positive index) (tS given)
__global__ void dist_combine(int nb, const double *tmax, const double *tS, const double *tE,
                             const int *tlp, double shift_h, const double *shift_p, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = -DBL_MAX, S = 0.0, SE = 0.0;
  int l = -1;
  for (int b = 0; b < nb; ++b) {
    if (tmax) m = tmax[b] > m ? tmax[b] : m;
    if (tS) {
      S += tS[b];
      SE += tE[b];
      l = tlp[b] > l ? tlp[b] : l;
    }
  }
  if (tmax) {
    out[0] = m;
    return;
  }
  out[0] = dist_shift(shift_h, shift_p);
  out[1] = S;
  out[2] = SE;
  out[3] = (double)l;
}

// cdf of the local walkers in global weight units (offset: the earlier ranks')
__global__ void dist_cdf(int n, int nb, const double *lw, double shift, double offset,
                         const double *tS, double *cdf, double *wbuf) {
  __shared__ double s_scan[DT / 32];
  __shared__ double s_off;
  if (threadIdx.x == 0) {
    double pre = 0.0;
    for (int b = 0; b < (int)blockIdx.x && b < nb; ++b) pre += tS[b];
    s_off = offset + pre;
  }
  __syncthreads();
  const int base = blockIdx.x * DTILE + threadIdx.x * DPT;
  double w[DPT], loc[DPT], acc = 0.0;
  for (int j = 0; j < DPT; ++j) {
    const int k = base + j;
    const double wk = k < n ? exp(lw[k] - shift) : 0.0;
    w[j] = wk;
    acc += wk;
    loc[j] = acc;
  }
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  const double inc = warp_inclusive_scan(acc, lane);
  if (lane == 31) s_scan[wi] = inc;
  __syncthreads();
  double wpre = 0.0;
  for (int i = 0; i < wi; ++i) wpre += s_scan[i];
  const double excl = wpre + inc - acc;
  for (int j = 0; j < DPT; ++j) {
    const int k = base + j;
    if (k < n) {
      cdf[k] = s_off + (excl + loc[j]);
      wbuf[k] = w[j];
    }
  }
}

// local parents of the global slots [i_lo, i_lo + count): searchsorted(cdf,
// U, right), capped at the last positive weight, stepped back off zero weights
__global__ void dist_parents(int n, const double *cdf, const double *wbuf, double psi,
                             double S_total, long long N_total, long long i_lo, int count,
                             int last_pos, int *parents) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const double U = ((double)(i_lo + t) + psi) / (double)N_total * S_total;
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cdf[mid] <= U) lo = mid + 1;
    else hi = mid;
  }
  int k = lo < last_pos ? lo : last_pos;
  while (k > 0 && !(wbuf[k] > 0.0)) --k;
  parents[t] = k;
}

}  // namespace

int dist_tiles(int n) { return (n + DTILE - 1) / DTILE; }

cudaError_t launch_dist_max(int n, const double *lw, double *tmax, double *out, cudaStream_t s) {
  const int nb = dist_tiles(n);
  dist_tile_max<<<nb, DT, 0, s>>>(n, lw, tmax);
  dist_combine<<<1, 32, 0, s>>>(nb, tmax, nullptr, nullptr, nullptr, 0.0, nullptr, out);
  return cudaGetLastError();
}

cudaError_t launch_dist_sums(int n, const double *lw, const double *e, double shift,
                             const double *shift_dev, double *tS, double *tE, int *tlp,
                             double *out, cudaStream_t s) {
  const int nb = dist_tiles(n);
  dist_tile_sums<<<nb, DT, 0, s>>>(n, lw, e, shift, shift_dev, tS, tE, tlp);
  dist_combine<<<1, 32, 0, s>>>(nb, nullptr, tS, tE, tlp, shift, shift_dev, out);
  return cudaGetLastError();
}

cudaError_t launch_dist_parents(int n, const double *lw, double shift, double offset,
                                const double *tS, double *cdf, double *wbuf, double psi,
                                double S_total, long long N_total, long long i_lo, int count,
                                int last_pos, int *parents, cudaStream_t s) {
  const int nb = dist_tiles(n);
  dist_cdf<<<nb, DT, 0, s>>>(n, nb, lw, shift, offset, tS, cdf, wbuf);
  if (count > 0)
    dist_parents<<<(count + 255) / 256, 256, 0, s>>>(n, cdf, wbuf, psi, S_total, N_total, i_lo,
                                                      count, last_pos, parents);
  return cudaGetLastError();
}

}  // namespace gfmc

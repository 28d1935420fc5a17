// Population control of GFMC on B200: systematic resampling
// (walkers/reconfiguration.py:9-62) in float64, in three launches per step:
//
//   recon_sum      per tile of 1024 walkers: s_b = sum exp(log_w - max)
//   recon_cdf      log G = log(sum_b s_b) + max, w = exp(log_w - log G),
//                  the tile's inclusive prefix of w offset by the canonical
//                  prefix of the tile sums, sum e_loc * w, last positive w
//   recon_parents  one thread per output slot i: u = (i + psi) / N, the
//                  first walker whose cdf exceeds u (binary search), capped
//                  at the last positive weight
//
// The configuration gather is not a pass of its own: the next evolve
// kernel loads walker i from parents[i].  The weighted energy of each step is
// left as per-tile partials and reduced, in a fixed order, once per chunk.
// Also here: the explicit gather (end of a run), configuration packing, and
// the windowed energy estimator (engine/estimators.py:268-305) in float64.
#include <cfloat>

#include "engine.cuh"

namespace gfmc {
namespace {

constexpr int RT = 256;          // threads per reconfiguration block
constexpr int RPT = 4;           // walkers per thread
constexpr int TILE = RT * RPT;   // walkers per tile

__device__ __forceinline__ double block_reduce_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
    sh[32] = r;
  }
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double global_max(const double *pm, int n, double *sh) {
  double v = -DBL_MAX;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v = pm[i] > v ? pm[i] : v;
  v = warp_max(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = -DBL_MAX;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = sh[i] > r ? sh[i] : r;
    sh[32] = r;
  }
  __syncthreads();
  v = sh[32];
  __syncthreads();
  return v;
}

// The shift jax.scipy.special.logsumexp uses: the max when finite, else 0.
__device__ __forceinline__ double lse_shift(double gmax) {
  return (gmax > -DBL_MAX && gmax < DBL_MAX) ? gmax : 0.0;
}

__global__ void __launch_bounds__(RT) recon_sum(ReconArgs a) {
  __shared__ double sh[33];
  const double gmax = global_max(a.partial_max, a.n_partial_max, sh);
  const double shift = lse_shift(gmax);
  const int base = blockIdx.x * TILE;
  double s = 0.0;
  for (int j = 0; j < RPT; ++j) {
    int k = base + j * RT + threadIdx.x;
    if (k < a.n) s += exp(a.log_w[k] - shift);
  }
  s = block_reduce_sum(s, sh);
  if (threadIdx.x == 0) a.psum[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RT) recon_cdf(ReconArgs a, int nb) {
  __shared__ double sh[33];
  __shared__ double s_scan[RT / 32];
  __shared__ double s_tot[3];
  __shared__ int s_lp[RT / 32];
  const double gmax = global_max(a.partial_max, a.n_partial_max, sh);
  const double shift = lse_shift(gmax);
  if (threadIdx.x == 0) {
    // canonical, sequential prefix of the tile sums (identical in every block)
    double S = 0.0, pre = 0.0;
    for (int b = 0; b < nb; ++b) {
      if (b == (int)blockIdx.x) pre = S;
      S += a.psum[b];
    }
    s_tot[0] = S;
    s_tot[1] = log(S) + shift;   // log G_n
    s_tot[2] = pre / S;          // cdf offset of this tile
  }
  __syncthreads();
  const double lG = s_tot[1], off = s_tot[2];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.logG_out = lG - log((double)a.n);
    if (!(lG > -DBL_MAX && lG < DBL_MAX)) atomicOr(a.status, ST_NONFINITE);
  }
  // thread t owns walkers base + RPT t .. + RPT - 1 (contiguous)
  const int base = blockIdx.x * TILE + threadIdx.x * RPT;
  double w[RPT], loc[RPT];
  double acc = 0.0, eacc = 0.0;
  int lp = -1;
  for (int j = 0; j < RPT; ++j) {
    int k = base + j;
    double wk = 0.0;
    if (k < a.n) {
      wk = exp(a.log_w[k] - lG);
      eacc += a.e_loc[k] * wk;
      if (wk > 0.0) lp = k;
    }
    w[j] = wk;
    acc += wk;
    loc[j] = acc;
  }
  // block exclusive scan of the per-thread totals
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  double inc = warp_inclusive_scan(acc, lane);
  if (lane == 31) s_scan[wi] = inc;
  int lpw = warp_max(lp);
  if (lane == 0) s_lp[wi] = lpw;
  __syncthreads();
  double wpre = 0.0;
  for (int i = 0; i < wi; ++i) wpre += s_scan[i];
  const double excl = wpre + inc - acc;
  for (int j = 0; j < RPT; ++j) {
    int k = base + j;
    if (k < a.n) {
      a.cdf[k] = off + (excl + loc[j]);
      a.wbuf[k] = w[j];
    }
  }
  double e = block_reduce_sum(eacc, sh);
  if (threadIdx.x == 0) {
    a.pE[blockIdx.x] = e;
    int l = -1;
    for (int i = 0; i < RT / 32; ++i) l = s_lp[i] > l ? s_lp[i] : l;
    a.plp[blockIdx.x] = l;
  }
}

__global__ void __launch_bounds__(RT) recon_parents(ReconArgs a, int nb) {
  __shared__ int s_lp;
  __shared__ double s_psi;
  if (threadIdx.x == 0) {
    int l = -1;
    for (int b = 0; b < nb; ++b) l = a.plp[b] > l ? a.plp[b] : l;
    s_lp = l < 0 ? 0 : l;   // max(where(w > 0, arange, 0)): 0 when none
    s_psi = uniform_f64(a.key);
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double u = ((double)i + s_psi) / (double)a.n;
  int lo = 0, hi = a.n;   // searchsorted(cdf, u, side="right")
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a.cdf[mid] <= u) lo = mid + 1;
    else hi = mid;
  }
  int k = lo < s_lp ? lo : s_lp;
  while (k > 0 && !(a.wbuf[k] > 0.0)) --k;   // never a zero-weight parent
  a.parents[i] = k;
}

// ---- the three phases in one cooperative launch ----------------------------
// One block of TILE threads per tile (one walker or output slot per thread);
// the phases are separated by grid barriers on a counter that only grows
// (the host passes its value at launch, bar_base): barrier k of the launch
// waits until every block has arrived, i.e. the counter reaches
// bar_base + k nb.  Each wait is bounded; one that runs out sets ST_TIMEOUT
// (the host then reports the error) and the block carries on.  The
// arithmetic is that of the three launches with one walker per thread.
constexpr int FT = TILE;                 // threads per block of the fused launch
constexpr uint32_t BAR_LIMIT = 1u << 22;

__device__ __forceinline__ void grid_barrier(unsigned *ctr, unsigned target, int *status) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    uint32_t it = 0;
    while ((int)(*(volatile unsigned *)ctr - target) < 0 && ++it < BAR_LIMIT) __nanosleep(32);
    if (it >= BAR_LIMIT) atomicOr(status, ST_TIMEOUT);
    __threadfence();
  }
  __syncthreads();
}

__device__ __forceinline__ double block_sum_f(double v, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < FT / 32; ++i) r += sh[i];
    sh[32] = r;
  }
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(FT) recon_fused(ReconArgs a, int nb, unsigned *ctr,
                                                  unsigned bar_base) {
  __shared__ double sh[33];
  __shared__ double s_scan[FT / 32];
  __shared__ int s_lp[FT / 32];
  __shared__ double s_tot[3];
  __shared__ int s_last;
  __shared__ double s_psi;
  const int tid = threadIdx.x, lane = tid & 31, wi = tid >> 5;
  const int k = blockIdx.x * FT + tid;
  const double gmax = global_max(a.partial_max, a.n_partial_max, sh);
  const double shift = lse_shift(gmax);
  const double lwk = k < a.n ? a.log_w[k] : 0.0;
  // phase 1: the tile's sum of exp(log_w - shift)
  const double s = block_sum_f(k < a.n ? exp(lwk - shift) : 0.0, sh);
  if (tid == 0) a.psum[blockIdx.x] = s;
  grid_barrier(ctr, bar_base + (unsigned)nb, a.status);
  // phase 2: log G, the weights and the cdf (canonical prefix of the tile sums)
  if (tid == 0) {
    double S = 0.0, pre = 0.0;
    for (int b = 0; b < nb; ++b) {   // (other blocks' values: L2 loads)
      if (b == (int)blockIdx.x) pre = S;
      S += __ldcg(a.psum + b);
    }
    s_tot[0] = S;
    s_tot[1] = log(S) + shift;
    s_tot[2] = pre / S;
  }
  __syncthreads();
  const double lG = s_tot[1], off = s_tot[2];
  if (blockIdx.x == 0 && tid == 0) {
    *a.logG_out = lG - log((double)a.n);
    if (!(lG > -DBL_MAX && lG < DBL_MAX)) atomicOr(a.status, ST_NONFINITE);
  }
  double wk = 0.0, ek = 0.0;
  int lp = -1;
  if (k < a.n) {
    wk = exp(lwk - lG);
    ek = a.e_loc[k] * wk;
    if (wk > 0.0) lp = k;
  }
  const double inc = warp_inclusive_scan(wk, lane);
  if (lane == 31) s_scan[wi] = inc;
  const int lpw = warp_max(lp);
  if (lane == 0) s_lp[wi] = lpw;
  __syncthreads();
  double wpre = 0.0;
  for (int i = 0; i < wi; ++i) wpre += s_scan[i];
  if (k < a.n) {
    a.cdf[k] = off + (wpre + inc);
    a.wbuf[k] = wk;
  }
  const double e = block_sum_f(ek, sh);
  if (tid == 0) {
    a.pE[blockIdx.x] = e;
    int l = -1;
    for (int i = 0; i < FT / 32; ++i) l = s_lp[i] > l ? s_lp[i] : l;
    a.plp[blockIdx.x] = l;
  }
  grid_barrier(ctr, bar_base + 2u * (unsigned)nb, a.status);
  // the step's E_n: the tile partials in tile order (series_reduce's sum)
  if (a.E_step && blockIdx.x == 0 && tid == 0) {
    double es = 0.0;
    for (int b = 0; b < nb; ++b) es += __ldcg(a.pE + b);
    *a.E_step = es;
  }
  // phase 3: the parent of output slot k
  if (tid == 0) {
    int l = -1;
    for (int b = 0; b < nb; ++b) {
      const int pl = __ldcg(a.plp + b);
      l = pl > l ? pl : l;
    }
    s_last = l < 0 ? 0 : l;
    s_psi = uniform_f64(a.key);
  }
  __syncthreads();
  if (k >= a.n) return;
  const double u = ((double)k + s_psi) / (double)a.n;
  int lo = 0, hi = a.n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldcg(a.cdf + mid) <= u) lo = mid + 1;
    else hi = mid;
  }
  int q = lo < s_last ? lo : s_last;
  while (q > 0 && !(__ldcg(a.wbuf + q) > 0.0)) --q;
  a.parents[k] = q;
}

__global__ void series_reduce(const double *pE, int nb, int n_steps, double *E_out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_steps) return;
  double e = 0.0;
  for (int b = 0; b < nb; ++b) e += pE[(size_t)s * nb + b];
  E_out[s] = e;
}

__global__ void gather_kernel(int n, int cfg_bytes, const int *parents, const void *cfg_in,
                              void *cfg_out, const double *e_in, double *e_out, double *log_w) {
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  if (i >= n) return;
  const int p = parents ? parents[i] : i;
  const uint32_t *src = reinterpret_cast<const uint32_t *>(
      reinterpret_cast<const uint8_t *>(cfg_in) + (size_t)p * cfg_bytes);
  uint32_t *dst = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(cfg_out) +
                                               (size_t)i * cfg_bytes);
  for (int k = threadIdx.x; k < cfg_bytes / 4; k += blockDim.x) dst[k] = src[k];
  if (threadIdx.x == 0) {
    if (e_out) e_out[i] = e_in[p];
    if (log_w) log_w[i] = 0.0;
  }
}

// engine/estimators.py _energy_and_diagonal_estimates:268-305 (energy part):
// L = cumsum(log G); log G_p(i) = L[i+p] - L[i]; E_p = sum G_p E[i+p] / sum G_p.
// One block per window p; the prefix sum is sequential (thread 0) so that the
// window products are the float64 differences of one canonical cumulative sum.
// L is the prefix written by prefix_kernel in the preceding launch.
__global__ void windowed_kernel(const double *E, int n, const int *p_arr, const double *L,
                                double *out) {
  __shared__ double sh[33];
  const int p = p_arr[blockIdx.x];
  const int cnt = n - p;
  double mx = -DBL_MAX;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    double v = L[i + p] - L[i];
    mx = v > mx ? v : mx;
  }
  mx = warp_max(mx);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = -DBL_MAX;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = sh[i] > r ? sh[i] : r;
    sh[32] = r;
  }
  __syncthreads();
  mx = sh[32];
  __syncthreads();
  double num = 0.0, den = 0.0;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    double g = exp((L[i + p] - L[i]) - mx);
    num += g * E[i + p];
    den += g;
  }
  num = block_reduce_sum(num, sh);
  den = block_reduce_sum(den, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = num / den;
}

__global__ void prefix_kernel(const double *logG, int n, double *L) {
  double acc = 0.0;
  for (int i = 0; i < n; ++i) { acc += logG[i]; L[i] = acc; }
}

__global__ void pack_spin(int n, int N, int NW, const double *cfg, uint64_t *out, int *status) {
  const int w = blockIdx.x * blockDim.y + threadIdx.y;
  if (w >= n) return;
  for (int word = threadIdx.x; word < NW; word += blockDim.x) {
    uint64_t bits = 0;
    for (int b = 0; b < 64; ++b) {
      int k = word * 64 + b;
      if (k < N) {
        double x = cfg[(size_t)w * N + k];
        if (x == 1.0) bits |= 1ull << b;
        else if (x != -1.0) atomicOr(status, ST_BAD_CONFIG);
      }
    }
    out[(size_t)w * NW + word] = bits;
  }
}

__global__ void unpack_spin(int n, int N, int NW, const uint64_t *in, double *cfg) {
  const int w = blockIdx.x * blockDim.y + threadIdx.y;
  if (w >= n) return;
  for (int k = threadIdx.x; k < N; k += blockDim.x)
    cfg[(size_t)w * N + k] = ((in[(size_t)w * NW + (k >> 6)] >> (k & 63)) & 1ull) ? 1.0 : -1.0;
}

__global__ void pack_bose(int n, int N, int CB, const double *cfg, uint8_t *out, int n_max,
                          int *status) {
  const int w = blockIdx.x * blockDim.y + threadIdx.y;
  if (w >= n) return;
  for (int k = threadIdx.x; k < CB; k += blockDim.x) {
    uint8_t v = 0;
    if (k < N) {
      double x = cfg[(size_t)w * N + k];
      if (!(x >= 0.0 && x <= (double)n_max && x == floor(x))) atomicOr(status, ST_BAD_CONFIG);
      else v = (uint8_t)x;
    }
    out[(size_t)w * CB + k] = v;
  }
}

__global__ void unpack_bose(int n, int N, int CB, const uint8_t *in, double *cfg) {
  const int w = blockIdx.x * blockDim.y + threadIdx.y;
  if (w >= n) return;
  for (int k = threadIdx.x; k < N; k += blockDim.x)
    cfg[(size_t)w * N + k] = (double)in[(size_t)w * CB + k];
}

}  // namespace

int recon_tiles(int n) { return (n + TILE - 1) / TILE; }

cudaError_t launch_reconfigure(const ReconArgs &a, cudaStream_t s) {
  const int nb = recon_tiles(a.n);
  recon_sum<<<nb, RT, 0, s>>>(a);
  recon_cdf<<<nb, RT, 0, s>>>(a, nb);
  recon_parents<<<(a.n + RT - 1) / RT, RT, 0, s>>>(a, nb);
  return cudaGetLastError();
}

int recon_fused_max_tiles() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, recon_fused, FT, 0) != cudaSuccess)
    return 0;
  return sms * per_sm;
}

cudaError_t launch_reconfigure_fused(const ReconArgs &a, unsigned *ctr, unsigned bar_base,
                                     cudaStream_t s) {
  int nb = recon_tiles(a.n);
  ReconArgs aa = a;
  void *args[] = {&aa, &nb, &ctr, &bar_base};
  return cudaLaunchCooperativeKernel((const void *)recon_fused, dim3(nb), dim3(FT), args, 0, s);
}

cudaError_t launch_series_reduce(const double *pE, int nb, int n_steps, double *E_out,
                                 cudaStream_t s) {
  if (n_steps <= 0) return cudaSuccess;
  series_reduce<<<(n_steps + 127) / 128, 128, 0, s>>>(pE, nb, n_steps, E_out);
  return cudaGetLastError();
}

cudaError_t launch_gather(int n, int cfg_bytes, const int *parents, const void *cfg_in,
                          void *cfg_out, const double *e_in, double *e_out, double *log_w,
                          cudaStream_t s) {
  dim3 blk(32, 8);
  gather_kernel<<<(n + 7) / 8, blk, 0, s>>>(n, cfg_bytes, parents, cfg_in, cfg_out, e_in, e_out,
                                            log_w);
  return cudaGetLastError();
}

cudaError_t launch_windowed(const double *logG, const double *E, int n_steps, const int *p,
                            int n_p, double *work, cudaStream_t s) {
  // work: n_steps doubles (prefix) followed by n_p doubles (results)
  prefix_kernel<<<1, 1, 0, s>>>(logG, n_steps, work);
  windowed_kernel<<<n_p, 256, 0, s>>>(E, n_steps, p, work, work + n_steps);
  return cudaGetLastError();
}

cudaError_t launch_pack(int family, int n, int N, int cfg_bytes, const double *cfg, void *packed,
                        int n_max, int *status, cudaStream_t s) {
  dim3 blk(32, 8);
  if (family == SPIN_HALF)
    pack_spin<<<(n + 7) / 8, blk, 0, s>>>(n, N, cfg_bytes / 8, cfg,
                                          reinterpret_cast<uint64_t *>(packed), status);
  else
    pack_bose<<<(n + 7) / 8, blk, 0, s>>>(n, N, cfg_bytes, cfg, reinterpret_cast<uint8_t *>(packed),
                                          n_max, status);
  return cudaGetLastError();
}

cudaError_t launch_unpack(int family, int n, int N, int cfg_bytes, const void *packed,
                          double *cfg, cudaStream_t s) {
  dim3 blk(32, 8);
  if (family == SPIN_HALF)
    unpack_spin<<<(n + 7) / 8, blk, 0, s>>>(n, N, cfg_bytes / 8,
                                            reinterpret_cast<const uint64_t *>(packed), cfg);
  else
    unpack_bose<<<(n + 7) / 8, blk, 0, s>>>(n, N, cfg_bytes,
                                            reinterpret_cast<const uint8_t *>(packed), cfg);
  return cudaGetLastError();
}

}  // namespace gfmc

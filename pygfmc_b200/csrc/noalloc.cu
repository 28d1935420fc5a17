// gfmc_reconfigure_noalloc: systematic resampling of a walker population
// that allocates no device memory.
//
// Who needs it: callers that must not allocate device memory inside a call.
// A host framework that owns the whole device through its own pool
// allocator can see a plugin's cudaMalloc fail (or fragment its arena), and
// cudaMalloc / cudaFree synchronise the device, which stalls every stream of
// a latency-critical loop.  This entry point takes its scratch from a fixed,
// file-scope device array instead.
//
// Limits and behaviour:
//  * at most GFMC_NOALLOC_MAX_WALKERS (131072) walkers per call; larger
//    populations are refused with GFMC_ERR_INVALID before any GPU work;
//  * the array (~2 MB) is held by every GPU that loads the library, until
//    the process exits;
//  * every call on a device shares the array and it keeps the last call's
//    contents: calls whose kernels overlap on the GPU (on different streams
//    without ordering between them) race on it.  Nothing in it needs to
//    start at zero: each pass writes every entry the next pass reads;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make
//    that first call before any stream capture;
//  * the call does not wait for the GPU and returns no status: the status
//    word the resampling kernels write lives in the array and is never read.
//    The one condition it records (weights that sum to zero or overflow) is
//    exactly a non-finite *logG_out, which is the caller's signal.
#include <cfloat>
#include <mutex>

#include "../../include/gfmc_b200.h"
#include "engine.cuh"

namespace {

constexpr int kMaxWalkers = GFMC_NOALLOC_MAX_WALKERS;
constexpr int kTile = 1024;                       // walkers per reconfiguration tile
constexpr int kMaxTiles = kMaxWalkers / kTile;    // 128
// layout (doubles): cdf[kMaxWalkers] | wbuf[kMaxWalkers] | tile max | tile sums |
// tile energies | tile last-positive (as int) | status (as int)
constexpr size_t kScratchDoubles = 2 * (size_t)kMaxWalkers + 4 * (size_t)kMaxTiles + 2;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_dev_ptr[kMaxDevices] = {nullptr};

// Per-tile maximum of log_w (the role the evolve kernel's per-warp maxima
// play in gfmc_run_steps).
__global__ void tile_max_kernel(const double *log_w, int n, double *tile_max) {
  __shared__ double sh[8];
  const int base = blockIdx.x * kTile;
  double v = -DBL_MAX;
  for (int j = threadIdx.x; j < kTile; j += blockDim.x) {
    const int k = base + j;
    if (k < n && log_w[k] > v) v = log_w[k];
  }
  v = gfmc::warp_max(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = -DBL_MAX;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r = sh[i] > r ? sh[i] : r;
    tile_max[blockIdx.x] = r;
  }
}

}  // namespace

namespace gfmc {
int record_error(int code, const char *msg);   // capi.cu: the gfmc_last_error message
}

namespace {
int set_err(int code, const char *msg) { return gfmc::record_error(code, msg); }
}  // namespace

extern "C" int gfmc_reconfigure_noalloc(int n_walkers, const double *log_w, const double *e_loc,
                                        const uint32_t key[2], int32_t *parents_out,
                                        double *logG_out, double *E_out, void *stream) {
  if (n_walkers <= 0 || !log_w || !e_loc || !key || !parents_out || !logG_out || !E_out)
    return set_err(GFMC_ERR_INVALID, "gfmc_reconfigure_noalloc: null or empty argument");
  if (n_walkers > kMaxWalkers)
    return set_err(GFMC_ERR_INVALID,
                   "gfmc_reconfigure_noalloc: n_walkers exceeds GFMC_NOALLOC_MAX_WALKERS (131072)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_err(GFMC_ERR_CUDA, "gfmc_reconfigure_noalloc: no usable current device");
  double *base;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_ptr[dev]) {
      // the array's device address on this (current) device; host code may not
      // use the symbol itself as a device pointer
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return set_err(GFMC_ERR_CUDA, "gfmc_reconfigure_noalloc: cudaGetSymbolAddress failed");
      g_dev_ptr[dev] = static_cast<double *>(p);
    }
    base = g_dev_ptr[dev];
  }
  const int nb = (n_walkers + kTile - 1) / kTile;
  double *cdf = base;
  double *wbuf = base + kMaxWalkers;
  double *tmax = base + 2 * (size_t)kMaxWalkers;
  double *tsum = tmax + kMaxTiles;
  double *tE = tsum + kMaxTiles;
  int *tlp = reinterpret_cast<int *>(tE + kMaxTiles);
  int *status = reinterpret_cast<int *>(tE + 2 * kMaxTiles);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  tile_max_kernel<<<nb, 256, 0, s>>>(log_w, n_walkers, tmax);
  gfmc::ReconArgs r{};
  r.n = n_walkers;
  r.log_w = log_w;
  r.e_loc = e_loc;
  r.partial_max = tmax;
  r.n_partial_max = nb;
  r.key = gfmc::Key{key[0], key[1]};
  r.psum = tsum;
  r.pE = tE;
  r.plp = tlp;
  r.cdf = cdf;
  r.wbuf = wbuf;
  r.parents = parents_out;
  r.logG_out = logG_out;
  r.status = status;
  e = gfmc::launch_reconfigure(r, s);
  if (e == cudaSuccess) e = gfmc::launch_series_reduce(tE, nb, 1, E_out, s);
  if (e != cudaSuccess) return set_err(GFMC_ERR_CUDA, "gfmc_reconfigure_noalloc: launch failed");
  return GFMC_OK;
}

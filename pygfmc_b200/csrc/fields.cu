// Guide state of a whole population at once, for dense Jastrow couplings:
//   F[w, k] = sum_p Jd[p, k] x_p(w)       (x = +-1 spins or occupations)
// and, for spin-1/2, the signed ratio factors s_k = x_k exp(-2 x_k (F_k + h_k))
// the step kernel carries (JastrowSpinHalf; jastrow_spin_half.py:290-353).
//
// The step kernel rebuilds this state per walker when it has none to carry
// (a fresh population, every refresh); with a dense coupling matrix that is
// N^2 multiply-adds per walker through L2.  Here the population's fields are
// one (walkers x N) x (N x N) product.  A block takes 64 walkers and 128
// output sites (blockIdx.y picks the sites): the walkers' configurations are
// staged in shared memory once, J comes in chunks of 16 rows x 128 columns
// through a two-stage cp.async ring (the next chunk lands while the current
// one is used), and each thread accumulates 4 walkers x 8 sites in
// registers, adding the sites p = 0 .. N-1 in order with one fused
// multiply-add each -- the order and rounding of the step kernel's own
// rebuild, so the carried state is bit-identical to it.  Rows are indexed
// like the configurations (the step reads them through the parent map).
#include "engine.cuh"

namespace gfmc {
namespace {

constexpr int FW = 64;    // walkers per block
constexpr int FS = 128;   // output sites per block
constexpr int FK = 16;    // sites p per chunk of J
constexpr int CFG_STAGE_MAX = 64 * 1024;   // staged configuration bytes per block at most

__device__ __forceinline__ uint32_t sh_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One element of J into shared memory (zero-filled when it lies outside J).
template <int SZ>
__device__ __forceinline__ void cp_el(void *dst, const void *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(sh_addr(dst)), "l"(src),
               "n"(SZ), "r"(valid ? SZ : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND> __device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

// +-1 from bit b of a spin word.
template <typename T> __device__ __forceinline__ T spin_of(uint32_t word, int b) {
  return ((word >> b) & 1u) ? T(1) : T(-1);
}

template <typename T, int FAM>
__global__ void __launch_bounds__(256) fields_kernel(DevModel<T> m, DevGuide<T> g, int n,
                                                     const void *cfg, T *out, int stage_cfg) {
  extern __shared__ __align__(16) unsigned char fsm[];
  T *Js = reinterpret_cast<T *>(fsm);                                    // [2][FK][FS]
  unsigned char *cs = fsm + (size_t)2 * FK * FS * sizeof(T);             // [FW][cfgb]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int N = m.N, NW = (N + 63) / 64, CB = ((N + 15) / 16) * 16;
  const int cfgb = FAM == SPIN_HALF ? NW * 8 : CB;
  const int w0 = blockIdx.x * FW, s0 = blockIdx.y * FS;
  const int nwb = n - w0 < FW ? n - w0 : FW;
  const unsigned char *cg = reinterpret_cast<const unsigned char *>(cfg) + (size_t)w0 * cfgb;
  if (stage_cfg) {
    const uint64_t *src = reinterpret_cast<const uint64_t *>(cg);
    uint64_t *dst = reinterpret_cast<uint64_t *>(cs);
    for (int i = tid; i < nwb * cfgb / 8; i += 256) dst[i] = src[i];
  }
  const unsigned char *cw = stage_cfg ? cs : cg;   // the block's configurations

  T acc[4][8];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = T(0);

  const int nch = (N + FK - 1) / FK;
  auto load_chunk = [&](int c) {
    T *dst = Js + (c & 1) * FK * FS;
    const int p0 = c * FK;
    for (int i = tid; i < FK * FS; i += 256) {
      const int p = p0 + i / FS, k = s0 + i % FS;
      const bool ok = p < N && k < N;
      cp_el<sizeof(T)>(dst + i, ok ? g.Jd + (size_t)p * N + k : g.Jd, ok);
    }
    cp_commit();
  };
  load_chunk(0);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      load_chunk(c + 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const T *J = Js + (c & 1) * FK * FS;
    const int p0 = c * FK;
    const int kmax = N - p0 < FK ? N - p0 : FK;
    if (FAM == SPIN_HALF) {
      // the 16 spins p0 .. p0+15 of each of the thread's walkers (0 past n)
      uint32_t xb[4];
      bool xv_ok[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int wl = 4 * ty + a;
        xv_ok[a] = wl < nwb;
        const uint64_t wd =
            xv_ok[a] ? reinterpret_cast<const uint64_t *>(cw + (size_t)wl * cfgb)[p0 >> 6] : 0ull;
        xb[a] = (uint32_t)(wd >> (p0 & 63));
      }
#pragma unroll
      for (int kk = 0; kk < FK; ++kk) {
        if (kk < kmax) {
          T xv[4], jv[8];
#pragma unroll
          for (int a = 0; a < 4; ++a) xv[a] = xv_ok[a] ? spin_of<T>(xb[a], kk) : T(0);
#pragma unroll
          for (int b = 0; b < 8; ++b) jv[b] = J[kk * FS + tx + 16 * b];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = fma(jv[b], xv[a], acc[a][b]);
        }
      }
    } else {
#pragma unroll 4
      for (int kk = 0; kk < kmax; ++kk) {
        T xv[4], jv[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const int wl = 4 * ty + a;
          xv[a] = wl < nwb ? T(cw[(size_t)wl * cfgb + p0 + kk]) : T(0);
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) jv[b] = J[kk * FS + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = fma(jv[b], xv[a], acc[a][b]);
      }
    }
    __syncthreads();   // the next iteration's prefetch overwrites this buffer
  }

#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int wl = 4 * ty + a;
    if (wl >= nwb) continue;
    const int w = w0 + wl;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int k = s0 + tx + 16 * b;
      if (k >= N) continue;
      T v = acc[a][b];
      if (FAM == SPIN_HALF) {
        const uint64_t wd = reinterpret_cast<const uint64_t *>(cw + (size_t)wl * cfgb)[k >> 6];
        const T x = ((wd >> (k & 63)) & 1ull) ? T(1) : T(-1);
        v = x * math_exp(T(-2) * x * (g.has_h ? v + g.h[k] : v));
      }
      out[(size_t)w * N + k] = v;
    }
  }
}

}  // namespace

template <typename T>
cudaError_t launch_fields(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg,
                          T *out, cudaStream_t s) {
  if (!g.dense || !g.Jd || g.kind == GUIDE_NONE) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  const int N = m.N;
  const size_t cfgb = m.family == SPIN_HALF ? (size_t)((N + 63) / 64) * 8 : (size_t)((N + 15) / 16) * 16;
  const int stage_cfg = FW * cfgb <= (size_t)CFG_STAGE_MAX;
  const size_t smem = (size_t)2 * FK * FS * sizeof(T) + (stage_cfg ? FW * cfgb : 0);
  const dim3 grid((n + FW - 1) / FW, (N + FS - 1) / FS);
  auto kern = m.family == SPIN_HALF ? fields_kernel<T, SPIN_HALF> : fields_kernel<T, BOSE_HUBBARD>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, 256, smem, s>>>(m, g, n, cfg, out, stage_cfg);
  return cudaGetLastError();
}

template cudaError_t launch_fields<double>(const DevModel<double> &, const DevGuide<double> &, int,
                                           const void *, double *, cudaStream_t);
template cudaError_t launch_fields<float>(const DevModel<float> &, const DevGuide<float> &, int,
                                          const void *, float *, cudaStream_t);

}  // namespace gfmc

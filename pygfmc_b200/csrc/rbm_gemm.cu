// RBM hidden pre-activations of a whole population on the 5th-generation
// tensor cores: theta[w, h] = b[h] + sum_i s_wi W[h, i], s = +-1.
//
// One CTA (4 warps) per 128 walkers.  Per 64-site chunk of the visible axis
// the CTA expands its walkers' spin words into a bf16 +-1 tile A (128 x 64)
// and copies the matching W columns into a tile B (up to 512 hidden rows x
// 64), both K-major in the 128-byte swizzled canonical layout; thread 0
// issues tcgen05.mma (kind::f16, bf16 x bf16 -> f32, M = 128, N = 256, K = 16)
// into a TMEM accumulator of up to 512 columns and commits to an mbarrier.
// The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31 = walkers), adds b and writes theta in float32.  Hidden axes
// above 512 run in passes of 512 columns.  Every wait is bounded: a wait that
// runs out sets GFMC status bit 8 and the CTA still frees its TMEM.
//
// Roofline: tensor bound at 2 * 128 * Hp * Np flops per CTA; bytes per
// walker: Np / 8 of spins in, 4 Hp of theta out, W re-read from L2 per CTA.
#include <cuda_bf16.h>

#include "rbm.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

constexpr int GT = 128;            // threads = walkers per CTA = UMMA M
constexpr int KC = 64;             // visible sites per chunk (one 128-byte swizzle row)
constexpr int MAXN = 512;          // TMEM columns per pass
using namespace tc;

// D f32, A and B bf16, both K-major, M = 128, N = 256.
constexpr uint32_t IDESC = idesc_m128(256u);

__global__ void __launch_bounds__(GT, 1)
rbm_theta_kernel(const uint64_t *cfg, const int *parents, int NW, int n, int Np,
                 const __nv_bfloat16 *W, const float *b, int Hp, float *theta, int *status) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  unsigned char *A = base;                       // 128 x 64 bf16 = 16 KB
  unsigned char *B = base + GT * 128;            // up to 512 x 64 bf16 = 64 KB
  uint64_t *bar = reinterpret_cast<uint64_t *>(B + MAXN * 128);
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
  volatile int *flag = reinterpret_cast<volatile int *>(slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncols = Hp < MAXN ? Hp : MAXN;       // 256 or 512 (a power of two)

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *slot;

  const int row = tid;                           // walker row of the tile
  const int w = blockIdx.x * GT + row;
  const int src = w < n ? (parents ? parents[w] : w) : 0;
  uint32_t phase = 0;
  bool ok = true;
  const int nk = Np / KC;

  for (int hb = 0; hb < Hp && ok; hb += MAXN) {
    const int nc = (Hp - hb) < MAXN ? (Hp - hb) : MAXN;   // 256 or 512
    for (int kc = 0; kc < nk && ok; ++kc) {
      // A: the walker's 64 spins of this chunk as bf16 +-1 (0 past the sites)
      {
        const uint64_t word = w < n && kc < NW ? cfg[(size_t)src * NW + kc] : 0ull;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          uint32_t q[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k0 = 8 * c + 2 * e;
            const uint32_t lo = ((word >> k0) & 1ull) ? 0x3F80u : 0xBF80u;
            const uint32_t hi = ((word >> (k0 + 1)) & 1ull) ? 0x3F80u : 0xBF80u;
            q[e] = w < n ? (lo | (hi << 16)) : 0u;
          }
          *reinterpret_cast<uint4 *>(sw_chunk(A, row, c)) = make_uint4(q[0], q[1], q[2], q[3]);
        }
      }
      // B: W[hb + r, 64 kc .. 64 kc + 63] for the pass's rows
      for (int r = tid; r < nc; r += GT) {
        const uint4 *srcw =
            reinterpret_cast<const uint4 *>(W + (size_t)(hb + r) * Np + (size_t)kc * KC);
#pragma unroll
        for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4 *>(sw_chunk(B, r, c)) = __ldg(srcw + c);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
        for (int sub = 0; sub < nc / 256; ++sub) {
#pragma unroll
          for (int kk = 0; kk < KC / 16; ++kk) {
            const uint64_t ad = sw128_desc(a0 + 32u * kk);
            const uint64_t bd = sw128_desc(b0 + (uint32_t)sub * 256u * 128u + 32u * kk);
            mma_bf16(tmem + (uint32_t)sub * 256u, ad, bd, IDESC, (kc > 0 || kk > 0) ? 1u : 0u);
          }
        }
        mma_commit(bar);
      }
      // the tiles may be overwritten once the MMAs have read them
      if (!cta_wait(bar, phase, flag)) {
        if (tid == 0) atomicOr(status, 8);
        ok = false;
      }
      phase ^= 1u;
    }
    if (!ok) break;
    // epilogue: warp owns TMEM lanes 32 warp .. 32 warp + 31
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    for (int c0 = 0; c0 < nc; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (w < n) {
        float *out = theta + (size_t)w * Hp + hb + c0;
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
          const float4 o = make_float4(v[i] + b[hb + c0 + i], v[i + 1] + b[hb + c0 + i + 1],
                                       v[i + 2] + b[hb + c0 + i + 2], v[i + 3] + b[hb + c0 + i + 3]);
          *reinterpret_cast<float4 *>(out + i) = o;
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  (void)lane;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
}

size_t theta_smem_bytes() { return 1024 + GT * 128 + MAXN * 128 + 16; }

}  // namespace

cudaError_t launch_rbm_theta(const RbmTables &r, int n, const void *cfg, const int *parents,
                             int NW, float *theta, int *status, cudaStream_t s) {
  const size_t smem = theta_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(rbm_theta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int grid = (n + GT - 1) / GT;
  rbm_theta_kernel<<<grid, GT, smem, s>>>(reinterpret_cast<const uint64_t *>(cfg), parents, NW, n,
                                          r.Np, r.W, r.b, r.Hp, theta, status);
  return cudaGetLastError();
}

}  // namespace gfmc

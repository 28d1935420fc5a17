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

namespace gfmc {
namespace {

constexpr int GT = 128;            // threads = walkers per CTA = UMMA M
constexpr int KC = 64;             // visible sites per chunk (one 128-byte swizzle row)
constexpr int MAXN = 512;          // TMEM columns per pass
constexpr uint32_t WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on the mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// CTA-uniform bounded wait: thread 0 waits, every thread gets its verdict
// (so all threads leave or stay in the loops together).
__device__ __forceinline__ bool cta_wait(uint64_t *bar, uint32_t parity, volatile int *flag) {
  if (threadIdx.x == 0) *flag = mbar_wait(bar, parity) ? 1 : 0;
  __syncthreads();
  const bool r = *flag != 0;
  __syncthreads();
  return r;
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                 // LBO (unused by swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;       // SBO
  d |= (uint64_t)1u << 46;                 // version
  d |= (uint64_t)2u << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = 256.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) |
                           ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Row r of a 128-byte-swizzled K-major tile: logical 16-byte chunk c lives
// at chunk c ^ (r & 7).
__device__ __forceinline__ unsigned char *sw_chunk(unsigned char *tile, int r, int c) {
  return tile + (size_t)r * 128 + (size_t)((c ^ (r & 7)) * 16);
}

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
            mma_bf16(tmem + (uint32_t)sub * 256u, ad, bd, (kc > 0 || kk > 0) ? 1u : 0u);
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

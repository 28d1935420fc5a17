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
// Roofline: 2 Np Hp flops and 4 Hp bytes of theta written per walker: the
// float32 output bounds it (HBM), the tensor work is half that time.  The
// persistent kernel below (one CTA per SM, W resident per pass, A in a
// two-stage ring, two TMEM accumulators) is the one launched whenever a
// pass's W tile fits in shared memory; the one-CTA-per-tile kernel above
// takes the rest.
#include <atomic>

#include <cuda.h>
#include <cudaTypedefs.h>
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

// ---------------------------------------------------------------------------
// Persistent version: one CTA of 9 warps per SM.  The hidden axis runs in
// passes of PW columns (256, or 128 / 64 when a pass's W tile would not fit);
// the pass's W tile (PW rows x Np sites, bf16, K-chunks of 64 sites in the
// 128-byte swizzled K-major layout) stays in shared memory while the CTA
// walks its walker tiles (128 walkers each):
//  * warps 0-3 (one walker row per thread) expand the spin words of each
//    64-site chunk into a two-stage ring of A tiles (bf16 +-1);
//  * warp 8 waits for each chunk (lane 0 waits, the other lanes hold at a
//    shuffle, so the warp never spins divergently) and its lane 0 issues the
//    chunk's four MMAs (K = 16 each, N = PW) into one of two TMEM
//    accumulators, commits them to the ring stage's "free" mbarrier, and
//    after a tile's last chunk to the accumulator's "full" one;
//  * warps 4-7 (warp 4 + q reads TMEM lanes 32 q .. 32 q + 31) add b and
//    write theta while the next tile accumulates in the other buffer: each
//    32 x 32 block goes into one of the warp's two staging boxes in shared
//    memory (128-byte swizzled rows, the layout of the output's tensor map)
//    and leaves by one TMA tensor store (this GPU's own memory, no
//    multicast), so the stores stream while the warp reads the next block.
// The tiles of a pass go round the CTAs from an offset that advances by
// n_tiles mod grid per pass, so the CTAs that took one tile more in one pass
// take one less in the next.  Every wait is bounded (status bit 8); a wait
// that runs out stops every role at its next wait, and the CTA frees its
// TMEM.
constexpr int PT = 288;   // threads: 4 producer, 4 epilogue and 1 MMA warp

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// TMA tensor store of one box at (x, y) from shared memory, and the bulk
// groups of the issuing thread: commit, wait until at most one group is
// still reading shared memory, wait until every group has read it / has
// completed.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, uint32_t saddr, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// TMA tensor load of one box at (x, y) into shared memory, completing on
// mbarrier bar (whose expected bytes the issuer has armed).
__device__ __forceinline__ void tma_load_2d(const CUtensorMap *map, uint32_t saddr, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(saddr), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

constexpr int STAGE_BYTES = 32 * 128;   // one 32 x 32 float box

// Bounded wait of one thread on completion `k` (parity k & 1); false (and
// the CTA's abort flag set) when the limit ran out or another role aborted.
__device__ __forceinline__ bool bwait(uint64_t *bar, uint32_t k, volatile int *abort_flag) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try_wait(bar, k & 1u)) return true;
    if ((it & 1023u) == 0 && *abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}

// First tile of this CTA in pass p: the tiles go round the CTAs from an
// offset that advances by n_tiles mod G per pass.
__device__ __forceinline__ int first_tile(int p, int n_tiles, int G) {
  const long long rot = n_tiles % G;
  return (int)((((long long)blockIdx.x - (long long)p * rot) % G + G) % G);
}

__global__ void __launch_bounds__(PT, 1)
rbm_theta_persist(const uint64_t *cfg, const int *parents, int NW, int n, int Np,
                  const __nv_bfloat16 *W, const float *b, int Hp, int PW,
                  const __grid_constant__ CUtensorMap tmap,
                  const __grid_constant__ CUtensorMap wmap, int *status) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int nk = Np / KC;
  unsigned char *Bt = base;                                   // nk x PW x 128 bytes
  unsigned char *At = Bt + (size_t)nk * PW * 128;             // 2 stages x 128 x 128 bytes
  // epilogue staging: per epilogue warp two boxes (1024-byte aligned, as the
  // 128-byte swizzle wants), then the pass's biases
  unsigned char *St = At + 2 * GT * 128;
  float *bsm = reinterpret_cast<float *>(St + 4 * 2 * STAGE_BYTES);   // every bias
  uint64_t *bar = reinterpret_cast<uint64_t *>(bsm + 1024);
  uint64_t *a_full = bar, *a_free = bar + 2, *acc_full = bar + 4, *acc_free = bar + 6;
  uint64_t *w_full = bar + 8;   // the pass's W tile has landed (one phase per pass)
  uint64_t *w_free = bar + 9;   // the pass's MMAs are done with it (one phase per pass)
  uint64_t *fin = bar + 10;     // every MMA of the CTA is done (one phase)
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 11);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = 2u * (uint32_t)PW;                   // two accumulators

  if (warp == 0) tmem_alloc(slot, ncols);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(a_full + i, GT);
      mbar_init(a_free + i, 1);
      mbar_init(acc_full + i, 1);
      mbar_init(acc_free + i, GT);
    }
    mbar_init(w_full, 1);
    mbar_init(w_free, 1);
    mbar_init(fin, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t idesc = idesc_m128((uint32_t)PW);
  const int n_tiles = (n + GT - 1) / GT;
  const int G = (int)gridDim.x;
  const int n_pass = Hp / PW;
  // every bias once (Hp <= 1024)
  for (int i = tid; i < Hp; i += PT) bsm[i] = b[i];
  __syncthreads();

  if (warp < 4) {
    // ---- producers
    uint32_t gg = 0;
    for (int pass = 0; pass < n_pass && !*abort_flag; ++pass) {
      for (int t = first_tile(pass, n_tiles, G); t < n_tiles && !*abort_flag; t += G) {
        const int w = t * GT + tid;
        const int src = w < n ? (parents ? parents[w] : w) : 0;
        // the walker's spin words of up to 8 chunks at once (one load latency
        // per tile instead of one per chunk)
        uint64_t words[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
          words[k] = (w < n && k < NW && k < nk) ? cfg[(size_t)src * NW + k] : 0ull;
        for (int kc = 0; kc < nk; ++kc, ++gg) {
          const uint32_t s = gg & 1u, u = gg >> 1;
          if (u >= 1 && !bwait(a_free + s, u - 1, abort_flag)) break;
          unsigned char *A = At + (size_t)s * GT * 128;
          uint64_t word = 0ull;
          if (kc < 8) {
#pragma unroll
            for (int k = 0; k < 8; ++k)
              if (k == kc) word = words[k];
          } else if (w < n && kc < NW) {
            word = cfg[(size_t)src * NW + kc];
          }
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
            *reinterpret_cast<uint4 *>(sw_chunk(A, tid, c)) = make_uint4(q[0], q[1], q[2], q[3]);
          }
          fence_async_smem();
          mbar_arrive(a_full + s);
        }
      }
    }
  } else if (warp == 8) {
    // ---- the MMA issuer, which also brings in each pass's W tile (by TMA,
    //      in the 128-byte swizzled layout the MMA descriptors expect) as soon
    //      as the previous pass's MMAs have finished reading the last one
    const int lane = tid & 31;
    uint32_t gg = 0, TT = 0;
    int w_issued = 0;
    bool ok = true;
    for (int pass = 0; pass < n_pass && ok; ++pass) {
      const int hb = pass * PW;
      if (lane == 0) {
        if (pass > 0) {
          mma_commit(w_free);
          ok = bwait(w_free, (uint32_t)(pass - 1), abort_flag);
        }
        if (ok) {
          mbar_expect_tx(w_full, (uint32_t)(nk * PW * 128));
          for (int kc = 0; kc < nk; ++kc)
            tma_load_2d(&wmap, smem_u32(Bt + (size_t)kc * PW * 128), kc * KC, hb, w_full);
          ++w_issued;
          ok = bwait(w_full, (uint32_t)pass, abort_flag);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      for (int t = first_tile(pass, n_tiles, G); t < n_tiles && ok; t += G, ++TT) {
        const uint32_t buf = TT & 1u, use = TT >> 1;
        for (int kc = 0; kc < nk; ++kc, ++gg) {
          const uint32_t s = gg & 1u, u = gg >> 1;
          if (lane == 0)
            ok = bwait(a_full + s, u, abort_flag) &&
                 (kc != 0 || use < 1 || bwait(acc_free + buf, use - 1, abort_flag));
          ok = __shfl_sync(0xffffffffu, ok, 0);
          if (!ok) break;
          fence_after();
          if (lane == 0) {
            const uint32_t a0 = smem_u32(At + (size_t)s * GT * 128);
            const uint32_t b0 = smem_u32(Bt + (size_t)kc * PW * 128);
            const uint32_t d = tmem + buf * (uint32_t)PW;
#pragma unroll
            for (int kk = 0; kk < KC / 16; ++kk)
              mma_bf16(d, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), idesc,
                       (kc > 0 || kk > 0) ? 1u : 0u);
            mma_commit(a_free + s);
            if (kc == nk - 1) mma_commit(acc_full + buf);
          }
          __syncwarp();
        }
      }
    }
    if (lane == 0) {
      // every MMA this warp issued and, after a wait that ran out, the last
      // W copies finish (bounded) before the CTA frees its memory
      mma_commit(fin);
      for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(fin, 0u)) break;
      if (!ok && w_issued > 0)
        for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
          if (mbar_try_wait(w_full, (uint32_t)(w_issued - 1) & 1u)) break;
    }
    __syncwarp();
  } else {
    // ---- epilogue: theta = accumulator + b
    const int q = warp - 4, lane = tid & 31;
    unsigned char *S0 = St + (size_t)q * 2 * STAGE_BYTES;
    uint32_t nst = 0;   // boxes this warp has stored
    uint32_t TT = 0;
    for (int pass = 0; pass < n_pass && !*abort_flag; ++pass) {
      const int hb = pass * PW;
      for (int t = first_tile(pass, n_tiles, G); t < n_tiles && !*abort_flag; t += G, ++TT) {
        const uint32_t buf = TT & 1u, use = TT >> 1;
        if (!bwait(acc_full + buf, use, abort_flag)) break;
        fence_after();
        // this warp's 32 walkers (one per lane) x 32 columns at a time
        const int w0 = t * GT + 32 * q;
        for (int cb = 0; cb < PW / 32; ++cb) {
          const int c0 = 32 * cb;
          uint32_t v[32];
          tmem_ld32_async(tmem + ((uint32_t)(32 * q) << 16) + buf * (uint32_t)PW + (uint32_t)c0, v);
          tmem_ld_wait(v);
          if (w0 >= n) continue;   // (the last tile's rows past the population)
          unsigned char *S = S0 + (size_t)(nst & 1u) * STAGE_BYTES;
          // the box stored two blocks ago has left this buffer
          if (nst >= 2 && lane == 0) bulk_wait_read1();
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float4 bj = *reinterpret_cast<const float4 *>(bsm + hb + c0 + 4 * j);
            *reinterpret_cast<float4 *>(sw_chunk(S, lane, j)) =
                make_float4(__uint_as_float(v[4 * j]) + bj.x, __uint_as_float(v[4 * j + 1]) + bj.y,
                            __uint_as_float(v[4 * j + 2]) + bj.z, __uint_as_float(v[4 * j + 3]) + bj.w);
          }
          fence_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(&tmap, smem_u32(S), hb + c0, w0);
            bulk_commit();
          }
          ++nst;
        }
        fence_before();
        mbar_arrive(acc_free + buf);
      }
    }
    // the output boxes in flight have landed before the CTA leaves
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }
  fence_before();
  __syncthreads();
  if (*abort_flag && tid == 0) atomicOr(status, 8);
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// Pass width of the persistent kernel for Np padded sites: the widest of
// 256, 128, 64 columns whose W tile fits beside the A ring; 0 when none does.
int theta_pass_width(int Np, int Hp) {
  for (int pw = 256; pw >= 64; pw /= 2) {
    if (Hp % pw) continue;
    const size_t bytes = 1024 + (size_t)(Np / KC) * pw * 128 + 2 * GT * 128 + 8 * STAGE_BYTES + 4096 + 128;
    if (bytes <= (size_t)227 * 1024) return pw;
  }
  return 0;
}

size_t theta_persist_smem(int Np, int PW) {
  return 1024 + (size_t)(Np / KC) * PW * 128 + 2 * GT * 128 + 8 * STAGE_BYTES + 4096 + 128;
}

// cuTensorMapEncodeTiled from the driver, looked up once (no link against
// the driver library); nullptr when unavailable.
PFN_cuTensorMapEncodeTiled encode_tiled() {
  // (a function-local static: initialised once, also under concurrent callers)
  static const PFN_cuTensorMapEncodeTiled fn = []() -> PFN_cuTensorMapEncodeTiled {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
    return nullptr;
  }();
  return fn;
}

// Tensor map of W (Hp rows of Np bf16) in boxes of 64 sites x PW rows with
// the 128-byte swizzle; false when the driver refuses it.
bool w_tensor_map(const __nv_bfloat16 *W, int Hp, int Np, int PW, CUtensorMap *tm) {
  PFN_cuTensorMapEncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Np, (cuuint64_t)Hp};
  const cuuint64_t stride[1] = {(cuuint64_t)Np * sizeof(__nv_bfloat16)};
  const cuuint32_t box[2] = {(cuuint32_t)KC, (cuuint32_t)PW}, es[2] = {1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(W), dims, stride, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of theta (n rows of Hp floats) in 32 x 32 boxes with the
// 128-byte swizzle; false when the driver refuses it.
bool theta_tensor_map(float *theta, int n, int Hp, CUtensorMap *tm) {
  PFN_cuTensorMapEncodeTiled enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Hp, (cuuint64_t)n};
  const cuuint64_t stride[1] = {(cuuint64_t)Hp * sizeof(float)};
  const cuuint32_t box[2] = {32, 32}, es[2] = {1, 1};
  return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, theta, dims, stride, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

cudaError_t launch_rbm_theta(const RbmTables &r, int n, const void *cfg, const int *parents,
                             int NW, float *theta, int *status, cudaStream_t s) {
  const int PW = theta_pass_width(r.Np, r.Hp);
  CUtensorMap tm, wm;
  if (PW > 0 && n > 0 && r.Hp <= 1024 && theta_tensor_map(theta, n, r.Hp, &tm) &&
      w_tensor_map(r.W, r.Hp, r.Np, PW, &wm)) {
    const size_t smem = theta_persist_smem(r.Np, PW);
    // the kernel's shared-memory limit (its largest size) and the SM count,
    // once per device
    // (several host threads may launch at once: the per-device entries are
    // atomics, and a race only repeats the idempotent attribute calls)
    static std::atomic<int> sms_of[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int sms = (dev >= 0 && dev < 64) ? sms_of[dev].load(std::memory_order_acquire) : 0;
    if (sms == 0) {
      e = cudaFuncSetAttribute(rbm_theta_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               227 * 1024);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) sms_of[dev].store(sms, std::memory_order_release);
    }
    const int tiles = (n + GT - 1) / GT;
    const int grid = tiles < sms ? tiles : sms;
    rbm_theta_persist<<<grid, PT, smem, s>>>(reinterpret_cast<const uint64_t *>(cfg), parents, NW,
                                             n, r.Np, r.W, r.b, r.Hp, PW, tm, wm, status);
    return cudaGetLastError();
  }
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

// Guide state of a whole population at once, for dense Jastrow couplings:
//   F[w, k] = sum_p Jd[p, k] x_p(w)       (x = +-1 spins or occupations)
// and, for spin-1/2, the signed ratio factors s_k = x_k exp(-2 x_k (F_k + h_k))
// the step kernel carries (JastrowSpinHalf; jastrow_spin_half.py:290-353).
//
// The step kernel would otherwise rebuild this state per walker (a fresh
// population, every refresh): N^2 multiply-adds per walker through L2.  Here
// it is one (walkers x N) x (N x N) product on the 5th-generation tensor
// cores with exact integer arithmetic:
//
// * the couplings are split once, on the host, into D balanced base-128
//   digits, Jd[p, k] = S sum_d j_d[k, p] 128^-(d+1) + r, j_d in [-64, 64],
//   S a power of two with |Jd| <= S / 2, |r| <= S 2^-(7D+1) (D = 8 in the
//   float64 build, 56 bits; D = 4 in the float32 build);
// * x (+-1, or an occupation 0..n_max) is an int8, so every digit's product
//   I_d[w, k] = sum_p x_p j_d[k, p] is exact in int32 (tcgen05.mma
//   kind::i8, s8 x s8 -> s32);
// * the epilogue combines the digits exactly in int64, four at a time, and
//   the two groups of the float64 build with one rounding (combine_digits),
//   F = acc S / 128 -- closer to the exact sum than a sequential float64
//   accumulation of the N terms (and two int-to-float64 conversions per
//   output instead of eight).
//
// A CTA (8 warps) takes 128 walkers (TMEM lanes) and 256 / D output sites;
// the B operand holds all D digits of those sites (row d (256 / D) + j), so
// one MMA of N = 256 covers every digit and the accumulator is 256 int32
// columns.  K runs in chunks of 128 sites (one 128-byte swizzled row of
// int8) through a two-stage ring: the CTA expands its walkers'
// configurations into the int8 A tile (128 x 128) and copies the digit rows
// into the B tile (256 x 128); thread 0 issues four MMAs of K = 32 per chunk
// and commits to the stage's mbarrier.  Every wait is bounded: one that runs
// out sets status bit ST_TIMEOUT, and the CTA still frees its TMEM.
#include <atomic>
#include <cstdint>

#include "engine.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

using namespace tc;

constexpr int MT = 128;     // walkers per CTA = UMMA M = TMEM lanes
constexpr int KCH = 128;    // sites per K chunk (128 int8 = one swizzled row)
constexpr int BN = 256;     // B rows = UMMA N = TMEM columns
constexpr int FT = 256;     // threads per CTA
constexpr int STAGE = MT * KCH + BN * KCH;   // A + B bytes per stage (48 KB)

// D s32, A and B s8, both K-major, M = 128, N = 256.
constexpr uint32_t IDESC_I8 =
    (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(IDESC_I8), "r"(accum));
}

// Four TMEM columns of this warp's 32 lanes (no wait).
__device__ __forceinline__ void tmem_ld4_async(uint32_t taddr, int32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}

__device__ __forceinline__ void cp16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND> __device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

// Spins (bits b0..b3 of b4) as four int8 bytes, 1 for up and -1 for down:
// the multiply spreads bit i to bit 8 i, the mask keeps those, and each
// byte becomes ~(bit * 0xFE).
__device__ __forceinline__ uint32_t spin_bytes4(uint32_t b4) {
  return ~(((b4 * 0x00204081u) & 0x01010101u) * 0xFEu);
}

// 16 sites p0 .. p0+15 of a walker (row pointer crow, nullptr past the
// population) as int8 x, 0 past N.  Spin-1/2: wd is the walker's 64-bit
// word holding p0.
template <int FAM>
__device__ __forceinline__ uint4 x_chunk(const unsigned char *crow, uint64_t wd, int N, int p0) {
  if (crow == nullptr || p0 >= N) return make_uint4(0u, 0u, 0u, 0u);
  uint32_t q[4];
  if (FAM == SPIN_HALF) {
    const uint32_t bits = (uint32_t)(wd >> (p0 & 63));
#pragma unroll
    for (int e = 0; e < 4; ++e) q[e] = spin_bytes4((bits >> (4 * e)) & 0xFu);
  } else {
    const uint4 o = *reinterpret_cast<const uint4 *>(crow + p0);
    q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = o.w;
  }
  if (p0 + 16 > N) {
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (p0 + 4 * e + b >= N) q[e] &= ~(0xFFu << (8 * b));
  }
  return make_uint4(q[0], q[1], q[2], q[3]);
}

// sum_d I_d 128^-d of output e from its D digit products: four digits at a
// time exactly in int64 (|I_d| < 2^23, so each group stays far below 2^53),
// then one rounding when the two groups of the float64 build meet (the
// float32 build's four digits give the sum exactly).
template <int D>
__device__ __forceinline__ double combine_digits(const int32_t (&I)[D][4], int e) {
  long long hi = I[0][e];
#pragma unroll
  for (int d = 1; d < 4; ++d) hi = hi * 128 + I[d][e];
  if (D == 8) {
    long long lo = I[4 % D][e];
#pragma unroll
    for (int d = 5; d < 8; ++d) lo = lo * 128 + I[d % D][e];
    return fma((double)lo, 0x1p-28, (double)hi) * 0x1p-21;
  }
  return (double)hi * 0x1p-21;
}

template <typename T, int FAM, int D>
__global__ void __launch_bounds__(FT, 1) fields_i8_kernel(DevModel<T> m, DevGuide<T> g, int n,
                                                           const void *cfg_v, T *out, int *status) {
  constexpr int NT = BN / D;   // output sites per CTA
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * STAGE);   // [2]
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
  volatile int *flag = reinterpret_cast<volatile int *>(slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int N = m.N, Kp = g.jdig_kp, nk = Kp / KCH;
  const int cfgb = FAM == SPIN_HALF ? ((N + 63) / 64) * 8 : ((N + 15) / 16) * 16;
  const unsigned char *cfg = reinterpret_cast<const unsigned char *>(cfg_v);
  const int w0 = blockIdx.x * MT, k0 = blockIdx.y * NT;
  const int8_t *Bg = g.jdig + (size_t)blockIdx.y * BN * Kp;

  if (warp == 0) tmem_alloc(slot, BN);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;

  // B: the CTA's 256 digit rows of chunk kc into its stage (the digit
  // buffer is padded to whole chunks and tiles)
  auto issue_b = [&](int kc) {
    unsigned char *B = base + (kc & 1) * STAGE + MT * KCH;
    const int8_t *src = Bg + (size_t)kc * KCH;
#pragma unroll
    for (int q = 0; q < (BN * 8) / FT; ++q) {
      const int i = tid + FT * q, r = i >> 3, c = i & 7;
      cp16(sw_chunk(B, r, c), src + (size_t)r * Kp + 16 * c);
    }
    cp_commit();
  };
  issue_b(0);
  if (nk > 1) issue_b(1);

  const int ar = tid & (MT - 1), ac0 = (tid >> 7) * 4;     // A row and first 16-site piece
  const unsigned char *crow = w0 + ar < n ? cfg + (size_t)(w0 + ar) * cfgb : nullptr;
  bool ok = true;
  int last = -1;   // last chunk whose MMAs were committed
  for (int kc = 0; kc < nk && ok; ++kc) {
    const int st = kc & 1;
    unsigned char *A = base + st * STAGE;
    unsigned char *B = A + MT * KCH;
    if (kc >= 2) {
      // the MMAs of chunk kc - 2 have read this stage
      if (!cta_wait(&bar[st], (uint32_t)(((kc - 2) >> 1) & 1), flag)) {
        if (tid == 0) atomicOr(status, ST_TIMEOUT);
        ok = false;
        break;
      }
      issue_b(kc);
    }
    // A: row ar = walker w0 + ar, four 16-site pieces (64 sites) per thread
    {
      const int p0 = kc * KCH + 16 * ac0;
      uint64_t wd = 0;
      if (FAM == SPIN_HALF && crow != nullptr && p0 < N)
        wd = reinterpret_cast<const uint64_t *>(crow)[p0 >> 6];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4 *>(sw_chunk(A, ar, ac0 + c)) = x_chunk<FAM>(crow, wd, N, p0 + 16 * c);
    }
    // this chunk's B has landed (the newest group, B of chunk 1, may still be
    // in flight while chunk 0 is used)
    if (kc == 0 && nk > 1)
      cp_wait<1>();
    else
      cp_wait<0>();
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
#pragma unroll
      for (int kk = 0; kk < KCH / 32; ++kk)
        mma_i8(tmem, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), (kc > 0 || kk > 0) ? 1u : 0u);
      mma_commit(&bar[st]);
    }
    last = kc;
  }
  // every MMA done: the last commit arrives after all earlier ones complete
  if (ok && !cta_wait(&bar[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1), flag)) {
    if (tid == 0) atomicOr(status, ST_TIMEOUT);
    ok = false;
  } else if (!ok && last >= 0 && tid == 0) {
    // a wait ran out: give the committed MMAs one more bounded wait before
    // the accumulator is freed
    for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
      if (mbar_try_wait(&bar[last & 1], (uint32_t)((last >> 1) & 1))) break;
  }
  cp_wait<0>();

  if (ok) {
    fence_after();
    const int q = warp & 3, half = warp >> 2;
    const int wl = 32 * q + lane, w = w0 + wl;
    const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
    const double scale = g.jdig_scale;   // S / 128
    // the tile's NT sites lie in one 64-bit spin word
    uint64_t wb = 0;
    if (FAM == SPIN_HALF && w < n && k0 < N)
      wb = reinterpret_cast<const uint64_t *>(cfg + (size_t)w * cfgb)[k0 >> 6];
    const bool vec = (N % 4) == 0;
    for (int j0 = half * (NT / 2); j0 < (half + 1) * (NT / 2); j0 += 4) {
      int32_t I[D][4];
#pragma unroll
      for (int d = 0; d < D; ++d) tmem_ld4_async(trow + (uint32_t)(d * NT + j0), I[d]);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      T v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double acc = combine_digits<D>(I, e);
        const int k = k0 + j0 + e;
        v[e] = (T)(acc * scale);
        if (FAM == SPIN_HALF) {
          const T x = ((wb >> (k & 63)) & 1ull) ? T(1) : T(-1);
          const T hk = (g.has_h && k < N) ? g.h[k] : T(0);
          v[e] = x * math_exp(T(-2) * x * (v[e] + hk));
        }
      }
      const int kb = k0 + j0;
      if (w < n) {
        T *o = out + (size_t)w * N + kb;
        if (vec && kb + 3 < N) {
          if (sizeof(T) == 8) {
            reinterpret_cast<double2 *>(o)[0] = make_double2((double)v[0], (double)v[1]);
            reinterpret_cast<double2 *>(o)[1] = make_double2((double)v[2], (double)v[3]);
          } else {
            *reinterpret_cast<float4 *>(o) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (kb + e < N) o[e] = v[e];
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, BN);
}


// ---------------------------------------------------------------------------
// Persistent version (when the digit rows of a site tile fit in shared memory
// beside the A ring): a CTA keeps one site tile's digit rows resident and
// walks its walker tiles with 21 warps in three roles:
//   warps 0-3  expand the walkers' configurations (one row per thread) into a
//              two-stage ring of int8 A chunks;
//   warp 20    issues the four K = 32 MMAs of each chunk (lane 0) into one of
//              two TMEM accumulators (256 columns each);
//   warps 4-19 form F and the factors of the other accumulator (the same
//              digit recombination and exp as the kernel above, so the
//              outputs are identical), four warps per TMEM lane quarter, a
//              quarter of the tile's sites each: the float64 recombination
//              and exp of every output are the kernel's work, and they need
//              the warps to hide their latency.
// Every wait is bounded; a wait that runs out stops every role at its next
// wait, sets ST_TIMEOUT, and the CTA frees its TMEM after its MMAs end.
constexpr int PEW = 16;              // epilogue warps
constexpr int PFT = (5 + PEW) * 32;

__device__ __forceinline__ bool pwait(uint64_t *bar, uint32_t k, volatile int *abort_flag) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try_wait(bar, k & 1u)) return true;
    if ((it & 1023u) == 0 && *abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}
__device__ __forceinline__ void pbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__host__ __device__ inline size_t persist_smem(int Kp) {
  return 1024 + (size_t)(Kp / KCH) * BN * KCH + 2 * (size_t)MT * KCH + 128;
}

template <typename T, int FAM, int D>
__global__ void __launch_bounds__(PFT, 1)
fields_i8_persist(DevModel<T> m, DevGuide<T> g, int n, const void *cfg_v, T *out, int *status,
                  int n_st, int cps) {
  constexpr int NT = BN / D;   // output sites per site tile
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int N = m.N, Kp = g.jdig_kp, nk = Kp / KCH;
  unsigned char *Bs = base;                               // nk x BN rows x 128 bytes, resident
  unsigned char *As = Bs + (size_t)nk * BN * KCH;         // 2 stages x MT rows x 128 bytes
  uint64_t *bar = reinterpret_cast<uint64_t *>(As + 2 * MT * KCH);
  uint64_t *a_full = bar, *a_free = bar + 2, *acc_full = bar + 4, *acc_free = bar + 6;
  uint64_t *fin = bar + 8;
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 9);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cfgb = FAM == SPIN_HALF ? ((N + 63) / 64) * 8 : ((N + 15) / 16) * 16;
  const unsigned char *cfg = reinterpret_cast<const unsigned char *>(cfg_v);
  const int y = (int)blockIdx.x % n_st, c0 = (int)blockIdx.x / n_st;   // site tile, first walker tile
  const int k0 = y * NT;
  const int n_wt = (n + MT - 1) / MT;

  if (warp == 0) tmem_alloc(slot, 2 * BN);
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(a_full + i, MT);
      mbar_init(a_free + i, 1);
      mbar_init(acc_full + i, 1);
      mbar_init(acc_free + i, PEW * 32);
    }
    mbar_init(fin, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the site tile's digit rows of every chunk (the digit buffer is padded to
  // whole chunks and tiles)
  const int8_t *Bg = g.jdig + (size_t)y * BN * Kp;
  for (int i = tid; i < nk * BN * 8; i += PFT) {
    const int kc = i / (BN * 8), rem = i - kc * (BN * 8), r = rem >> 3, c = rem & 7;
    cp16(sw_chunk(Bs + (size_t)kc * BN * KCH, r, c), Bg + (size_t)r * Kp + (size_t)kc * KCH + 16 * c);
  }
  cp_commit();
  cp_wait<0>();
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;

  if (warp < 4) {
    // ---- producers: walker row tid of each tile, 128 sites per chunk
    uint32_t gg = 0;
    for (int t = c0; t < n_wt && !*abort_flag; t += cps) {
      const int w = t * MT + tid;
      const unsigned char *crow = w < n ? cfg + (size_t)w * cfgb : nullptr;
      for (int kc = 0; kc < nk; ++kc, ++gg) {
        const uint32_t st = gg & 1u, u = gg >> 1;
        if (u >= 1 && !pwait(a_free + st, u - 1, abort_flag)) break;
        unsigned char *A = As + (size_t)st * MT * KCH;
        const int p0 = kc * KCH;
        uint64_t wd0 = 0, wd1 = 0;
        if (FAM == SPIN_HALF && crow != nullptr) {
          if (p0 < N) wd0 = reinterpret_cast<const uint64_t *>(crow)[p0 >> 6];
          if (p0 + 64 < N) wd1 = reinterpret_cast<const uint64_t *>(crow)[(p0 >> 6) + 1];
        }
#pragma unroll
        for (int c = 0; c < 8; ++c)
          *reinterpret_cast<uint4 *>(sw_chunk(A, tid, c)) =
              x_chunk<FAM>(crow, c < 4 ? wd0 : wd1, N, p0 + 16 * c);
        fence_async_smem();
        pbar_arrive(a_full + st);
      }
    }
  } else if (warp == 4 + PEW) {
    // ---- the MMA issuer (lane 0 waits and issues, the warp stays converged)
    uint32_t gg = 0, TT = 0;
    bool ok = true;
    for (int t = c0; t < n_wt && ok; t += cps, ++TT) {
      const uint32_t buf = TT & 1u, use = TT >> 1;
      for (int kc = 0; kc < nk; ++kc, ++gg) {
        const uint32_t st = gg & 1u, u = gg >> 1;
        if (lane == 0)
          ok = pwait(a_full + st, u, abort_flag) &&
               (kc != 0 || use < 1 || pwait(acc_free + buf, use - 1, abort_flag));
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        fence_after();
        if (lane == 0) {
          const uint32_t a0 = smem_u32(As + (size_t)st * MT * KCH);
          const uint32_t b0 = smem_u32(Bs + (size_t)kc * BN * KCH);
#pragma unroll
          for (int kk = 0; kk < KCH / 32; ++kk)
            mma_i8(tmem + buf * BN, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk),
                   (kc > 0 || kk > 0) ? 1u : 0u);
          mma_commit(a_free + st);
          if (kc == nk - 1) mma_commit(acc_full + buf);
        }
        __syncwarp();
      }
    }
    if (lane == 0) {
      // every MMA of the CTA has ended (bounded) before the TMEM is freed
      mma_commit(fin);
      for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(fin, 0u)) break;
    }
    __syncwarp();
  } else {
    // ---- epilogue: F and the factors of one accumulator
    const int ew = warp - 4, q = ew & 3, part = ew >> 2;
    const double scale = g.jdig_scale;   // S / 128
    uint32_t TT = 0;
    for (int t = c0; t < n_wt && !*abort_flag; t += cps, ++TT) {
      const uint32_t buf = TT & 1u, use = TT >> 1;
      if (!pwait(acc_full + buf, use, abort_flag)) break;
      fence_after();
      const int w = t * MT + 32 * q + lane;
      const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16) + buf * BN;
      // the tile's NT sites lie in one 64-bit spin word
      uint64_t wb = 0;
      if (FAM == SPIN_HALF && w < n && k0 < N)
        wb = reinterpret_cast<const uint64_t *>(cfg + (size_t)w * cfgb)[k0 >> 6];
      const bool vec = (N % 4) == 0;
      for (int j0 = part * (NT / 4); j0 < (part + 1) * (NT / 4); j0 += 4) {
        int32_t I[D][4];
#pragma unroll
        for (int d = 0; d < D; ++d) tmem_ld4_async(trow + (uint32_t)(d * NT + j0), I[d]);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        T v[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double acc = combine_digits<D>(I, e);
          const int k = k0 + j0 + e;
          v[e] = (T)(acc * scale);
          if (FAM == SPIN_HALF) {
            const T x = ((wb >> (k & 63)) & 1ull) ? T(1) : T(-1);
            const T hk = (g.has_h && k < N) ? g.h[k] : T(0);
            v[e] = x * math_exp(T(-2) * x * (v[e] + hk));
          }
        }
        const int kb = k0 + j0;
        if (w < n) {
          T *o = out + (size_t)w * N + kb;
          if (vec && kb + 3 < N) {
            if (sizeof(T) == 8) {
              reinterpret_cast<double2 *>(o)[0] = make_double2((double)v[0], (double)v[1]);
              reinterpret_cast<double2 *>(o)[1] = make_double2((double)v[2], (double)v[3]);
            } else {
              *reinterpret_cast<float4 *>(o) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
            }
          } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
              if (kb + e < N) o[e] = v[e];
          }
        }
      }
      fence_before();
      pbar_arrive(acc_free + buf);
    }
  }
  fence_before();
  __syncthreads();
  if (*abort_flag && tid == 0) atomicOr(status, ST_TIMEOUT);
  if (warp == 0) tmem_dealloc(tmem, 2 * BN);
}

constexpr size_t I8_SMEM = 1024 + 2 * (size_t)STAGE + 32;

template <typename T, int D>
cudaError_t launch_d(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg, T *out,
                     int *status, cudaStream_t s) {
  const size_t psmem = persist_smem(g.jdig_kp);
  if (psmem <= (size_t)227 * 1024) {
    // persistent: CTAs per site tile from the SM count (cached per device;
    // a race between host threads only repeats the idempotent calls)
    auto pk = m.family == SPIN_HALF ? fields_i8_persist<T, SPIN_HALF, D>
                                    : fields_i8_persist<T, BOSE_HUBBARD, D>;
    static std::atomic<int> sms_of[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int sms = (dev >= 0 && dev < 64) ? sms_of[dev].load(std::memory_order_acquire) : 0;
    if (sms == 0) {
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) sms_of[dev].store(sms, std::memory_order_release);
    }
    // at least 120 KB: one CTA per SM, so that no two CTAs contend for the
    // 512 TMEM columns each allocates
    const size_t lsmem = psmem > (size_t)120 * 1024 ? psmem : (size_t)120 * 1024;
    e = cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem);
    if (e != cudaSuccess) return e;
    const int NT = BN / D;
    const int n_st = (m.N + NT - 1) / NT, n_wt = (n + MT - 1) / MT;
    int cps = sms / n_st;
    if (cps < 1) cps = 1;
    if (cps > n_wt) cps = n_wt;
    pk<<<n_st * cps, PFT, lsmem, s>>>(m, g, n, cfg, out, status, n_st, cps);
    return cudaGetLastError();
  }
  auto kern = m.family == SPIN_HALF ? fields_i8_kernel<T, SPIN_HALF, D>
                                    : fields_i8_kernel<T, BOSE_HUBBARD, D>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)I8_SMEM);
  if (e != cudaSuccess) return e;
  const dim3 grid((n + MT - 1) / MT, (m.N + BN / D - 1) / (BN / D));
  kern<<<grid, FT, I8_SMEM, s>>>(m, g, n, cfg, out, status);
  return cudaGetLastError();
}

}  // namespace

template <typename T>
cudaError_t launch_fields(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg,
                          T *out, int *status, cudaStream_t s) {
  if (!g.dense || !g.Jd || !g.jdig || g.kind == GUIDE_NONE) return cudaErrorInvalidValue;
  if (g.jdig_d != fields_digits<T>()) return cudaErrorInvalidValue;
  if (n <= 0) return cudaSuccess;
  return launch_d<T, fields_digits<T>()>(m, g, n, cfg, out, status, s);
}

template cudaError_t launch_fields<double>(const DevModel<double> &, const DevGuide<double> &, int,
                                           const void *, double *, int *, cudaStream_t);
template cudaError_t launch_fields<float>(const DevModel<float> &, const DevGuide<float> &, int,
                                          const void *, float *, int *, cudaStream_t);

}  // namespace gfmc

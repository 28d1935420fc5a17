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
// * the epilogue combines the digits from the least significant one,
//   acc = I_d + acc / 128 in float64 (each step exact until the bits run
//   past 53; about 1.5 ulp in all), F = acc S / 128 -- closer to the exact
//   sum than a sequential float64 accumulation of the N terms.
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
        double acc = (double)I[D - 1][e];
#pragma unroll
        for (int d = D - 2; d >= 0; --d) acc = (double)I[d][e] + acc * (1.0 / 128.0);
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

constexpr size_t I8_SMEM = 1024 + 2 * (size_t)STAGE + 32;

template <typename T, int D>
cudaError_t launch_d(const DevModel<T> &m, const DevGuide<T> &g, int n, const void *cfg, T *out,
                     int *status, cudaStream_t s) {
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

// Variance minimisation of the RBM guide on GFMC walkers (no PyGFMC
// counterpart: PyGFMC trains its guides by NetKet VMC).
//
// Loss over a population x_w with weights omega_w (1 after resampling):
//   L = sum_w omega_w (e_w - E)^2 / sum_w omega_w,   E = sum omega e / sum omega,
//   e_w = H_ww + sum_s r_ws,  r_ws = coupling_s psi(x'_s) / psi(x_w).
// dL/dp = sum_w g_w sum_s r_ws (O_p(x'_s) - O_p(x_w)),  g_w = 2 omega_w (e_w - E) / sum omega,
// with O_W[h, i] = tanh(theta_h) s_i, O_b = tanh(theta), O_a = s.  So
//   dL/dW = sum over rows r of U_r (x) V_r:
//     slot rows (w, s): U = g_w r_ws tanh(theta'_ws), V = s'_ws (x_w with the move's flips)
//     base rows (w):    U = -g_w R_w tanh(theta_w),  V = s_w,  R_w = sum_s r_ws
//   dL/db = sum_r U_r,   dL/da_i = sum_(w,s) g_w r_ws (-2 s_wi) [i flipped by s].
//
// Up to 256 padded sites the contraction runs in float32 without row tiles
// (rbm_grad_acc_kernel, below); wider lattices use the tensor-core
// contraction:
// rbm_grad_kernel: one CTA per (128-unit hidden tile, block of walkers).
// Each 64-row chunk: 64 threads decode the rows (sites, coefficient, spins)
// into shared memory; every thread then produces its hidden unit's 64 values
// of U (tanh.approx of theta' built from the staged W^T tile) as bf16 into the
// swizzled K-major A tile, and two site rows of V (+-1 as bf16) into the B
// tile; thread 0 issues tcgen05.mma (M = 128 hidden, N = sites, K = 64 rows)
// accumulating dL/dW of the tile in TMEM.  Two stages: the MMAs of one chunk
// run while the next is produced.  Up to 256 sites both tiles are double
// buffered; above (at most 448 padded sites) the B tile has one buffer, which
// its producers refill once the previous chunk's MMAs are done, and each K
// step is two MMAs (sites 0..255 and 256..Np-1 into TMEM columns of their
// own, 512 in all).  The epilogue adds the tile into the global float32
// gradient (atomics; one CTA per walker block and tile).
#include <cuda_bf16.h>

#include "rbm.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

constexpr int TT = 128;     // threads = hidden units per tile = UMMA M
constexpr int KR = 64;      // rows per chunk = UMMA K per chunk
using namespace tc;

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&p);
}

}  // namespace



namespace {

// Row records of the gradient contraction, one per (walker, slot) and one
// base row per walker, in row order r = w (n_off + 1) + s:
//   x: coefficient c (slot: g_w r_ws; base: -g_w R_w; 0 for a zero rate)
//   y, z: -2 s_i, -2 s_j of the flipped sites (0 when absent)
//   w: code = i | j << 9 | (walker & 0x3FFF) << 18, absent sites = Np (a
//      zero row of the staged weight tile)
// rbm_records_kernel also accumulates dL/da (per-block shared sums, then one
// global atomic per site and block).
__global__ void rbm_records_kernel(GradArgs g, float4 *recs) {
  extern __shared__ float acc[];   // (Np,)
  const int rows_per_w = g.n_off + 1;
  for (int i = threadIdx.x; i < g.Np; i += blockDim.x) acc[i] = 0.0f;
  __syncthreads();
  const int wb0 = blockIdx.x * 16;
  int wb1 = wb0 + 16;
  if (wb1 > g.n) wb1 = g.n;
  const long long r0 = (long long)wb0 * rows_per_w, r1 = (long long)wb1 * rows_per_w;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const int w = (int)(r / rows_per_w);
    const int s = (int)(r - (long long)w * rows_per_w);
    int i = g.Np, j = g.Np;
    float c, m2si = 0.0f, m2sj = 0.0f;
    if (s < g.n_off) {
      c = g.gw[w] * g.rates[(size_t)w * g.n_off + s];
      if (c != 0.0f) {
        if (s < g.n_hx) {
          i = s;
        } else {
          const uint32_t pe = g.edge[s - g.n_hx];
          i = (int)(pe & 0xFFFF);
          j = (int)(pe >> 16);
        }
        const uint64_t *x = g.cfg + (size_t)w * g.NW;
        const float si = ((x[i >> 6] >> (i & 63)) & 1ull) ? 1.0f : -1.0f;
        m2si = -2.0f * si;
        atomicAdd(&acc[i], c * m2si);
        if (j < g.Np) {
          const float sj = ((x[j >> 6] >> (j & 63)) & 1ull) ? 1.0f : -1.0f;
          m2sj = -2.0f * sj;
          atomicAdd(&acc[j], c * m2sj);
        }
      }
    } else {
      c = -g.gw[w] * g.rsum[w];
    }
    const uint32_t code = (uint32_t)i | ((uint32_t)j << 9) | (((uint32_t)w & 0x3FFFu) << 18);
    recs[r] = make_float4(c, m2si, m2sj, __uint_as_float(code));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < g.Np; i += blockDim.x)
    if (acc[i] != 0.0f) atomicAdd(&g.grad_a[i], acc[i]);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void bgroup_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Shared-memory plan of the gradient kernel (offsets from a 1024-aligned base).
struct GradSmem {
  size_t A0, A1, B0, B1, WTs, recs, th, wd, bar, total;
  int maxw;
};

__host__ __device__ inline GradSmem grad_smem_plan(int Np, int n_off, int NW) {
  GradSmem p;
  const int rows_per_w = n_off + 1;
  p.maxw = (KR - 1) / rows_per_w + 2;
  size_t o = 0;
  p.A0 = o; o += 16384;
  p.A1 = o; o += 16384;
  p.B0 = o; o += (size_t)Np * 128;
  p.B1 = p.B0;
  if (Np <= 256) { p.B1 = o; o += (size_t)Np * 128; }     // wider tiles: one B buffer
  p.WTs = o; o += (size_t)(Np + 1) * TT * 2;                 // + one zero row
  o = (o + 15) & ~(size_t)15;
  p.recs = o; o += 3 * (size_t)KR * 16;                      // three chunks in flight
  p.th = o; o += 3 * (size_t)p.maxw * TT * 4;
  p.wd = o; o += 3 * (size_t)p.maxw * NW * 8;
  o = (o + 7) & ~(size_t)7;
  p.bar = o; o += 32;
  p.total = o;
  return p;
}

// The copies of chunk ch into buffer b (run by the 128 B-group threads): its
// 64 row records, and the theta rows (this tile's units) and spin words of
// the walkers it spans.  Rows past the end get zero records.
__device__ __forceinline__ void issue_chunk(const GradArgs &g, const float4 *recs_g,
                                            unsigned char *base, const GradSmem &P, int b,
                                            long long R0, long long R1, int ch, int h0, int t) {
  const int rows_per_w = g.n_off + 1;
  const long long r0 = R0 + (long long)ch * KR;
  float4 *rs = reinterpret_cast<float4 *>(base + P.recs) + (size_t)b * KR;
  if (t < KR) {
    if (r0 + t < R1) cp_async16(rs + t, recs_g + r0 + t);
    else rs[t] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
  }
  const int wbase = (int)(r0 / rows_per_w);
  long long rl = r0 + KR - 1;
  if (rl > R1 - 1) rl = R1 - 1;
  const int nw = (int)(rl / rows_per_w) - wbase + 1;
  float *th = reinterpret_cast<float *>(base + P.th) + (size_t)b * P.maxw * TT;
  for (int k = t; k < nw * (TT / 4); k += 128) {
    const int wi = k / (TT / 4), c4 = k % (TT / 4);
    cp_async16(th + (size_t)wi * TT + 4 * c4, g.theta + (size_t)(wbase + wi) * g.Hp + h0 + 4 * c4);
  }
  uint64_t *wd = reinterpret_cast<uint64_t *>(base + P.wd) + (size_t)b * P.maxw * g.NW;
  for (int k = t; k < nw * g.NW; k += 128)
    cp_async8(wd + k, g.cfg + (size_t)(wbase + k / g.NW) * g.NW + (k % g.NW));
}

__global__ void __launch_bounds__(3 * TT, 1) rbm_grad_kernel(GradArgs g, const float4 *recs_g) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int Np = g.Np;
  const GradSmem P = grad_smem_plan(Np, g.n_off, g.NW);
  __nv_bfloat16 *WTs = reinterpret_cast<__nv_bfloat16 *>(base + P.WTs);   // (Np + 1, 128)
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + P.bar);
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
  volatile int *flag = reinterpret_cast<volatile int *>(slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const bool groupA = tid < 2 * TT;       // A producers: two threads per hidden unit
  const int hl = tid & (TT - 1), half = (tid >> 7) & 1;
  const int tb = tid - 2 * TT;            // B group: sites and the copies
  const int h0 = blockIdx.x * TT;
  const int w0 = blockIdx.y * g.walkers_per_cta;
  int w1 = w0 + g.walkers_per_cta;
  if (w1 > g.n) w1 = g.n;
  const int rows_per_w = g.n_off + 1;
  const long long R0 = (long long)w0 * rows_per_w, R1 = (long long)w1 * rows_per_w;
  const int nchunks = R1 > R0 ? (int)((R1 - R0 + KR - 1) / KR) : 0;
  const uint32_t ncols =
      Np <= 32 ? 32u : (Np <= 64 ? 64u : (Np <= 128 ? 128u : (Np <= 256 ? 256u : 512u)));
  const bool oneB = Np > 256;

  for (int idx = tid; idx < (Np + 1) * (TT / 8); idx += 3 * TT) {
    const int i = idx / (TT / 8), c = idx % (TT / 8);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (i < g.N) v = __ldg(reinterpret_cast<const uint4 *>(g.WT + (size_t)i * g.Hp + h0) + c);
    reinterpret_cast<uint4 *>(WTs + (size_t)i * TT)[c] = v;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    flag[2] = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (!groupA) {
    if (nchunks > 0) issue_chunk(g, recs_g, base, P, 0, R0, R1, 0, h0, tb);
    cp_commit();
    if (nchunks > 1) issue_chunk(g, recs_g, base, P, 1, R0, R1, 1, h0, tb);
    cp_commit();
    cp_wait1();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *slot;

  float acc_b = 0.0f;
  uint32_t cnt0 = 0u, cnt1 = 0u;
  bool ok = true;

  for (int ch = 0; ch < nchunks && ok; ++ch) {
    const int st = ch & 1, b = ch % 3;
    const uint32_t cst = st ? cnt1 : cnt0;
    if (cst > 0 && !cta_wait(&bar[st], (cst - 1u) & 1u, flag)) {
      if (tid == 0) atomicOr(g.status, 8);
      ok = false;
      break;
    }
    const long long r0 = R0 + (long long)ch * KR;
    const int wbase_lo = (int)((r0 / rows_per_w) & 0x3FFF);
    const float4 *rs = reinterpret_cast<const float4 *>(base + P.recs) + (size_t)b * KR;
    if (groupA) {
      // U[h, r] = c_r tanh(theta_w,h - 2 s_i W[h, i] - 2 s_j W[h, j]), rows 32 half ..
      const float *th = reinterpret_cast<const float *>(base + P.th) + (size_t)b * P.maxw * TT;
      unsigned char *A = base + (st ? P.A1 : P.A0);
#pragma unroll 1
      for (int cc = 4 * half; cc < 4 * half + 4; ++cc) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          float u2[2];
#pragma unroll
          for (int t2 = 0; t2 < 2; ++t2) {
            const float4 rec = rs[8 * cc + 2 * e + t2];
            float u = 0.0f;
            if (rec.x != 0.0f) {
              const uint32_t code = __float_as_uint(rec.w);
              const int i = (int)(code & 0x1FFu), j = (int)((code >> 9) & 0x1FFu);
              const int wr = (int)(((code >> 18) - (uint32_t)wbase_lo) & 0x3FFFu);
              float t = th[(size_t)wr * TT + hl];
              t = fmaf(rec.y, __bfloat162float(WTs[(size_t)i * TT + hl]), t);
              t = fmaf(rec.z, __bfloat162float(WTs[(size_t)j * TT + hl]), t);
              u = rec.x * tanh_approx(t);
              acc_b += u;
            }
            u2[t2] = u;
          }
          q[e] = bf16_pair(u2[0], u2[1]);
        }
        *reinterpret_cast<uint4 *>(sw_chunk(A, hl, cc)) = make_uint4(q[0], q[1], q[2], q[3]);
      }
    } else {
      // copies of chunk ch + 2 (its buffer held chunk ch - 1, consumed)
      if (ch + 2 < nchunks) issue_chunk(g, recs_g, base, P, (ch + 2) % 3, R0, R1, ch + 2, h0, tb);
      cp_commit();
      // V: each site row holds the spin of the row's walker (one run per
      // walker), then the moves' flips are patched in
      unsigned char *B = base + (st ? P.B1 : P.B0);
      bool writeB = true;
      if (oneB && ch > 0) {
        // the single B buffer still feeds chunk ch - 1's MMAs (stage 1 - st,
        // its commit number (ch + 1) / 2 on that barrier)
        const uint32_t prev = (uint32_t)((ch + 1) / 2);
        if (tb == 0) {
          int okw = 0;
          for (uint32_t it = 0; it < WAIT_LIMIT && !okw; ++it)
            okw = mbar_try_wait(&bar[1 - st], (prev - 1u) & 1u) ? 1 : 0;
          flag[1] = okw;
        }
        bgroup_sync();
        const bool okb = flag[1] != 0;
        bgroup_sync();
        if (!okb) {
          // the whole CTA leaves after the barrier below; B is not touched
          if (tb == 0) {
            atomicOr(g.status, 8);
            flag[2] = 1;
          }
          writeB = false;
        }
      }
      const uint64_t *wd = reinterpret_cast<const uint64_t *>(base + P.wd) + (size_t)b * P.maxw * g.NW;
      const long long rend = R1 - r0;                 // valid rows of this chunk
      const int first = (int)(r0 % rows_per_w);       // row offset inside the first walker
      for (int i = tb; writeB && i < Np; i += TT) {
        const bool real = i < g.N;
        // walker segments: row rr belongs to walker wr; the next one starts at nextb
        int wr = 0, nextb = rows_per_w - first;
        uint32_t val = real ? (((wd[i >> 6] >> (i & 63)) & 1ull) ? 0x3F80u : 0xBF80u) : 0u;
#pragma unroll 1
        for (int cc = 0; cc < KR / 8; ++cc) {
          uint32_t q[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            uint32_t hv[2];
#pragma unroll
            for (int t2 = 0; t2 < 2; ++t2) {
              const int rr = 8 * cc + 2 * e + t2;
              if (rr == nextb) {
                ++wr;
                nextb += rows_per_w;
                val = (real && rr < rend)
                          ? (((wd[(size_t)wr * g.NW + (i >> 6)] >> (i & 63)) & 1ull) ? 0x3F80u : 0xBF80u)
                          : 0u;
              }
              hv[t2] = rr < rend ? val : 0u;
            }
            q[e] = hv[0] | (hv[1] << 16);
          }
          *reinterpret_cast<uint4 *>(sw_chunk(B, i, cc)) = make_uint4(q[0], q[1], q[2], q[3]);
        }
      }
      bgroup_sync();
      if (writeB && tb < KR) {
        const float4 rec = rs[tb];
        if (rec.x != 0.0f) {
          const uint32_t code = __float_as_uint(rec.w);
          const int i = (int)(code & 0x1FFu), j = (int)((code >> 9) & 0x1FFu);
          // the flipped spin -s = m2s / 2
          const int cc = tb >> 3, e = tb & 7;
          if (i < Np) {
            unsigned short *p = reinterpret_cast<unsigned short *>(sw_chunk(B, i, cc)) + e;
            *p = rec.y > 0.0f ? 0x3F80u : 0xBF80u;
          }
          if (j < Np) {
            unsigned short *p = reinterpret_cast<unsigned short *>(sw_chunk(B, j, cc)) + e;
            *p = rec.z > 0.0f ? 0x3F80u : 0xBF80u;
          }
        }
      }
      cp_wait1();   // chunk ch + 1 has landed (this thread's copies)
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (flag[2]) {
      ok = false;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(base + (st ? P.A1 : P.A0));
      const uint32_t b0 = smem_u32(base + (st ? P.B1 : P.B0));
      // sites 0..255 into TMEM columns 0..255, the rest into 256..Np-1
      const int n0 = Np < 256 ? Np : 256;
      const uint32_t id0 = idesc_m128((uint32_t)n0);
      const uint32_t id1 = idesc_m128((uint32_t)(Np > 256 ? Np - 256 : 16));
#pragma unroll
      for (int kk = 0; kk < KR / 16; ++kk) {
        mma_bf16(tmem, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), id0,
                 (ch > 0 || kk > 0) ? 1u : 0u);
        if (Np > 256)
          mma_bf16(tmem + 256u, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 256u * 128u + 32u * kk),
                   id1, (ch > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(&bar[st]);
    }
    if (st) ++cnt1; else ++cnt0;
  }
  if (!groupA) cp_wait0();
  if (ok && cnt0 > 0 && !cta_wait(&bar[0], (cnt0 - 1u) & 1u, flag)) {
    if (tid == 0) atomicOr(g.status, 8);
    ok = false;
  }
  if (ok && cnt1 > 0 && !cta_wait(&bar[1], (cnt1 - 1u) & 1u, flag)) {
    if (tid == 0) atomicOr(g.status, 8);
    ok = false;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && nchunks > 0) {
    // warp w reads TMEM lanes 32 (w % 4) ..; the three warps of a lane
    // quarter split the columns
    const int q4 = warp & 3, part = warp >> 2;
    const int per = ((Np / 16 + 2) / 3) * 16;
    const int cbeg = part * per;
    const int cend = cbeg + per < Np ? cbeg + per : Np;
    for (int c0 = cbeg; c0 < cend; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)c0, v);
      float *out = g.grad_W + (size_t)(h0 + q4 * 32 + (tid & 31)) * Np + c0;
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (v[k] != 0.0f) atomicAdd(out + k, v[k]);
    }
    if (groupA && acc_b != 0.0f) atomicAdd(&g.grad_b[h0 + hl], acc_b);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
}

// ---- the gradient in float32 without row tiles (Np <= 256) -----------------------
// Every slot row's V is its walker's spins with the move's sites flipped
// (V_r = s_w + Delta_r, Delta_r = the record's y, z at sites i, j), and the
// base row is -(sum of the slot coefficients) tanh(theta) against s_w, so
//   dL/dW = sum_w ub_w s_w^T + sum_(w,s) T_ws Delta_ws^T,
//   ub_w = sum_s c_ws (tanh theta'_ws - tanh theta_w),  T_ws = c_ws tanh theta'_ws:
// the cancellation between a walker's base row and its slot rows happens in
// float32 inside ub_w, before any rounding (the tensor-core contraction
// below rounds U to bf16 first, which leaves dW about 1e-2 off at 256
// sites).  A CTA takes 128 hidden units and a block of walkers; each of its
// four groups of 128 threads (one unit per thread) holds theta, tanh theta
// and ub of 16 walkers in registers and runs over the slots (each group from
// its own starting slot), summing T Delta for the slot's two sites over its
// walkers in registers and adding that into the CTA's float32 dW tile in
// shared memory; after the slots, the rank-1 terms ub_w s_w^T go into the
// tile (each thread its own sites, no atomics).  The tile goes into grad_W
// at the end.
constexpr int AG = 4;          // walker groups per CTA
constexpr int AW = 16;         // walkers per thread per chunk
constexpr int ACW = AG * AW;   // walkers per chunk

__host__ __device__ inline size_t acc_smem(int Np, int NW) {
  return 1024 + (size_t)Np * TT * 4 + (size_t)ACW * TT * 4 + (size_t)ACW * NW * 8;
}

__global__ void __launch_bounds__(AG * TT, 1) rbm_grad_acc_kernel(GradArgs g, const float4 *recs) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int Np = g.Np, N = g.N, NW = g.NW;
  float *dWs = reinterpret_cast<float *>(base);                         // (Np, 128)
  float *ubs = dWs + (size_t)Np * TT;                                   // (ACW, 128)
  uint64_t *xs = reinterpret_cast<uint64_t *>(ubs + (size_t)ACW * TT);  // (ACW, NW)
  const int tid = threadIdx.x, h = tid & (TT - 1), grp = tid / TT;
  const int h0 = blockIdx.x * TT;
  const int w0 = blockIdx.y * g.walkers_per_cta;
  int w1 = w0 + g.walkers_per_cta;
  if (w1 > g.n) w1 = g.n;
  const int rows_per_w = g.n_off + 1, n_off = g.n_off;
  for (int k = tid; k < Np * TT; k += AG * TT) dWs[k] = 0.0f;
  __syncthreads();
  float acc_b = 0.0f;
  for (int c0 = w0; c0 < w1; c0 += ACW) {
    // this thread's walkers: c0 + grp * AW + q
    float th[AW], tt[AW], ub[AW];
#pragma unroll
    for (int q = 0; q < AW; ++q) {
      const int w = c0 + grp * AW + q;
      th[q] = w < w1 ? g.theta[(size_t)w * g.Hp + h0 + h] : 0.0f;
      tt[q] = tanh_approx(th[q]);
      ub[q] = 0.0f;
    }
    for (int k = tid; k < ACW * NW; k += AG * TT) {
      const int wl = k / NW, wi = k - wl * NW;
      xs[k] = c0 + wl < w1 ? g.cfg[(size_t)(c0 + wl) * NW + wi] : 0ull;
    }
    // slots, each group from its own starting point (the groups rarely add
    // into the same sites at once)
    for (int so = 0; so < n_off; ++so) {
      int sl = so + grp * (n_off / AG);
      if (sl >= n_off) sl -= n_off;
      int i, j;
      if (sl < g.n_hx) { i = sl; j = Np; }
      else { const uint32_t pe = g.edge[sl - g.n_hx]; i = (int)(pe & 0xFFFF); j = (int)(pe >> 16); }
      const float Wi = __bfloat162float(g.WT[(size_t)i * g.Hp + h0 + h]);
      const float Wj = j < Np ? __bfloat162float(g.WT[(size_t)j * g.Hp + h0 + h]) : 0.0f;
      float yi = 0.0f, yj = 0.0f;
#pragma unroll
      for (int q = 0; q < AW; ++q) {
        const int w = c0 + grp * AW + q;
        if (w < w1) {
          const float4 rec = __ldg(recs + (size_t)w * rows_per_w + sl);
          if (rec.x != 0.0f) {
            const float t = tanh_approx(fmaf(rec.z, Wj, fmaf(rec.y, Wi, th[q])));
            ub[q] = fmaf(rec.x, t - tt[q], ub[q]);
            const float T = rec.x * t;
            yi = fmaf(T, rec.y, yi);
            yj = fmaf(T, rec.z, yj);
          }
        }
      }
      if (yi != 0.0f) atomicAdd(&dWs[(size_t)i * TT + h], yi);
      if (j < Np && yj != 0.0f) atomicAdd(&dWs[(size_t)j * TT + h], yj);
    }
#pragma unroll
    for (int q = 0; q < AW; ++q) {
      ubs[(size_t)(grp * AW + q) * TT + h] = ub[q];
      acc_b += ub[q];
    }
    __syncthreads();
    // the rank-1 terms sum_w ub_w s_w over this chunk: thread (h, grp) owns
    // the sites k = grp, grp + AG, ...
    for (int k = grp; k < N; k += AG) {
      float a = 0.0f;
      for (int wl = 0; wl < ACW; ++wl) {
        const float u = ubs[(size_t)wl * TT + h];
        a += ((xs[(size_t)wl * NW + (k >> 6)] >> (k & 63)) & 1ull) ? u : -u;
      }
      dWs[(size_t)k * TT + h] += a;
    }
    __syncthreads();
  }
  for (int k = grp; k < Np; k += AG) {
    const float v = dWs[(size_t)k * TT + h];
    if (v != 0.0f) atomicAdd(&g.grad_W[(size_t)(h0 + h) * Np + k], v);
  }
  if (acc_b != 0.0f) atomicAdd(&g.grad_b[h0 + h], acc_b);
}

// Per-walker coefficients g_w = 2 omega_w (e_w - E) / sum omega and the
// weighted mean and variance of e (one block; float64 sums in a fixed order).
__global__ void train_coeff_kernel(int n, const double *e, const double *omega, float *gw,
                                   double *stats) {
  __shared__ double s1[1024], s2[1024];
  const int t = threadIdx.x;
  double a = 0.0, b = 0.0;
  for (int i = t; i < n; i += blockDim.x) {
    const double o = omega ? omega[i] : 1.0;
    a += o * e[i];
    b += o;
  }
  s1[t] = a;
  s2[t] = b;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (t < k) {
      s1[t] += s1[t + k];
      s2[t] += s2[t + k];
    }
    __syncthreads();
  }
  const double W = s2[0], E = s1[0] / W;
  __syncthreads();
  double v = 0.0;
  for (int i = t; i < n; i += blockDim.x) {
    const double o = omega ? omega[i] : 1.0;
    const double d = e[i] - E;
    v += o * d * d;
    gw[i] = (float)(2.0 * o * d / W);
  }
  s1[t] = v;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (t < k) s1[t] += s1[t + k];
    __syncthreads();
  }
  if (t == 0) {
    stats[0] = E;
    stats[1] = s1[0] / W;
  }
}

// Adam on the float32 master parameters (W (H, N), b (H), a (N)), gradients
// in the padded layouts; then the bf16 / float tables of the guide.
__global__ void adam_kernel(int H, int N, int Hp, int Np, float *W, float *b, float *a,
                            const float *gW, const float *gb, const float *ga, float *m, float *v,
                            float lr, float b1, float b2, float eps, float c1, float c2,
                            __nv_bfloat16 *WT_t, __nv_bfloat16 *W_t, float *b_t, float *a_t) {
  const int P = H * N + H + N;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x) {
    float *p;
    float gr;
    int hh = -1, ii = -1;
    if (k < H * N) {
      hh = k / N;
      ii = k % N;
      p = W + k;
      gr = gW[(size_t)hh * Np + ii];
    } else if (k < H * N + H) {
      hh = k - H * N;
      p = b + hh;
      gr = gb[hh];
    } else {
      ii = k - H * N - H;
      p = a + ii;
      gr = ga[ii];
    }
    const float mk = b1 * m[k] + (1.0f - b1) * gr;
    const float vk = b2 * v[k] + (1.0f - b2) * gr * gr;
    m[k] = mk;
    v[k] = vk;
    const float val = *p - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    *p = val;
    if (k < H * N) {
      const __nv_bfloat16 q = __float2bfloat16_rn(val);
      WT_t[(size_t)ii * Hp + hh] = q;
      W_t[(size_t)hh * Np + ii] = q;
    } else if (k < H * N + H) {
      b_t[hh] = val;
    } else {
      a_t[ii] = val;
    }
  }
}

__global__ void master_init_kernel(int H, int N, int Np, const __nv_bfloat16 *Wt, const float *bt,
                                   const float *at, float *W, float *b, float *a) {
  const int P = H * N + H + N;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x) {
    if (k < H * N) W[k] = __bfloat162float(Wt[(size_t)(k / N) * Np + (k % N)]);
    else if (k < H * N + H) b[k - H * N] = bt[k - H * N];
    else a[k - H * N - H] = at[k - H * N - H];
  }
}

}  // namespace

cudaError_t launch_rbm_master_init(const RbmTables &r, int N, float *W, float *b, float *a,
                                   cudaStream_t s) {
  const int P = r.H * N + r.H + N;
  int grid = (P + 255) / 256;
  if (grid > 4096) grid = 4096;
  master_init_kernel<<<grid, 256, 0, s>>>(r.H, N, r.Np, r.W, r.b, r.a, W, b, a);
  return cudaGetLastError();
}

cudaError_t launch_rbm_grad(const GradArgs &a, void *recs, int sms, cudaStream_t s) {
  const size_t smem = 1024 + grad_smem_plan(a.Np, a.n_off, a.NW).total;
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  // the row records (and dL/da)
  rbm_records_kernel<<<(a.n + 15) / 16, 256, sizeof(float) * a.Np, s>>>(a, (float4 *)recs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int tiles = a.Hp / TT;
  const size_t asmem = acc_smem(a.Np, a.NW);
  if (a.Np <= 256 && asmem <= 227 * 1024) {
    e = cudaFuncSetAttribute(rbm_grad_acc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)asmem);
    if (e != cudaSuccess) return e;
    int blocks = (sms + tiles - 1) / tiles;
    if (blocks > a.n) blocks = a.n;
    if (blocks < 1) blocks = 1;
    GradArgs g = a;
    g.walkers_per_cta = (a.n + blocks - 1) / blocks;
    blocks = (a.n + g.walkers_per_cta - 1) / g.walkers_per_cta;
    rbm_grad_acc_kernel<<<dim3(tiles, blocks), AG * TT, asmem, s>>>(g, (const float4 *)recs);
    return cudaGetLastError();
  }
  e = cudaFuncSetAttribute(rbm_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int blocks = (2 * sms + tiles - 1) / tiles;
  if (blocks > a.n) blocks = a.n;
  if (blocks < 1) blocks = 1;
  GradArgs g = a;
  g.walkers_per_cta = (a.n + blocks - 1) / blocks;
  blocks = (a.n + g.walkers_per_cta - 1) / g.walkers_per_cta;
  rbm_grad_kernel<<<dim3(tiles, blocks), 3 * TT, smem, s>>>(g, (const float4 *)recs);
  return cudaGetLastError();
}

cudaError_t launch_train_coeff(int n, const double *e, const double *omega, float *gw,
                               double *stats, cudaStream_t s) {
  train_coeff_kernel<<<1, 1024, 0, s>>>(n, e, omega, gw, stats);
  return cudaGetLastError();
}

cudaError_t launch_adam(int H, int N, int Hp, int Np, float *W, float *b, float *a, const float *gW,
                        const float *gb, const float *ga, float *m, float *v, float lr, float b1,
                        float b2, float eps, int step, __nv_bfloat16 *WT_t, __nv_bfloat16 *W_t,
                        float *b_t, float *a_t, cudaStream_t s) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  const int P = H * N + H + N;
  int grid = (P + 255) / 256;
  if (grid > 4096) grid = 4096;
  adam_kernel<<<grid, 256, 0, s>>>(H, N, Hp, Np, W, b, a, gW, gb, ga, m, v, lr, b1, b2, eps, c1, c2,
                                   WT_t, W_t, b_t, a_t);
  return cudaGetLastError();
}

}  // namespace gfmc

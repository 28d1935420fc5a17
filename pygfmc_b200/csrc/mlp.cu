// The GFMC step with a dense MLP guide for Bose-Hubbard occupations (no
// PyGFMC counterpart), float32 with a bf16 tensor-core second layer.
//
//   x = one-hot occupations, z1 = W1 x + b1, h1 = tanh(z1),
//   log psi = w3 . tanh(W2 bf16(h1) + b2) + b3
//
// One CTA per SM, persistent over walkers (atomic work counter), running two
// independent walker pipelines of 8 warps each (named barriers), so that one
// pipeline computes while the other waits on its tensor-core work or draws
// its move.  W2 (H2 x H1, bf16) is staged once per CTA in shared memory in
// the 128-byte swizzled K-major layout (the MMA's B operand, shared by both
// pipelines).  For a walker, z1 is carried from step to step through the
// parent map (field_in / field_out, with log psi: H1 + 1 floats per walker;
// rebuilt from the W1 columns of the occupations when the engine refreshes
// the carried state) and updated per move.  A rate evaluation takes the
// moves in tiles of 128 rows, two threads per row (warps w and w + 4 of the
// pipeline share TMEM lanes 32 (w % 4)):
//   1. one thread per row decodes its move (sites, W1 columns, unguided
//      element);
//   2. per chunk of 64 inputs, the two threads write half the row of the A
//      chunk each,
//      the activations h1' = tanh(z1 + W1[:, new] - W1[:, old]) as bf16
//      (four W1 columns for a two-site move, read as 16-byte vectors); the
//      chunks go through a ring of two buffers, and the pipeline's leader
//      issues tcgen05.mma (kind::f16, M = 128 moves, N = H2, K = 64) on a
//      chunk while the next one is built;
//   3. the epilogue (tcgen05.ld, each thread half the columns of its row)
//      forms log psi(x') = w3 . tanh(v + b2) (up to the constant b3 + sum w3,
//      which cancels in
//      every ratio) and the guided element coupling * exp(log psi(x') -
//      log psi(x)).
// Rows of moves with no element are neither built nor read.  The walker's
// own log psi comes from the same path (a tile whose row 0 is the current
// configuration), so every ratio is a ratio of one function.  The
// pipeline's first warp then forms the diagonal element, scans the rates
// and draws the move and the hold as the cont_time propagator of evolve.cu
// does (the same per-walker Threefry streams).
//
// Roofline: per tile 2 * 128 * H1 * H2 tensor flops, 128 (H1 + H2) tanh (two
// MUFU operations each) and 128 x 4 W1 columns (2 H1 bytes each) from L2.
#include <cfloat>
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "mlp_dev.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

using namespace tc;
using namespace mlpdev;

constexpr int ROWS = 128;               // moves per tile = UMMA M = TMEM lanes
constexpr int PT = 2 * ROWS;            // threads per pipeline: two per row
constexpr int NP = 2;                   // walker pipelines per CTA
constexpr int MT = PT * NP;
constexpr int KC = 64;                  // inputs per A chunk (one 128-byte swizzle row)
constexpr int NBUF = 2;                 // A chunk buffers per pipeline
constexpr unsigned FULLW = 0xffffffffu;

// acc + sum_i wm_i / (1 + 2^{K v_i + bk_i}) over 32 accumulator columns.
__device__ __forceinline__ float reduce32(const uint32_t (&r)[32], const float *bk, const float *wm,
                                          float acc) {
#pragma unroll
  for (int i = 0; i < 32; i += 4) {
    const float4 b = *reinterpret_cast<const float4 *>(bk + i);
    const float4 w = *reinterpret_cast<const float4 *>(wm + i);
    acc = fmaf(w.x, sig2(fmaf(__uint_as_float(r[i]), KT, b.x)), acc);
    acc = fmaf(w.y, sig2(fmaf(__uint_as_float(r[i + 1]), KT, b.y)), acc);
    acc = fmaf(w.z, sig2(fmaf(__uint_as_float(r[i + 2]), KT, b.z)), acc);
    acc = fmaf(w.w, sig2(fmaf(__uint_as_float(r[i + 3]), KT, b.w)), acc);
  }
  return acc;
}

// Shared memory: W2 and the epilogue constants (CTA), then one region per
// pipeline: the A chunk ring, z1, the tile's row records, the rates and
// log amplitudes of the moves, the occupations and the pipeline's
// mbarriers and broadcast words.
struct PipeSmem {
  size_t A, z1, rc, rv, part, rates, lps, occ, misc, bytes;
};
struct MlpSmem {
  size_t W2s, b2, w3, pipe0;
  PipeSmem p;
  size_t total;
};

__host__ __device__ inline MlpSmem mlp_plan(int H1, int H2, int n_off, int N) {
  MlpSmem s;
  size_t o = 0;
  s.W2s = o; o += (size_t)H2 * H1 * 2;
  s.b2 = o; o += (size_t)H2 * 4;
  s.w3 = o; o += (size_t)H2 * 4;
  o = (o + 1023) & ~(size_t)1023;
  s.pipe0 = o;
  PipeSmem &p = s.p;
  size_t q = 0;
  p.A = q; q += (size_t)NBUF * ROWS * 128;
  p.z1 = q; q += (size_t)H1 * 4;
  p.rc = q; q += (size_t)ROWS * 16;
  p.rv = q; q += (size_t)ROWS * 4;
  p.part = q; q += (size_t)2 * ROWS * 4;
  p.rates = q; q += (size_t)(n_off + 1) * 4;
  p.lps = q; q += (size_t)(n_off + 1) * 4;
  p.occ = q; q += (size_t)((N + 15) / 16) * 16;
  q = (q + 15) & ~(size_t)15;
  p.misc = q; q += 128;
  p.bytes = (q + 1023) & ~(size_t)1023;
  s.total = o + NP * p.bytes;
  return s;
}

__device__ __forceinline__ void pipe_sync(int s) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + s), "r"(PT) : "memory");
}

// Pipeline-uniform bounded wait on an mbarrier phase: the leader waits, the
// pipeline's threads get the verdict (false when the limit ran out).
__device__ __forceinline__ bool pipe_wait(uint64_t *bar, uint32_t parity, volatile int *flag, int s,
                                          bool leader) {
  if (leader) {
    int ok = 0;
    for (uint32_t it = 0; it < WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(bar, parity) ? 1 : 0;
    *flag = ok;
  }
  pipe_sync(s);
  const bool r = *flag != 0;
  pipe_sync(s);
  return r;
}

__global__ void __launch_bounds__(MT, 1) mlp_evolve_kernel(DevModel<float> m, MlpTables t,
                                                           EvolveArgs a) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int H1 = t.H1, H2 = t.H2, np1 = t.np1;
  const MlpSmem S = mlp_plan(H1, H2, m.n_off, m.N);
  unsigned char *W2s = base + S.W2s;
  float *b2s = reinterpret_cast<float *>(base + S.b2);
  float *w3s = reinterpret_cast<float *>(base + S.w3);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = tid / PT, tp = tid % PT;             // pipeline, thread in it
  const int ridx = tp & (ROWS - 1), half = tp / ROWS; // row (TMEM lane), row half
  const bool leader = tp == 0;
  unsigned char *pb = base + S.pipe0 + (size_t)s * S.p.bytes;
  unsigned char *Ar = pb + S.p.A;
  float *z1 = reinterpret_cast<float *>(pb + S.p.z1);
  int4 *rc = reinterpret_cast<int4 *>(pb + S.p.rc);
  float *rv = reinterpret_cast<float *>(pb + S.p.rv);
  float *part = reinterpret_cast<float *>(pb + S.p.part);
  float *rates = reinterpret_cast<float *>(pb + S.p.rates);
  float *lps = reinterpret_cast<float *>(pb + S.p.lps);
  uint8_t *occ = pb + S.p.occ;
  uint64_t *freeb = reinterpret_cast<uint64_t *>(pb + S.p.misc);       // NBUF
  uint64_t *done = freeb + NBUF;
  volatile int *flag = reinterpret_cast<volatile int *>(pb + S.p.misc + 32);
  volatile int *bi = reinterpret_cast<volatile int *>(pb + S.p.misc + 48);      // 4 ints
  volatile float *bf = reinterpret_cast<volatile float *>(pb + S.p.misc + 64);  // 4 floats
  uint32_t *slot = reinterpret_cast<uint32_t *>(base + S.pipe0 + S.p.misc + 96);
  const uint32_t dcols = H2 <= 32 ? 32u : (H2 <= 64 ? 64u : (H2 <= 128 ? 128u : 256u));
  const uint32_t ncols = NP * dcols;

  // W2 into the swizzled K-major B layout: K chunk kc (64 inputs) holds the
  // H2 rows, 128 bytes each.  log psi = b3 + sum_j w3_j tanh(v_j + b2_j) =
  // const + sum_j (-2 w3_j) / (1 + 2^{K v_j + K b2_j}).
  for (int idx = tid; idx < H2 * (H1 / 8); idx += MT) {
    const int j = idx / (H1 / 8), c8 = idx % (H1 / 8);
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(t.W2 + (size_t)j * H1) + c8);
    *reinterpret_cast<uint4 *>(sw_chunk(W2s + (size_t)(c8 / 8) * H2 * 128, j, c8 % 8)) = v;
  }
  for (int j = tid; j < H2; j += MT) {
    b2s[j] = KT * t.b2[j];
    w3s[j] = -2.0f * t.w3[j];
  }
  if (warp == 0) tmem_alloc(slot, ncols);
  if (leader) {
    for (int b = 0; b < NBUF; ++b) mbar_init(freeb + b, 1);
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t tD = tmem + (uint32_t)s * dcols;                    // this pipeline's accumulator
  const uint32_t tl = tD + ((uint32_t)(32 * (warp & 3)) << 16);     // this warp's lanes
  const uint32_t idesc = idesc_m128((uint32_t)H2);
  const int CB = ((m.N + 15) / 16) * 16;
  const int C = (m.n_off + 31) / 32;   // rate slots per lane of the sampling warp
  const bool sampler = tp < 32;
  uint32_t use[NBUF] = {};             // commits per A buffer
  uint32_t dphase = 0;
  bool ok = true;
  double wmax = -DBL_MAX;
  unsigned long long hop_acc = 0;

  // One tile: the moves tb .. tb + 127 (current: row 0 is the configuration
  // itself).  Writes rates[o] / lps[o] of the moves, or bf[0] = log psi(x)
  // for the current-configuration tile.
  auto tile = [&](int tb, bool current, float lpx) -> bool {
    if (half == 0) {
      const int o = tb + ridx;
      float v = 0.0f;
      int4 c = make_int4(-1, -1, -1, -1);
      if (current) {
        v = ridx == 0 ? 1.0f : 0.0f;
      } else if (o < m.n_off) {
        const Mv mv = mlp_move(m, occ, o);
        v = mv.v;
        if (v != 0.0f) c = move_cols(mv, occ, np1);
      }
      rv[ridx] = v;
      rc[ridx] = c;
    }
    pipe_sync(s);
    const bool act = rv[ridx] != 0.0f;
    const int4 c = rc[ridx];
    const uint4 *W = reinterpret_cast<const uint4 *>(t.W1T);
    const int rs = H1 / 8;             // uint4 per W1 column
    for (int kc = 0; kc < H1 / KC; ++kc) {
      const int b = kc & (NBUF - 1);
      if (use[b] > 0 && !pipe_wait(freeb + b, (use[b] - 1) & 1u, flag, s, leader)) return false;
      unsigned char *Ab = Ar + (size_t)b * ROWS * 128;
      if (act) {
#pragma unroll 2
        for (int pc = 4 * half; pc < 4 * half + 4; ++pc) {
          const int q = kc * 8 + pc;   // 8-input piece of the row
          float z[8];
          const float4 z0 = *reinterpret_cast<const float4 *>(z1 + 8 * q);
          const float4 z4 = *reinterpret_cast<const float4 *>(z1 + 8 * q + 4);
          z[0] = z0.x; z[1] = z0.y; z[2] = z0.z; z[3] = z0.w;
          z[4] = z4.x; z[5] = z4.y; z[6] = z4.z; z[7] = z4.w;
          if (c.x >= 0) {
            const uint4 pa = __ldg(W + (size_t)c.y * rs + q), qa = __ldg(W + (size_t)c.x * rs + q);
            uint4 pb4 = make_uint4(0, 0, 0, 0), qb4 = make_uint4(0, 0, 0, 0);
            if (c.z >= 0) {
              pb4 = __ldg(W + (size_t)c.w * rs + q);
              qb4 = __ldg(W + (size_t)c.z * rs + q);
            }
            float p8[8], q8[8];
            bf8(pa, p8);
            bf8(qa, q8);
#pragma unroll
            for (int i = 0; i < 8; ++i) z[i] = (z[i] + p8[i]) - q8[i];
            if (c.z >= 0) {
              bf8(pb4, p8);
              bf8(qb4, q8);
#pragma unroll
              for (int i = 0; i < 8; ++i) z[i] = (z[i] + p8[i]) - q8[i];
            }
          }
          uint4 o4;
          uint32_t *ow = reinterpret_cast<uint32_t *>(&o4);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(tanh_h1(z[2 * i]), tanh_h1(z[2 * i + 1]));
            ow[i] = *reinterpret_cast<const uint32_t *>(&h);
          }
          *reinterpret_cast<uint4 *>(sw_chunk(Ab, ridx, pc)) = o4;
        }
      }
      fence_async_smem();
      pipe_sync(s);
      if (leader) {
        fence_after();
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          mma_bf16(tD, sw128_desc(smem_u32(Ab) + 32u * kk),
                   sw128_desc(smem_u32(W2s + (size_t)kc * H2 * 128) + 32u * kk), idesc,
                   (kc > 0 || kk > 0) ? 1u : 0u);
        mma_commit(freeb + b);
        if (kc == H1 / KC - 1) mma_commit(done);
      }
      ++use[b];
    }
    if (!pipe_wait(done, dphase, flag, s, leader)) return false;
    dphase ^= 1u;
    fence_after();
    float acc = 0.0f;
    if (__any_sync(FULLW, rv[ridx] != 0.0f)) {
      if ((H2 & 63) == 0) {
        // this thread's column half in loads of 32 columns
        const int cb = half * (H2 / 2);
        for (int cc = cb; cc < cb + H2 / 2; cc += 32) {
          uint32_t ra[32];
          tmem_ld32_async(tl + (uint32_t)cc, ra);
          tmem_ld_wait(ra);
          acc = reduce32(ra, b2s + cc, w3s + cc, acc);
        }
      } else {
        for (int c0 = 16 * half; c0 < H2; c0 += 32) {
          float v[16];
          tmem_ld16(tl + (uint32_t)c0, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc = fmaf(w3s[c0 + i], sig2(fmaf(v[i], KT, b2s[c0 + i])), acc);
        }
      }
    }
    part[half * ROWS + ridx] = acc;
    fence_before();
    pipe_sync(s);
    if (half == 0) {
      const float lp = part[ridx] + part[ROWS + ridx];
      if (current) {
        if (ridx == 0) bf[0] = lp;
      } else {
        const int o = tb + ridx;
        if (o < m.n_off) {
          const float v = rv[ridx];
          lps[o] = lp;
          rates[o] = v != 0.0f ? v * __expf(lp - lpx) : 0.0f;
        }
      }
    }
    fence_before();
    pipe_sync(s);
    return true;
  };

  // H_xx (BoseHubbard diagonal, bose_hubbard.py:271-281) in the step
  // kernel's lane order, by the sampling warp
  auto diag0 = [&]() -> float {
    float su = 0.0f, sm = 0.0f;
    for (int k = lane; k < m.N; k += 32) {
      const float n = (float)occ[k];
      if (m.has_U) su += m.U[k] * n * (n - 1.0f);
      if (m.has_mu) sm += m.mu[k] * n;
    }
    float d = 0.0f;
    if (m.has_U) d = d + 0.5f * warp_sum(su);
    if (m.has_mu) d = d - warp_sum(sm);
    return d;
  };

  // Sampling warp: this lane's chunk sum of the weights -rates (C slots per
  // lane) into *own; returns its inclusive scan over the lanes.
  auto scan0 = [&](float *own) -> float {
    float sum = 0.0f;
    const int lo = lane * C, hi = min(lo + C, m.n_off);
    for (int o = lo; o < hi; ++o) sum += -rates[o];
    *own = sum;
    return warp_inclusive_scan(sum, lane);
  };

  for (;;) {
    if (leader) bi[0] = atomicAdd(a.work_ctr, 1);
    pipe_sync(s);
    const int walker = bi[0];
    pipe_sync(s);
    if (walker >= a.n_walkers) break;
    const int src = a.parents ? a.parents[walker] : walker;
    const uint32_t *in = reinterpret_cast<const uint32_t *>(
        reinterpret_cast<const uint8_t *>(a.cfg_in) + (size_t)src * CB);
    for (int k = tp; k < CB / 4; k += PT) reinterpret_cast<uint32_t *>(occ)[k] = in[k];
    pipe_sync(s);
    // an occupation above n_max is flagged and clamped (W1 has n_max + 1
    // columns per site)
    for (int k = tp; k < m.N; k += PT)
      if (occ[k] > m.n_max) {
        atomicOr(a.status, ST_BAD_CONFIG);
        occ[k] = (uint8_t)m.n_max;
      }
    pipe_sync(s);
    // z1 and log psi: carried from the parent (H1 + 1 floats per walker), or
    // z1 = b1 + the W1 columns of the occupations and log psi through a tile
    const float *fin =
        a.field_in ? reinterpret_cast<const float *>(a.field_in) + (size_t)src * (H1 + 1) : nullptr;
    for (int j = tp; j < H1; j += PT) {
      float z;
      if (fin) {
        z = fin[j];
      } else {
        z = t.b1[j];
        for (int k = 0; k < m.N; ++k) z += __bfloat162float(t.W1T[(size_t)(k * np1 + occ[k]) * H1 + j]);
      }
      z1[j] = z;
    }
    pipe_sync(s);
    float lpx;
    if (fin) {
      lpx = fin[H1];
    } else {
      if (!tile(0, true, 0.0f)) { ok = false; break; }
      lpx = bf[0];
    }

    const Key kw = fold(a.key, (uint32_t)(a.walker_offset + walker));
    double lw = a.lw_in ? a.lw_in[src] : 0.0;
    float eloc = 0.0f;
    int hops = 0;
    if (a.method == CONT_TIME) {
      const float beta = (float)a.step;
      float tcur = 0.0f;
      uint32_t it = 0;
      while (tcur < beta) {
        for (int tb = 0; tb < m.n_off && ok; tb += ROWS) ok = tile(tb, false, lpx);
        if (!ok) break;
        if (sampler) {
          // evolution.sample_index:30-59: the first slot whose cdf exceeds u,
          // stepped back to the nearest slot at or before it with positive
          // weight
          const float d = diag0();
          float own;
          const float cum = scan0(&own);
          const float R = __shfl_sync(FULLW, cum, 31);
          const float U1 = uniform<float>(fold(kw, 2u * it));
          const float psi = uniform<float>(fold(kw, 2u * it + 1u));
          int si = 0;
          if (R > 0.0f) {   // (R is the same in every lane)
            float u = U1 * R;
            const float cap = nextafterf(R, 0.0f);
            u = u < cap ? u : cap;
            const unsigned bal = __ballot_sync(FULLW, cum > u);
            const int Lh = bal ? __ffs(bal) - 1 : 31;
            if (lane == Lh) {
              int hit = m.n_off - 1;
              if (bal) {
                float cu = cum - own;
                const int lo = Lh * C, hi = min(lo + C, m.n_off);
                for (int o = lo; o < hi; ++o) {
                  cu += -rates[o];
                  if (cu > u) { hit = o; break; }
                }
              }
              si = hit;
              for (int o = hit; o >= 0; --o)
                if (-rates[o] > 0.0f) { si = o; break; }
            }
            si = __shfl_sync(FULLW, si, Lh);
          }
          if (lane == 0) {
            const float tau_raw = R > 0.0f ? -log1pf(-psi) / R : __int_as_float(0x7F800000);
            const float rem = beta - tcur;
            bi[2] = si;
            bi[1] = (tau_raw < rem) ? 1 : 0;
            bf[1] = tau_raw < rem ? tau_raw : rem;
            bf[0] = d - R;
          }
        }
        pipe_sync(s);
        const float tau = bf[1], eL = bf[0];
        const int hop = bi[1], si = bi[2];
        lw = lw - (double)eL * (double)tau;
        tcur = tcur + tau;
        if (hop) {
          const Mv mv = mlp_move(m, occ, si);
          const int4 c = move_cols(mv, occ, np1);
          for (int j = tp; j < H1; j += PT) {
            float z = z1[j];
            z = (z + __bfloat162float(t.W1T[(size_t)c.y * H1 + j])) -
                __bfloat162float(t.W1T[(size_t)c.x * H1 + j]);
            if (c.z >= 0)
              z = (z + __bfloat162float(t.W1T[(size_t)c.w * H1 + j])) -
                  __bfloat162float(t.W1T[(size_t)c.z * H1 + j]);
            z1[j] = z;
          }
          lpx = lps[si];
          pipe_sync(s);
          if (leader) {
            occ[mv.a] = (uint8_t)(occ[mv.a] + mv.da);
            if (mv.b != mv.a) occ[mv.b] = (uint8_t)(occ[mv.b] + mv.db);
          }
          ++hops;
        }
        eloc = eL;
        pipe_sync(s);
        if (++it >= (uint32_t)a.max_iters) {
          if (leader) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      lw -= a.alw * a.step;
    } else {   // EVALUATE: E_L = H_xx + sum of the guided off-diagonal elements
      for (int tb = 0; tb < m.n_off && ok; tb += ROWS) ok = tile(tb, false, lpx);
      if (!ok) break;
      if (sampler) {
        const float d = diag0();
        float own;
        const float R = __shfl_sync(FULLW, scan0(&own), 31);
        if (lane == 0) {
          bf[0] = d - R;
          bf[3] = d;
          if (a.rsum_out) a.rsum_out[walker] = -R;
        }
      }
      pipe_sync(s);
      eloc = bf[0];
      if (leader && a.diag_out) a.diag_out[walker] = (double)bf[3];
      // the guided elements of every move (the trainer's row coefficients)
      if (a.rates_out)
        for (int o = tp; o < m.n_off; o += PT) a.rates_out[(size_t)walker * m.n_off + o] = rates[o];
    }
    if (!ok) break;
    if (a.cfg_out) {
      uint32_t *out = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(a.cfg_out) +
                                                   (size_t)walker * CB);
      for (int k = tp; k < CB / 4; k += PT) out[k] = reinterpret_cast<const uint32_t *>(occ)[k];
    }
    if (a.field_out) {
      float *fo = reinterpret_cast<float *>(a.field_out) + (size_t)walker * (H1 + 1);
      for (int j = tp; j < H1; j += PT) fo[j] = z1[j];
      if (leader) fo[H1] = lpx;
    }
    if (leader) {
      if (a.method == CONT_TIME) a.log_w[walker] = lw;
      a.e_loc[walker] = (double)eloc;
    }
    if (a.method == CONT_TIME) wmax = lw > wmax ? lw : wmax;
    hop_acc += (unsigned long long)hops;
    pipe_sync(s);
  }
  if (!ok && leader) atomicOr(a.status, ST_TIMEOUT);
  if (leader) {
    if (a.partial_max) a.partial_max[(size_t)blockIdx.x * NP + s] = wmax;
    if (a.hops && hop_acc) atomicAdd(a.hops, hop_acc);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace

size_t mlp_smem_bytes(int H1, int H2, int n_off, int N) {
  return 1024 + mlp_plan(H1, H2, n_off, N).total;
}

int mlp_partials(int grid, int n_walkers) {
  return NP * (grid < n_walkers ? grid : (n_walkers > 0 ? n_walkers : 1));
}

int mlp_grid() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

cudaError_t launch_mlp_evolve(const DevModel<float> &m, const MlpTables &t, const EvolveArgs &a,
                              int grid, cudaStream_t s) {
  // at least half an SM's shared memory, so that one CTA per SM holds TMEM
  size_t smem = mlp_smem_bytes(t.H1, t.H2, m.n_off, m.N);
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  if (smem < 120 * 1024) smem = 120 * 1024;
  cudaError_t e = cudaFuncSetAttribute(mlp_evolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  if (grid > a.n_walkers) grid = a.n_walkers;
  if (grid < 1) grid = 1;
  mlp_evolve_kernel<<<grid, MT, smem, s>>>(m, t, a);
  return cudaGetLastError();
}

}  // namespace gfmc

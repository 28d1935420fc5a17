// The GFMC step with an RBM guide, float32 build: the walkers of a block
// evaluate their rates in lockstep, over tables staged once per block.
//
// Ratio of a move.  With theta' = theta + u_i + u_j, u_ih = -2 s_i W_hi (an
// edge flip; a site flip has no j), the addition theorems give per hidden
// unit
//   cosh(theta'_h) / cosh(theta_h)
//     = c_ih c_jh [1 + s_i s_j tau_ih tau_jh - t_h (s_i tau_ih + s_j tau_jh)],
// c = cosh(2 W), tau = tanh(2 W) (spin-independent weight tables) and
// t_h = tanh(theta_h) (once per walker and evaluation).  So a (slot, unit)
// pair costs three FMA-pipe operations and a product instead of a log cosh
// (the units go in pairs through packed float32x2 instructions): the
// product of the bracket over a lane's units, plus the lane's
// log2 prod c_ih (tabulated per site and lane), gives one lg2 per lane and
// slot, and a warp sum the slot's log2 ratio.  Should a lane's product leave
// the normal float range (weights far beyond the guide's usual scale), the
// slot is evaluated term by term instead (log cosh differences from W).
// Each slot's sites, staged rows, couplings and a terms come from one
// 32-byte record; the walker's spins are kept as +-1 floats in shared
// memory beside its spin words.
//
// Staging.  The slots are split into chunks whose flipped sites' rows
// (tau of every unit, then the 32 lane sums of log2 c) fit in shared memory
// (at most 16 sites, double buffered); the block's 8 warps, one walker each,
// evaluate chunk by chunk between block barriers while the next chunk's rows
// arrive by cp.async, so each row crosses L2 once per block and evaluation
// instead of once per walker and slot.  A round is one rate evaluation of
// every warp's walker; between rounds each warp draws its move, holds or
// finishes its walker and takes the next one (dynamic assignment), as the
// float64 kernel does per walker (rbm.cu).  The propagators, random streams,
// draws and outputs are those of rbm.cu.
#include "rbm_dev.cuh"

namespace gfmc {
namespace {

constexpr int RBF_THREADS = RBF_WARPS * 32;

__host__ __device__ inline size_t rbf_stage_bytes(int U, int RS) {
  return (size_t)U * RS * sizeof(float);
}

// Per-warp region: the float64 kernel's (spin words, rate row), then the
// walker's spins as +-1 floats.
__host__ __device__ inline size_t rbf_warp_bytes(int N, int M) {
  return rb_warp_bytes<float>(N, M) + (((size_t)N * sizeof(float) + 15) & ~(size_t)15);
}

// Stages chunk c's rows into buf (all threads; 16-byte cp.async pieces).
__device__ __forceinline__ void stage_chunk(const RbmTables &r, int c, float *buf) {
  const int nrow = r.ch_n[c];
  const int pieces = r.RS / 4;   // RS is a multiple of 32 floats
  const int *sites = r.ch_sites + (size_t)c * r.ch_U;
  for (int p = threadIdx.x; p < nrow * pieces; p += RBF_THREADS) {
    const int row = p / pieces, col = p - row * pieces;
    const float *src = r.RT + (size_t)sites[row] * r.RS + 4 * col;
    const unsigned dst = (unsigned)__cvta_generic_to_shared(buf + (size_t)row * r.RS + 4 * col);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Packed float pairs (two IEEE single-precision operations per instruction).
__device__ __forceinline__ uint64_t pk2(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 upk2(uint64_t v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

// The lane's product over its HPL units of the bracket of slot (i, j):
// KIND 0 a site flip, 1 an anti-parallel edge, 2 a parallel edge; SI the
// sign of s_i (an edge's s_j is -s_i for KIND 1, s_i for KIND 2).
// ti / tj: the staged rows at this lane's first float4 (the rows hold the
// lane's units k4 * 4 .. k4 * 4 + 3 at float4 k4 * 32 + lane, so a warp's
// loads are consecutive 16-byte pieces, free of bank conflicts); t2 the
// lane's tanh(theta) as pairs of units.  The units go in pairs through
// packed float32x2 operations, the even units into the low half of the
// product and the odd ones into the high half.  Where a bracket is formed
// negated (-B, one operation shorter), every unit's is, and each half
// multiplies an even number of them (HPL / 2 of 4, 8, 12, 16), so the
// product is the same.
template <int HPL, int KIND, bool SI>
__device__ __forceinline__ float bracket_product(const float *ti, const float *tj,
                                                 const uint64_t (&t2)[HPL / 2]) {
  const uint64_t one2 = pk2(1.0f, 1.0f), mone2 = pk2(-1.0f, -1.0f);
  uint64_t pr = one2;
#pragma unroll
  for (int k4 = 0; k4 < HPL / 4; ++k4) {
    const ulonglong2 A = reinterpret_cast<const ulonglong2 *>(ti)[32 * k4];
    ulonglong2 Bv = make_ulonglong2(0ull, 0ull);
    if (KIND != 0) Bv = reinterpret_cast<const ulonglong2 *>(tj)[32 * k4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint64_t a = h ? A.y : A.x, b = h ? Bv.y : Bv.x, t = t2[2 * k4 + h];
      uint64_t B;
      if (KIND == 0) {
        // 1 - t s_i tau_i (as t tau_i - 1 = -B for s_i = +1)
        B = SI ? fma2(t, a, mone2) : fma2(t, a, one2);
      } else if (KIND == 1) {
        // s_i s_j = -1: -B = t s_i (tau_i - tau_j) + tau_i tau_j - 1
        const uint64_t d = SI ? sub2(a, b) : sub2(b, a);
        B = fma2(t, d, fma2(a, b, mone2));
      } else {
        // s_i s_j = +1: 1 + tau_i tau_j - t s_i (tau_i + tau_j)
        const uint64_t e = fma2(a, b, one2), u = add2(a, b);
        B = SI ? sub2(e, mul2(t, u)) : fma2(t, u, e);
      }
      pr = mul2(pr, B);
    }
  }
  const float2 p = upk2(pr);
  return p.x * p.y;
}

// log cosh(theta') - log cosh(theta) summed over the lane's units, term by
// term from the weight rows (the slow path for products out of range).
template <int HPL>
__device__ __forceinline__ float direct_difference(const RbmTables &r, const float (&th)[HPL],
                                                   int i, int j, float si, float sj, int lane) {
  float wi[HPL], wj[HPL];
  load_row<HPL>(r.WT + (size_t)i * r.Hp + lane * HPL, wi);
  if (j >= 0) {
    load_row<HPL>(r.WT + (size_t)j * r.Hp + lane * HPL, wj);
  } else {
#pragma unroll
    for (int k = 0; k < HPL; ++k) wj[k] = 0.0f;
  }
  float acc = 0.0f;
#pragma unroll
  for (int k = 0; k < HPL; ++k)
    acc += lncosh<float>(th[k] - 2.0f * si * wi[k] - 2.0f * sj * wj[k]) - lncosh<float>(th[k]);
  return acc;
}

// The rates of the chunk's slots for this warp's walker into q[1 + o]; sg:
// the walker's spins as +-1 floats.
template <int HPL>
__device__ __forceinline__ void chunk_rates(const RbmTables &r, int c, const float *buf,
                                            const float *sg, const float (&th)[HPL],
                                            const uint64_t (&t)[HPL / 2], float *q, int lane) {
  constexpr float LOG2E = 1.4426950408889634f;
  const int o1 = r.ch_start[c + 1];
  for (int o = r.ch_start[c]; o < o1; ++o) {
    const int4 r0 = __ldg(r.ch_rec + 2 * o);
    const int i = r0.x & 0xFFFF, j = r0.y & 0xFFFF;
    const float si = sg[i];
    const bool site = j == 0xFFFF;
    const float sj = site ? 0.0f : sg[j];
    const bool anti = si != sj;
    const float cpl = __int_as_float(anti ? r0.z : r0.w);
    float rate = cpl;
    if (cpl != 0.0f) {
      const float *ri = buf + (size_t)(r0.x >> 16) * r.RS;
      const float *rj = buf + (size_t)(r0.y >> 16) * r.RS;
      const float *a = ri + 4 * lane, *b = rj + 4 * lane;
      const bool up = si > 0.0f;
      float prod;
      if (site)
        prod = up ? bracket_product<HPL, 0, true>(a, b, t) : bracket_product<HPL, 0, false>(a, b, t);
      else if (anti)
        prod = up ? bracket_product<HPL, 1, true>(a, b, t) : bracket_product<HPL, 1, false>(a, b, t);
      else
        prod = up ? bracket_product<HPL, 2, true>(a, b, t) : bracket_product<HPL, 2, false>(a, b, t);
      const bool ok = prod >= FLT_MIN && prod <= FLT_MAX;
      float l2;
      if (__all_sync(FULLM, ok)) {
        l2 = __log2f(prod) + ri[r.Hp + lane] + (site ? 0.0f : rj[r.Hp + lane]);
      } else {
        l2 = LOG2E * direct_difference<HPL>(r, th, i, site ? -1 : j, si, sj, lane);
      }
      const float4 r1 = __ldg(reinterpret_cast<const float4 *>(r.ch_rec) + 2 * o + 1);
      const float d2 = fmaf(-r1.y, sj, fmaf(-r1.x, si, warp_sum(l2)));
      rate = cpl * ex2_approx(d2);
    }
    if (lane == 0) q[1 + o] = rate;
  }
}

// Off-diagonal move o of the walker: theta and the spin words (rbm_move),
// then the +-1 spins.
template <int HPL>
__device__ __forceinline__ void rbf_move(const DevModel<float> &m, const RbmTables &r,
                                         uint64_t *bits, float *sg, float (&th)[HPL], int o,
                                         int lane) {
  const int4 r0 = __ldg(r.ch_rec + 2 * o);
  rbm_move<float, HPL>(m, r, bits, th, o, lane);
  if (lane == 0) {
    const int i = r0.x & 0xFFFF, j = r0.y & 0xFFFF;
    sg[i] = -sg[i];
    if (j != 0xFFFF) sg[j] = -sg[j];
  }
  __syncwarp();
}

// Diagonal element q[0] (SpinHalf.diagonal_weight:291-314).
__device__ __forceinline__ void rbf_diag(const DevModel<float> &m, const uint64_t *bits, float *q,
                                         int lane) {
  float dg = 0.0f;
  if (m.has_jz) {
    int na = 0;
    float jzs = 0.0f;
    for (int e = lane; e < m.E; e += 32) {
      const uint32_t pe = m.edge[e];
      const bool anti = spin_bit(bits, (int)(pe & 0xFFFF)) != spin_bit(bits, (int)(pe >> 16));
      if (m.uniform_jz) na += anti;
      else jzs += anti ? -m.jz[e] / 4.0f : m.jz[e] / 4.0f;
    }
    if (m.uniform_jz) dg = (m.jz[0] / 4.0f) * (float)(m.E - 2 * warp_sum(na));
    else dg = warp_sum(jzs);
  }
  if (m.has_hz) {
    float hzs = 0.0f;
    for (int k = lane; k < m.N; k += 32) hzs += m.hz[k] * (spin_bit(bits, k) ? 1.0f : -1.0f);
    dg = dg + warp_sum(hzs) / 2.0f;
  }
  if (lane == 0) q[0] = dg;
}

// Per-warp walker state between rounds.
struct Walk {
  int active, walker, src;
  double lw;
  float eloc, t, draws;
  uint32_t it;
  int hops, phase;   // discrete methods: sub-steps done (single) / used (multi)
  Key kw;
};

template <int HPL>
__global__ void __launch_bounds__(RBF_THREADS, 2)
rbm_evolve_f32_kernel(DevModel<float> m, RbmTables r, EvolveArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int NW = rb_words(m.N);
  const size_t sb = rbf_stage_bytes(r.ch_U, r.RS);
  float *const stage0 = reinterpret_cast<float *>(smem);
  const size_t stage_stride = sb / sizeof(float);   // the second buffer follows the first
  unsigned char *wb = smem + 2 * sb + (size_t)wib * rbf_warp_bytes(m.N, m.M);
  uint64_t *bits = reinterpret_cast<uint64_t *>(wb);
  float *q = reinterpret_cast<float *>(wb + (size_t)NW * 8);
  float *sg = reinterpret_cast<float *>(wb + rb_warp_bytes<float>(m.N, m.M));
  const int method = a.method;
  const float lam = (float)a.lam;
  const int hoff = lane * HPL;
  double wmax = -DBL_MAX;
  unsigned long long hop_acc = 0;
  float th[HPL];
  Walk w{};

  // takes the next walker (or none): configuration through the parent map, theta
  auto fetch = [&]() {
    int wk = 0;
    if (lane == 0) wk = atomicAdd(a.work_ctr, 1);
    wk = __shfl_sync(FULLM, wk, 0);
    w.active = wk < a.n_walkers;
    if (!w.active) return;
    w.walker = wk;
    w.src = a.parents ? a.parents[wk] : wk;
    const uint64_t *in = reinterpret_cast<const uint64_t *>(a.cfg_in) + (size_t)w.src * NW;
    for (int k = lane; k < NW; k += 32) bits[k] = in[k];
    __syncwarp();
    for (int k = lane; k < m.N; k += 32) sg[k] = spin_bit(bits, k) ? 1.0f : -1.0f;
    __syncwarp();
    if (a.field_in) {
      const float *fin = reinterpret_cast<const float *>(a.field_in) + (size_t)w.src * r.Hp + hoff;
#pragma unroll
      for (int k = 0; k < HPL; ++k) th[k] = fin[k];
    } else {
#pragma unroll
      for (int k = 0; k < HPL; ++k) th[k] = r.b[hoff + k];
      for (int i = 0; i < m.N; ++i) {
        const float si = spin_bit(bits, i) ? 1.0f : -1.0f;
        float wv[HPL];
        load_row<HPL>(r.WT + (size_t)i * r.Hp + hoff, wv);
#pragma unroll
        for (int k = 0; k < HPL; ++k) th[k] = th[k] + si * wv[k];
      }
    }
    w.kw = fold(a.key, (uint32_t)(a.walker_offset + wk));
    w.lw = a.lw_in ? a.lw_in[w.src] : 0.0;
    w.eloc = 0.0f;
    w.t = 0.0f;
    w.draws = 0.0f;
    w.it = 0;
    w.hops = 0;
    w.phase = 0;
  };

  // writes the finished walker
  auto finish = [&]() {
    if (a.cfg_out) {
      uint64_t *out = reinterpret_cast<uint64_t *>(a.cfg_out) + (size_t)w.walker * NW;
      for (int k = lane; k < NW; k += 32) out[k] = bits[k];
    }
    if (a.field_out) {
      float *fout = reinterpret_cast<float *>(a.field_out) + (size_t)w.walker * r.Hp + hoff;
#pragma unroll
      for (int k = 0; k < HPL; ++k) fout[k] = th[k];
    }
    if (lane == 0) {
      if (method <= MULTI_STEP) a.log_w[w.walker] = w.lw;
      a.e_loc[w.walker] = (double)w.eloc;
    }
    if (method <= MULTI_STEP) wmax = w.lw > wmax ? w.lw : wmax;
    hop_acc += (unsigned long long)w.hops;
    __syncwarp();
  };

  fetch();
  for (;;) {
    if (!__syncthreads_or(w.active)) break;
    // ---- one rate evaluation of every active warp's walker, chunk by chunk
    uint64_t t[HPL / 2];
    if (w.active) {
#pragma unroll
      for (int k = 0; k < HPL / 2; ++k) t[k] = pk2(tanhf(th[2 * k]), tanhf(th[2 * k + 1]));
    }
    if (r.n_chunks > 0) stage_chunk(r, 0, stage0);
    for (int c = 0; c < r.n_chunks; ++c) {
      stage_wait();
      __syncthreads();   // chunk c landed; every warp is done with chunk c - 1
      if (c + 1 < r.n_chunks) stage_chunk(r, c + 1, stage0 + ((c + 1) & 1) * stage_stride);
      if (w.active) chunk_rates<HPL>(r, c, stage0 + (c & 1) * stage_stride, sg, th, t, q, lane);
    }
    if (!w.active) continue;
    rbf_diag(m, bits, q, lane);
    __syncwarp();

    // ---- this walker's use of the evaluation
    bool done = false;
    if (method == CONT_TIME) {
      const float beta = (float)a.step;
      const RScan<float> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      const float R = sc.total;
      const float eL = q[0] - R;
      if ((w.it & 15u) == 0) w.draws = uniform<float>(fold(w.kw, 2u * w.it + (uint32_t)lane));
      const float U1 = __shfl_sync(FULLM, w.draws, (int)(2u * (w.it & 15u)));
      const float psi = __shfl_sync(FULLM, w.draws, (int)(2u * (w.it & 15u) + 1u));
      int si = 0;
      if (R > 0.0f) {
        const float u = U1 * R, cap = next_below(R);
        si = rbm_pick(q, sc, RB_OFF, lam, u < cap ? u : cap, lane);
      }
      const float tau_raw = (R > 0.0f) ? -math_log1p(-psi) / R : pos_inf<float>();
      const float rem = beta - w.t;
      const float tau = tau_raw < rem ? tau_raw : rem;
      w.lw = w.lw - (double)eL * (double)tau;
      w.t = w.t + tau;
      if (tau_raw < rem) {
        rbf_move<HPL>(m, r, bits, sg, th, si, lane);
        ++w.hops;
      }
      w.eloc = eL;
      if (++w.it >= (uint32_t)a.max_iters) {
        if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
        done = true;
      }
      if (!(w.t < beta)) done = true;
      if (done) w.lw -= a.alw * a.step;
    } else if (method == SINGLE_STEP) {
      const int n_bra = (int)a.step;
      if (w.phase < n_bra) {
        const int sidx = w.phase;
        const RScan<float> sc = rbm_scan(q, m.n_off, RB_LAM, lane);
        const float bx = lam - sc.total;
        if ((sidx & 31) == 0) w.draws = uniform<float>(fold(w.kw, (uint32_t)(sidx + lane)));
        const float U = __shfl_sync(FULLM, w.draws, sidx & 31);
        const float u = U * bx, cap = next_below(bx);
        const int idx = rbm_pick(q, sc, RB_LAM, lam, u < cap ? u : cap, lane);
        if (idx != 0) {
          rbf_move<HPL>(m, r, bits, sg, th, idx - 1, lane);
          ++w.hops;
        }
        w.lw = w.lw + (double)math_log(bx);
        ++w.phase;
      } else {
        const RScan<float> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
        w.eloc = q[0] - sc.total;
        w.lw -= a.alw * (double)n_bra;
        done = true;
      }
    } else if (method == MULTI_STEP) {
      const int n_bra = (int)a.step;
      const RScan<float> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      if (w.phase < n_bra) {
        const float R = sc.total;
        const float bx = lam - q[0] + R;
        if ((w.it & 15u) == 0) w.draws = uniform<float>(fold(w.kw, 2u * w.it + (uint32_t)lane));
        const float U1 = __shfl_sync(FULLM, w.draws, (int)(2u * (w.it & 15u)));
        const float psi = __shfl_sync(FULLM, w.draws, (int)(2u * (w.it & 15u) + 1u));
        int si = 0;
        if (R > 0.0f) {
          const float u = U1 * R, cap = next_below(R);
          si = rbm_pick(q, sc, RB_OFF, lam, u < cap ? u : cap, lane);
        }
        const int remaining = n_bra - w.phase;
        const float hp = R / bx;
        const bool can_hop = hp > 0.0f;
        const float log_pd = can_hop ? math_log1p(-hp) : -1.0f;
        const float hold = floorf(math_log1p(-psi) / log_pd) + 1.0f;
        const float capk = (float)(remaining + 1);
        const float hm = hold < capk ? hold : capk;
        const int k_raw = can_hop ? (int)hm : remaining + 1;
        const int k = k_raw < remaining ? k_raw : remaining;
        w.lw = w.lw + (double)math_log(bx) * (double)k;
        w.phase += k;
        if (k_raw <= remaining) {
          rbf_move<HPL>(m, r, bits, sg, th, si, lane);
          ++w.hops;
        }
        if (++w.it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          w.phase = n_bra;   // the next round is the final evaluation
        }
      } else {
        w.eloc = q[0] - sc.total;
        w.lw -= a.alw * (double)n_bra;
        done = true;
      }
    } else {  // EVALUATE
      const RScan<float> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      w.eloc = q[0] - sc.total;
      if (a.rates_out)
        for (int o = lane; o < m.n_off; o += 32)
          a.rates_out[(size_t)w.walker * m.n_off + o] = q[1 + o];
      if (a.rsum_out && lane == 0) a.rsum_out[w.walker] = -sc.total;
      if (a.diag_out && lane == 0) a.diag_out[w.walker] = (double)q[0];
      done = true;
    }
    if (done) {
      finish();
      fetch();
    }
    __syncwarp();
  }
  if (lane == 0) {
    if (a.partial_max) a.partial_max[(size_t)blockIdx.x * RBF_WARPS + wib] = wmax;
    if (a.hops && hop_acc) atomicAdd(a.hops, hop_acc);
  }
}

using RbfKernel = void (*)(DevModel<float>, RbmTables, EvolveArgs);

RbfKernel pick_rbf(int hpl) {
  switch (hpl) {
    case 8: return rbm_evolve_f32_kernel<8>;
    case 16: return rbm_evolve_f32_kernel<16>;
    case 24: return rbm_evolve_f32_kernel<24>;
    default: return rbm_evolve_f32_kernel<32>;
  }
}

size_t rbf_smem(const DevModel<float> &m, const RbmTables &r) {
  return 2 * rbf_stage_bytes(r.ch_U, r.RS) + RBF_WARPS * rbf_warp_bytes(m.N, m.M);
}

// RT row i: tanh(2 W[h, i]) for h < Hp, interleaved by lane (unit h =
// l HPL + 4 k4 + q of lane l at float 4 (32 k4 + l) + q), then per lane l the
// log2 of the product of cosh(2 W[h, i]) over the lane's units (evaluated in
// float64).
__global__ void rbm_derive_kernel(const __nv_bfloat16 *WT, int Hp, int RS, float *RT) {
  const int i = blockIdx.x;
  const __nv_bfloat16 *row = WT + (size_t)i * Hp;
  float *out = RT + (size_t)i * RS;
  const int hpl = Hp / 32;
  for (int h = threadIdx.x; h < Hp; h += blockDim.x) {
    const int l = h / hpl, k = h - l * hpl;
    out[4 * (32 * (k >> 2) + l) + (k & 3)] = (float)tanh(2.0 * (double)__bfloat162float(row[h]));
  }
  for (int l = threadIdx.x; l < 32; l += blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < hpl; ++k) s += log(cosh(2.0 * (double)__bfloat162float(row[l * hpl + k])));
    out[Hp + l] = (float)(s * 1.4426950408889634);
  }
}

// The slot records' a terms 2 log2(e) a_i, 2 log2(e) a_j from the guide's a.
__global__ void rbm_derive_rec_kernel(const float *a, int n_rec, int4 *rec) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_rec) return;
  const int4 r0 = rec[2 * o];
  const int i = r0.x & 0xFFFF, j = r0.y & 0xFFFF;
  int4 r1 = rec[2 * o + 1];
  const float l2a = 2.0f * 1.4426950408889634f;
  r1.x = __float_as_int(l2a * a[i]);
  r1.y = __float_as_int(j == 0xFFFF ? 0.0f : l2a * a[j]);
  rec[2 * o + 1] = r1;
}

}  // namespace

int rbm_chunk_sites(int Hp, int N, int M) {
  const size_t RS = (size_t)Hp + 32;
  const size_t budget = (size_t)227 * 1024 / 2;   // two blocks per SM
  const size_t warps = (size_t)RBF_WARPS * rbf_warp_bytes(N, M);
  if (warps >= budget) return 0;
  size_t U = (budget - warps) / (2 * RS * sizeof(float));
  if (U > 16) U = 16;
  return U >= 2 ? (int)U : 0;
}

void rbm_build_chunks(int N, int n_hx, int n_edges, const int *edge_i, const int *edge_j, int U,
                      std::vector<int> &start, std::vector<int> &sites, std::vector<int> &nsites,
                      std::vector<uint16_t> &pos) {
  start.clear();
  sites.clear();
  nsites.clear();
  pos.assign((size_t)n_hx + n_edges, 0);
  std::vector<int> cur;
  auto find = [&](int s) {
    for (size_t k = 0; k < cur.size(); ++k)
      if (cur[k] == s) return (int)k;
    return -1;
  };
  auto close = [&]() {
    nsites.push_back((int)cur.size());
    for (int k = 0; k < U; ++k) sites.push_back(k < (int)cur.size() ? cur[k] : 0);
    cur.clear();
  };
  start.push_back(0);
  const int n_off = n_hx + n_edges;
  for (int o = 0; o < n_off; ++o) {
    const int i = o < n_hx ? o : edge_i[o - n_hx];
    const int j = o < n_hx ? -1 : edge_j[o - n_hx];
    const int add = (find(i) < 0) + (j >= 0 && j != i && find(j) < 0);
    if ((int)cur.size() + add > U) {
      close();
      start.push_back(o);
    }
    if (find(i) < 0) cur.push_back(i);
    if (j >= 0 && find(j) < 0) cur.push_back(j);
    pos[o] = (uint16_t)(find(i) | ((j >= 0 ? find(j) : 255) << 8));
  }
  if (n_off > 0) {
    close();
    start.push_back(n_off);
  }
  (void)N;
}

cudaError_t launch_rbm_derive(const RbmTables &r, int N, cudaStream_t s) {
  if (N <= 0) return cudaSuccess;
  rbm_derive_kernel<<<N, 256, 0, s>>>(r.WT, r.Hp, r.RS, r.RT);
  if (r.n_rec > 0) rbm_derive_rec_kernel<<<(r.n_rec + 255) / 256, 256, 0, s>>>(r.a, r.n_rec, r.ch_rec);
  return cudaGetLastError();
}

int rbm_grid_f32(const DevModel<float> &m, const RbmTables &r) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = rbf_smem(m, r);
  RbfKernel k = pick_rbf(rbm_hpl(r.Hp));
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, RBF_THREADS, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

cudaError_t launch_rbm_evolve_f32(const DevModel<float> &m, const RbmTables &r,
                                  const EvolveArgs &a, int grid, cudaStream_t s) {
  const size_t smem = rbf_smem(m, r);
  int need = (a.n_walkers + RBF_WARPS - 1) / RBF_WARPS;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  pick_rbf(rbm_hpl(r.Hp))<<<grid, RBF_THREADS, smem, s>>>(m, r, a);
  return cudaGetLastError();
}

}  // namespace gfmc

// The per-walker propagation step of GFMC on B200: one warp per walker.
//
// Per warp, in shared memory, the walker's state.  A spin-1/2 walker is held
// as signed ratio factors s_k = x_k A_k, A_k = exp(-2 x_k (W_k + h_k)) with
// W_k = sum_p J_kp x_p the Jastrow field (A = 1 without a guide): the sign is
// the spin, an edge is anti-parallel iff s_i s_j < 0, and the guide ratio of
// flipping it is |s_i s_j| times a per-edge constant, so a rate costs two
// shared loads and two multiplies and the hop loop evaluates no exp; a flip
// updates s multiplicatively (s_k *= exp(+-4 J_ak), s_a -> -1/s_a).  A
// Bose-Hubbard walker is held as uint8 occupations plus its Jastrow fields
// S_k = sum_p w_kp n_p, updated additively.  Per CTA, in shared memory: the edge list, the
// couplings and, when they fit, the guide's partner tables.
//
// A rate evaluation enumerates the off-diagonal moves (the Green's-function
// elements tau |H_x'x| psi(x')/psi(x), i.e. the rates of
// engine/evolution.py transition_rates:205-261) with each lane owning a
// contiguous chunk of C slots (C odd, so the chunk-strided shared-memory
// accesses are conflict-free): the lane sums its chunk in order, one warp
// shuffle scan combines the 32 chunk totals, and the inverse-CDF draw
// (sample_index:30-59) finds its lane by ballot and its slot by a warp scan
// of that lane's chunk, re-evaluated by C lanes at once.  The propagators follow engine/evolution.py:
// cont_time (559-721), single_step (322-406), multi_step (409-556); each
// walker consumes the JAX Threefry stream split(key, N_walkers)[w] with
// fold_in(., 2 i) / fold_in(., 2 i + 1) per hold (single_step: fold_in(., i)).
#include <cfloat>

#include "engine.cuh"
#include "bose_moves.cuh"

namespace gfmc {
namespace {

constexpr unsigned FULL = 0xffffffffu;

template <typename X>
__host__ __device__ inline X *stage_arr(const X *src, int n, unsigned char *base, size_t &off,
                                        bool copy) {
  if (src == nullptr || n <= 0) return const_cast<X *>(src);
  size_t o = (off + 15) & ~size_t(15);
  off = o + (size_t)n * sizeof(X);
#ifdef __CUDA_ARCH__
  if (copy) {
    X *dst = reinterpret_cast<X *>(base + o);
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    return dst;
  }
#endif
  return const_cast<X *>(src);
}

// A pointer into this block's dynamic shared memory rebuilt from the shared
// array, so that the compiler addresses it as shared memory.
template <typename X>
__device__ __forceinline__ const X *as_shared(const X *p, const unsigned char *smem) {
  const size_t o = __cvta_generic_to_shared(p) - __cvta_generic_to_shared(smem);
  return reinterpret_cast<const X *>(smem + o);
}

// Stages the CTA-shared tables (in a fixed order) and rewrites the pointers
// to their shared copies.  The host runs the same function with copy=false
// to size the region.
template <typename T>
__host__ __device__ inline size_t stage_tables(DevModel<T> &m, DevGuide<T> &g, int stage_nbr,
                                               unsigned char *base, bool copy) {
  size_t off = 0;
  m.edge = stage_arr(m.edge, m.E, base, off, copy);
  if (m.family == SPIN_HALF) {
    m.jpm = stage_arr(m.jpm, (m.n_jpm && !m.uniform_pm) ? m.E : 0, base, off, copy);
    m.jpmpm = stage_arr(m.jpmpm, (m.n_jpm && !m.uniform_pm) ? m.E : 0, base, off, copy);
    m.jz = stage_arr(m.jz, m.has_jz ? (m.uniform_jz ? 1 : m.E) : 0, base, off, copy);
    m.hz = stage_arr(m.hz, m.has_hz ? m.N : 0, base, off, copy);
    m.hx_half = stage_arr(m.hx_half, m.n_hx ? m.N : 0, base, off, copy);
    if (g.kind == GUIDE_JASTROW_SPIN) {
      g.h = stage_arr(g.h, g.has_h ? m.N : 0, base, off, copy);
      g.c_anti = stage_arr(g.c_anti, g.uniform_c ? 0 : m.E, base, off, copy);
      g.c_par = stage_arr(g.c_par, g.uniform_c ? 0 : m.E, base, off, copy);
    }
  } else {
    m.t = stage_arr(m.t, m.n_hop ? m.E : 0, base, off, copy);
    m.eta = stage_arr(m.eta, m.n_eta ? m.E : 0, base, off, copy);
    m.U = stage_arr(m.U, m.has_U ? m.N : 0, base, off, copy);
    m.mu = stage_arr(m.mu, m.has_mu ? m.N : 0, base, off, copy);
    m.hpm = stage_arr(m.hpm, m.n_hpm ? m.N : 0, base, off, copy);
    {
      const int nsq = (m.n_max + 1) * (m.n_max + 1) + 1;   // staged when small (n_max <= 21)
      m.sqrt_tab = stage_arr(m.sqrt_tab, nsq <= 513 ? nsq : 0, base, off, copy);
    }
    if (g.kind == GUIDE_JASTROW_BOSE) {
      g.slot_q = stage_arr(g.slot_q, m.M, base, off, copy);
      {
        const int nst = m.N * (m.n_max + 1) * 2;   // staged when small
        g.site_t = stage_arr(g.site_t, nst <= 1024 ? nst : 0, base, off, copy);
      }
      g.h = stage_arr(g.h, g.h_mode == 2 ? m.N : 0, base, off, copy);
      g.d = stage_arr(g.d, g.d_mode == 2 ? m.N : 0, base, off, copy);
    }
  }
  if (g.kind == GUIDE_JASTROW_SPIN && g.ti) {
    g.tE = stage_arr(g.tE, 8 * m.N, base, off, copy);
    g.tq = stage_arr(g.tq, m.N, base, off, copy);
  }
  if (g.kind != GUIDE_NONE && stage_nbr && !g.dense) {
    g.nbr = stage_arr(g.nbr, m.N * g.deg, base, off, copy);
    g.nbr_w = stage_arr(g.nbr_w, m.N * g.deg, base, off, copy);
    g.nbr_cnt = stage_arr(g.nbr_cnt, m.N, base, off, copy);
    if (g.kind == GUIDE_JASTROW_SPIN) {
      g.nbr_ep = stage_arr(g.nbr_ep, m.N * g.deg, base, off, copy);
      g.nbr_em = stage_arr(g.nbr_em, m.N * g.deg, base, off, copy);
    }
  }
  return (off + 15) & ~size_t(15);
}

__host__ __device__ inline int spin_words(int N) { return (N + 63) / 64; }
__host__ __device__ inline int bose_bytes(int N) { return ((N + 15) / 16) * 16; }

// Slots per lane for n_slots moves: ceil(n/32), rounded up to odd.
__host__ __device__ inline int chunk_of(int n_slots) {
  int c = (n_slots + 31) / 32;
  if (c < 1) c = 1;
  return c | 1;
}

struct WarpLayout {
  size_t fa, bytes;
};

// Per-warp shared region (configuration words or occupations, then the
// per-site state: the signed ratio factors s_k = x_k A_k of a spin-1/2 walker,
// or the Jastrow fields of a Bose-Hubbard walker), sized on the host by the
// same function.
template <typename T>
__host__ __device__ inline WarpLayout warp_layout(const DevModel<T> &m, const DevGuide<T> &g) {
  WarpLayout L;
  size_t off = (m.family == SPIN_HALF) ? (size_t)spin_words(m.N) * 8 : (size_t)bose_bytes(m.N);
  off = (off + 15) & ~size_t(15);
  L.fa = off;
  if (m.family == SPIN_HALF || g.kind != GUIDE_NONE) off += (size_t)m.N * sizeof(T);
  // Bose-Hubbard guide: the factors exp(+beta_scale F_k), exp(-beta_scale F_k)
  if (m.family != SPIN_HALF && g.kind != GUIDE_NONE) off += 2 * (size_t)m.N * sizeof(T);
  L.bytes = (off + 15) & ~size_t(15);
  return L;
}

// ---- configuration access ---------------------------------------------------
template <typename T> __device__ __forceinline__ T spin_x(const uint64_t *bits, int k) {
  return ((bits[k >> 6] >> (k & 63)) & 1ull) ? T(1) : T(-1);
}

// Basis index of a spin-1/2 walker under the exact-amplitude guide
// (ExactGroundState.basis_index, wavefunction/exact_ground_state.py:141-147,
// digits over SpinHalf.local_hilbert_space (1, -1)): bit N-1-k is set for a
// down spin at site k.  S holds the plain spins; N <= 26, one site per lane.
template <typename T>
__device__ __forceinline__ int exact_index(int N, const T *S, int lane) {
  const unsigned down = __ballot_sync(FULL, lane < N && S[lane < N ? lane : 0] < T(0));
  return (int)(__brev(down) >> (32 - N));
}

// psi(y) / psi(x) under the exact-amplitude guide, y = x with the index bits
// `flip` toggled: exp(log_amp[y] - log_amp[x]) (log_diff_from_configs:150-190).
template <typename T>
__device__ __forceinline__ T exact_ratio(const DevGuide<T> &g, int gx, int flip) {
  return math_exp(g.lamp[gx ^ flip] - g.lamp[gx]);
}

template <typename T, int FAM>
__device__ __forceinline__ T site_val(const uint64_t *bits, const uint8_t *occ, int k) {
  if (FAM == SPIN_HALF) return spin_x<T>(bits, k);
  return T(occ[k]);
}

// Off-diagonal element of Bose-Hubbard move o (<= 0), guide ratio folded in:
// BoseHubbard.get_rates:285-393, JastrowBoseHubbard.log_diff_from_operator:253-286.
template <typename T>
__device__ __forceinline__ T bose_offdiag(const DevModel<T> &m, const DevGuide<T> &g,
                                          const uint8_t *occ, const T *F, int o) {
  BoseMove mv = bose_decode(m, o);
  const T na = T(occ[mv.a]), nb = T(occ[mv.b]);
  T v = bose_element<T>(m, occ, mv);
  if (g.kind && v != T(0)) {
    // exp(out) of JastrowBoseHubbard.log_diff_from_operator as the product of
    // its factors (DevGuide::slot_q, site_t and the walker's Gs)
    const T *Gp = F + m.N, *Gm = F + 2 * m.N;
    const int np1 = m.n_max + 1;
    const int oa = occ[mv.a] < m.n_max ? occ[mv.a] : m.n_max;   // (clamped: table bounds)
    const int ob = occ[mv.b] < m.n_max ? occ[mv.b] : m.n_max;
    T f = g.slot_q[o + 1] * (mv.da > 0 ? Gp[mv.a] : Gm[mv.a]) *
          g.site_t[((size_t)mv.a * np1 + oa) * 2 + (mv.da > 0)];
    if (mv.db != 0)
      f = f * (mv.db > 0 ? Gp[mv.b] : Gm[mv.b]) *
          g.site_t[((size_t)mv.b * np1 + ob) * 2 + (mv.db > 0)];
    v *= f;
  }
  (void)na;
  (void)nb;
  return v;
}

// ---- guide state ---------------------------------------------------------------
// Field of every site from scratch into F.  Dense couplings accumulate the
// rows of J (coalesced, fixed order p = 0..N-1); sparse ones walk the
// partner lists.
template <typename T, int FAM>
__device__ __forceinline__ void field_init(const DevModel<T> &m, const DevGuide<T> &g,
                                           const uint64_t *bits, const uint8_t *occ, T *F,
                                           int lane) {
  if (g.dense) {
    for (int k = lane; k < m.N; k += 32) F[k] = T(0);
    for (int p = 0; p < m.N; ++p) {
      const T xp = site_val<T, FAM>(bits, occ, p);
      const T *row = g.Jd + (size_t)p * m.N;
      for (int k = lane; k < m.N; k += 32) F[k] += row[k] * xp;
    }
    return;
  }
  for (int k = lane; k < m.N; k += 32) {
    T s = T(0);
    const int c = g.nbr_cnt[k];
    const uint32_t *nb = g.nbr + (size_t)k * g.deg;
    const T *nw = g.nbr_w + (size_t)k * g.deg;
    for (int d = 0; d < c; ++d) s += nw[d] * site_val<T, FAM>(bits, occ, (int)nb[d]);
    F[k] = s;
  }
}

// Signed ratio factors of a spin-1/2 walker from its configuration:
// s_k = x_k A_k, A_k = exp(-2 x_k (W_k + h_k)) the exp of
// JastrowSpinHalf._site_log_diff:290-297 (A = 1 without a guide).
template <typename T>
__device__ __forceinline__ void signed_init(const DevModel<T> &m, const DevGuide<T> &g,
                                            const uint64_t *bits, T *S, int lane) {
  if (g.kind != GUIDE_JASTROW_SPIN) {   // no guide, or exact amplitudes: the spins
    for (int k = lane; k < m.N; k += 32) S[k] = spin_x<T>(bits, k);
    __syncwarp();
    return;
  }
  field_init<T, SPIN_HALF>(m, g, bits, nullptr, S, lane);
  __syncwarp();
  for (int k = lane; k < m.N; k += 32) {
    const T x = spin_x<T>(bits, k);
    S[k] = x * math_exp(T(-2) * x * (g.has_h ? S[k] + g.h[k] : S[k]));
  }
  __syncwarp();
}

// Flip of spin a (the sequential update of one flip): its partners k get
// A_k *= exp(4 x_k x_a J_ak) (x_a before the flip), then s_a -> -1 / s_a.
template <typename T>
__device__ __forceinline__ void flip_one(const DevModel<T> &m, const DevGuide<T> &g, T *S, int a,
                                         int lane) {
  const T sa = S[a];
  if (g.kind == GUIDE_JASTROW_SPIN) {
    const bool ua = sa > T(0);
    if (g.ti) {
      const int ca = g.tE_off - g.tq[a];
#pragma unroll 8
      for (int k = lane; k < m.N; k += 32) {
        const T sk = S[k];
        S[k] = sk * g.tE[g.tq[k] + ca + ((sk > T(0)) != ua)];
      }
    } else if (g.dense) {
      const T *ep = g.Ep + (size_t)a * m.N, *em = g.Em + (size_t)a * m.N;
      for (int k = lane; k < m.N; k += 32) {
        const T sk = S[k];
        S[k] = sk * (((sk > T(0)) == ua) ? ep[k] : em[k]);
      }
    } else {
      const int c = g.nbr_cnt[a];
      const uint32_t *nb = g.nbr + (size_t)a * g.deg;
      const T *ep = g.nbr_ep + (size_t)a * g.deg, *em = g.nbr_em + (size_t)a * g.deg;
      for (int d = lane; d < c; d += 32) {
        const int k = (int)nb[d];
        const T sk = S[k];
        S[k] = sk * (((sk > T(0)) == ua) ? ep[d] : em[d]);
      }
    }
    __syncwarp();
    if (lane == 0) S[a] = -math_rcp(sa);
  } else {
    if (lane == 0) S[a] = -sa;
  }
  __syncwarp();
}

// Flip of the pair (a, b): for dense couplings both rows in one pass (their
// loads overlap), with the two endpoints fixed up as the sequential flips
// a-then-b would leave them; sparse couplings flip one after the other.
template <typename T>
__device__ __forceinline__ void flip_pair(const DevModel<T> &m, const DevGuide<T> &g, T *S, int a,
                                          int b, int lane) {
  if (g.kind != GUIDE_JASTROW_SPIN || !g.dense) {
    flip_one(m, g, S, a, lane);
    flip_one(m, g, S, b, lane);
    return;
  }
  const T sa = S[a], sb = S[b];
  const bool ua = sa > T(0), ub = sb > T(0);
  if (g.ti) {
    const int qa = g.tq[a], qb = g.tq[b];
    const int ca = g.tE_off - qa, cb = g.tE_off - qb;
#pragma unroll 8
    for (int k = lane; k < m.N; k += 32) {
      const T sk = S[k];
      const bool uk = sk > T(0);
      const int qk = g.tq[k];
      const T fa = g.tE[qk + ca + (uk != ua)];
      const T fb = g.tE[qk + cb + (uk != ub)];
      S[k] = sk * fa * fb;
    }
    __syncwarp();
    if (lane == 0) {
      const T fba = g.tE[qa + cb + ((!ua) != ub)];   // row b at a, x_a after its flip
      const T fab = g.tE[qb + ca + (ub != ua)];      // row a at b, x_b before its flip
      S[a] = -math_rcp(sa) * fba;
      S[b] = -math_rcp(sb * fab);
    }
    __syncwarp();
    return;
  }
  const T *epa = g.Ep + (size_t)a * m.N, *ema = g.Em + (size_t)a * m.N;
  const T *epb = g.Ep + (size_t)b * m.N, *emb = g.Em + (size_t)b * m.N;
  for (int k = lane; k < m.N; k += 32) {
    const T sk = S[k];
    const bool uk = sk > T(0);
    const T fa = (uk == ua) ? epa[k] : ema[k];
    const T fb = (uk == ub) ? epb[k] : emb[k];
    S[k] = sk * fa * fb;
  }
  __syncwarp();
  if (lane == 0) {
    const T fba = ((!ua) == ub) ? epb[a] : emb[a];   // row b at a, x_a after its flip
    const T fab = (ub == ua) ? epa[b] : ema[b];      // row a at b, x_b before its flip
    S[a] = -math_rcp(sa) * fba;
    S[b] = -math_rcp(sb * fab);
  }
  __syncwarp();
}

// Bose-Hubbard Jastrow field update after site k changed by delta.
template <typename T>
__device__ __forceinline__ void field_update(const DevGuide<T> &g, T *F, int N, int k, T delta,
                                             int lane) {
  const int c = g.nbr_cnt[k];
  const uint32_t *nb = g.nbr + (size_t)k * g.deg;
  const T *nw = g.nbr_w + (size_t)k * g.deg;
  for (int d = lane; d < c; d += 32) {
    const int q = (int)nb[d];
    const T fq = F[q] + nw[d] * delta;
    F[q] = fq;
    F[N + q] = math_exp(g.beta_scale * fq);       // the partner's ratio factors
    F[2 * N + q] = math_exp(-g.beta_scale * fq);
  }
  __syncwarp();
}

// The Bose-Hubbard ratio factors exp(+-beta_scale F_k) of every site from F.
template <typename T>
__device__ __forceinline__ void bose_factors(const DevGuide<T> &g, T *F, int N, int lane) {
  for (int k = lane; k < N; k += 32) {
    F[N + k] = math_exp(g.beta_scale * F[k]);
    F[2 * N + k] = math_exp(-g.beta_scale * F[k]);
  }
  __syncwarp();
}

// Apply move o (off-diagonal index) to the walker's state.
template <typename T, int FAM>
__device__ __forceinline__ void apply_move(const DevModel<T> &m, const DevGuide<T> &g,
                                           uint8_t *occ, T *SF, int o, int lane) {
  if (FAM == SPIN_HALF) {
    if (o < m.n_hx) {
      flip_one(m, g, SF, o, lane);
    } else {
      const uint32_t pe = m.edge[o - m.n_hx];
      flip_pair(m, g, SF, (int)(pe & 0xFFFF), (int)(pe >> 16), lane);
    }
  } else {
    BoseMove mv = bose_decode(m, o);
    __syncwarp();
    if (lane == 0) {
      occ[mv.a] = (uint8_t)(occ[mv.a] + mv.da);
      occ[mv.b] = (uint8_t)(occ[mv.b] + mv.db);
    }
    __syncwarp();
    if (g.kind != GUIDE_NONE) {
      field_update(g, SF, m.N, mv.a, T(mv.da), lane);
      if (mv.db != 0) field_update(g, SF, m.N, mv.b, T(mv.db), lane);
    }
  }
}

// The walker's basis index when the exact-amplitude guide is on (general
// spin layout; a warp-uniform branch), else 0.
template <typename T, int FAM, int FAST>
__device__ __forceinline__ int exact_gx(const DevModel<T> &m, const DevGuide<T> &g, const T *SF,
                                        int lane) {
  if (FAST || FAM != SPIN_HALF || g.kind != GUIDE_EXACT_SPIN) return 0;
  return exact_index(m.N, SF, lane);
}

// Off-diagonal element of move o (<= 0 for a sign-free model) with the
// guide ratio folded in (evolution.transition_rates:255-260).  Spin-1/2: a
// site flip costs -h_x/2 A_k = hx_half |s_k|; an edge flip the coupling of
// its spin alignment times A_i A_j c_e = |s_i s_j| c_e (c_e = exp(4 Jsum_e
// x_i x_j), the pair's own term).  *anti: the edge's spins are anti-parallel.
// Under the exact-amplitude guide (general layout only) the ratio is
// exact_ratio at the walker's basis index gx; zero elements stay zero
// without looking the ratio up (transition_rates:252-260).
template <typename T, int FAM, int FAST>
__device__ __forceinline__ T offdiag(const DevModel<T> &m, const DevGuide<T> &g,
                                     const uint8_t *occ, const T *SF, int o, int *anti_out,
                                     int gx) {
  if (FAM == SPIN_HALF) {
    if (!FAST && o < m.n_hx) {
      const T v = m.hx_half[o];
      if (v != T(0) && g.kind == GUIDE_EXACT_SPIN) return v * exact_ratio(g, gx, 1 << (m.N - 1 - o));
      return v != T(0) ? v * fabs(SF[o]) : v;
    }
    const int e = FAST ? o : o - m.n_hx;
    const uint32_t pe = m.edge[e];
    const T p = SF[pe & 0xFFFF] * SF[pe >> 16];
    const bool anti = p < T(0);
    *anti_out = anti;
    // (k_anti (-p) and k_par p as one product: negation and the order of a
    // product's factors do not change its rounding; with k_par = 0 the
    // parallel edges' +0 comes from min(p, 0) instead of a select)
    if (FAST == 1) return (-m.k_anti) * math_min(p, T(0));
    if (FAST == 2) return (anti ? -m.k_anti : m.k_par) * p;
    const T b = m.uniform_pm ? (anti ? m.jpm0 : m.jpmpm0) : (anti ? m.jpm[e] : m.jpmpm[e]);
    if (g.kind == GUIDE_EXACT_SPIN) {
      if (b == T(0)) return b;
      const int i = (int)(pe & 0xFFFF), j = (int)(pe >> 16);
      return b * exact_ratio(g, gx, (1 << (m.N - 1 - i)) ^ (1 << (m.N - 1 - j)));
    }
    if (g.kind != GUIDE_NONE && b != T(0)) {
      const T c = g.uniform_c ? (anti ? g.c_anti0 : g.c_par0) : (anti ? g.c_anti[e] : g.c_par[e]);
      return b * fabs(p) * c;
    }
    return b;
  }
  return bose_offdiag<T>(m, g, occ, SF, o);
}

// Result of one rate evaluation, per lane.
template <typename T> struct Eval {
  T diag;    // H_xx (warp-uniform)
  T excl;    // scanned total of the lanes before this one
  T end;     // excl + this lane's chunk total
  T total;   // scanned total of all slots (warp-uniform)
  int C;     // slots per lane
};

// Slot layouts of a rate evaluation:
//  MODE_OFF (cont_time, multi_step): the off-diagonal moves, scanned values
//    their weights -rates, cdf = cumsum(weights);
//  MODE_LAM (single_step): slot 0 the diagonal, scanned values the rates,
//    cdf = lam - cumsum(rates), weights (lam - H_xx, -rates);
//  MODE_POS (applying a measurement operator, apply_operator_one:849-888):
//    slot 0 the diagonal, scanned values and weights the (non-negative)
//    rates, cdf = cumsum(rates).
enum SlotMode { MODE_OFF = 0, MODE_LAM = 1, MODE_POS = 2 };

// One rate evaluation in slot layout `mode`.
template <typename T, int FAM, int FAST>
__device__ __forceinline__ Eval<T> evaluate(const DevModel<T> &m, const DevGuide<T> &g,
                                            const uint8_t *occ, const T *SF, int n_slots,
                                            int mode, int lane) {
  const bool lamform = mode != MODE_OFF;   // slot 0 is the diagonal
  Eval<T> ev;
  const int C = chunk_of(n_slots);
  ev.C = C;
  const bool spin = FAM == SPIN_HALF;
  const bool fused_diag = spin && m.has_jz && m.n_jpm == m.E && m.E > 0;
  const int gx = exact_gx<T, FAM, FAST>(m, g, SF, lane);
  int na = 0;
  T jzs = T(0);
  T acc = T(0);
  const int s0 = lane * C;
  int jmax = n_slots - s0;
  jmax = jmax < 0 ? 0 : (jmax > C ? C : jmax);
#pragma unroll 8
  for (int j = 0; j < jmax; ++j) {
    const int o = lamform ? s0 + j - 1 : s0 + j;
    if (!lamform || o >= 0) {
      int anti = -1;
      const T v = offdiag<T, FAM, FAST>(m, g, occ, SF, o, &anti, gx);
      if (fused_diag && anti >= 0) {
        if (FAST || m.uniform_jz) na += anti;
        else jzs += anti ? -m.jz[o - m.n_hx] / T(4) : m.jz[o - m.n_hx] / T(4);
      }
      acc += lamform ? v : -v;
    }
  }
  // diagonal element: SpinHalf.diagonal_weight:291-314, BoseHubbard:271-281
  T d = T(0);
  if (spin) {
    if (!FAST && m.has_jz && !fused_diag) {
      for (int e = lane; e < m.E; e += 32) {
        const uint32_t pe = m.edge[e];
        const bool anti = SF[pe & 0xFFFF] * SF[pe >> 16] < T(0);
        if (m.uniform_jz) na += anti;
        else jzs += anti ? -m.jz[e] / T(4) : m.jz[e] / T(4);
      }
    }
    if (m.has_jz) {
      if (FAST || m.uniform_jz) d = (m.jz[0] / T(4)) * T(m.E - 2 * warp_sum(na));
      else d = warp_sum(jzs);
    }
    if (!FAST && m.has_hz) {
      T hzs = T(0);
      for (int k = lane; k < m.N; k += 32) hzs += m.hz[k] * (SF[k] > T(0) ? T(1) : T(-1));
      d = d + warp_sum(hzs) / T(2);
    }
  } else {
    T su = T(0), sm = T(0);
    for (int k = lane; k < m.N; k += 32) {
      const T n = T(occ[k]);
      if (m.has_U) su += m.U[k] * n * (n - T(1));
      if (m.has_mu) sm += m.mu[k] * n;
    }
    if (m.has_U) d = d + T(0.5) * warp_sum(su);
    if (m.has_mu) d = d - warp_sum(sm);
  }
  ev.diag = d;
  if (lamform && lane == 0) acc = d + acc;   // slot 0 carries the diagonal
  const T inc = warp_inclusive_scan(acc, lane);
  T excl = __shfl_up_sync(FULL, inc, 1);
  if (lane == 0) excl = T(0);
  ev.excl = excl;
  ev.end = excl + acc;
  const int last_lane = n_slots > 0 ? (n_slots - 1) / C : 0;
  ev.total = __shfl_sync(FULL, ev.end, last_lane);
  return ev;
}

// Scanned value and weight of slot s (valid slots only).
template <typename T, int FAM, int FAST>
__device__ __forceinline__ T slot_q(const DevModel<T> &m, const DevGuide<T> &g, const uint8_t *occ,
                                    const T *SF, int s, int mode, T diag, int gx) {
  const bool lamform = mode != MODE_OFF;
  if (lamform && s == 0) return diag;
  int anti;
  const T v = offdiag<T, FAM, FAST>(m, g, occ, SF, lamform ? s - 1 : s, &anti, gx);
  return lamform ? v : -v;
}

// Weight of slot s with scanned value q.
template <typename T>
__device__ __forceinline__ T slot_w(int mode, int s, T q, T lam) {
  if (mode == MODE_LAM) return s == 0 ? (-q + lam) : -q;
  return q;
}

// evolution.sample_index: the first slot whose cdf exceeds u, stepped back to
// the nearest slot at or before it with positive weight.  The lane whose
// chunk holds the crossing is found by ballot; its chunk is re-evaluated by
// C lanes at once and scanned.  The step-back past that chunk (a zero-weight
// crossing with no positive slot before it in the chunk) re-evaluates the
// earlier chunks the same way.
template <typename T, int FAM, int FAST>
__device__ __forceinline__ int sample_slot(const DevModel<T> &m, const DevGuide<T> &g,
                                           const uint8_t *occ, const T *SF, const Eval<T> &ev,
                                           int n_slots, int mode, T lam, T u, int lane) {
  const int C = ev.C;
  const int last_lane = (n_slots - 1) / C;
  const bool lamc = mode == MODE_LAM;   // cdf = lam - cumsum
  const int gx = exact_gx<T, FAM, FAST>(m, g, SF, lane);
  const T cend = lamc ? lam - ev.end : ev.end;
  const unsigned bal = __ballot_sync(FULL, lane <= last_lane && cend > u);
  const int L = bal ? __ffs(bal) - 1 : last_lane;
  const T exclL = __shfl_sync(FULL, ev.excl, L);
  int s = L * C + lane;
  bool valid = lane < C && s < n_slots;
  T qv = valid ? slot_q<T, FAM, FAST>(m, g, occ, SF, s, mode, ev.diag, gx) : T(0);
  const T pre = warp_inclusive_scan(qv, lane);
  const T c = lamc ? lam - (exclL + pre) : exclL + pre;
  const unsigned hit = __ballot_sync(FULL, valid && c > u);
  const int nvalid = (n_slots - L * C) < C ? (n_slots - L * C) : C;
  const int jh = hit ? __ffs(hit) - 1 : nvalid - 1;
  T w = slot_w(mode, s, qv, lam);
  unsigned bk = __ballot_sync(FULL, valid && lane <= jh && w > T(0));
  if (bk) return L * C + 31 - __clz(bk);
  for (int L2 = L - 1; L2 >= 0; --L2) {
    s = L2 * C + lane;
    valid = lane < C && s < n_slots;
    qv = valid ? slot_q<T, FAM, FAST>(m, g, occ, SF, s, mode, ev.diag, gx) : T(0);
    w = slot_w(mode, s, qv, lam);
    bk = __ballot_sync(FULL, valid && w > T(0));
    if (bk) return L2 * C + 31 - __clz(bk);
  }
  return L * C + jh;
}

// 256 threads and 4 blocks per SM: 64 registers, 32 resident warps per SM
// (a warp's shared state is ~2 KB, so registers bound the occupancy).
// KIND selects the instantiation: 0 cont_time and EVALUATE, 1 the discrete
// propagators single_step and multi_step, 2 the measurement-operator modes
// APPLY and MIN_RATE (kept apart so that the code of one does not weigh on
// another's register allocation).
// (The Bose-Hubbard instantiations too: at 4 blocks they spill a little but
// ran 34 % faster on the 64-site ring than at 2 blocks and 128 registers.)
template <typename T, int FAM, int FAST, int KIND>
__global__ void __launch_bounds__(256, 4)
evolve_kernel(DevModel<T> m, DevGuide<T> g, EvolveArgs a, int stage_nbr, int cta_bytes) {
  extern __shared__ __align__(16) unsigned char smem[];
  stage_tables(m, g, stage_nbr, smem, true);
  // the tables every staging copies, as pointers derived from the shared
  // array itself (shared-memory loads, 32-bit addresses); absent tables stay
  // unused
  m.edge = as_shared(m.edge, smem);
  g.tE = as_shared(g.tE, smem);
  g.tq = as_shared(g.tq, smem);
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const WarpLayout WL = warp_layout(m, g);
  unsigned char *wb = smem + cta_bytes + (size_t)wib * WL.bytes;
  uint64_t *bits = reinterpret_cast<uint64_t *>(wb);
  uint8_t *occ = wb;
  T *SF = reinterpret_cast<T *>(wb + WL.fa);

  const int NW = spin_words(m.N);
  const int CB = bose_bytes(m.N);
  const int method = a.method;
  const bool guided = g.kind != GUIDE_NONE;
  const T lam = T(a.lam);
  double wmax = -DBL_MAX;
  unsigned long long hop_acc = 0;

  for (;;) {
    int walker = 0;
    if (lane == 0) walker = atomicAdd(a.work_ctr, 1);
    walker = __shfl_sync(FULL, walker, 0);
    if (walker >= a.n_walkers) break;

    // ---- load (fused gather through the previous step's parent map)
    const int src = a.parents ? a.parents[walker] : walker;
    if (guided && a.field_in) {
      const T *fin = reinterpret_cast<const T *>(a.field_in) + (size_t)src * m.N;
      for (int k = lane; k < m.N; k += 32) SF[k] = fin[k];
      if (FAM != SPIN_HALF) {
        const uint32_t *in = reinterpret_cast<const uint32_t *>(
            reinterpret_cast<const uint8_t *>(a.cfg_in) + (size_t)src * CB);
        uint32_t *o32 = reinterpret_cast<uint32_t *>(occ);
        for (int k = lane; k < CB / 4; k += 32) o32[k] = in[k];
      }
      __syncwarp();
    } else if (FAM == SPIN_HALF) {
      const uint64_t *in = reinterpret_cast<const uint64_t *>(a.cfg_in) + (size_t)src * NW;
      for (int k = lane; k < NW; k += 32) bits[k] = in[k];
      __syncwarp();
      signed_init<T>(m, g, bits, SF, lane);
    } else {
      const uint32_t *in = reinterpret_cast<const uint32_t *>(
          reinterpret_cast<const uint8_t *>(a.cfg_in) + (size_t)src * CB);
      uint32_t *o32 = reinterpret_cast<uint32_t *>(occ);
      for (int k = lane; k < CB / 4; k += 32) o32[k] = in[k];
      __syncwarp();
      if (guided) {
        field_init<T, FAM>(m, g, bits, occ, SF, lane);
        __syncwarp();
      }
    }
    if (FAM != SPIN_HALF && guided) bose_factors(g, SF, m.N, lane);

    const Key kw = fold(a.key, (uint32_t)(a.walker_offset + walker));
    double lw = a.lw_in ? a.lw_in[src] : 0.0;
    T eloc = T(0);
    int hops = 0;
    T draws = T(0);   // draws of 16 holds (cont/multi) or uniforms of 32 sub-steps (single)

    if (KIND == 0 && method == CONT_TIME) {
      const T beta = T(a.step);
      T t = T(0);
      uint32_t it = 0;
      // the previous step's evaluation of this configuration, when carried
      const T *rec = a.eval_in ? reinterpret_cast<const T *>(a.eval_in) + (size_t)src * EVAL_REC
                               : nullptr;
      bool carried = rec != nullptr && rec[66] != T(0);
      while (t < beta) {
        Eval<T> ev;
        if (carried) {
          ev.excl = rec[lane];
          ev.end = rec[32 + lane];
          ev.diag = rec[64];
          ev.total = rec[65];
          ev.C = chunk_of(m.n_off);
          carried = false;
        } else {
          ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.n_off, MODE_OFF, lane);
        }
        const T R = ev.total;
        const T eL = ev.diag - R;
        if ((it & 15u) == 0) {
          // even lanes keep the move uniform, odd lanes turn the hold uniform
          // psi into the exponential variate -log1p(-psi) for its hold
          const T d = uniform<T>(fold(kw, 2u * it + (uint32_t)lane));
          const T ex = -math_log1p(-d);
          draws = (lane & 1) ? ex : d;
        }
        const T U1 = __shfl_sync(FULL, draws, (int)(2u * (it & 15u)));
        const T ex = __shfl_sync(FULL, draws, (int)(2u * (it & 15u) + 1u));
        int si = 0;
        if (R > T(0)) {
          const T u = U1 * R, cap = next_below(R);
          si = sample_slot<T, FAM, FAST>(m, g, occ, SF, ev, m.n_off, MODE_OFF, lam,
                                         u < cap ? u : cap, lane);
        }
        const T tau_raw = (R > T(0)) ? ex / R : pos_inf<T>();
        const T rem = beta - t;
        const T tau = tau_raw < rem ? tau_raw : rem;
        lw = lw - (double)eL * (double)tau;
        t = t + tau;
        if (tau_raw < rem) {
          apply_move<T, FAM>(m, g, occ, SF, si, lane);
          ++hops;
        } else if (a.eval_out) {
          // the final configuration's evaluation, for the next step
          T *out = reinterpret_cast<T *>(a.eval_out) + (size_t)walker * EVAL_REC;
          out[lane] = ev.excl;
          out[32 + lane] = ev.end;
          if (lane == 0) {
            out[64] = ev.diag;
            out[65] = ev.total;
            out[66] = T(1);
          }
        }
        eloc = eL;
        if (++it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          if (a.eval_out && lane == 0)   // (the configuration moved after ev)
            reinterpret_cast<T *>(a.eval_out)[(size_t)walker * EVAL_REC + 66] = T(0);
          break;
        }
      }
      lw -= a.alw * a.step;
    } else if (KIND == 1 && method == SINGLE_STEP) {
      const int n_bra = (int)a.step;
      for (int sidx = 0; sidx < n_bra; ++sidx) {
        const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.M, MODE_LAM, lane);
        const T bx = lam - ev.total;
        if ((sidx & 31) == 0) draws = uniform<T>(fold(kw, (uint32_t)(sidx + lane)));
        const T U = __shfl_sync(FULL, draws, sidx & 31);
        const T u = U * bx, cap = next_below(bx);
        const int idx = sample_slot<T, FAM, FAST>(m, g, occ, SF, ev, m.M, MODE_LAM, lam,
                                                  u < cap ? u : cap, lane);
        if (idx != 0) {
          apply_move<T, FAM>(m, g, occ, SF, idx - 1, lane);
          ++hops;
        }
        lw = lw + (double)math_log(bx);
      }
      const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.n_off, MODE_OFF, lane);
      eloc = ev.diag - ev.total;
      lw -= a.alw * (double)n_bra;
    } else if (KIND == 1 && method == MULTI_STEP) {
      const int n_bra = (int)a.step;
      int used = 0;
      uint32_t it = 0;
      while (used < n_bra) {
        const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.n_off, MODE_OFF, lane);
        const T R = ev.total;
        const T bx = lam - ev.diag + R;
        if ((it & 15u) == 0) {
          // odd lanes hold log1p(-psi) of their hold uniform
          const T d = uniform<T>(fold(kw, 2u * it + (uint32_t)lane));
          const T lp = math_log1p(-d);
          draws = (lane & 1) ? lp : d;
        }
        const T U1 = __shfl_sync(FULL, draws, (int)(2u * (it & 15u)));
        const T lpsi = __shfl_sync(FULL, draws, (int)(2u * (it & 15u) + 1u));
        int si = 0;
        if (R > T(0)) {
          const T u = U1 * R, cap = next_below(R);
          si = sample_slot<T, FAM, FAST>(m, g, occ, SF, ev, m.n_off, MODE_OFF, lam,
                                         u < cap ? u : cap, lane);
        }
        const int remaining = n_bra - used;
        const T hp = R / bx;
        const bool can_hop = hp > T(0);
        const T log_pd = can_hop ? math_log1p(-hp) : T(-1);
        const T hold = floor(lpsi / log_pd) + T(1);
        const T capk = T(remaining + 1);
        const T hm = hold < capk ? hold : capk;
        const int k_raw = can_hop ? (int)hm : remaining + 1;
        const int k = k_raw < remaining ? k_raw : remaining;
        lw = lw + (double)math_log(bx) * (double)k;
        used += k;
        if (k_raw <= remaining) {
          apply_move<T, FAM>(m, g, occ, SF, si, lane);
          ++hops;
        }
        if (++it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.n_off, MODE_OFF, lane);
      eloc = ev.diag - ev.total;
      lw -= a.alw * (double)n_bra;
    } else if (KIND == 2 && method == APPLY) {
      // apply_operator_one:849-888: draw the successor in proportion to the
      // operator's guided rates (slot 0 the diagonal, i.e. stay); the value
      // is their sum, 0 when it is not positive; a purely diagonal operator
      // keeps the configuration and returns its diagonal element
      if (m.M == 1) {
        const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, 0, MODE_OFF, lane);
        eloc = ev.diag;
      } else {
        const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.M, MODE_POS, lane);
        const T total = ev.total;
        if (total <= T(0)) {
          eloc = T(0);
        } else {
          const T U = uniform<T>(kw);
          const T u = U * total, cap = next_below(total);
          const int idx = sample_slot<T, FAM, FAST>(m, g, occ, SF, ev, m.M, MODE_POS, lam,
                                                    u < cap ? u : cap, lane);
          if (idx != 0) apply_move<T, FAM>(m, g, occ, SF, idx - 1, lane);
          eloc = total;
        }
      }
    } else if (KIND == 2 && method == MIN_RATE) {
      // check_off_diag_operator_positivity (engine/estimators.py:631-681):
      // the smallest guide-transformed rate over all M_total slots, NaN when
      // one is not finite (the full evaluation gives the diagonal element)
      const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.M, MODE_POS, lane);
      T mn = ev.diag;
      bool bad = !isfinite(ev.diag);
      const int gx = exact_gx<T, FAM, FAST>(m, g, SF, lane);
      for (int o = lane; o < m.n_off; o += 32) {
        int anti;
        const T v = offdiag<T, FAM, FAST>(m, g, occ, SF, o, &anti, gx);
        mn = v < mn ? v : mn;
        bad = bad || !isfinite(v);
      }
      mn = -warp_max(-mn);
      eloc = __any_sync(FULL, bad) ? T(NAN) : mn;
    } else {  // EVALUATE: local energy of the loaded configuration
      const Eval<T> ev = evaluate<T, FAM, FAST>(m, g, occ, SF, m.n_off, MODE_OFF, lane);
      eloc = ev.diag - ev.total;
      if (a.diag_out && lane == 0) a.diag_out[walker] = (double)ev.diag;
    }

    // ---- store
    if (a.cfg_out) {
      if (FAM == SPIN_HALF) {
        uint64_t *out = reinterpret_cast<uint64_t *>(a.cfg_out) + (size_t)walker * NW;
        for (int w = 0; w < NW; ++w) {
          const int k0 = 64 * w + lane, k1 = k0 + 32;
          const unsigned lo = __ballot_sync(FULL, k0 < m.N && SF[k0 < m.N ? k0 : 0] > T(0));
          const unsigned hi = __ballot_sync(FULL, k1 < m.N && SF[k1 < m.N ? k1 : 0] > T(0));
          if (lane == 0) out[w] = (uint64_t)lo | ((uint64_t)hi << 32);
        }
      } else {
        uint32_t *out = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(a.cfg_out) +
                                                     (size_t)walker * CB);
        const uint32_t *o32 = reinterpret_cast<const uint32_t *>(occ);
        for (int k = lane; k < CB / 4; k += 32) out[k] = o32[k];
      }
    }
    if (guided && a.field_out) {
      T *fout = reinterpret_cast<T *>(a.field_out) + (size_t)walker * m.N;
      for (int k = lane; k < m.N; k += 32) fout[k] = SF[k];
    }
    if (lane == 0) {
      if (method <= MULTI_STEP) a.log_w[walker] = lw;
      a.e_loc[walker] = (double)eloc;
    }
    if (method <= MULTI_STEP) wmax = lw > wmax ? lw : wmax;
    hop_acc += (unsigned long long)hops;
    __syncwarp();
  }

  // ---- per-warp max of log_w and hop count (no block barrier: warps that
  //      run out of walkers leave at once)
  if (lane == 0) {
    if (a.partial_max) a.partial_max[(size_t)blockIdx.x * (blockDim.x >> 5) + wib] = wmax;
    if (a.hops && hop_acc) atomicAdd(a.hops, hop_acc);
  }
}

template <typename T>
void staging_plan(const DevModel<T> &m, const DevGuide<T> &g, int *stage_nbr, size_t *cta) {
  const bool jastrow = g.kind == GUIDE_JASTROW_SPIN || g.kind == GUIDE_JASTROW_BOSE;
  size_t nbr_bytes =
      jastrow ? (size_t)m.N * g.deg * (sizeof(uint32_t) + 3 * sizeof(T)) + m.N * 4 : 0;
  // (translation-invariant dense tables are staged by stage_tables itself)
  *stage_nbr = jastrow && !g.dense && nbr_bytes <= 48 * 1024;
  DevModel<T> mm = m;
  DevGuide<T> gg = g;
  *cta = stage_tables(mm, gg, *stage_nbr, nullptr, false);
}

template <typename T>
using KernelFn = void (*)(DevModel<T>, DevGuide<T>, EvolveArgs, int, int);

// Instantiation of a method (the KIND parameter of evolve_kernel).
inline int kind_of(int method) {
  return (method == CONT_TIME || method == EVALUATE) ? 0 : (method <= MULTI_STEP ? 1 : 2);
}

template <typename T, int KIND> KernelFn<T> pick_kind(const DevModel<T> &m) {
  if (m.family == SPIN_HALF) {
    if constexpr (sizeof(T) == 4) {   // (float64 builds use fast = 2 only)
      if (m.fast == 1) return evolve_kernel<T, SPIN_HALF, 1, KIND>;
    }
    if (m.fast == 2) return evolve_kernel<T, SPIN_HALF, 2, KIND>;
    return evolve_kernel<T, SPIN_HALF, 0, KIND>;
  }
  return evolve_kernel<T, BOSE_HUBBARD, 0, KIND>;
}

template <typename T> KernelFn<T> pick_kernel(const DevModel<T> &m, int kind) {
  return kind == 0 ? pick_kind<T, 0>(m) : (kind == 1 ? pick_kind<T, 1>(m) : pick_kind<T, 2>(m));
}

}  // namespace

template <typename T>
cudaError_t plan_evolve(const DevModel<T> &m, const DevGuide<T> &g, int n_slots_max,
                        LaunchPlan *plan) {
  (void)n_slots_max;
  int dev = 0, sms = 0, max_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int stage_nbr;
  size_t cta;
  staging_plan(m, g, &stage_nbr, &cta);
  const size_t warp_bytes = warp_layout(m, g).bytes;
  KernelFn<T> kern = pick_kernel(m, 0);
  cudaError_t err = cudaSuccess;
  for (int kind = 0; kind < 3; ++kind) {
    err = cudaFuncSetAttribute(pick_kernel(m, kind), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               max_smem);
    if (err != cudaSuccess) return err;
  }
  // the warps-per-block choice with the most resident warps per SM
  int best_w = 0, best = -1;
  for (int wpb = 8; wpb >= 1; wpb >>= 1) {
    size_t smem = cta + wpb * warp_bytes;
    if (smem > (size_t)max_smem) continue;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpb * 32, smem);
    if (err != cudaSuccess) return err;
    if (per_sm * wpb > best) { best = per_sm * wpb; best_w = wpb; }
  }
  if (best <= 0) return cudaErrorInvalidConfiguration;
  plan->wpb = best_w;
  plan->block = best_w * 32;
  plan->smem = cta + best_w * warp_bytes;
  plan->grid = sms * (best / best_w);
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_evolve(const DevModel<T> &m, const DevGuide<T> &g, const LaunchPlan &plan,
                          const EvolveArgs &a, cudaStream_t s) {
  int stage_nbr;
  size_t cta;
  staging_plan(m, g, &stage_nbr, &cta);
  int grid = plan.grid;
  int need = (a.n_walkers + plan.wpb - 1) / plan.wpb;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  pick_kernel(m, kind_of(a.method))<<<grid, plan.block, plan.smem, s>>>(m, g, a, stage_nbr,
                                                                         (int)cta);
  return cudaGetLastError();
}

int evolve_partials(const LaunchPlan &plan, int n_walkers) {
  int grid = plan.grid;
  int need = (n_walkers + plan.wpb - 1) / plan.wpb;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  return grid * plan.wpb;
}

template cudaError_t plan_evolve<double>(const DevModel<double> &, const DevGuide<double> &, int,
                                         LaunchPlan *);
template cudaError_t plan_evolve<float>(const DevModel<float> &, const DevGuide<float> &, int,
                                        LaunchPlan *);
template cudaError_t launch_evolve<double>(const DevModel<double> &, const DevGuide<double> &,
                                           const LaunchPlan &, const EvolveArgs &, cudaStream_t);
template cudaError_t launch_evolve<float>(const DevModel<float> &, const DevGuide<float> &,
                                          const LaunchPlan &, const EvolveArgs &, cudaStream_t);

}  // namespace gfmc

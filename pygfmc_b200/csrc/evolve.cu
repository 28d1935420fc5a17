// The per-walker propagation step of GFMC on B200: one warp per walker.
//
// Per warp, in shared memory: the walker configuration (bit-packed spins or
// uint8 occupations), the guide's local fields (W_k = sum_p J_kp x_p for the
// spin-1/2 Jastrow, S_k = sum_p w_kp n_p for the Bose-Hubbard Jastrow,
// updated incrementally after every move), and the scanned transition
// weights of the current configuration.  Per CTA, in shared memory: the edge
// list, the couplings and, when they fit, the guide's partner tables.
//
// Each rate evaluation enumerates the off-diagonal moves in rows of 32 slots
// (one slot per lane), computes the guide-transformed Green's-function
// elements tau |H_x'x| psi(x')/psi(x) (here: the rates of
// engine/evolution.py transition_rates:205-261), scans them with warp
// shuffles and draws the move by inverse CDF (sample_index:30-59).  The
// propagators follow engine/evolution.py: cont_time (559-721), single_step
// (322-406), multi_step (409-556); each walker consumes the JAX Threefry
// stream split(key, N_walkers)[w] with fold_in(., 2 i) / fold_in(., 2 i + 1)
// per hold (single_step: fold_in(., i) per sub-step).
#include <cfloat>

#include "engine.cuh"

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

// Stages the CTA-shared tables (in a fixed order) and rewrites the pointers
// to their shared copies.  The host runs the same function with copy=false
// to size the region.
template <typename T>
__host__ __device__ inline size_t stage_tables(DevModel<T> &m, DevGuide<T> &g, int stage_nbr,
                                               unsigned char *base, bool copy) {
  size_t off = 0;
  m.edge = stage_arr(m.edge, m.E, base, off, copy);
  if (m.family == SPIN_HALF) {
    m.jpm = stage_arr(m.jpm, m.n_jpm ? m.E : 0, base, off, copy);
    m.jpmpm = stage_arr(m.jpmpm, m.n_jpm ? m.E : 0, base, off, copy);
    m.jz = stage_arr(m.jz, m.has_jz ? (m.uniform_jz ? 1 : m.E) : 0, base, off, copy);
    m.hz = stage_arr(m.hz, m.has_hz ? m.N : 0, base, off, copy);
    m.hx_half = stage_arr(m.hx_half, m.n_hx ? m.N : 0, base, off, copy);
    if (g.kind == GUIDE_JASTROW_SPIN) {
      g.h = stage_arr(g.h, m.N, base, off, copy);
      g.edge_jsum = stage_arr(g.edge_jsum, m.E, base, off, copy);
    }
  } else {
    m.t = stage_arr(m.t, m.n_hop ? m.E : 0, base, off, copy);
    m.eta = stage_arr(m.eta, m.n_eta ? m.E : 0, base, off, copy);
    m.U = stage_arr(m.U, m.has_U ? m.N : 0, base, off, copy);
    m.mu = stage_arr(m.mu, m.has_mu ? m.N : 0, base, off, copy);
    m.hpm = stage_arr(m.hpm, m.n_hpm ? m.N : 0, base, off, copy);
    if (g.kind == GUIDE_JASTROW_BOSE) {
      g.trans_pw = stage_arr(g.trans_pw, m.M, base, off, copy);
      g.h = stage_arr(g.h, g.h_mode == 2 ? m.N : 0, base, off, copy);
      g.d = stage_arr(g.d, g.d_mode == 2 ? m.N : 0, base, off, copy);
    }
  }
  if (g.kind != GUIDE_NONE && stage_nbr) {
    g.nbr = stage_arr(g.nbr, m.N * g.deg, base, off, copy);
    g.nbr_w = stage_arr(g.nbr_w, m.N * g.deg, base, off, copy);
    g.nbr_cnt = stage_arr(g.nbr_cnt, m.N, base, off, copy);
  }
  return (off + 15) & ~size_t(15);
}

__host__ __device__ inline int spin_words(int N) { return (N + 63) / 64; }
__host__ __device__ inline int bose_bytes(int N) { return ((N + 15) / 16) * 16; }

// Per-warp shared region, sized on the host by the same function.
template <typename T>
__host__ __device__ inline size_t warp_region(const DevModel<T> &m, const DevGuide<T> &g,
                                              int n_slots_max, size_t *o_field, size_t *o_q,
                                              size_t *o_rowend) {
  size_t off = (m.family == SPIN_HALF) ? (size_t)spin_words(m.N) * 8 : (size_t)bose_bytes(m.N);
  off = (off + 15) & ~size_t(15);
  *o_field = off;
  if (g.kind != GUIDE_NONE) off += (size_t)m.N * sizeof(T);
  off = (off + 15) & ~size_t(15);
  *o_q = off;
  int rows = (n_slots_max + 31) / 32;
  off += (size_t)rows * 32 * sizeof(T);
  *o_rowend = off;
  off += (size_t)rows * sizeof(T);
  return (off + 15) & ~size_t(15);
}

// ---- configuration access ---------------------------------------------------
template <typename T> __device__ __forceinline__ T spin_x(const uint64_t *bits, int k) {
  return ((bits[k >> 6] >> (k & 63)) & 1ull) ? T(1) : T(-1);
}

template <typename T, int FAM>
__device__ __forceinline__ T site_val(const uint64_t *bits, const uint8_t *occ, int k) {
  if (FAM == SPIN_HALF) return spin_x<T>(bits, k);
  return T(occ[k]);
}

// ---- diagonal element -------------------------------------------------------
// SpinHalf.diagonal_weight:291-314, BoseHubbard.diagonal_weight:271-281.
template <typename T, int FAM>
__device__ __forceinline__ T diag_elem(const DevModel<T> &m, const uint64_t *bits,
                                       const uint8_t *occ, int lane) {
  if (FAM == SPIN_HALF) {
    int na = 0;
    T jzs = T(0), hzs = T(0);
    if (m.has_jz) {
      for (int e = lane; e < m.E; e += 32) {
        uint32_t pe = m.edge[e];
        int i = pe & 0xFFFF, j = pe >> 16;
        bool anti = (((bits[i >> 6] >> (i & 63)) ^ (bits[j >> 6] >> (j & 63))) & 1ull) != 0;
        if (m.uniform_jz) na += anti;
        else jzs += anti ? -m.jz[e] / T(4) : m.jz[e] / T(4);
      }
    }
    if (m.has_hz)
      for (int k = lane; k < m.N; k += 32) hzs += m.hz[k] * spin_x<T>(bits, k);
    T d = T(0);
    if (m.has_jz) {
      if (m.uniform_jz) {
        na = warp_sum(na);
        d = (m.jz[0] / T(4)) * T(m.E - 2 * na);
      } else {
        d = warp_sum(jzs);
      }
    }
    if (m.has_hz) d = d + warp_sum(hzs) / T(2);
    return d;
  } else {
    T su = T(0), sm = T(0);
    for (int k = lane; k < m.N; k += 32) {
      T n = T(occ[k]);
      if (m.has_U) su += m.U[k] * n * (n - T(1));
      if (m.has_mu) sm += m.mu[k] * n;
    }
    T d = T(0);
    if (m.has_U) d = d + T(0.5) * warp_sum(su);
    if (m.has_mu) d = d - warp_sum(sm);
    return d;
  }
}

// ---- Bose-Hubbard transition layout (bose_hubbard.py module docstring;
//      _common.two_site_move:34-72) -------------------------------------------
struct BoseMove {
  int a, b, da, db, blk, idx;  // blk: 0 hop fwd, 1 hop bwd, 2 pair up, 3 pair dn, 4 b+, 5 b
};

template <typename T>
__device__ __forceinline__ BoseMove bose_decode(const DevModel<T> &m, int o) {
  BoseMove mv;
  int E = m.E;
  if (m.n_hop) {
    if (o < 2 * E) {
      int e = o < E ? o : o - E;
      uint32_t pe = m.edge[e];
      mv.a = pe & 0xFFFF; mv.b = pe >> 16; mv.idx = e;
      if (o < E) { mv.da = -1; mv.db = +1; mv.blk = 0; }
      else { mv.da = +1; mv.db = -1; mv.blk = 1; }
      return mv;
    }
    o -= 2 * E;
  }
  if (m.n_eta) {
    if (o < 2 * E) {
      int e = o < E ? o : o - E;
      uint32_t pe = m.edge[e];
      mv.a = pe & 0xFFFF; mv.b = pe >> 16; mv.idx = e;
      if (o < E) { mv.da = +1; mv.db = +1; mv.blk = 2; }
      else { mv.da = -1; mv.db = -1; mv.blk = 3; }
      return mv;
    }
    o -= 2 * E;
  }
  int k = o < m.N ? o : o - m.N;
  mv.a = mv.b = k; mv.idx = k; mv.db = 0;
  if (o < m.N) { mv.da = +1; mv.blk = 4; } else { mv.da = -1; mv.blk = 5; }
  return mv;
}

// The off-diagonal matrix element of move o (<= 0 for a sign-free model),
// with the guide ratio folded in (evolution.transition_rates:255-260).
template <typename T, int FAM>
__device__ __forceinline__ T offdiag(const DevModel<T> &m, const DevGuide<T> &g,
                                     const uint64_t *bits, const uint8_t *occ, const T *F, int o) {
  if (FAM == SPIN_HALF) {
    if (o < m.n_hx) {
      T v = m.hx_half[o];
      if (g.kind && v != T(0)) {
        T x = spin_x<T>(bits, o);
        T ld = T(-2) * x * F[o] - T(2) * g.h[o] * x;           // _site_log_diff:290-297
        v *= math_exp(ld);
      }
      return v;
    }
    int e = o - m.n_hx;
    uint32_t pe = m.edge[e];
    int i = pe & 0xFFFF, j = pe >> 16;
    T xi = spin_x<T>(bits, i), xj = spin_x<T>(bits, j);
    T v = (xi != xj) ? m.jpm[e] : m.jpmpm[e];
    if (g.kind && v != T(0)) {
      // _edge_log_diff_from_cache:462-472 with sum_{b!=j} J_ib x_b = W_i - Jsum_ij x_j
      T pair = xi * F[i] + xj * F[j] - T(2) * g.edge_jsum[e] * xi * xj;
      T ld = T(-2) * pair - T(2) * (g.h[i] * xi + g.h[j] * xj);
      v *= math_exp(ld);
    }
    return v;
  } else {
    BoseMove mv = bose_decode(m, o);
    T na = T(occ[mv.a]), nb = T(occ[mv.b]);
    T nmax = T(m.n_max);
    T v;
    switch (mv.blk) {
      case 0: v = -m.t[mv.idx] * math_sqrt(na * (nb + T(1))) * (nb < nmax ? T(1) : T(0)); break;
      case 1: v = -m.t[mv.idx] * math_sqrt((na + T(1)) * nb) * (na < nmax ? T(1) : T(0)); break;
      case 2:
        v = -m.eta[mv.idx] * math_sqrt((na + T(1)) * (nb + T(1))) *
            ((na < nmax && nb < nmax) ? T(1) : T(0));
        break;
      case 3: v = -m.eta[mv.idx] * math_sqrt(na * nb); break;
      case 4: v = m.hpm[mv.idx] * math_sqrt(na + T(1)) * (na < nmax ? T(1) : T(0)); break;
      default: v = m.hpm[mv.idx] * math_sqrt(na); break;
    }
    if (g.kind && v != T(0)) {
      // JastrowBoseHubbard.log_diff_from_operator:253-286
      T da = T(mv.da), db = T(mv.db);
      T out = T(0);
      if (g.d_mode) {
        T dsa = (na + da) * (na + da) - na * na, dsb = (nb + db) * (nb + db) - nb * nb;
        out = (g.d_mode == 2) ? -(g.d[mv.a] * dsa + g.d[mv.b] * dsb) : -g.d0 * (dsa + dsb);
      }
      T pw = g.trans_pw[o + 1];
      if (g.beta_scale == T(1)) out = out + da * F[mv.a] + db * F[mv.b] + da * db * pw;
      else out = out + g.beta_scale * (da * F[mv.a] + db * F[mv.b] + da * db * pw);
      if (g.h_mode == 2) out = out + (g.h[mv.a] * da + g.h[mv.b] * db);
      else if (g.h_mode == 1) out = out + g.h0 * (da + db);
      v *= math_exp(out);
    }
    return v;
  }
}

// Field of every site from scratch: W_k / S_k.
template <typename T, int FAM>
__device__ __forceinline__ void field_init(const DevModel<T> &m, const DevGuide<T> &g,
                                           const uint64_t *bits, const uint8_t *occ, T *F,
                                           int lane) {
  for (int k = lane; k < m.N; k += 32) {
    T s = T(0);
    const int c = g.nbr_cnt[k];
    const uint32_t *nb = g.nbr + (size_t)k * g.deg;
    const T *nw = g.nbr_w + (size_t)k * g.deg;
    for (int d = 0; d < c; ++d) s += nw[d] * site_val<T, FAM>(bits, occ, (int)nb[d]);
    F[k] = s;
  }
}

// Field update after site k changed by delta (spin: delta = -2 x_old).
template <typename T>
__device__ __forceinline__ void field_update(const DevGuide<T> &g, T *F, int k, T delta, int lane) {
  const int c = g.nbr_cnt[k];
  const uint32_t *nb = g.nbr + (size_t)k * g.deg;
  const T *nw = g.nbr_w + (size_t)k * g.deg;
  for (int d = lane; d < c; d += 32) F[nb[d]] += nw[d] * delta;
  __syncwarp();
}

// Apply move o (off-diagonal index) to the warp's configuration and fields.
template <typename T, int FAM>
__device__ __forceinline__ void apply_move(const DevModel<T> &m, const DevGuide<T> &g,
                                           uint64_t *bits, uint8_t *occ, T *F, int o, int lane) {
  if (FAM == SPIN_HALF) {
    int s0, s1;
    if (o < m.n_hx) { s0 = o; s1 = -1; }
    else { uint32_t pe = m.edge[o - m.n_hx]; s0 = pe & 0xFFFF; s1 = pe >> 16; }
    T x0 = spin_x<T>(bits, s0);
    T x1 = s1 >= 0 ? spin_x<T>(bits, s1) : T(0);
    __syncwarp();
    if (lane == 0) {
      bits[s0 >> 6] ^= 1ull << (s0 & 63);
      if (s1 >= 0) bits[s1 >> 6] ^= 1ull << (s1 & 63);
    }
    __syncwarp();
    if (g.kind) {
      field_update(g, F, s0, T(-2) * x0, lane);
      if (s1 >= 0) field_update(g, F, s1, T(-2) * x1, lane);
    }
  } else {
    BoseMove mv = bose_decode(m, o);
    __syncwarp();
    if (lane == 0) {
      occ[mv.a] = (uint8_t)(occ[mv.a] + mv.da);
      occ[mv.b] = (uint8_t)(occ[mv.b] + mv.db);
    }
    __syncwarp();
    if (g.kind) {
      field_update(g, F, mv.a, T(mv.da), lane);
      if (mv.db != 0) field_update(g, F, mv.b, T(mv.db), lane);
    }
  }
}

// Pass 1: fill q[s] for every slot and scan.  lamform (single_step): slot 0
// is the diagonal, q = rates, cdf = lam - cumsum(q); otherwise q = -rates
// of the off-diagonal moves and cdf = cumsum(q).  Returns the scanned total.
template <typename T, int FAM>
__device__ __forceinline__ T scan_pass(const DevModel<T> &m, const DevGuide<T> &g,
                                       const uint64_t *bits, const uint8_t *occ, const T *F,
                                       T *q, T *rowend, int n_slots, bool lamform, T diag,
                                       int lane) {
  const int rows = (n_slots + 31) >> 5;
  T carry = T(0);
  for (int r = 0; r < rows; ++r) {
    const int s = (r << 5) + lane;
    T v = T(0);
    if (s < n_slots) {
      if (lamform) v = (s == 0) ? diag : offdiag<T, FAM>(m, g, bits, occ, F, s - 1);
      else v = -offdiag<T, FAM>(m, g, bits, occ, F, s);
    }
    q[s] = v;
    T inc = warp_inclusive_scan(v, lane) + carry;
    carry = __shfl_sync(FULL, inc, 31);
    if (lane == 0) rowend[r] = carry;
  }
  __syncwarp();
  return carry;
}

// Pass 2: evolution.sample_index on the scanned slots for the threshold u:
// the first slot whose cdf exceeds u, stepped back to the nearest slot at or
// before it with positive weight.
template <typename T>
__device__ __forceinline__ int warp_sample(const T *q, const T *rowend, int n_slots,
                                           bool lamform, T lam, T u, int lane) {
  const int rows = (n_slots + 31) >> 5;
  int rstar = rows - 1;
  for (int base = 0; base < rows; base += 32) {
    int r = base + lane;
    bool hit = false;
    if (r < rows) {
      T c = lamform ? lam - rowend[r] : rowend[r];
      hit = c > u;
    }
    unsigned bal = __ballot_sync(FULL, hit);
    if (bal) { rstar = base + __ffs(bal) - 1; break; }
  }
  T carry = rstar > 0 ? rowend[rstar - 1] : T(0);
  int s = (rstar << 5) + lane;
  T inc = warp_inclusive_scan(q[s], lane) + carry;
  T c = lamform ? lam - inc : inc;
  unsigned bal = __ballot_sync(FULL, s < n_slots && c > u);
  int idx = bal ? (rstar << 5) + __ffs(bal) - 1 : (rstar << 5) + 31;
  if (idx > n_slots - 1) idx = n_slots - 1;
  for (int r = idx >> 5; r >= 0; --r) {
    int s2 = (r << 5) + lane;
    T q2 = q[s2];
    T w2 = lamform ? (s2 == 0 ? (-q2 + lam) : -q2) : q2;
    unsigned b2 = __ballot_sync(FULL, s2 <= idx && s2 < n_slots && w2 > T(0));
    if (b2) return (r << 5) + 31 - __clz(b2);
  }
  return idx;
}

template <typename T, int FAM>
__global__ void __launch_bounds__(256)
evolve_kernel(DevModel<T> m, DevGuide<T> g, EvolveArgs a, int stage_nbr, int n_slots_max,
              int cta_bytes, int warp_bytes) {
  extern __shared__ __align__(16) unsigned char smem[];
  stage_tables(m, g, stage_nbr, smem, true);
  __syncthreads();

  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  size_t o_field, o_q, o_rowend;
  warp_region(m, g, n_slots_max, &o_field, &o_q, &o_rowend);
  unsigned char *wb = smem + cta_bytes + (size_t)wib * warp_bytes;
  uint64_t *bits = reinterpret_cast<uint64_t *>(wb);
  uint8_t *occ = wb;
  T *F = reinterpret_cast<T *>(wb + o_field);
  T *q = reinterpret_cast<T *>(wb + o_q);
  T *rowend = reinterpret_cast<T *>(wb + o_rowend);

  const int NW = spin_words(m.N);
  const int CB = bose_bytes(m.N);
  const int method = a.method;
  const bool guided = g.kind != GUIDE_NONE;
  const T lam = T(a.lam);
  double wmax = -DBL_MAX;
  bool any_walker = false;
  unsigned long long hop_acc = 0;

  for (;;) {
    int walker = 0;
    if (lane == 0) walker = atomicAdd(a.work_ctr, 1);
    walker = __shfl_sync(FULL, walker, 0);
    if (walker >= a.n_walkers) break;

    // ---- load (fused gather through the previous step's parent map)
    const int src = a.parents ? a.parents[walker] : walker;
    if (FAM == SPIN_HALF) {
      const uint64_t *in = reinterpret_cast<const uint64_t *>(a.cfg_in) + (size_t)src * NW;
      for (int k = lane; k < NW; k += 32) bits[k] = in[k];
    } else {
      const uint32_t *in =
          reinterpret_cast<const uint32_t *>(reinterpret_cast<const uint8_t *>(a.cfg_in) + (size_t)src * CB);
      uint32_t *o32 = reinterpret_cast<uint32_t *>(occ);
      for (int k = lane; k < CB / 4; k += 32) o32[k] = in[k];
    }
    __syncwarp();
    if (guided) {
      field_init<T, FAM>(m, g, bits, occ, F, lane);
      __syncwarp();
    }

    const Key kw = fold(a.key, (uint32_t)walker);
    double lw = 0.0;
    T eloc = T(0);
    int hops = 0;

    if (method == CONT_TIME) {
      const T beta = T(a.step);
      T t = T(0);
      uint32_t it = 0;
      while (t < beta) {
        const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
        const T R = scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.n_off, false, diag, lane);
        const T eL = diag - R;
        const T dr = uniform<T>(fold(kw, 2u * it + (uint32_t)(lane & 1)));
        const T U1 = __shfl_sync(FULL, dr, 0), psi = __shfl_sync(FULL, dr, 1);
        int si = 0;
        if (R > T(0)) {
          T u = U1 * R, cap = next_below(R);
          si = warp_sample(q, rowend, m.n_off, false, lam, u < cap ? u : cap, lane);
        }
        const T tau_raw = (R > T(0)) ? -math_log1p(-psi) / R : pos_inf<T>();
        const T rem = beta - t;
        const T tau = tau_raw < rem ? tau_raw : rem;
        lw = lw - (double)eL * (double)tau;
        t = t + tau;
        if (tau_raw < rem) {
          apply_move<T, FAM>(m, g, bits, occ, F, si, lane);
          ++hops;
        }
        eloc = eL;
        if (++it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      lw -= a.alw * a.step;
    } else if (method == SINGLE_STEP) {
      const int n_bra = (int)a.step;
      for (int sidx = 0; sidx < n_bra; ++sidx) {
        const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
        const T Q = scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.M, true, diag, lane);
        const T bx = lam - Q;
        const T U = uniform<T>(fold(kw, (uint32_t)sidx));
        T u = U * bx, cap = next_below(bx);
        const int idx = warp_sample(q, rowend, m.M, true, lam, u < cap ? u : cap, lane);
        if (idx != 0) {
          apply_move<T, FAM>(m, g, bits, occ, F, idx - 1, lane);
          ++hops;
        }
        lw = lw + (double)math_log(bx);
      }
      const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
      const T R = scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.n_off, false, diag, lane);
      eloc = diag - R;
      lw -= a.alw * (double)n_bra;
    } else if (method == MULTI_STEP) {
      const int n_bra = (int)a.step;
      int used = 0;
      uint32_t it = 0;
      while (used < n_bra) {
        const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
        const T R = scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.n_off, false, diag, lane);
        const T bx = lam - diag + R;
        const T dr = uniform<T>(fold(kw, 2u * it + (uint32_t)(lane & 1)));
        const T U1 = __shfl_sync(FULL, dr, 0), psi = __shfl_sync(FULL, dr, 1);
        int si = 0;
        if (R > T(0)) {
          T u = U1 * R, cap = next_below(R);
          si = warp_sample(q, rowend, m.n_off, false, lam, u < cap ? u : cap, lane);
        }
        const int remaining = n_bra - used;
        const T hp = R / bx;
        const bool can_hop = hp > T(0);
        const T log_pd = can_hop ? math_log1p(-hp) : T(-1);
        const T hold = floor(math_log1p(-psi) / log_pd) + T(1);
        const T capk = T(remaining + 1);
        const T hm = hold < capk ? hold : capk;
        const int k_raw = can_hop ? (int)hm : remaining + 1;
        const int k = k_raw < remaining ? k_raw : remaining;
        lw = lw + (double)math_log(bx) * (double)k;
        used += k;
        if (k_raw <= remaining) {
          apply_move<T, FAM>(m, g, bits, occ, F, si, lane);
          ++hops;
        }
        if (++it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
      const T R = scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.n_off, false, diag, lane);
      eloc = diag - R;
      lw -= a.alw * (double)n_bra;
    } else {  // EVALUATE: local energy of the loaded configuration
      const T diag = diag_elem<T, FAM>(m, bits, occ, lane);
      const T R = m.n_off > 0
                      ? scan_pass<T, FAM>(m, g, bits, occ, F, q, rowend, m.n_off, false, diag, lane)
                      : T(0);
      eloc = diag - R;
    }

    // ---- store
    if (a.cfg_out) {
      if (FAM == SPIN_HALF) {
        uint64_t *out = reinterpret_cast<uint64_t *>(a.cfg_out) + (size_t)walker * NW;
        for (int k = lane; k < NW; k += 32) out[k] = bits[k];
      } else {
        uint32_t *out = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(a.cfg_out) +
                                                     (size_t)walker * CB);
        const uint32_t *o32 = reinterpret_cast<const uint32_t *>(occ);
        for (int k = lane; k < CB / 4; k += 32) out[k] = o32[k];
      }
    }
    if (lane == 0) {
      if (method != EVALUATE) a.log_w[walker] = lw;
      a.e_loc[walker] = (double)eloc;
    }
    wmax = lw > wmax ? lw : wmax;
    any_walker = true;
    hop_acc += (unsigned long long)hops;
    __syncwarp();
  }

  // ---- block max of log_w and hop count
  __shared__ double s_max[32];
  __shared__ unsigned long long s_hops[32];
  if (lane == 0) {
    s_max[wib] = any_walker ? wmax : -DBL_MAX;
    s_hops[wib] = hop_acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = -DBL_MAX;
    unsigned long long h = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      mx = s_max[i] > mx ? s_max[i] : mx;
      h += s_hops[i];
    }
    if (a.partial_max) a.partial_max[blockIdx.x] = mx;
    if (a.hops && h) atomicAdd(a.hops, h);
  }
}

}  // namespace

template <typename T>
cudaError_t plan_evolve(const DevModel<T> &m, const DevGuide<T> &g, int n_slots_max,
                        LaunchPlan *plan) {
  int dev = 0, sms = 0, max_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  DevModel<T> mm = m;
  DevGuide<T> gg = g;
  size_t of, oq, orr;
  size_t warp_bytes = warp_region(m, g, n_slots_max, &of, &oq, &orr);
  // Partner tables go to shared memory when they fit a 64 KB budget.
  size_t nbr_bytes = g.kind ? (size_t)m.N * g.deg * (sizeof(uint32_t) + sizeof(T)) + m.N * 4 : 0;
  int stage_nbr = (g.kind != GUIDE_NONE) && nbr_bytes <= 64 * 1024;
  size_t cta = stage_tables(mm, gg, stage_nbr, nullptr, false);
  int wpb = 8;
  while (wpb > 1 && cta + wpb * warp_bytes > (size_t)max_smem) wpb >>= 1;
  if (cta + wpb * warp_bytes > (size_t)max_smem) return cudaErrorInvalidConfiguration;
  plan->wpb = wpb;
  plan->block = wpb * 32;
  plan->smem = cta + wpb * warp_bytes;
  int per_sm = 0;
  cudaError_t err;
  if (m.family == SPIN_HALF) {
    err = cudaFuncSetAttribute(evolve_kernel<T, SPIN_HALF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)plan->smem);
    if (err != cudaSuccess) return err;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, evolve_kernel<T, SPIN_HALF>,
                                                        plan->block, plan->smem);
  } else {
    err = cudaFuncSetAttribute(evolve_kernel<T, BOSE_HUBBARD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)plan->smem);
    if (err != cudaSuccess) return err;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, evolve_kernel<T, BOSE_HUBBARD>,
                                                        plan->block, plan->smem);
  }
  if (err != cudaSuccess) return err;
  if (per_sm < 1) per_sm = 1;
  plan->grid = sms * per_sm;
  // stash the table staging decision and region sizes in the plan's upper bits
  plan->smem = cta + wpb * warp_bytes;
  (void)stage_nbr;
  return cudaSuccess;
}

template <typename T>
cudaError_t launch_evolve(const DevModel<T> &m, const DevGuide<T> &g, const LaunchPlan &plan,
                          const EvolveArgs &a, cudaStream_t s) {
  size_t of, oq, orr;
  int n_slots_max = m.M;
  size_t warp_bytes = warp_region(m, g, n_slots_max, &of, &oq, &orr);
  size_t nbr_bytes = g.kind ? (size_t)m.N * g.deg * (sizeof(uint32_t) + sizeof(T)) + m.N * 4 : 0;
  int stage_nbr = (g.kind != GUIDE_NONE) && nbr_bytes <= 64 * 1024;
  DevModel<T> mm = m;
  DevGuide<T> gg = g;
  size_t cta = stage_tables(mm, gg, stage_nbr, nullptr, false);
  int grid = plan.grid;
  int need = (a.n_walkers + plan.wpb - 1) / plan.wpb;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  if (m.family == SPIN_HALF)
    evolve_kernel<T, SPIN_HALF><<<grid, plan.block, plan.smem, s>>>(
        m, g, a, stage_nbr, n_slots_max, (int)cta, (int)warp_bytes);
  else
    evolve_kernel<T, BOSE_HUBBARD><<<grid, plan.block, plan.smem, s>>>(
        m, g, a, stage_nbr, n_slots_max, (int)cta, (int)warp_bytes);
  return cudaGetLastError();
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

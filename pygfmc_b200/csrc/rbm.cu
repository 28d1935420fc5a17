// The GFMC step with an RBM guide: one warp per walker.
//
// Each lane owns HPL = Hp / 32 consecutive hidden units and keeps their
// theta in registers.  A rate evaluation loops over the move slots (site
// flips, then edges): for a slot with a nonzero coupling the warp loads the
// flipped sites' weight rows W[:, i], W[:, j] (bf16, 16-byte vector loads of
// the lane's HPL units, read-only cache), sums log cosh(theta' ) over its
// units with theta' = theta - 2 s_i W_i - 2 s_j W_j, and reduces over the
// warp; rate = coupling * exp(sum - sum_h log cosh(theta_h) - 2 a_i s_i -
// 2 a_j s_j).  Zero couplings (parallel spins without J_pmpm) are skipped,
// as the reference masks zero rates (engine/evolution.py:260).  The rates go
// to the warp's shared-memory row; the draw scans lane chunks of it and
// steps back off zero weights exactly as sample_index
// (engine/evolution.py:30-59).  A move updates theta in registers with the
// same expression the rate used, so the state and the ratios agree bit for
// bit.  The propagators are those of the Jastrow kernel (evolve.cu), with the
// same per-walker Threefry streams.
//
// Roofline: special-function bound.  Per evaluation and slot: HPL log cosh
// per lane (two MUFU ops each in float: ex2, lg2), against 2 x 2 Hp bytes of
// weight rows from L1/L2.
#include <cfloat>

#include "rbm_dev.cuh"

namespace gfmc {
namespace {

constexpr int RB_WARPS = 4;   // warps per block

// q[0] = H_xx, q[1 + o] = guide-transformed rate of slot o.
//
// float64: sum_h lncosh(theta') - sum_h lncosh(theta) term by term (the
// reference form).  float32: the same difference as
//   sum_h (|theta'_h| - |theta_h|) + log prod_h (1 + e'_h) / (1 + e_h),
//   e = exp(-2 |x|),
// with 1 / (1 + e_h) computed once per evaluation, so a (slot, unit) pair
// costs one ex2 instead of an ex2 and a lg2; each factor lies in (1/2, 2),
// so the lane's product of HPL factors stays in range, and one lg2 per
// lane and slot closes it.
template <typename T, int HPL>
__device__ void rbm_rates(const DevModel<T> &m, const RbmTables &r, const uint64_t *bits,
                          const T (&th)[HPL], T *q, int lane) {
  constexpr bool F32 = sizeof(T) == 4;
  T lcs = T(0);
  float binv[F32 ? HPL : 1];
  if constexpr (F32) {
#pragma unroll
    for (int k = 0; k < HPL; ++k)
      binv[k] = __fdividef(1.0f, 1.0f + ex2_approx(-2.8853900817779268f * fabsf((float)th[k])));
  } else {
    T l = T(0);
#pragma unroll
    for (int k = 0; k < HPL; ++k) l += lncosh<T>(th[k]);
    lcs = warp_sum(l);
  }
  const int hoff = lane * HPL;
  for (int o = 0; o < m.n_off; ++o) {
    int i, j;
    const T c = slot_coupling(m, bits, o, &i, &j);
    T rate = c;
    if (c != T(0)) {
      const T si = spin_bit(bits, i) ? T(1) : T(-1);
      const T sj = j >= 0 ? (spin_bit(bits, j) ? T(1) : T(-1)) : T(0);
      float wi[HPL], wj[HPL];
      load_row<HPL>(r.WT + (size_t)i * r.Hp + hoff, wi);
      if (j >= 0) {
        load_row<HPL>(r.WT + (size_t)j * r.Hp + hoff, wj);
      } else {
#pragma unroll
        for (int k = 0; k < HPL; ++k) wj[k] = 0.0f;
      }
      T d;
      if constexpr (F32) {
        float sd = 0.0f, pr = 1.0f;
#pragma unroll
        for (int k = 0; k < HPL; ++k) {
          const float t = th[k] - 2.0f * si * wi[k] - 2.0f * sj * wj[k];
          const float y = fabsf(t);
          sd += y - fabsf(th[k]);
          pr *= (1.0f + ex2_approx(-2.8853900817779268f * y)) * binv[k];
        }
        d = warp_sum(sd + 0.69314718f * __log2f(pr));
      } else {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < HPL; ++k)
          acc += lncosh<T>(th[k] - T(2) * si * T(wi[k]) - T(2) * sj * T(wj[k]));
        d = warp_sum(acc) - lcs;
      }
      d = d - T(2) * T(r.a[i]) * si;
      if (j >= 0) d = d - T(2) * T(r.a[j]) * sj;
      rate = c * math_exp<T>(d);
    }
    if (lane == 0) q[1 + o] = rate;
  }
  // diagonal element: SpinHalf.diagonal_weight:291-314
  T dg = T(0);
  if (m.has_jz) {
    int na = 0;
    T jzs = T(0);
    for (int e = lane; e < m.E; e += 32) {
      const uint32_t pe = m.edge[e];
      const bool anti = spin_bit(bits, (int)(pe & 0xFFFF)) != spin_bit(bits, (int)(pe >> 16));
      if (m.uniform_jz) na += anti;
      else jzs += anti ? -m.jz[e] / T(4) : m.jz[e] / T(4);
    }
    if (m.uniform_jz) dg = (m.jz[0] / T(4)) * T(m.E - 2 * warp_sum(na));
    else dg = warp_sum(jzs);
  }
  if (m.has_hz) {
    T hzs = T(0);
    for (int k = lane; k < m.N; k += 32) hzs += m.hz[k] * (spin_bit(bits, k) ? T(1) : T(-1));
    dg = dg + warp_sum(hzs) / T(2);
  }
  if (lane == 0) q[0] = dg;
  __syncwarp();
}

template <typename T, int HPL>
__global__ void __launch_bounds__(RB_WARPS * 32)
rbm_evolve_kernel(DevModel<T> m, RbmTables r, EvolveArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int NW = rb_words(m.N);
  unsigned char *wb = smem + (size_t)wib * rb_warp_bytes<T>(m.N, m.M);
  uint64_t *bits = reinterpret_cast<uint64_t *>(wb);
  T *q = reinterpret_cast<T *>(wb + (size_t)NW * 8);
  const int method = a.method;
  const T lam = T(a.lam);
  const int hoff = lane * HPL;
  double wmax = -DBL_MAX;
  unsigned long long hop_acc = 0;

  for (;;) {
    int walker = 0;
    if (lane == 0) walker = atomicAdd(a.work_ctr, 1);
    walker = __shfl_sync(FULLM, walker, 0);
    if (walker >= a.n_walkers) break;

    // ---- load: configuration (through the parent map) and theta
    const int src = a.parents ? a.parents[walker] : walker;
    const uint64_t *in = reinterpret_cast<const uint64_t *>(a.cfg_in) + (size_t)src * NW;
    for (int k = lane; k < NW; k += 32) bits[k] = in[k];
    __syncwarp();
    T th[HPL];
    if (a.field_in) {
      const T *fin = reinterpret_cast<const T *>(a.field_in) + (size_t)src * r.Hp + hoff;
#pragma unroll
      for (int k = 0; k < HPL; ++k) th[k] = fin[k];
    } else {
#pragma unroll
      for (int k = 0; k < HPL; ++k) th[k] = T(r.b[hoff + k]);
      for (int i = 0; i < m.N; ++i) {
        const T si = spin_bit(bits, i) ? T(1) : T(-1);
        float w[HPL];
        load_row<HPL>(r.WT + (size_t)i * r.Hp + hoff, w);
#pragma unroll
        for (int k = 0; k < HPL; ++k) th[k] = th[k] + si * T(w[k]);
      }
    }

    const Key kw = fold(a.key, (uint32_t)(a.walker_offset + walker));
    double lw = a.lw_in ? a.lw_in[src] : 0.0;
    T eloc = T(0);
    int hops = 0;
    T draws = T(0);

    if (method == CONT_TIME) {
      const T beta = T(a.step);
      T t = T(0);
      uint32_t it = 0;
      while (t < beta) {
        rbm_rates<T, HPL>(m, r, bits, th, q, lane);
        const RScan<T> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
        const T R = sc.total;
        const T eL = q[0] - R;
        if ((it & 15u) == 0) draws = uniform<T>(fold(kw, 2u * it + (uint32_t)lane));
        const T U1 = __shfl_sync(FULLM, draws, (int)(2u * (it & 15u)));
        const T psi = __shfl_sync(FULLM, draws, (int)(2u * (it & 15u) + 1u));
        int si = 0;
        if (R > T(0)) {
          const T u = U1 * R, cap = next_below(R);
          si = rbm_pick(q, sc, RB_OFF, lam, u < cap ? u : cap, lane);
        }
        const T tau_raw = (R > T(0)) ? -math_log1p(-psi) / R : pos_inf<T>();
        const T rem = beta - t;
        const T tau = tau_raw < rem ? tau_raw : rem;
        lw = lw - (double)eL * (double)tau;
        t = t + tau;
        if (tau_raw < rem) {
          rbm_move<T, HPL>(m, r, bits, th, si, lane);
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
        rbm_rates<T, HPL>(m, r, bits, th, q, lane);
        const RScan<T> sc = rbm_scan(q, m.n_off, RB_LAM, lane);
        const T bx = lam - sc.total;
        if ((sidx & 31) == 0) draws = uniform<T>(fold(kw, (uint32_t)(sidx + lane)));
        const T U = __shfl_sync(FULLM, draws, sidx & 31);
        const T u = U * bx, cap = next_below(bx);
        const int idx = rbm_pick(q, sc, RB_LAM, lam, u < cap ? u : cap, lane);
        if (idx != 0) {
          rbm_move<T, HPL>(m, r, bits, th, idx - 1, lane);
          ++hops;
        }
        lw = lw + (double)math_log(bx);
      }
      rbm_rates<T, HPL>(m, r, bits, th, q, lane);
      const RScan<T> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      eloc = q[0] - sc.total;
      lw -= a.alw * (double)n_bra;
    } else if (method == MULTI_STEP) {
      const int n_bra = (int)a.step;
      int used = 0;
      uint32_t it = 0;
      while (used < n_bra) {
        rbm_rates<T, HPL>(m, r, bits, th, q, lane);
        const RScan<T> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
        const T R = sc.total;
        const T bx = lam - q[0] + R;
        if ((it & 15u) == 0) draws = uniform<T>(fold(kw, 2u * it + (uint32_t)lane));
        const T U1 = __shfl_sync(FULLM, draws, (int)(2u * (it & 15u)));
        const T psi = __shfl_sync(FULLM, draws, (int)(2u * (it & 15u) + 1u));
        int si = 0;
        if (R > T(0)) {
          const T u = U1 * R, cap = next_below(R);
          si = rbm_pick(q, sc, RB_OFF, lam, u < cap ? u : cap, lane);
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
          rbm_move<T, HPL>(m, r, bits, th, si, lane);
          ++hops;
        }
        if (++it >= (uint32_t)a.max_iters) {
          if (lane == 0) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      rbm_rates<T, HPL>(m, r, bits, th, q, lane);
      const RScan<T> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      eloc = q[0] - sc.total;
      lw -= a.alw * (double)n_bra;
    } else {  // EVALUATE
      rbm_rates<T, HPL>(m, r, bits, th, q, lane);
      const RScan<T> sc = rbm_scan(q, m.n_off, RB_OFF, lane);
      eloc = q[0] - sc.total;
      if (a.rates_out)
        for (int o = lane; o < m.n_off; o += 32)
          a.rates_out[(size_t)walker * m.n_off + o] = (float)q[1 + o];
      if (a.rsum_out && lane == 0) a.rsum_out[walker] = (float)(-sc.total);
      if (a.diag_out && lane == 0) a.diag_out[walker] = (double)q[0];
    }

    // ---- store
    if (a.cfg_out) {
      uint64_t *out = reinterpret_cast<uint64_t *>(a.cfg_out) + (size_t)walker * NW;
      for (int k = lane; k < NW; k += 32) out[k] = bits[k];
    }
    if (a.field_out) {
      T *fout = reinterpret_cast<T *>(a.field_out) + (size_t)walker * r.Hp + hoff;
#pragma unroll
      for (int k = 0; k < HPL; ++k) fout[k] = th[k];
    }
    if (lane == 0) {
      if (method <= MULTI_STEP) a.log_w[walker] = lw;
      a.e_loc[walker] = (double)eloc;
    }
    if (method <= MULTI_STEP) wmax = lw > wmax ? lw : wmax;
    hop_acc += (unsigned long long)hops;
    __syncwarp();
  }
  if (lane == 0) {
    if (a.partial_max) a.partial_max[(size_t)blockIdx.x * RB_WARPS + wib] = wmax;
    if (a.hops && hop_acc) atomicAdd(a.hops, hop_acc);
  }
}

template <typename T>
using RbmKernel = void (*)(DevModel<T>, RbmTables, EvolveArgs);

template <typename T> RbmKernel<T> pick_rbm(int hpl) {
  switch (hpl) {
    case 8: return rbm_evolve_kernel<T, 8>;
    case 16: return rbm_evolve_kernel<T, 16>;
    case 24: return rbm_evolve_kernel<T, 24>;
    default: return rbm_evolve_kernel<T, 32>;
  }
}

}  // namespace

template <typename T> int rbm_grid(const DevModel<T> &m, const RbmTables &r) {
  if constexpr (sizeof(T) == 4) return rbm_grid_f32(m, r);
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t smem = RB_WARPS * rb_warp_bytes<T>(m.N, m.M);
  RbmKernel<T> k = pick_rbm<T>(rbm_hpl(r.Hp));
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, RB_WARPS * 32, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

template <typename T>
cudaError_t launch_rbm_evolve(const DevModel<T> &m, const RbmTables &r, const EvolveArgs &a,
                              int grid, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) return launch_rbm_evolve_f32(m, r, a, grid, s);
  const size_t smem = RB_WARPS * rb_warp_bytes<T>(m.N, m.M);
  int need = (a.n_walkers + RB_WARPS - 1) / RB_WARPS;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  pick_rbm<T>(rbm_hpl(r.Hp))<<<grid, RB_WARPS * 32, smem, s>>>(m, r, a);
  return cudaGetLastError();
}

// per-warp partial maxima a launch over n walkers writes
int rbm_partials(int grid, int n_walkers, bool f32) {
  const int wpb = f32 ? RBF_WARPS : RB_WARPS;
  int need = (n_walkers + wpb - 1) / wpb;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  return grid * wpb;
}

template int rbm_grid<double>(const DevModel<double> &, const RbmTables &);
template int rbm_grid<float>(const DevModel<float> &, const RbmTables &);
template cudaError_t launch_rbm_evolve<double>(const DevModel<double> &, const RbmTables &,
                                               const EvolveArgs &, int, cudaStream_t);
template cudaError_t launch_rbm_evolve<float>(const DevModel<float> &, const RbmTables &,
                                              const EvolveArgs &, int, cudaStream_t);

}  // namespace gfmc

// Device helpers of the RBM step kernels (rbm.cu: float64; rbm_f32.cu:
// float32): slot couplings, weight rows, the slot scan and draw of
// sample_index (engine/evolution.py:30-59), and a move's theta update.
#pragma once
#include <cfloat>

#include "rbm.cuh"

namespace gfmc {
namespace {

constexpr unsigned FULLM = 0xffffffffu;

__host__ __device__ inline int rb_words(int N) { return (N + 63) / 64; }

__host__ __device__ inline int rb_chunk(int n_slots) {
  int c = (n_slots + 31) / 32;
  if (c < 1) c = 1;
  return c | 1;
}

enum RbMode { RB_OFF = 0, RB_LAM = 1 };

template <typename T> __device__ __forceinline__ T lncosh(T x);
// log cosh x - log 2 = |x| + log1p(exp(-2|x|)) - log 2
template <> __device__ __forceinline__ double lncosh<double>(double x) {
  const double y = fabs(x);
  return y + log1p(exp(-2.0 * y)) - 0.6931471805599453;
}
template <> __device__ __forceinline__ float lncosh<float>(float x) {
  const float y = fabsf(x);
  return y + __logf(1.0f + __expf(-2.0f * y)) - 0.69314718f;
}

__device__ __forceinline__ int spin_bit(const uint64_t *bits, int k) {
  return (int)((bits[k >> 6] >> (k & 63)) & 1ull);
}

// The lane's HPL weights of one row of WT (bf16 -> float, exact).
template <int HPL>
__device__ __forceinline__ void load_row(const __nv_bfloat16 *row, float (&w)[HPL]) {
  const uint4 *p = reinterpret_cast<const uint4 *>(row);
#pragma unroll
  for (int c = 0; c < HPL / 8; ++c) {
    const uint4 u = __ldg(p + c);
    const uint32_t v[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      w[8 * c + 2 * q] = __uint_as_float(v[q] << 16);
      w[8 * c + 2 * q + 1] = __uint_as_float(v[q] & 0xFFFF0000u);
    }
  }
}

// Coupling of off-diagonal slot o (site flips first, then edges) at the
// current spins, and the flipped sites (j = -1 for a site flip).
template <typename T>
__device__ __forceinline__ T slot_coupling(const DevModel<T> &m, const uint64_t *bits, int o,
                                           int *i, int *j) {
  if (o < m.n_hx) {
    *i = o;
    *j = -1;
    return m.hx_half[o];
  }
  const int e = o - m.n_hx;
  const uint32_t pe = m.edge[e];
  *i = (int)(pe & 0xFFFF);
  *j = (int)(pe >> 16);
  const bool anti = spin_bit(bits, *i) != spin_bit(bits, *j);
  return m.uniform_pm ? (anti ? m.jpm0 : m.jpmpm0) : (anti ? m.jpm[e] : m.jpmpm[e]);
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Scanned value of slot s: RB_OFF the weights -rates of the off-diagonal
// slots; RB_LAM slot 0 = H_xx and the rates (cdf = lam - cumsum).
template <typename T>
__device__ __forceinline__ T slot_val(const T *q, int mode, int s) {
  return mode == RB_LAM ? q[s] : -q[1 + s];
}
template <typename T>
__device__ __forceinline__ T slot_weight(const T *q, int mode, int s, T lam) {
  if (mode == RB_LAM) return s == 0 ? lam - q[0] : -q[s];
  return -q[1 + s];
}

template <typename T> struct RScan {
  T excl, end, total;
  int C, n_slots;
};

template <typename T>
__device__ __forceinline__ RScan<T> rbm_scan(const T *q, int n_off, int mode, int lane) {
  RScan<T> sc;
  sc.n_slots = mode == RB_LAM ? n_off + 1 : n_off;
  sc.C = rb_chunk(sc.n_slots);
  const int s0 = lane * sc.C;
  T acc = T(0);
  for (int j = 0; j < sc.C; ++j) {
    const int s = s0 + j;
    if (s < sc.n_slots) acc += slot_val(q, mode, s);
  }
  const T inc = warp_inclusive_scan(acc, lane);
  T ex = __shfl_up_sync(FULLM, inc, 1);
  if (lane == 0) ex = T(0);
  sc.excl = ex;
  sc.end = ex + acc;
  const int last = sc.n_slots > 0 ? (sc.n_slots - 1) / sc.C : 0;
  sc.total = __shfl_sync(FULLM, sc.end, last);
  return sc;
}

// sample_index over the scanned slots: the first slot whose cdf exceeds u,
// clamped to the last slot, stepped back to the nearest positive weight.
template <typename T>
__device__ __forceinline__ int rbm_pick(const T *q, const RScan<T> &sc, int mode, T lam, T u,
                                        int lane) {
  const int C = sc.C, n = sc.n_slots;
  const int last = (n - 1) / C;
  const bool lamc = mode == RB_LAM;
  const T cend = lamc ? lam - sc.end : sc.end;
  const unsigned bal = __ballot_sync(FULLM, lane <= last && cend > u);
  const int L = bal ? __ffs(bal) - 1 : last;
  int res = 0;
  if (lane == L) {
    const int s0 = L * C;
    const int s1 = (s0 + C < n) ? s0 + C : n;
    T c = sc.excl;
    int hit = s1 - 1;
    for (int s = s0; s < s1; ++s) {
      c += slot_val(q, mode, s);
      if ((lamc ? lam - c : c) > u) {
        hit = s;
        break;
      }
    }
    res = hit;
    for (int s = hit; s >= 0; --s)
      if (slot_weight(q, mode, s, lam) > T(0)) {
        res = s;
        break;
      }
  }
  return __shfl_sync(FULLM, res, L);
}

// Off-diagonal move o: theta -= 2 s_i W_i (+ 2 s_j W_j), then the flips.
template <typename T, int HPL>
__device__ __forceinline__ void rbm_move(const DevModel<T> &m, const RbmTables &r,
                                         uint64_t *bits, T (&th)[HPL], int o, int lane) {
  int i, j;
  (void)slot_coupling(m, bits, o, &i, &j);
  const int hoff = lane * HPL;
  const T si = spin_bit(bits, i) ? T(1) : T(-1);
  float wi[HPL];
  load_row<HPL>(r.WT + (size_t)i * r.Hp + hoff, wi);
  if (j >= 0) {
    const T sj = spin_bit(bits, j) ? T(1) : T(-1);
    float wj[HPL];
    load_row<HPL>(r.WT + (size_t)j * r.Hp + hoff, wj);
#pragma unroll
    for (int k = 0; k < HPL; ++k) th[k] = th[k] - T(2) * si * T(wi[k]) - T(2) * sj * T(wj[k]);
  } else {
#pragma unroll
    for (int k = 0; k < HPL; ++k) th[k] = th[k] - T(2) * si * T(wi[k]);
  }
  __syncwarp();
  if (lane == 0) {
    bits[i >> 6] ^= 1ull << (i & 63);
    if (j >= 0) bits[j >> 6] ^= 1ull << (j & 63);
  }
  __syncwarp();
}

template <typename T>
__host__ __device__ inline size_t rb_warp_bytes(int N, int M) {
  return (((size_t)rb_words(N) * 8 + (size_t)M * sizeof(T)) + 15) & ~(size_t)15;
}

}  // namespace
}  // namespace gfmc

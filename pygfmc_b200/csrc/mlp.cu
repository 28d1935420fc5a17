// The GFMC step with a dense MLP guide for Bose-Hubbard occupations (no
// PyGFMC counterpart), float32 with a bf16 tensor-core second layer.
//
//   x = one-hot occupations, z1 = W1 x + b1, h1 = tanh(z1),
//   log psi = w3 . tanh(W2 bf16(h1) + b2) + b3
//
// One CTA (4 warps) per SM, persistent over walkers (atomic work counter).
// W2 (H2 x H1, bf16) is staged once per CTA in shared memory in the 128-byte
// swizzled K-major layout (the MMA's B operand).  For a walker, z1 is built
// from the W1 columns of its occupations and updated per move.  A rate
// evaluation takes the moves in tiles of 128: the moves' first-layer
// activations h1' = tanh(z1 + W1[:, new] - W1[:, old]) (two sites, four
// columns) are written as bf16 rows of the A tile, one tcgen05.mma
// (kind::f16, M = 128 moves, N = H2, K = H1) per tile computes every
// successor's second-layer pre-activations into TMEM, and the epilogue
// (tcgen05.ld, thread = move) forms log psi(x') and the guided rate
// coupling * exp(log psi(x') - log psi(x)).  The walker's own log psi comes
// from the same path (a tile whose row 0 is the current configuration), so
// every ratio is a ratio of one function.  The draw and the hold follow the
// cont_time propagator of evolve.cu (same per-walker Threefry streams).
//
// Roofline: tensor + special-function bound: 2 * 128 * H1 * H2 flops and
// 128 (H1 + H2) tanh per tile, W1 columns (4 x H1 bf16 per move) from L1/L2.
#include <cfloat>
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

using namespace tc;

constexpr int MT = 128;                 // threads = moves per tile = UMMA M

// Moves of the Bose-Hubbard layout (bose_hubbard.py; _common.two_site_move):
// sites a, b, occupation changes da, db (b == a, db = 0 for the single-site
// h_pm moves) and the unguided off-diagonal element.
struct Mv {
  int a, b, da, db;
  float v;
};

__device__ __forceinline__ Mv mlp_move(const DevModel<float> &m, const uint8_t *occ, int o) {
  Mv mv;
  const int E = m.E;
  const float nmax = (float)m.n_max;
  int blk;
  int idx;
  if (m.n_hop && o < 2 * E) {
    const int e = o < E ? o : o - E;
    const uint32_t pe = m.edge[e];
    mv.a = pe & 0xFFFF; mv.b = pe >> 16; idx = e;
    if (o < E) { mv.da = -1; mv.db = 1; blk = 0; } else { mv.da = 1; mv.db = -1; blk = 1; }
  } else {
    if (m.n_hop) o -= 2 * E;
    if (m.n_eta && o < 2 * E) {
      const int e = o < E ? o : o - E;
      const uint32_t pe = m.edge[e];
      mv.a = pe & 0xFFFF; mv.b = pe >> 16; idx = e;
      if (o < E) { mv.da = 1; mv.db = 1; blk = 2; } else { mv.da = -1; mv.db = -1; blk = 3; }
    } else {
      if (m.n_eta) o -= 2 * E;
      const int k = o < m.N ? o : o - m.N;
      mv.a = mv.b = k; idx = k; mv.db = 0;
      if (o < m.N) { mv.da = 1; blk = 4; } else { mv.da = -1; blk = 5; }
    }
  }
  const float na = (float)occ[mv.a], nb = (float)occ[mv.b];
  switch (blk) {
    case 0: mv.v = -m.t[idx] * sqrtf(na * (nb + 1.0f)) * (nb < nmax ? 1.0f : 0.0f); break;
    case 1: mv.v = -m.t[idx] * sqrtf((na + 1.0f) * nb) * (na < nmax ? 1.0f : 0.0f); break;
    case 2:
      mv.v = -m.eta[idx] * sqrtf((na + 1.0f) * (nb + 1.0f)) * ((na < nmax && nb < nmax) ? 1.0f : 0.0f);
      break;
    case 3: mv.v = -m.eta[idx] * sqrtf(na * nb); break;
    case 4: mv.v = m.hpm[idx] * sqrtf(na + 1.0f) * (na < nmax ? 1.0f : 0.0f); break;
    default: mv.v = m.hpm[idx] * sqrtf(na); break;
  }
  // a move that leaves [0, n_max] has no element (and reads no W1 column),
  // whatever the couplings hold
  const int a1 = (int)occ[mv.a] + mv.da, b1 = (int)occ[mv.b] + mv.db;
  if (a1 < 0 || a1 > m.n_max || b1 < 0 || b1 > m.n_max) mv.v = 0.0f;
  return mv;
}

// z1 after move mv for the units j, j + 1 (the same expression as the rows
// of the A tile, so state and ratios agree bit for bit)
__device__ __forceinline__ float2 z1_moved(const MlpTables &t, const uint8_t *occ, const Mv &mv,
                                           int np1, float2 z, int j) {
  const int ca0 = mv.a * np1 + occ[mv.a], ca1 = ca0 + mv.da;
  const __nv_bfloat162 wa1 = *reinterpret_cast<const __nv_bfloat162 *>(t.W1T + (size_t)ca1 * t.H1 + j);
  const __nv_bfloat162 wa0 = *reinterpret_cast<const __nv_bfloat162 *>(t.W1T + (size_t)ca0 * t.H1 + j);
  z.x = (z.x + __low2float(wa1)) - __low2float(wa0);
  z.y = (z.y + __high2float(wa1)) - __high2float(wa0);
  if (mv.b != mv.a) {
    const int cb0 = mv.b * np1 + occ[mv.b], cb1 = cb0 + mv.db;
    const __nv_bfloat162 wb1 = *reinterpret_cast<const __nv_bfloat162 *>(t.W1T + (size_t)cb1 * t.H1 + j);
    const __nv_bfloat162 wb0 = *reinterpret_cast<const __nv_bfloat162 *>(t.W1T + (size_t)cb0 * t.H1 + j);
    z.x = (z.x + __low2float(wb1)) - __low2float(wb0);
    z.y = (z.y + __high2float(wb1)) - __high2float(wb0);
  }
  return z;
}

struct MlpSmem {
  size_t W2s, As, z1, b2, w3, rates, lps, rv, occ, misc, total;
};

__host__ __device__ inline MlpSmem mlp_plan(int H1, int H2, int n_off, int N) {
  MlpSmem p;
  size_t o = 0;
  p.W2s = o; o += (size_t)H2 * H1 * 2;
  p.As = o; o += (size_t)MT * H1 * 2;
  p.z1 = o; o += (size_t)H1 * 4;
  p.b2 = o; o += (size_t)H2 * 4;
  p.w3 = o; o += (size_t)H2 * 4;
  p.rates = o; o += (size_t)(n_off + 1) * 4;
  p.lps = o; o += (size_t)(n_off + 1) * 4;
  p.rv = o; o += (size_t)MT * 4;
  p.occ = o; o += (size_t)((N + 15) / 16) * 16;
  o = (o + 15) & ~(size_t)15;
  p.misc = o; o += 128;
  p.total = o;
  return p;
}

__global__ void __launch_bounds__(MT, 1) mlp_evolve_kernel(DevModel<float> m, MlpTables t,
                                                           EvolveArgs a) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int H1 = t.H1, H2 = t.H2, np1 = t.np1;
  const MlpSmem P = mlp_plan(H1, H2, m.n_off, m.N);
  unsigned char *W2s = base + P.W2s;
  unsigned char *As = base + P.As;
  float *z1 = reinterpret_cast<float *>(base + P.z1);
  float *b2s = reinterpret_cast<float *>(base + P.b2);
  float *w3s = reinterpret_cast<float *>(base + P.w3);
  float *rates = reinterpret_cast<float *>(base + P.rates);
  float *lps = reinterpret_cast<float *>(base + P.lps);
  float *rv = reinterpret_cast<float *>(base + P.rv);
  uint8_t *occ = base + P.occ;
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + P.misc);
  uint32_t *slot = reinterpret_cast<uint32_t *>(base + P.misc + 8);
  volatile int *flag = reinterpret_cast<volatile int *>(base + P.misc + 12);
  volatile int *bi = reinterpret_cast<volatile int *>(base + P.misc + 16);      // 4 ints
  volatile float *bf = reinterpret_cast<volatile float *>(base + P.misc + 32);  // 4 floats
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = H2 <= 32 ? 32u : (H2 <= 64 ? 64u : (H2 <= 128 ? 128u : 256u));

  // W2 into the swizzled K-major B layout: K chunk kc (64 inputs) holds the
  // H2 rows, 128 bytes each
  for (int idx = tid; idx < H2 * (H1 / 8); idx += MT) {
    const int j = idx / (H1 / 8), c8 = idx % (H1 / 8);
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(t.W2 + (size_t)j * H1) + c8);
    *reinterpret_cast<uint4 *>(sw_chunk(W2s + (size_t)(c8 / 8) * H2 * 128, j, c8 % 8)) = v;
  }
  for (int j = tid; j < H2; j += MT) {
    b2s[j] = t.b2[j];
    w3s[j] = t.w3[j];
  }
  if (warp == 0) tmem_alloc(slot, ncols);
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t idesc = idesc_m128((uint32_t)H2);
  const int CB = ((m.N + 15) / 16) * 16;
  uint32_t phase = 0;
  bool ok = true;
  double wmax = -DBL_MAX;
  unsigned long long hop_acc = 0;
  const int j2 = 2 * tid;            // this thread's unit pair (j2, j2 + 1) when j2 < H1

  // One tile of 128 rows, the moves tb .. tb + 127 (current: row 0 is the
  // configuration itself).  Writes rates[o] / lps[o] of the moves, or
  // bf[0] = log psi(x) for the current-configuration tile.
  auto tile = [&](int tb, bool current, float lpx) -> bool {
    {
      const int o = tb + tid;
      float v = 0.0f;
      if (current) v = tid == 0 ? 1.0f : 0.0f;
      else if (o < m.n_off) v = mlp_move(m, occ, o).v;
      rv[tid] = v;
    }
    __syncthreads();
    if (j2 < H1) {
      const float2 zc = make_float2(z1[j2], z1[j2 + 1]);
      unsigned char *Ac = As + (size_t)(j2 / 64) * MT * 128;
      const int c16 = (j2 % 64) / 8, e2 = (j2 % 8) * 2;
      for (int r = 0; r < MT; ++r) {
        uint32_t q = 0u;
        if (rv[r] != 0.0f) {
          float2 z = zc;
          if (!current) z = z1_moved(t, occ, mlp_move(m, occ, tb + r), np1, zc, j2);
          const __nv_bfloat162 h = __floats2bfloat162_rn(tanhf(z.x), tanhf(z.y));
          q = *reinterpret_cast<const uint32_t *>(&h);
        }
        *reinterpret_cast<uint32_t *>(sw_chunk(Ac, r, c16) + e2) = q;
      }
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      for (int kc = 0; kc < H1 / 64; ++kc)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          mma_bf16(tmem, sw128_desc(smem_u32(As + (size_t)kc * MT * 128) + 32u * kk),
                   sw128_desc(smem_u32(W2s + (size_t)kc * H2 * 128) + 32u * kk), idesc,
                   (kc > 0 || kk > 0) ? 1u : 0u);
      mma_commit(bar);
    }
    const bool done = cta_wait(bar, phase, flag);
    phase ^= 1u;
    if (!done) return false;
    fence_after();
    float acc = 0.0f;
    for (int c0 = 0; c0 < H2; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) acc = fmaf(w3s[c0 + i], tanhf(v[i] + b2s[c0 + i]), acc);
    }
    const float lp = t.b3 + acc;
    if (current) {
      if (tid == 0) bf[0] = lp;
    } else {
      const int o = tb + tid;
      if (o < m.n_off) {
        const float v = rv[tid];
        lps[o] = lp;
        rates[o] = v != 0.0f ? v * __expf(lp - lpx) : 0.0f;
      }
    }
    fence_before();
    __syncthreads();
    return true;
  };

  // H_xx (BoseHubbard diagonal, bose_hubbard.py:271-281) by warp 0 in the
  // step kernel's lane order, into bf[3]
  auto diag = [&]() {
    if (warp == 0) {
      float su = 0.0f, sm = 0.0f;
      for (int k = lane; k < m.N; k += 32) {
        const float n = (float)occ[k];
        if (m.has_U) su += m.U[k] * n * (n - 1.0f);
        if (m.has_mu) sm += m.mu[k] * n;
      }
      float d = 0.0f;
      if (m.has_U) d = d + 0.5f * warp_sum(su);
      if (m.has_mu) d = d - warp_sum(sm);
      if (lane == 0) bf[3] = d;
    }
  };

  for (;;) {
    if (tid == 0) bi[0] = atomicAdd(a.work_ctr, 1);
    __syncthreads();
    const int walker = bi[0];
    __syncthreads();
    if (walker >= a.n_walkers) break;
    const int src = a.parents ? a.parents[walker] : walker;
    const uint32_t *in = reinterpret_cast<const uint32_t *>(
        reinterpret_cast<const uint8_t *>(a.cfg_in) + (size_t)src * CB);
    for (int k = tid; k < CB / 4; k += MT) reinterpret_cast<uint32_t *>(occ)[k] = in[k];
    __syncthreads();
    // an occupation above n_max is flagged and clamped (W1 has n_max + 1
    // columns per site)
    for (int k = tid; k < m.N; k += MT)
      if (occ[k] > m.n_max) {
        atomicOr(a.status, ST_BAD_CONFIG);
        occ[k] = (uint8_t)m.n_max;
      }
    __syncthreads();
    // z1 of the configuration: b1 + the W1 columns of its occupations
    if (j2 < H1) {
      float zx = t.b1[j2], zy = t.b1[j2 + 1];
      for (int k = 0; k < m.N; ++k) {
        const __nv_bfloat162 w = *reinterpret_cast<const __nv_bfloat162 *>(
            t.W1T + (size_t)(k * np1 + occ[k]) * H1 + j2);
        zx += __low2float(w);
        zy += __high2float(w);
      }
      z1[j2] = zx;
      z1[j2 + 1] = zy;
    }
    __syncthreads();
    if (!tile(0, true, 0.0f)) { ok = false; break; }
    float lpx = bf[0];

    const Key kw = fold(a.key, (uint32_t)(a.walker_offset + walker));
    double lw = 0.0;
    float eloc = 0.0f;
    int hops = 0;
    if (a.method == CONT_TIME) {
      const float beta = (float)a.step;
      float tcur = 0.0f;
      uint32_t it = 0;
      while (tcur < beta) {
        for (int tb = 0; tb < m.n_off && ok; tb += MT) ok = tile(tb, false, lpx);
        if (!ok) break;
        diag();
        __syncthreads();
        if (tid == 0) {
          // cumulative weights -rates in move order; evolution.sample_index:30-59
          float R = 0.0f;
          for (int o = 0; o < m.n_off; ++o) R += -rates[o];
          const float U1 = uniform<float>(fold(kw, 2u * it));
          const float psi = uniform<float>(fold(kw, 2u * it + 1u));
          int si = 0;
          if (R > 0.0f) {
            float u = U1 * R;
            const float cap = nextafterf(R, 0.0f);
            u = u < cap ? u : cap;
            float c = 0.0f;
            int hit = m.n_off - 1;
            for (int o = 0; o < m.n_off; ++o) {
              c += -rates[o];
              if (c > u) { hit = o; break; }
            }
            si = hit;
            for (int o = hit; o >= 0; --o)
              if (-rates[o] > 0.0f) { si = o; break; }
          }
          const float tau_raw = R > 0.0f ? -log1pf(-psi) / R : __int_as_float(0x7F800000);
          const float rem = beta - tcur;
          bi[1] = (tau_raw < rem) ? 1 : 0;
          bi[2] = si;
          bf[1] = tau_raw < rem ? tau_raw : rem;
          bf[0] = bf[3] - R;
        }
        __syncthreads();
        const float tau = bf[1], eL = bf[0];
        const int hop = bi[1], si = bi[2];
        lw = lw - (double)eL * (double)tau;
        tcur = tcur + tau;
        if (hop) {
          const Mv mv = mlp_move(m, occ, si);
          if (j2 < H1) {
            const float2 zn = z1_moved(t, occ, mv, np1, make_float2(z1[j2], z1[j2 + 1]), j2);
            z1[j2] = zn.x;
            z1[j2 + 1] = zn.y;
          }
          lpx = lps[si];
          __syncthreads();
          if (tid == 0) {
            occ[mv.a] = (uint8_t)(occ[mv.a] + mv.da);
            if (mv.b != mv.a) occ[mv.b] = (uint8_t)(occ[mv.b] + mv.db);
          }
          ++hops;
        }
        eloc = eL;
        __syncthreads();
        if (++it >= (uint32_t)a.max_iters) {
          if (tid == 0) atomicOr(a.status, ST_HOP_CAP);
          break;
        }
      }
      lw -= a.alw * a.step;
    } else {   // EVALUATE: E_L = H_xx + sum of the guided off-diagonal elements
      for (int tb = 0; tb < m.n_off && ok; tb += MT) ok = tile(tb, false, lpx);
      if (!ok) break;
      diag();
      __syncthreads();
      if (tid == 0) {
        float s = 0.0f;
        for (int o = 0; o < m.n_off; ++o) s += rates[o];
        bf[0] = bf[3] + s;
      }
      __syncthreads();
      eloc = bf[0];
      if (tid == 0 && a.diag_out) a.diag_out[walker] = (double)bf[3];
    }
    if (!ok) break;
    if (a.cfg_out) {
      uint32_t *out = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(a.cfg_out) +
                                                   (size_t)walker * CB);
      for (int k = tid; k < CB / 4; k += MT) out[k] = reinterpret_cast<const uint32_t *>(occ)[k];
    }
    if (tid == 0) {
      if (a.method == CONT_TIME) a.log_w[walker] = lw;
      a.e_loc[walker] = (double)eloc;
    }
    if (a.method == CONT_TIME) wmax = lw > wmax ? lw : wmax;
    hop_acc += (unsigned long long)hops;
    __syncthreads();
  }
  if (!ok && tid == 0) atomicOr(a.status, ST_TIMEOUT);
  if (tid == 0) {
    if (a.partial_max) a.partial_max[blockIdx.x] = wmax;
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

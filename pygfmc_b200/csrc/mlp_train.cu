// Variance minimisation of the MLP guide on GFMC walkers (no PyGFMC
// counterpart).
//
// Loss and gradient as for the RBM guide: with rows r = every walker's
// connected configurations x'_s (coefficient c = g_w r_ws) and a base row per
// walker (x_w, c = -g_w R_w), g_w = 2 omega_w (e_w - E) / sum omega,
//   dL/dp = sum_r c_r O_p(x_r),  O = d log psi / dp.
// For log psi = w3 . h2 + b3, h2 = tanh(W2 h1 + b2), h1 = bf16(tanh(W1 x + b1))
// (the rounding passed straight through):
//   d2_r = c_r w3 (1 - h2_r^2)               dw3 = sum c_r h2_r,  db2 = sum d2_r
//          (a bf16 pair hi + lo as the tensor-core operand: a walker's rows
//          have coefficients summing to zero, and the sums below cancel)
//   dW2  = sum_r d2_r h1_r^T                 (tensor cores, K = rows)
//   d1_r = (W2^T d2_r) (1 - t1_r^2)          (tensor cores, K = H2), db1 = sum d1_r
//          (t1 = tanh(W1 x + b1) before the rounding, kept as h1 + its bf16
//          residual: the straight-through derivative)
//   dW1  = sum_r d1_r x_r^T                  (x one-hot: per walker, its N
//          columns get sum_r d1_r, each move row adds d1_r at the columns it
//          enters and subtracts it at the columns it leaves)
//
// Kernels (one training step): mlp_rows_kernel (row coefficients and h1 rows,
// row-major and transposed), mlp_gemm_kernel three times (the second layer
// forward with the d2 epilogue; d2 W2 with the d1 epilogue; d2^T h1 into dW2),
// mlp_dw1_kernel (the one-hot layer in shared memory), then Adam on float32
// master parameters and the guide's bf16 tables rewritten.
//
// mlp_gemm_kernel: C(M x N) = A(M x K) B(N x K)^T, A and B bf16 K-major in
// global memory, 128 threads, M tile 128 (TMEM lanes), N <= 256 (TMEM
// columns), K in chunks of 64 staged by cp.async into the 128-byte swizzled
// layout through a three-stage ring; thread 0 issues tcgen05.mma (kind::f16)
// per chunk and commits to the stage's mbarrier.  B stays resident in shared
// memory when it fits (the second-layer weights); every wait is bounded.
#include <cfloat>
#include <cuda_bf16.h>

#include "mlp.cuh"
#include "mlp_dev.cuh"
#include "tc05.cuh"

namespace gfmc {
namespace {

using namespace tc;
using namespace mlpdev;

constexpr int GT = 128;          // GEMM threads = M tile
constexpr int GSTAGES = 3;
constexpr int RB = 64;           // rows per block of the rows kernel
constexpr unsigned FULLW = 0xffffffffu;

__device__ __forceinline__ void cp16(void *dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND> __device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

__device__ __forceinline__ float tanh_k(float y) { return fmaf(-2.0f, sig2(KT * y), 1.0f); }

// 32 values per lane -> lane l holds the sum over the warp's lanes of value l
// (reduce-scatter in 31 shuffles).
__device__ __forceinline__ float reduce_scatter32(float (&v)[32], int lane) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool up = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < off; ++i) {
      const float send = up ? v[i] : v[i + off];
      const float keep = up ? v[i + off] : v[i];
      v[i] = keep + __shfl_xor_sync(FULLW, send, off);
    }
  }
  return v[0];
}

// ---- rows: coefficients and first-layer activations ------------------------
// Row r = w (n_off + 1) + s: s < n_off the move s of walker w, s = n_off the
// walker itself; rows past n (n_off + 1) up to Mpad are zero.  One block of
// 256 threads per 64 rows: threads 0..63 decode the rows (coefficient, the
// W1 columns the move exchanges, also written to rowcols for the one-hot
// layer); the z1 of each walker the block spans is built once in shared
// memory (thread i < H1 owns hidden unit i); the rows then go four at a
// time, their column loads issued together.
constexpr int RWMAX = 8;         // walkers one 64-row block can span (rows per walker >= 9)

__global__ void __launch_bounds__(256) mlp_rows_kernel(DevModel<float> m, MlpTables t,
                                                       const uint8_t *cfg, int CB, int n,
                                                       long long Mpad, const float *rates,
                                                       const float *rsum, const float *gw,
                                                       float *coef, int4 *rowcols,
                                                       __nv_bfloat16 *h1, __nv_bfloat16 *h1lo,
                                                       __nv_bfloat16 *h1T) {
  extern __shared__ unsigned char rsm[];
  __nv_bfloat16 *T = reinterpret_cast<__nv_bfloat16 *>(rsm);              // (H1, RB)
  float *zs = reinterpret_cast<float *>(rsm + (size_t)t.H1 * RB * 2);     // (RWMAX, H1)
  int4 *rcol = reinterpret_cast<int4 *>(zs + (size_t)RWMAX * t.H1);       // (RB,)
  int *rw = reinterpret_cast<int *>(rcol + RB);                           // (RB,) walker slot or -1
  const int H1 = t.H1, np1 = t.np1, rpw = m.n_off + 1;
  const long long r0 = (long long)blockIdx.x * RB;
  const long long R = (long long)n * rpw;
  const int tid = threadIdx.x;
  const int wfirst = (int)(r0 / rpw);
  if (tid < RB) {
    const long long r = r0 + tid;
    int w = -1;
    int4 c = make_int4(-1, -1, -1, -1);
    float co = 0.0f;
    if (r < R) {
      w = (int)(r / rpw);
      const int s = (int)(r - (long long)w * rpw);
      const uint8_t *occ = cfg + (size_t)w * CB;
      if (s == m.n_off) {
        co = -gw[w] * rsum[w];
      } else {
        const Mv mv = mlp_move(m, occ, s);
        if (mv.v != 0.0f) {
          c = move_cols(mv, occ, np1);
          co = gw[w] * rates[(size_t)w * m.n_off + s];
        } else {
          w = -1;             // no element: a zero row
        }
      }
    }
    coef[r] = co;
    rowcols[r] = c;
    rcol[tid] = c;
    rw[tid] = w >= 0 ? w - wfirst : -1;
  }
  // z1 of the walkers this block spans
  long long rl = r0 + RB - 1;
  if (rl > R - 1) rl = R - 1;
  const int nwb = r0 < R ? (int)(rl / rpw) - wfirst + 1 : 0;
  if (tid < H1) {
    for (int wi = 0; wi < nwb; ++wi) {
      const uint8_t *occ = cfg + (size_t)(wfirst + wi) * CB;
      float z = t.b1[tid];
#pragma unroll 8
      for (int k = 0; k < m.N; ++k) {
        const int o = occ[k] <= m.n_max ? occ[k] : m.n_max;   // (packed occupations are checked)
        z += __bfloat162float(t.W1T[(size_t)(k * np1 + o) * H1 + tid]);
      }
      zs[(size_t)wi * H1 + tid] = z;
    }
  }
  __syncthreads();
  if (tid < H1) {
    for (int rr0 = 0; rr0 < RB; rr0 += 4) {
      float w1v[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int4 c = rcol[rr0 + u];
        const bool on = rw[rr0 + u] >= 0 && c.x >= 0;
        w1v[u][0] = on ? __bfloat162float(t.W1T[(size_t)c.y * H1 + tid]) : 0.0f;
        w1v[u][1] = on ? __bfloat162float(t.W1T[(size_t)c.x * H1 + tid]) : 0.0f;
        const bool onb = on && c.z >= 0;
        w1v[u][2] = onb ? __bfloat162float(t.W1T[(size_t)c.w * H1 + tid]) : 0.0f;
        w1v[u][3] = onb ? __bfloat162float(t.W1T[(size_t)c.z * H1 + tid]) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int rr = rr0 + u, wi = rw[rr];
        __nv_bfloat16 hv = __float2bfloat16_rn(0.0f), lv = hv;
        if (wi >= 0) {
          float z = zs[(size_t)wi * H1 + tid];
          // ((z + new a) - old a), then b: the step kernel's order
          z = (z + w1v[u][0]) - w1v[u][1];
          z = (z + w1v[u][2]) - w1v[u][3];
          const float th = tanh_h1(z);   // the step kernel's first-layer activation
          hv = __float2bfloat16_rn(th);
          lv = __float2bfloat16_rn(th - __bfloat162float(hv));
        }
        h1[(size_t)(r0 + rr) * H1 + tid] = hv;
        h1lo[(size_t)(r0 + rr) * H1 + tid] = lv;
        T[(size_t)tid * RB + rr] = hv;
      }
    }
  }
  __syncthreads();
  if (tid < H1) {
    const uint4 *src = reinterpret_cast<const uint4 *>(T + (size_t)tid * RB);
    uint4 *dst = reinterpret_cast<uint4 *>(h1T + (size_t)tid * Mpad + r0);
#pragma unroll
    for (int k = 0; k < RB / 8; ++k) dst[k] = src[k];
  }
}

// ---- the tensor-core GEMM ----------------------------------------------------
struct GemmSmem {
  size_t B, A, red, bar, total;
  int bres;
};

__host__ __device__ inline GemmSmem gemm_plan(int N, int kb, int mode) {
  GemmSmem p;
  size_t o = 0;
  p.bres = (mode != MLP_EPI_ACC && (size_t)N * kb * 2 <= 128 * 1024) ? 1 : 0;
  p.B = o; o += p.bres ? (size_t)N * kb * 2 : (size_t)GSTAGES * N * 128;
  p.A = o; o += (size_t)GSTAGES * GT * 128;
  p.red = o; o += 2 * 256 * 4;
  p.bar = o; o += 64;
  p.total = o;
  return p;
}

__global__ void __launch_bounds__(GT, 1) mlp_gemm_kernel(MlpGemmArgs g) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int N = g.N;
  const int kb = g.kb > 0 ? g.kb : g.K, nkb = kb / 64;
  const GemmSmem P = gemm_plan(N, kb, g.mode);
  unsigned char *Bs = base + P.B;
  unsigned char *As = base + P.A;
  float *red0 = reinterpret_cast<float *>(base + P.red);
  float *red1 = red0 + 256;
  uint64_t *bar = reinterpret_cast<uint64_t *>(base + P.bar);   // GSTAGES + done
  uint64_t *done = bar + GSTAGES;
  uint32_t *slot = reinterpret_cast<uint32_t *>(done + 1);
  volatile int *flag = reinterpret_cast<volatile int *>(slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
  const int nk_all = g.K / 64;
  const int mtiles = (g.M + GT - 1) / GT;

  for (int j = tid; j < 512; j += GT) red0[j] = 0.0f;
  if (warp == 0) tmem_alloc(slot, ncols);
  if (tid == 0) {
    for (int k = 0; k <= GSTAGES; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (P.bres) {
    // B (N x K) resident: K chunk kc holds the N rows, 128 bytes each
    for (int q = tid; q < N * (kb / 8); q += GT) {
      const int n = q / (kb / 8), gq = q % (kb / 8);
      const int kc = gq >> 3, c = gq & 7;
      cp16(sw_chunk(Bs + (size_t)kc * N * 128, n, c), g.B + (size_t)n * g.ldb + 8 * gq, true);
    }
    cp_commit();
    cp_wait<0>();
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t idesc = idesc_m128((uint32_t)N);

  // chunk x (running sequence over this CTA's tiles) of tile m0, K chunk kc
  auto issue = [&](long long x, int m0, int kc) {
    const int st = (int)(x % GSTAGES);
    unsigned char *Ad = As + (size_t)st * GT * 128;
    for (int q = tid; q < GT * 8; q += GT) {
      const int r = q >> 3, c = q & 7;
      const int row = m0 + r;
      const bool v = row < g.M;
      cp16(sw_chunk(Ad, r, c), g.A + (size_t)(v ? row : 0) * g.lda + (size_t)kc * 64 + 8 * c, v);
    }
    if (!P.bres) {
      unsigned char *Bd = Bs + (size_t)st * N * 128;
      for (int q = tid; q < N * 8; q += GT) {
        const int n = q >> 3, c = q & 7;
        cp16(sw_chunk(Bd, n, c), g.B + (size_t)n * g.ldb + (size_t)(kc % nkb) * 64 + 8 * c, true);
      }
    }
  };

  bool ok = true;
  long long x0 = 0;        // chunks issued by earlier tiles
  uint32_t dphase = 0;
  const bool acc_mode = g.mode == MLP_EPI_ACC;
  const int t_first = acc_mode ? blockIdx.x : blockIdx.x;
  const int t_step = acc_mode ? mtiles : gridDim.x;
  for (int tile = t_first; tile < mtiles && ok; tile += t_step) {
    const int m0 = tile * GT;
    int kc0 = 0, nk = nk_all;
    if (acc_mode) {
      kc0 = blockIdx.y * g.kchunks_per_cta;
      nk = nk_all - kc0 < g.kchunks_per_cta ? nk_all - kc0 : g.kchunks_per_cta;
      if (nk <= 0) break;
    }
    for (int p = 0; p < GSTAGES - 1; ++p) {
      if (p < nk) issue(x0 + p, m0, kc0 + p);
      cp_commit();
    }
    for (int c = 0; c < nk; ++c) {
      const long long xn = x0 + c + GSTAGES - 1;
      if (c + GSTAGES - 1 < nk) {
        // the stage of chunk xn last held chunk xn - GSTAGES (the previous
        // iteration's): its MMAs must be done
        if (xn >= GSTAGES &&
            !cta_wait(bar + (xn % GSTAGES), (uint32_t)((xn / GSTAGES - 1) & 1), flag)) {
          ok = false;
          break;
        }
        issue(xn, m0, kc0 + c + GSTAGES - 1);
      }
      cp_commit();
      cp_wait<GSTAGES - 1>();
      fence_async_smem();
      __syncthreads();
      const long long xc = x0 + c;
      const int st = (int)(xc % GSTAGES);
      if (tid == 0) {
        fence_after();
        const uint32_t a0 = smem_u32(As + (size_t)st * GT * 128);
        const uint32_t b0 =
            smem_u32(Bs + (P.bres ? (size_t)((kc0 + c) % nkb) * N * 128 : (size_t)st * N * 128));
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          mma_bf16(tmem, sw128_desc(a0 + 32u * kk), sw128_desc(b0 + 32u * kk), idesc,
                   (c > 0 || kk > 0) ? 1u : 0u);
        mma_commit(bar + st);
        if (c == nk - 1) mma_commit(done);
      }
    }
    if (!ok) break;
    x0 += nk;
    if (!cta_wait(done, dphase, flag)) {
      ok = false;
      break;
    }
    dphase ^= 1u;
    fence_after();
    // ---- epilogue: warp w holds rows m0 + 32 w + lane
    const int lr = 32 * warp + lane;
    const long long row = (long long)m0 + lr;
    const bool valid = row < g.M;
    const uint32_t tl = tmem + ((uint32_t)(32 * warp) << 16);
    if (g.mode == MLP_EPI_FWD) {
      const float cr = valid ? g.coef[row] : 0.0f;
      for (int j0 = 0; j0 < N; j0 += 32) {
        uint32_t v[32];
        tmem_ld32_async(tl + (uint32_t)j0, v);
        tmem_ld_wait(v);
        float p[32], q[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const float h2 = tanh_k(__uint_as_float(v[i]) + __ldg(g.b2 + j0 + i));
          const float d = cr * (__ldg(g.w3 + j0 + i) * (1.0f - h2 * h2));
          p[i] = cr * h2;
          q[i] = d;
        }
        if (valid) {
          // d2 as hi + lo: [hi | lo] in the row, [hi^T | lo^T] in the column
          uint32_t ph[16], pl[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const __nv_bfloat162 hb = __floats2bfloat162_rn(q[2 * i], q[2 * i + 1]);
            const __nv_bfloat162 lb = __floats2bfloat162_rn(q[2 * i] - __low2float(hb),
                                                            q[2 * i + 1] - __high2float(hb));
            ph[i] = *reinterpret_cast<const uint32_t *>(&hb);
            pl[i] = *reinterpret_cast<const uint32_t *>(&lb);
          }
          uint4 *dh = reinterpret_cast<uint4 *>(g.d2 + (size_t)row * 2 * N + j0);
          uint4 *dl = reinterpret_cast<uint4 *>(g.d2 + (size_t)row * 2 * N + N + j0);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            dh[i] = make_uint4(ph[4 * i], ph[4 * i + 1], ph[4 * i + 2], ph[4 * i + 3]);
            dl[i] = make_uint4(pl[4 * i], pl[4 * i + 1], pl[4 * i + 2], pl[4 * i + 3]);
          }
          const unsigned short *hs = reinterpret_cast<const unsigned short *>(ph);
          const unsigned short *ls = reinterpret_cast<const unsigned short *>(pl);
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            unsigned short *col = reinterpret_cast<unsigned short *>(g.d2T + (size_t)(j0 + i) * g.ldT);
            col[row] = hs[i];
            col[g.M + row] = ls[i];
          }
        }
        const float sp = reduce_scatter32(p, lane);
        const float sq = reduce_scatter32(q, lane);
        atomicAdd(red0 + j0 + lane, sp);
        atomicAdd(red1 + j0 + lane, sq);
      }
    } else if (g.mode == MLP_EPI_BWD) {
      // the row's h1 and residual of the next 32 columns load while this
      // chunk is formed (the loads are the epilogue's latency)
      uint4 hn[4], ln[4];
      if (valid) {
        const uint4 *hs = reinterpret_cast<const uint4 *>(g.h1 + (size_t)row * N);
        const uint4 *ls = reinterpret_cast<const uint4 *>(g.h1lo + (size_t)row * N);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          hn[k] = hs[k];
          ln[k] = ls[k];
        }
      }
      for (int j0 = 0; j0 < N; j0 += 32) {
        uint32_t v[32];
        tmem_ld32_async(tl + (uint32_t)j0, v);
        uint4 hc[4], lc[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          hc[k] = hn[k];
          lc[k] = ln[k];
        }
        if (valid && j0 + 32 < N) {
          const uint4 *hs = reinterpret_cast<const uint4 *>(g.h1 + (size_t)row * N + j0 + 32);
          const uint4 *ls = reinterpret_cast<const uint4 *>(g.h1lo + (size_t)row * N + j0 + 32);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            hn[k] = hs[k];
            ln[k] = ls[k];
          }
        }
        tmem_ld_wait(v);
        float d[32];
        if (valid) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            float f[8], fl[8];
            bf8(hc[k], f);
            bf8(lc[k], fl);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const float t1 = f[e] + fl[e];
              d[8 * k + e] = __uint_as_float(v[8 * k + e]) * (1.0f - t1 * t1);
            }
          }
          float4 *dst = reinterpret_cast<float4 *>(g.d1 + (size_t)row * N + j0);
#pragma unroll
          for (int k = 0; k < 8; ++k) dst[k] = make_float4(d[4 * k], d[4 * k + 1], d[4 * k + 2], d[4 * k + 3]);
        } else {
#pragma unroll
          for (int i = 0; i < 32; ++i) d[i] = 0.0f;
        }
        const float sd = reduce_scatter32(d, lane);
        atomicAdd(red0 + j0 + lane, sd);
      }
    } else {
      for (int j0 = 0; j0 < N; j0 += 32) {
        uint32_t v[32];
        tmem_ld32_async(tl + (uint32_t)j0, v);
        tmem_ld_wait(v);
        if (valid) {
          float *out = g.C + (size_t)row * g.ldc + j0;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float f = __uint_as_float(v[i]);
            if (f != 0.0f) atomicAdd(out + i, f);
          }
        }
      }
    }
    fence_before();
    __syncthreads();
  }
  cp_wait<0>();
  if (!ok && tid == 0) atomicOr(g.status, ST_TIMEOUT);
  __syncthreads();
  if (ok && g.mode == MLP_EPI_FWD) {
    for (int j = tid; j < N; j += GT) {
      if (red0[j] != 0.0f) atomicAdd(g.g_w3 + j, red0[j]);
      if (red1[j] != 0.0f) atomicAdd(g.g_b2 + j, red1[j]);
    }
  } else if (ok && g.mode == MLP_EPI_BWD) {
    for (int j = tid; j < N; j += GT)
      if (red0[j] != 0.0f) atomicAdd(g.g_b1 + j, red0[j]);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// ---- the one-hot layer ---------------------------------------------------------
// Block (walker block, quarter of 64 hidden units): 4 groups of 64 threads,
// group g takes the block's walkers w = g (mod 4); thread t owns unit
// 64 q + t and accumulates its column of dW1 (D = N (n_max + 1) inputs) in
// shared memory; one global add per nonzero at the end.
__global__ void __launch_bounds__(256) mlp_dw1_kernel(DevModel<float> m, MlpTables t,
                                                      const uint8_t *cfg, int CB, int n,
                                                      int walkers_per_block, const float *d1,
                                                      const int4 *rowcols, float *gW1) {
  extern __shared__ float dacc[];   // (D, 64)
  const int H1 = t.H1, np1 = t.np1, D = m.N * np1, rpw = m.n_off + 1;
  const int tid = threadIdx.x, grp = tid >> 6, tt = tid & 63;
  const int unit = blockIdx.y * 64 + tt;
  for (int k = tid; k < D * 64; k += 256) dacc[k] = 0.0f;
  __syncthreads();
  const int w0 = blockIdx.x * walkers_per_block;
  const int w1 = min(w0 + walkers_per_block, n);
  for (int w = w0 + grp; w < w1; w += 4) {
    const uint8_t *occ = cfg + (size_t)w * CB;
    const float *dr = d1 + (size_t)w * rpw * H1 + unit;
    float S = 0.0f;
    // four rows per pass: their d1 values and decoded columns are loaded
    // together before they are used (S still adds the rows in order)
    for (int sl0 = 0; sl0 < rpw; sl0 += 4) {
      float d4[4];
      int4 c4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int sl = sl0 + q;
        d4[q] = sl < rpw ? dr[(size_t)sl * H1] : 0.0f;
        c4[q] = sl < m.n_off ? rowcols[(size_t)w * rpw + sl]   // the rows kernel's decode
                             : make_int4(-1, -1, -1, -1);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float d = d4[q];
        const int4 c = c4[q];
        S += d;
        // (c.x < 0: no element, its columns may not exist)
        if (d != 0.0f && c.x >= 0) {
          atomicAdd(dacc + (size_t)c.y * 64 + tt, d);
          atomicAdd(dacc + (size_t)c.x * 64 + tt, -d);
          if (c.z >= 0) {
            atomicAdd(dacc + (size_t)c.w * 64 + tt, d);
            atomicAdd(dacc + (size_t)c.z * 64 + tt, -d);
          }
        }
      }
    }
    if (S != 0.0f)
      for (int k = 0; k < m.N; ++k) {
        const int o = occ[k] <= m.n_max ? occ[k] : m.n_max;
        atomicAdd(dacc + (size_t)(k * np1 + o) * 64 + tt, S);
      }
  }
  __syncthreads();
  for (int k = tid; k < D * 64; k += 256) {
    const float v = dacc[k];
    if (v != 0.0f) atomicAdd(gW1 + (size_t)(blockIdx.y * 64 + (k & 63)) * D + (k >> 6), v);
  }
}

// ---- Adam and the guide's tables ------------------------------------------------
__global__ void mlp_adam_kernel(long long np, float *p, const float *gr, float *m1, float *m2,
                                float lr, float b1, float b2, float eps, float c1, float c2) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < np;
       k += (long long)gridDim.x * blockDim.x) {
    const float gk = gr[k];
    const float a = b1 * m1[k] + (1.0f - b1) * gk;
    const float v = b2 * m2[k] + (1.0f - b2) * gk * gk;
    m1[k] = a;
    m2[k] = v;
    p[k] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
  }
}

// Master parameters (W1 (H1, D), b1, W2 (H2, H1), b2, w3) -> the guide's
// tables (W1T (D, H1), W2 (H2, H1), W2T (H1, H2) bf16; b1, b2; w3 rounded).
__global__ void mlp_tables_kernel(int H1, int H2, int D, const float *p, __nv_bfloat16 *W1T,
                                  float *b1, __nv_bfloat16 *W2, __nv_bfloat16 *W2T, float *b2,
                                  float *w3) {
  const float *W1 = p, *pb1 = p + (size_t)H1 * D, *pW2 = pb1 + H1, *pb2 = pW2 + (size_t)H2 * H1,
              *pw3 = pb2 + H2;
  const long long tot = (long long)H1 * D + (long long)H2 * H1 + H1 + 2 * H2;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    if (k < (long long)H1 * D) {
      const int i = (int)(k / D), c = (int)(k % D);
      W1T[(size_t)c * H1 + i] = __float2bfloat16_rn(W1[k]);
      continue;
    }
    long long q = k - (long long)H1 * D;
    if (q < (long long)H2 * H1) {
      const int j = (int)(q / H1), i = (int)(q % H1);
      const __nv_bfloat16 v = __float2bfloat16_rn(pW2[q]);
      W2[q] = v;
      W2T[(size_t)i * H2 + j] = v;
      continue;
    }
    q -= (long long)H2 * H1;
    if (q < H1) { b1[q] = pb1[q]; continue; }
    q -= H1;
    if (q < H2) { b2[q] = pb2[q]; continue; }
    q -= H2;
    w3[q] = __bfloat162float(__float2bfloat16_rn(pw3[q]));
  }
}

__global__ void mlp_master_init_kernel(int H1, int H2, int D, const __nv_bfloat16 *W1T,
                                       const float *b1, const __nv_bfloat16 *W2, const float *b2,
                                       const float *w3, float *p) {
  const long long tot = (long long)H1 * D + (long long)H2 * H1 + H1 + 2 * H2;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    if (k < (long long)H1 * D) {
      const int i = (int)(k / D), c = (int)(k % D);
      p[k] = __bfloat162float(W1T[(size_t)c * H1 + i]);
      continue;
    }
    long long q = k - (long long)H1 * D;
    if (q < H1) { p[k] = b1[q]; continue; }
    q -= H1;
    if (q < (long long)H2 * H1) { p[k] = __bfloat162float(W2[q]); continue; }
    q -= (long long)H2 * H1;
    if (q < H2) { p[k] = b2[q]; continue; }
    q -= H2;
    p[k] = w3[q];
  }
}

int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

long long mlp_param_count(int H1, int H2, int D) {
  return (long long)H1 * D + H1 + (long long)H2 * H1 + H2 + H2;
}

cudaError_t launch_mlp_rows(const DevModel<float> &m, const MlpTables &t, const void *cfg, int CB,
                            int n, long long Mpad, const float *rates, const float *rsum,
                            const float *gw, float *coef, int4 *rowcols, __nv_bfloat16 *h1,
                            __nv_bfloat16 *h1lo, __nv_bfloat16 *h1T, cudaStream_t s) {
  if (m.n_off + 1 < (RB + RWMAX - 2) / (RWMAX - 1)) return cudaErrorInvalidValue;
  const size_t smem = (size_t)t.H1 * RB * 2 + (size_t)RWMAX * t.H1 * 4 + RB * 16 + RB * 4;
  const long long blocks = Mpad / RB;
  mlp_rows_kernel<<<(unsigned)blocks, 256, smem, s>>>(m, t, reinterpret_cast<const uint8_t *>(cfg),
                                                      CB, n, Mpad, rates, rsum, gw, coef, rowcols,
                                                      h1, h1lo, h1T);
  return cudaGetLastError();
}

cudaError_t launch_mlp_gemm(const MlpGemmArgs &g, cudaStream_t s) {
  if (g.N < 32 || g.N > 256 || (g.N & 31) || (g.K & 63) || g.M <= 0)
    return cudaErrorInvalidValue;
  const int kb = g.kb > 0 ? g.kb : g.K;
  if ((kb & 63) || g.K % kb) return cudaErrorInvalidValue;
  const size_t smem = 1024 + gemm_plan(g.N, kb, g.mode).total;
  if (smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(mlp_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int mtiles = (g.M + GT - 1) / GT;
  dim3 grid;
  MlpGemmArgs a = g;
  if (g.mode == MLP_EPI_ACC) {
    const int nk = g.K / 64;
    int parts = (2 * sm_count() + mtiles - 1) / mtiles;
    if (parts > nk) parts = nk;
    if (parts < 1) parts = 1;
    a.kchunks_per_cta = (nk + parts - 1) / parts;
    parts = (nk + a.kchunks_per_cta - 1) / a.kchunks_per_cta;
    grid = dim3(mtiles, parts);
  } else {
    const int sms = sm_count();
    grid = dim3(mtiles < sms ? mtiles : sms, 1);
  }
  mlp_gemm_kernel<<<grid, GT, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_mlp_dw1(const DevModel<float> &m, const MlpTables &t, const void *cfg, int CB,
                           int n, const float *d1, const int4 *rowcols, float *gW1, cudaStream_t s) {
  const int D = m.N * t.np1;
  const size_t smem = (size_t)D * 64 * 4;
  if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaFuncSetAttribute(mlp_dw1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int quarters = t.H1 / 64;
  int wpb = (int)((long long)n * quarters / (2 * sm_count()) + 1);
  if (wpb < 4) wpb = 4;
  const int blocks = (n + wpb - 1) / wpb;
  mlp_dw1_kernel<<<dim3(blocks, quarters), 256, smem, s>>>(
      m, t, reinterpret_cast<const uint8_t *>(cfg), CB, n, wpb, d1, rowcols, gW1);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(long long np, float *p, const float *g, float *m1, float *m2, float lr,
                            int step, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  mlp_adam_kernel<<<1024, 256, 0, s>>>(np, p, g, m1, m2, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_mlp_tables(const MlpTables &t, int D, const float *p, __nv_bfloat16 *W1T, float *b1,
                              __nv_bfloat16 *W2, __nv_bfloat16 *W2T, float *b2, float *w3,
                              cudaStream_t s) {
  mlp_tables_kernel<<<1024, 256, 0, s>>>(t.H1, t.H2, D, p, W1T, b1, W2, W2T, b2, w3);
  return cudaGetLastError();
}

cudaError_t launch_mlp_master_init(const MlpTables &t, int D, float *p, cudaStream_t s) {
  mlp_master_init_kernel<<<1024, 256, 0, s>>>(t.H1, t.H2, D, t.W1T, t.b1, t.W2, t.b2, t.w3, p);
  return cudaGetLastError();
}

}  // namespace gfmc

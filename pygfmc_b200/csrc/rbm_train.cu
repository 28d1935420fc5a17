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
// rbm_grad_kernel: one CTA per (128-unit hidden tile, block of walkers).
// Each 64-row chunk: 64 threads decode the rows (sites, coefficient, spins)
// into shared memory; every thread then produces its hidden unit's 64 values
// of U (tanh.approx of theta' built from the staged W^T tile) as bf16 into the
// swizzled K-major A tile, and two site rows of V (+-1 as bf16) into the B
// tile; thread 0 issues tcgen05.mma (M = 128 hidden, N = sites, K = 64 rows)
// accumulating dL/dW of the tile in TMEM.  Two stages: the MMAs of one chunk
// run while the next is produced.  The epilogue adds the tile into the global
// float32 gradient (atomics; one CTA per walker block and tile).
#include <cuda_bf16.h>

#include "rbm.cuh"

namespace gfmc {
namespace {

constexpr int TT = 128;     // threads = hidden units per tile = UMMA M
constexpr int KR = 64;      // rows per chunk = UMMA K per chunk
constexpr uint32_t WAIT_LIMIT = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// CTA-uniform bounded wait: thread 0 waits, every thread gets its verdict
// (so all threads leave or stay in the loops together).
__device__ __forceinline__ bool cta_wait(uint64_t *bar, uint32_t parity, volatile int *flag) {
  if (threadIdx.x == 0) *flag = mbar_wait(bar, parity) ? 1 : 0;
  __syncthreads();
  const bool r = *flag != 0;
  __syncthreads();
  return r;
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// D f32, A and B bf16, K-major, M = 128, N = n (multiple of 16, <= 256).
__device__ __forceinline__ uint32_t idesc_n(uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ unsigned char *sw_chunk(unsigned char *tile, int r, int c) {
  return tile + (size_t)r * 128 + (size_t)((c ^ (r & 7)) * 16);
}

__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&p);
}

}  // namespace



namespace {

__global__ void __launch_bounds__(TT, 1) rbm_grad_kernel(GradArgs g) {
  extern __shared__ unsigned char dsm[];
  unsigned char *base = (unsigned char *)(((uintptr_t)dsm + 1023) & ~(uintptr_t)1023);
  const int Np = g.Np;
  unsigned char *Ast[2], *Bst[2];
  Ast[0] = base;                                  // 128 x 64 bf16 = 16 KB
  Ast[1] = base + 16384;
  Bst[0] = base + 32768;                          // Np x 64 bf16
  Bst[1] = Bst[0] + (size_t)Np * 128;
  __nv_bfloat16 *WTs = reinterpret_cast<__nv_bfloat16 *>(Bst[1] + (size_t)Np * 128);  // (Np, 128)
  float *acc_a = reinterpret_cast<float *>(WTs + (size_t)Np * TT);                      // (Np,)
  int *m_w = reinterpret_cast<int *>(acc_a + Np);                                      // rows
  int *m_i = m_w + KR;
  int *m_j = m_i + KR;
  float *m_c = reinterpret_cast<float *>(m_j + KR);
  uint64_t *bar = reinterpret_cast<uint64_t *>(((uintptr_t)(m_c + KR) + 7) & ~(uintptr_t)7);
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
  volatile int *flag = reinterpret_cast<volatile int *>(slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int h0 = blockIdx.x * TT;
  const int w0 = blockIdx.y * g.walkers_per_cta;
  int w1 = w0 + g.walkers_per_cta;
  if (w1 > g.n) w1 = g.n;
  const int rows_per_w = g.n_off + 1;
  const long long R0 = (long long)w0 * rows_per_w, R1 = (long long)w1 * rows_per_w;
  const int nchunks = R1 > R0 ? (int)((R1 - R0 + KR - 1) / KR) : 0;
  const uint32_t ncols = Np <= 32 ? 32u : (Np <= 64 ? 64u : (Np <= 128 ? 128u : (Np <= 256 ? 256u : 512u)));
  const bool do_a = blockIdx.x == 0;

  // stage the W^T tile (sites x 128 hidden) and clear the a accumulator
  for (int idx = tid; idx < Np * (TT / 8); idx += TT) {
    const int i = idx / (TT / 8), c = idx % (TT / 8);
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (i < g.N) v = __ldg(reinterpret_cast<const uint4 *>(g.WT + (size_t)i * g.Hp + h0) + c);
    reinterpret_cast<uint4 *>(WTs + (size_t)i * TT)[c] = v;
  }
  for (int i = tid; i < Np; i += TT) acc_a[i] = 0.0f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *slot;

  const int h = h0 + tid;   // this thread's hidden unit
  float acc_b = 0.0f;
  uint32_t cnt[2] = {0u, 0u};
  bool ok = true;
  int th_w = -1;
  float th_v = 0.0f;

  for (int ch = 0; ch < nchunks && ok; ++ch) {
    const int st = ch & 1;
    // the stage's previous MMAs must have read it
    if (cnt[st] > 0 && !cta_wait(&bar[st], (cnt[st] - 1u) & 1u, flag)) {
      if (tid == 0) atomicOr(g.status, 8);
      ok = false;
      break;
    }
    // ---- decode the chunk's rows
    if (tid < KR) {
      const long long r = R0 + (long long)ch * KR + tid;
      int w = -1, i = -1, j = -1;
      float c = 0.0f;
      if (r < R1) {
        w = (int)(r / rows_per_w);
        const int s = (int)(r - (long long)w * rows_per_w);
        if (s < g.n_off) {
          c = g.gw[w] * g.rates[(size_t)w * g.n_off + s];
          if (s < g.n_hx) {
            i = s;
          } else {
            const uint32_t pe = g.edge[s - g.n_hx];
            i = (int)(pe & 0xFFFF);
            j = (int)(pe >> 16);
          }
          if (do_a && c != 0.0f) {
            const uint64_t *x = g.cfg + (size_t)w * g.NW;
            const float si = ((x[i >> 6] >> (i & 63)) & 1ull) ? 1.0f : -1.0f;
            atomicAdd(&acc_a[i], -2.0f * c * si);
            if (j >= 0) {
              const float sj = ((x[j >> 6] >> (j & 63)) & 1ull) ? 1.0f : -1.0f;
              atomicAdd(&acc_a[j], -2.0f * c * sj);
            }
          }
        } else {
          c = -g.gw[w] * g.rsum[w];   // base row
        }
      }
      m_w[tid] = w;
      m_i[tid] = i;
      m_j[tid] = j;
      m_c[tid] = c;
    }
    __syncthreads();
    // ---- A: U[h, r] = c_r tanh(theta'_r,h), this thread's hidden row
    unsigned char *A = Ast[st];
#pragma unroll 1
    for (int cc = 0; cc < KR / 8; ++cc) {
      uint32_t q[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float u2[2];
#pragma unroll
        for (int t2 = 0; t2 < 2; ++t2) {
          const int rr = 8 * cc + 2 * e + t2;
          const int w = m_w[rr];
          const float c = m_c[rr];
          float u = 0.0f;
          if (w >= 0 && c != 0.0f) {
            if (w != th_w) {
              th_v = g.theta[(size_t)w * g.Hp + h];
              th_w = w;
            }
            float t = th_v;
            const int i = m_i[rr], j = m_j[rr];
            if (i >= 0) {
              const uint64_t *x = g.cfg + (size_t)w * g.NW;
              const float si = ((x[i >> 6] >> (i & 63)) & 1ull) ? 1.0f : -1.0f;
              t = t - 2.0f * si * __bfloat162float(WTs[(size_t)i * TT + tid]);
              if (j >= 0) {
                const float sj = ((x[j >> 6] >> (j & 63)) & 1ull) ? 1.0f : -1.0f;
                t = t - 2.0f * sj * __bfloat162float(WTs[(size_t)j * TT + tid]);
              }
            }
            u = c * tanh_approx(t);
            acc_b += u;
          }
          u2[t2] = u;
        }
        q[e] = bf16_pair(u2[0], u2[1]);
      }
      *reinterpret_cast<uint4 *>(sw_chunk(A, tid, cc)) = make_uint4(q[0], q[1], q[2], q[3]);
    }
    // ---- B: V[i, r] = s'_r,i for the sites i = tid, tid + 128, ...
    unsigned char *B = Bst[st];
    for (int i = tid; i < Np; i += TT) {
      int lw = -1;
      uint64_t word = 0;
#pragma unroll 1
      for (int cc = 0; cc < KR / 8; ++cc) {
        uint32_t q[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          uint32_t hv[2];
#pragma unroll
          for (int t2 = 0; t2 < 2; ++t2) {
            const int rr = 8 * cc + 2 * e + t2;
            const int w = m_w[rr];
            uint32_t v = 0u;
            if (w >= 0 && i < g.N) {
              if (w != lw) {
                word = g.cfg[(size_t)w * g.NW + (i >> 6)];
                lw = w;
              }
              bool up = ((word >> (i & 63)) & 1ull) != 0ull;
              if (i == m_i[rr] || i == m_j[rr]) up = !up;
              v = up ? 0x3F80u : 0xBF80u;
            }
            hv[t2] = v;
          }
          q[e] = hv[0] | (hv[1] << 16);
        }
        *reinterpret_cast<uint4 *>(sw_chunk(B, i, cc)) = make_uint4(q[0], q[1], q[2], q[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
      for (int sub = 0; sub * 256 < Np; ++sub) {
        const int nn = (Np - sub * 256) < 256 ? (Np - sub * 256) : 256;
        const uint32_t id = idesc_n((uint32_t)nn);
#pragma unroll
        for (int kk = 0; kk < KR / 16; ++kk)
          mma_bf16(tmem + (uint32_t)sub * 256u, sw128_desc(a0 + 32u * kk),
                   sw128_desc(b0 + (uint32_t)sub * 256u * 128u + 32u * kk), id,
                   (ch > 0 || kk > 0) ? 1u : 0u);
      }
      mma_commit(&bar[st]);
    }
    cnt[st] += 1u;
  }
  // ---- the outstanding commits
  for (int st = 0; st < 2; ++st)
    if (ok && cnt[st] > 0 && !cta_wait(&bar[st], (cnt[st] - 1u) & 1u, flag)) {
      if (tid == 0) atomicOr(g.status, 8);
      ok = false;
    }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && nchunks > 0) {
    for (int c0 = 0; c0 < Np; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      float *out = g.grad_W + (size_t)(h0 + warp * 32 + (tid & 31)) * Np + c0;
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (v[k] != 0.0f) atomicAdd(out + k, v[k]);
    }
    atomicAdd(&g.grad_b[h], acc_b);
    if (do_a)
      for (int i = tid; i < Np; i += TT)
        if (acc_a[i] != 0.0f) atomicAdd(&g.grad_a[i], acc_a[i]);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols)
                 : "memory");
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

size_t rbm_grad_smem(int Np) {
  return 1024 + 32768 + 2 * (size_t)Np * 128 + (size_t)Np * TT * 2 + (size_t)Np * 4 + 4 * KR * 4 +
         64;
}

cudaError_t launch_rbm_grad(const GradArgs &a, int sms, cudaStream_t s) {
  const size_t smem = rbm_grad_smem(a.Np);
  cudaError_t e = cudaFuncSetAttribute(rbm_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int tiles = a.Hp / TT;
  int blocks = (2 * sms + tiles - 1) / tiles;
  if (blocks > a.n) blocks = a.n;
  if (blocks < 1) blocks = 1;
  GradArgs g = a;
  g.walkers_per_cta = (a.n + blocks - 1) / blocks;
  blocks = (a.n + g.walkers_per_cta - 1) / g.walkers_per_cta;
  rbm_grad_kernel<<<dim3(tiles, blocks), TT, smem, s>>>(g);
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

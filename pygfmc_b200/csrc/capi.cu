// C ABI of the engine (include/gfmc_b200.h): table construction, the host
// loop of a chunk of branching steps, and the small helpers around it.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/gfmc_b200.h"
#include "diag.cuh"
#include "fw.cuh"
#include "mlp.cuh"
#include "rbm.cuh"
#include "engine.cuh"

using namespace gfmc;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define GFMC_CUDA(expr)                                                                    \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return fail(GFMC_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(_e));          \
  } while (0)

// One device allocation holding every table; the builder appends arrays.
struct Arena {
  std::vector<unsigned char> host;
  size_t add(const void *p, size_t bytes) {
    size_t o = (host.size() + 255) & ~size_t(255);
    host.resize(o + bytes);
    if (bytes) memcpy(host.data() + o, p, bytes);
    return o;
  }
};

template <typename T> std::vector<T> conv(const double *src, size_t n) {
  std::vector<T> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = (T)src[i];
  return v;
}

}  // namespace

namespace gfmc {
// Records msg as the calling thread's gfmc_last_error message.
int record_error(int code, const char *msg) { return fail(code, "%s", msg); }
}  // namespace gfmc

struct gfmc_handle {
  int precision = 0;
  int family = 0;
  int max_iters = 1 << 22;
  int N = 0, E = 0, M = 0;
  int cfg_bytes = 0;
  int n_max = 0;
  void *d_tables = nullptr;
  DevModel<double> m64{};
  DevGuide<double> g64{};
  DevModel<float> m32{};
  DevGuide<float> g32{};
  LaunchPlan plan{};
  // scratch
  int cap_n = 0, cap_steps = 0;
  double *pmax = nullptr, *psum = nullptr, *pE = nullptr, *cdf = nullptr, *wbuf = nullptr;
  // grid-barrier counter of the one-launch resampling (grows by 2 tiles per
  // launch; rbase mirrors it) and the most tiles such a launch can hold
  unsigned *rctr = nullptr;
  unsigned rbase = 0;
  int fused_tiles = -1;
  int *plp = nullptr, *ctr = nullptr, *status = nullptr;
  unsigned long long *hops = nullptr;
  // carried guide fields (W / S per walker), double-buffered through the
  // parent map; rebuilt from scratch for a fresh population and every
  // refresh_every steps against rounding drift of the incremental updates
  int carry = 0;
  int refresh_every = 100;
  void *fbuf[2] = {nullptr, nullptr};
  int fcur = 0, field_valid = 0, since_refresh = 0;
  // evaluation records beside the carried fields (EvolveArgs::eval_in), plain
  // and Jastrow guides; eval_valid: ebuf[fcur] holds the last cont_time
  // step's records
  void *ebuf[2] = {nullptr, nullptr};
  int eval_valid = 0;
  int carry_optional = 0;   // carry chosen for speed only (the step can rebuild instead)
  int carry_pref = 0;       // the carry decision made at create
  int carry_mode = 1;       // gfmc_carry_mode: 1 carry the optional state when it fits, 0 rebuild
  const void *field_cfg = nullptr;
  int cap_field = 0;
  // diagonal observables (forward walking)
  DiagSet diag{};
  DiagOp *d_ops = nullptr;
  void *d_diag_tables = nullptr;
  int diag_cap_n = 0, diag_slot = 0, diag_ready = 0;
  double *diag_partial = nullptr;
  double *diag_out = nullptr;
  // RBM guide: bf16 weights (both layouts), biases; theta is the carried state
  int rbm_on = 0;
  RbmTables rbm{};
  void *d_rbm = nullptr;
  void *d_rbm_rt = nullptr, *d_rbm_ch = nullptr;   // the float32 RBM kernel's tables
  int rbm_grid = 0;
  int state_len = 0;     // carried state values per walker (N, or Hp for the RBM)
  // MLP guide (Bose-Hubbard, float32 build): bf16 layer weights, biases
  int mlp_on = 0;
  MlpTables mlp{};
  void *d_mlp = nullptr;
  int mlp_grid = 0;
  // MLP trainer: scratch sized for mtr_cap walkers / mtr_rows rows, float32
  // master parameters with their Adam moments, one gradient array
  int mtr_cap = 0;
  long long mtr_rows = 0;
  void *mtr_cfg = nullptr;
  float *mtr_rates = nullptr, *mtr_rsum = nullptr, *mtr_gw = nullptr, *mtr_coef = nullptr;
  double *mtr_e = nullptr, *mtr_stats = nullptr;
  __nv_bfloat16 *mtr_h1 = nullptr, *mtr_h1lo = nullptr, *mtr_h1T = nullptr, *mtr_d2 = nullptr,
                *mtr_d2T = nullptr;
  float *mtr_d1 = nullptr, *mtr_grad = nullptr, *mtr_p = nullptr, *mtr_m1 = nullptr,
        *mtr_m2 = nullptr;
  int4 *mtr_rowcols = nullptr;
  int mtr_step = 0;
  int mtr_ready = 0;   // MLP masters and Adam moments allocated and initialised
  // RBM variance-minimisation scratch (sized for train_cap walkers) and the
  // float32 master parameters with their Adam moments
  int train_cap = 0;
  uint64_t *tr_cfg = nullptr;
  float *tr_theta = nullptr, *tr_rates = nullptr, *tr_rsum = nullptr, *tr_gw = nullptr;
  double *tr_e = nullptr, *tr_stats = nullptr;
  float *tr_gW = nullptr, *tr_gb = nullptr, *tr_ga = nullptr;
  void *tr_recs = nullptr;
  // sharded reconfiguration: (max | S, S_e, last positive) on the device
  double *dist_out = nullptr;
  float *ms_W = nullptr, *ms_b = nullptr, *ms_a = nullptr, *ad_m = nullptr, *ad_v = nullptr;
  int adam_step = 0;
  int adam_ready = 0;  // RBM masters and Adam moments allocated and initialised
  // off-diagonal forward walking through this handle as the shadow chain
  FwHook *fw = nullptr;              // installed for the length of one walk
  int *ctr1 = nullptr;               // work counter of single launches (apply, min rate)
  double *fw_partial = nullptr, *fw_logG = nullptr, *fw_E = nullptr;
  int fw_cap_rows = 0, fw_cap_nb = 0;
};

namespace {

uint16_t bf16_bits(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);   // inf / nan kept
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);          // nearest, ties to even
}

// RBM tables: W rounded to bf16 in the site-major (N, Hp) and hidden-major
// (Hp, N) layouts, b and a in float; the hidden axis padded with zeros to a
// multiple of 256 (32 lanes x 8-element vector loads).
int build_rbm(gfmc_handle *h, const gfmc_model_desc *md, const gfmc_guide_desc *gd, int N) {
  const int H = gd->n_hidden;
  if (H < 1 || H > 1024) return fail(GFMC_ERR_INVALID, "n_hidden must be in [1, 1024], got %d", H);
  if (!gd->rbm_W || !gd->rbm_b || !gd->rbm_a)
    return fail(GFMC_ERR_INVALID, "RBM guide: rbm_W, rbm_b and rbm_a are required");
  const int Hp = ((H + 255) / 256) * 256;
  const int Np = ((N + 63) / 64) * 64;
  std::vector<uint16_t> WT((size_t)N * Hp, 0), W((size_t)Hp * Np, 0);
  std::vector<float> b(Hp, 0.0f), a(N);
  for (int hh = 0; hh < H; ++hh) {
    for (int i = 0; i < N; ++i) {
      const float w = gd->rbm_W[(size_t)hh * N + i];
      if (!std::isfinite(w)) return fail(GFMC_ERR_INVALID, "RBM weight (%d, %d) is not finite", hh, i);
      const uint16_t v = bf16_bits(w);
      WT[(size_t)i * Hp + hh] = v;
      W[(size_t)hh * Np + i] = v;
    }
    b[hh] = gd->rbm_b[hh];
  }
  for (int i = 0; i < N; ++i) a[i] = gd->rbm_a[i];
  const size_t sWT = WT.size() * 2, sW = W.size() * 2, sb = (size_t)Hp * 4, sa = (size_t)N * 4;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t oW = al(sWT), ob = oW + al(sW), oa = ob + al(sb), tot = oa + al(sa);
  std::vector<unsigned char> host(tot, 0);
  memcpy(host.data(), WT.data(), sWT);
  memcpy(host.data() + oW, W.data(), sW);
  memcpy(host.data() + ob, b.data(), sb);
  memcpy(host.data() + oa, a.data(), sa);
  GFMC_CUDA(cudaMalloc(&h->d_rbm, tot));
  GFMC_CUDA(cudaMemcpy(h->d_rbm, host.data(), tot, cudaMemcpyHostToDevice));
  unsigned char *base = (unsigned char *)h->d_rbm;
  h->rbm.WT = (const __nv_bfloat16 *)base;
  h->rbm.W = (const __nv_bfloat16 *)(base + oW);
  h->rbm.b = (const float *)(base + ob);
  h->rbm.a = (const float *)(base + oa);
  h->rbm.H = H;
  h->rbm.Hp = Hp;
  h->rbm.Np = Np;
  // the float32 kernel's derived tables (tanh(2 W) rows and the lanes'
  // log2 prod cosh(2 W)) and its slot chunks (rbm_f32.cu)
  const int n_hx = md->n_hx, n_edges = md->n_jpm ? md->n_edges : 0;
  const int M = 1 + n_hx + n_edges;
  const int U = rbm_chunk_sites(Hp, N, M);
  if (U < 2) return fail(GFMC_ERR_UNSUPPORTED, "RBM guide: %d moves exceed the shared memory of one SM", M - 1);
  h->rbm.RS = Hp + 32;
  GFMC_CUDA(cudaMalloc(&h->d_rbm_rt, sizeof(float) * (size_t)N * h->rbm.RS));
  h->rbm.RT = (float *)h->d_rbm_rt;
  std::vector<int> cstart, csites, cn;
  std::vector<uint16_t> cpos;
  rbm_build_chunks(N, n_hx, n_edges, md->edge_i, md->edge_j, U, cstart, csites, cn, cpos);
  // slot records: sites, staged rows, couplings, scaled a terms
  std::vector<int32_t> rec((size_t)8 * cpos.size(), 0);
  auto fbits = [](double v) {
    const float f = (float)v;
    int32_t b;
    memcpy(&b, &f, 4);
    return b;
  };
  const double l2a = 2.0 * 1.4426950408889634;
  for (size_t o = 0; o < cpos.size(); ++o) {
    int32_t *R = rec.data() + 8 * o;
    const int pi = cpos[o] & 255, pj = cpos[o] >> 8;
    if ((int)o < n_hx) {
      const double hx = md->hx_half ? md->hx_half[o] : 0.0;
      R[0] = (int32_t)o | (pi << 16);
      R[1] = 0xFFFF | (pi << 16);
      R[2] = R[3] = fbits(hx);
      R[4] = fbits(l2a * gd->rbm_a[o]);
    } else {
      const int e = (int)o - n_hx, i = md->edge_i[e], j = md->edge_j[e];
      R[0] = i | (pi << 16);
      R[1] = j | (pj << 16);
      R[2] = fbits(md->jpm[e]);
      R[3] = fbits(md->jpmpm[e]);
      R[4] = fbits(l2a * gd->rbm_a[i]);
      R[5] = fbits(l2a * gd->rbm_a[j]);
    }
  }
  const size_t s1 = cstart.size() * 4, s2 = csites.size() * 4, s3 = cn.size() * 4,
               s4 = rec.size() * 4;
  const size_t p2 = al(s1), p3 = p2 + al(s2), p4 = p3 + al(s3), ctot = p4 + al(s4) + 256;
  std::vector<unsigned char> ch(ctot, 0);
  memcpy(ch.data(), cstart.data(), s1);
  if (s2) memcpy(ch.data() + p2, csites.data(), s2);
  if (s3) memcpy(ch.data() + p3, cn.data(), s3);
  if (s4) memcpy(ch.data() + p4, rec.data(), s4);
  GFMC_CUDA(cudaMalloc(&h->d_rbm_ch, ctot));
  GFMC_CUDA(cudaMemcpy(h->d_rbm_ch, ch.data(), ctot, cudaMemcpyHostToDevice));
  unsigned char *cb = (unsigned char *)h->d_rbm_ch;
  h->rbm.ch_start = (const int *)cb;
  h->rbm.ch_sites = (const int *)(cb + p2);
  h->rbm.ch_n = (const int *)(cb + p3);
  h->rbm.ch_rec = (int4 *)(cb + p4);
  h->rbm.n_rec = (int)cpos.size();
  h->rbm.n_chunks = (int)cn.size();
  h->rbm.ch_U = U;
  GFMC_CUDA(launch_rbm_derive(h->rbm, N, 0));
  GFMC_CUDA(cudaDeviceSynchronize());
  h->rbm_on = 1;
  h->carry = 1;
  h->state_len = Hp;
  return GFMC_OK;
}

// MLP tables: W1 transposed to input-major (D, H1) and W2 (H2, H1), both
// rounded to bf16; b1, b2 and w3 (rounded to bf16 values) in float.
int build_mlp(gfmc_handle *h, const gfmc_guide_desc *gd, int N, int n_max) {
  const int H1 = gd->mlp_H1, H2 = gd->mlp_H2;
  if (H1 != 64 && H1 != 128 && H1 != 192 && H1 != 256)
    return fail(GFMC_ERR_INVALID, "mlp_H1 must be 64, 128, 192 or 256, got %d", H1);
  if (H2 < 16 || H2 > 256 || H2 % 16)
    return fail(GFMC_ERR_INVALID, "mlp_H2 must be a multiple of 16 in [16, 256], got %d", H2);
  if (!gd->mlp_W1 || !gd->mlp_b1 || !gd->mlp_W2 || !gd->mlp_b2 || !gd->mlp_w3)
    return fail(GFMC_ERR_INVALID, "MLP guide: mlp_W1, mlp_b1, mlp_W2, mlp_b2 and mlp_w3 are required");
  if (n_max < 1 || n_max > 254) return fail(GFMC_ERR_INVALID, "MLP guide: n_max must be in [1, 254]");
  const int np1 = n_max + 1;
  const size_t D = (size_t)N * np1;
  std::vector<uint16_t> W1T(D * H1), W2((size_t)H2 * H1), W2T((size_t)H1 * H2);
  std::vector<float> b1(H1), b2(H2), w3(H2);
  for (int j = 0; j < H1; ++j) {
    for (size_t c = 0; c < D; ++c) {
      const float w = gd->mlp_W1[(size_t)j * D + c];
      if (!std::isfinite(w)) return fail(GFMC_ERR_INVALID, "MLP W1 (%d, %zu) is not finite", j, c);
      W1T[c * H1 + j] = bf16_bits(w);
    }
    b1[j] = gd->mlp_b1[j];
  }
  for (int i = 0; i < H2; ++i) {
    for (int j = 0; j < H1; ++j) {
      const float w = gd->mlp_W2[(size_t)i * H1 + j];
      if (!std::isfinite(w)) return fail(GFMC_ERR_INVALID, "MLP W2 (%d, %d) is not finite", i, j);
      W2[(size_t)i * H1 + j] = bf16_bits(w);
      W2T[(size_t)j * H2 + i] = bf16_bits(w);
    }
    b2[i] = gd->mlp_b2[i];
    const uint32_t u = (uint32_t)bf16_bits(gd->mlp_w3[i]) << 16;
    memcpy(&w3[i], &u, 4);
  }
  const size_t s1 = W1T.size() * 2, s2 = W2.size() * 2;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o2 = al(s1), o2t = o2 + al(s2), ob1 = o2t + al(s2), ob2 = ob1 + al((size_t)H1 * 4),
               ow3 = ob2 + al((size_t)H2 * 4), tot = ow3 + al((size_t)H2 * 4);
  std::vector<unsigned char> host(tot, 0);
  memcpy(host.data(), W1T.data(), s1);
  memcpy(host.data() + o2, W2.data(), s2);
  memcpy(host.data() + o2t, W2T.data(), s2);
  memcpy(host.data() + ob1, b1.data(), (size_t)H1 * 4);
  memcpy(host.data() + ob2, b2.data(), (size_t)H2 * 4);
  memcpy(host.data() + ow3, w3.data(), (size_t)H2 * 4);
  GFMC_CUDA(cudaMalloc(&h->d_mlp, tot));
  GFMC_CUDA(cudaMemcpy(h->d_mlp, host.data(), tot, cudaMemcpyHostToDevice));
  unsigned char *base = (unsigned char *)h->d_mlp;
  h->mlp.W1T = (const __nv_bfloat16 *)base;
  h->mlp.W2 = (const __nv_bfloat16 *)(base + o2);
  h->mlp.W2T = (const __nv_bfloat16 *)(base + o2t);
  h->mlp.b1 = (const float *)(base + ob1);
  h->mlp.b2 = (const float *)(base + ob2);
  h->mlp.w3 = (const float *)(base + ow3);
  h->mlp.b3 = (float)gd->mlp_b3;
  h->mlp.H1 = H1;
  h->mlp.H2 = H2;
  h->mlp.np1 = np1;
  h->mlp_on = 1;
  h->mlp_grid = mlp_grid();
  h->carry = 1;            // z1 and log psi per walker (float32)
  h->state_len = H1 + 1;
  return GFMC_OK;
}

// The per-walker step kernel of the handle's guide.
template <typename T>
cudaError_t launch_step(gfmc_handle *h, const DevModel<T> &m, const DevGuide<T> &g,
                        const EvolveArgs &a, cudaStream_t s) {
  if (h->rbm_on) return launch_rbm_evolve<T>(m, h->rbm, a, h->rbm_grid, s);
  if constexpr (std::is_same<T, float>::value) {
    if (h->mlp_on) return launch_mlp_evolve(m, h->mlp, a, h->mlp_grid, s);
  }
  return launch_evolve<T>(m, g, h->plan, a, s);
}

// Per-block partial maxima of log_w a step launch over n walkers writes.
int step_partials(const gfmc_handle *h, int n) {
  if (h->rbm_on) return rbm_partials(h->rbm_grid, n, h->precision == GFMC_PRECISION_MIXED);
  if (h->mlp_on) return mlp_partials(h->mlp_grid, n);
  return evolve_partials(h->plan, n);
}

template <typename T>
int build_tables(gfmc_handle *h, const gfmc_model_desc *md, const gfmc_guide_desc *gd,
                 DevModel<T> &m, DevGuide<T> &g) {
  const int N = md->n_sites, E = md->n_edges;
  Arena A;
  std::vector<uint32_t> edge(E);
  for (int e = 0; e < E; ++e) {
    int i = md->edge_i[e], j = md->edge_j[e];
    if (i < 0 || j < 0 || i >= N || j >= N || i > 0xFFFF || j > 0xFFFF)
      return fail(GFMC_ERR_INVALID, "edge %d = (%d, %d) out of range for N=%d", e, i, j, N);
    edge[e] = (uint32_t)i | ((uint32_t)j << 16);
  }
  size_t o_edge = A.add(edge.data(), edge.size() * 4);
  memset(&m, 0, sizeof(m));
  memset(&g, 0, sizeof(g));
  m.family = md->kind;
  m.N = N;
  m.E = E;
  std::map<std::string, size_t> off;
  auto put = [&](const char *name, const double *src, size_t n) {
    if (src && n) {
      std::vector<T> v = conv<T>(src, n);
      off[name] = A.add(v.data(), n * sizeof(T));
    }
  };
  if (md->kind == GFMC_MODEL_SPIN_HALF) {
    m.n_hx = md->n_hx;
    m.n_jpm = md->n_jpm;
    m.has_jz = md->has_jz;
    m.uniform_jz = md->uniform_jz;
    m.has_hz = md->has_hz;
    if ((m.n_hx != 0 && m.n_hx != N) || (m.n_jpm != 0 && m.n_jpm != E))
      return fail(GFMC_ERR_INVALID, "SpinHalf layout: n_hx must be 0 or N, n_jpm 0 or n_edges");
    if (m.n_jpm && (!md->jpm || !md->jpmpm)) return fail(GFMC_ERR_INVALID, "jpm/jpmpm missing");
    if (m.n_hx && !md->hx_half) return fail(GFMC_ERR_INVALID, "hx_half missing");
    if (m.has_jz && !md->jz) return fail(GFMC_ERR_INVALID, "jz missing");
    if (m.has_hz && !md->hz) return fail(GFMC_ERR_INVALID, "hz missing");
    m.M = 1 + m.n_hx + m.n_jpm;
    put("jpm", md->jpm, m.n_jpm ? E : 0);
    put("jpmpm", md->jpmpm, m.n_jpm ? E : 0);
    put("jz", md->jz, m.has_jz ? (m.uniform_jz ? 1 : E) : 0);
    put("hz", md->hz, m.has_hz ? N : 0);
    put("hx_half", md->hx_half, m.n_hx ? N : 0);
    m.uniform_pm = 1;
    if (m.n_jpm) {
      for (int e = 1; e < E; ++e)
        if (md->jpm[e] != md->jpm[0] || md->jpmpm[e] != md->jpmpm[0]) m.uniform_pm = 0;
      m.jpm0 = (T)md->jpm[0];
      m.jpmpm0 = (T)md->jpmpm[0];
    }
    h->cfg_bytes = ((N + 63) / 64) * 8;
  } else if (md->kind == GFMC_MODEL_BOSE_HUBBARD) {
    m.n_max = md->n_max;
    m.n_hop = md->n_hop;
    m.n_eta = md->n_eta;
    m.n_hpm = md->n_hpm;
    m.has_U = md->has_U;
    m.has_mu = md->has_mu;
    if (m.n_max < 1 || m.n_max > 255) return fail(GFMC_ERR_INVALID, "n_max must be in [1, 255]");
    if ((m.n_hop != 0 && m.n_hop != 2 * E) || (m.n_eta != 0 && m.n_eta != 2 * E) ||
        (m.n_hpm != 0 && m.n_hpm != N))
      return fail(GFMC_ERR_INVALID, "BoseHubbard layout sizes inconsistent");
    if (m.n_hop && !md->t) return fail(GFMC_ERR_INVALID, "t missing");
    if (m.n_eta && !md->eta) return fail(GFMC_ERR_INVALID, "eta missing");
    if (m.has_U && !md->U) return fail(GFMC_ERR_INVALID, "U missing");
    if (m.has_mu && !md->mu) return fail(GFMC_ERR_INVALID, "mu missing");
    if (m.n_hpm && !md->hpm) return fail(GFMC_ERR_INVALID, "hpm missing");
    m.M = 1 + m.n_hop + m.n_eta + 2 * m.n_hpm;
    put("t", md->t, m.n_hop ? E : 0);
    put("eta", md->eta, m.n_eta ? E : 0);
    put("U", md->U, m.has_U ? N : 0);
    put("mu", md->mu, m.has_mu ? N : 0);
    put("hpm", md->hpm, m.n_hpm ? N : 0);
    {
      std::vector<T> sq((size_t)(m.n_max + 1) * (m.n_max + 1) + 1);
      for (size_t k = 0; k < sq.size(); ++k) sq[k] = std::sqrt((T)k);   // correctly rounded
      off["sqrt"] = A.add(sq.data(), sq.size() * sizeof(T));
    }
    h->cfg_bytes = ((N + 15) / 16) * 16;
  } else {
    return fail(GFMC_ERR_UNSUPPORTED, "unknown model kind %d", md->kind);
  }
  m.n_off = m.M - 1;

  // ---- guide
  int gk = gd ? gd->kind : GFMC_GUIDE_NONE;
  if (gk == GFMC_GUIDE_RBM_SPIN_HALF) {
    if (md->kind != GFMC_MODEL_SPIN_HALF)
      return fail(GFMC_ERR_INVALID, "the RBM guide needs a SpinHalf model");
    gk = GFMC_GUIDE_NONE;   // the Jastrow tables stay empty; rbm.cu evaluates the ratios
  }
  if (gk == GFMC_GUIDE_MLP_BOSE_HUBBARD) {
    if (md->kind != GFMC_MODEL_BOSE_HUBBARD)
      return fail(GFMC_ERR_INVALID, "the MLP guide needs a BoseHubbard model");
    if (h->precision != GFMC_PRECISION_MIXED)
      return fail(GFMC_ERR_UNSUPPORTED, "the MLP guide runs in the float32 (mixed) build");
    gk = GFMC_GUIDE_NONE;   // mlp.cu evaluates the ratios
  }
  if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF && md->kind != GFMC_MODEL_SPIN_HALF)
    return fail(GFMC_ERR_INVALID, "JastrowSpinHalf needs the SpinHalf transition layout");
  if (gk == GFMC_GUIDE_JASTROW_BOSE_HUBBARD && md->kind != GFMC_MODEL_BOSE_HUBBARD)
    return fail(GFMC_ERR_INVALID, "JastrowBoseHubbard needs a BoseHubbard operator");
  if (gk == GFMC_GUIDE_EXACT_SPIN_HALF) {
    if (md->kind != GFMC_MODEL_SPIN_HALF)
      return fail(GFMC_ERR_INVALID, "the exact-amplitude guide needs a SpinHalf model");
    if (gd->exact_n_sites != N || N < 1 || N > 26 || !gd->exact_log_amp)
      return fail(GFMC_ERR_INVALID, "exact-amplitude guide over %d sites (2^N amplitudes) for a "
                  "model of %d sites (N <= 26)", gd->exact_n_sites, N);
  }
  if (gk != GFMC_GUIDE_NONE && gk != GFMC_GUIDE_JASTROW_SPIN_HALF &&
      gk != GFMC_GUIDE_JASTROW_BOSE_HUBBARD && gk != GFMC_GUIDE_EXACT_SPIN_HALF)
    return fail(GFMC_ERR_UNSUPPORTED, "unknown guide kind %d", gk);
  g.kind = gk;
  const bool jastrow = gk == GFMC_GUIDE_JASTROW_SPIN_HALF || gk == GFMC_GUIDE_JASTROW_BOSE_HUBBARD;
  // exact amplitudes: one table of log |psi_0| in the build's precision, no
  // carried state (the ratio needs nothing but the configuration)
  if (gk == GFMC_GUIDE_EXACT_SPIN_HALF) put("lamp", gd->exact_log_amp, (size_t)1 << N);
  size_t o_jdig = 0, o_slq = 0, o_sit = 0;
  size_t o_nbr = 0, o_nbrw = 0, o_cnt = 0, o_tpw = 0, o_jd = 0, o_ep = 0, o_em = 0, o_tep = 0,
           o_xy = 0;
  if (jastrow) {
    // per-site partner lists, duplicates merged (each partner once per site)
    std::vector<std::map<int, double>> lists(N);
    for (int p = 0; p < gd->n_pairs; ++p) {
      int a = gd->pair_i[p], b = gd->pair_j[p];
      if (a < 0 || b < 0 || a >= N || b >= N || a == b)
        return fail(GFMC_ERR_INVALID, "pair %d = (%d, %d) invalid for N=%d", p, a, b, N);
      lists[a][b] += gd->pair_w[p];
      lists[b][a] += gd->pair_w[p];
    }
    int deg = 1;
    for (auto &l : lists) deg = (int)l.size() > deg ? (int)l.size() : deg;
    std::vector<uint32_t> nbr((size_t)N * deg, 0);
    std::vector<T> nbrw((size_t)N * deg, T(0));
    std::vector<int> cnt(N, 0);
    for (int k = 0; k < N; ++k) {
      int c = 0;
      for (auto &kv : lists[k]) {
        nbr[(size_t)k * deg + c] = (uint32_t)kv.first;
        nbrw[(size_t)k * deg + c] = (T)kv.second;
        ++c;
      }
      cnt[k] = c;
    }
    g.deg = deg;
    // dense couplings when most pairs are present: coalesced rows, no indices
    g.dense = (2 * deg > N) ? 1 : 0;
    if (g.dense) {
      std::vector<T> Jd((size_t)N * N, T(0));
      for (int k = 0; k < N; ++k)
        for (auto &kv : lists[k]) Jd[(size_t)k * N + kv.first] = (T)kv.second;
      o_jd = A.add(Jd.data(), Jd.size() * sizeof(T));
      // the population product's int8 digits of Jd (occupations must fit an int8)
      if (md->kind == GFMC_MODEL_SPIN_HALF || md->n_max <= 127) {
        const int D = fields_digits<T>(), NT = 256 / D;
        const int Kp = ((N + 127) / 128) * 128, ny = (N + NT - 1) / NT;
        double amax = 0.0;
        for (const T v : Jd) amax = std::max(amax, std::fabs((double)v));
        int ex = 0;
        if (amax > 0.0) std::frexp(amax, &ex);            // amax < 2^ex
        const double S = std::ldexp(1.0, ex + 1);         // |Jd| / S < 1/2
        std::vector<int8_t> dig((size_t)ny * 256 * Kp, 0);
        for (int k = 0; k < N; ++k) {
          const size_t row = (size_t)(k / NT) * 256 + (size_t)(k % NT);
          for (int p = 0; p < N; ++p) {
            double v = (double)Jd[(size_t)p * N + k] / S;   // exact: S is a power of two
            for (int d = 0; d < D; ++d) {
              const double t = v * 128.0, jd = std::nearbyint(t);   // |t| <= 64
              v = t - jd;                                           // exact, |v| <= 1/2
              dig[(row + (size_t)d * NT) * Kp + p] = (int8_t)jd;
            }
          }
        }
        o_jdig = A.add(dig.data(), dig.size());
        g.jdig_scale = S / 128.0;
        g.jdig_kp = Kp;
        g.jdig_d = D;
      }
      if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF) {
        // translation invariance on an Lx x Ly torus: J_ak = J_0[d(a, k)]
        // (its factor table, 8 N entries, is staged in shared memory: at most 48 KB)
        const bool ti_fits = (size_t)8 * N * sizeof(T) <= 48 * 1024;
        for (int Lx = 1; ti_fits && Lx <= N && !g.ti; ++Lx) {
          if (N % Lx) continue;
          const int Ly = N / Lx;
          bool ok = true;
          for (int a = 0; a < N && ok; ++a) {
            const int xa = a % Lx, ya = a / Lx;
            for (int k = 0; k < N; ++k) {
              const int d = (k % Lx - xa + Lx) % Lx + Lx * ((k / Lx - ya + Ly) % Ly);
              if (Jd[(size_t)a * N + k] != Jd[d]) { ok = false; break; }
            }
          }
          if (ok) {
            g.ti = 1;
            g.Lx = Lx;
            g.Ly = Ly;
          }
        }
        if (g.ti) {
          const int Lx = g.Lx, Ly = g.Ly;
          std::vector<T> te((size_t)8 * N);
          std::vector<int> tq(N);
          for (int uy = 0; uy < 2 * Ly; ++uy)
            for (int ux = 0; ux < 2 * Lx; ++ux) {
              const int d = (ux % Lx) + Lx * (uy % Ly);   // (ux - Lx) mod Lx, (uy - Ly) mod Ly
              const size_t i = 2 * ((size_t)ux + 2 * (size_t)Lx * uy);
              te[i] = (T)std::exp(4.0 * (double)Jd[d]);
              te[i + 1] = (T)std::exp(-4.0 * (double)Jd[d]);
            }
          for (int k = 0; k < N; ++k) tq[k] = 2 * (k % Lx + 2 * Lx * (k / Lx));
          g.tE_off = 2 * (Lx + 2 * Lx * Ly);
          o_tep = A.add(te.data(), te.size() * sizeof(T));
          o_xy = A.add(tq.data(), N * sizeof(int));
        }
        // multiplicative factor updates exp(+-4 J_kp) (1 where no pair)
        std::vector<T> ep((size_t)N * N, T(1)), em((size_t)N * N, T(1));
        for (int k = 0; k < N; ++k)
          for (auto &kv : lists[k]) {
            ep[(size_t)k * N + kv.first] = (T)std::exp(4.0 * kv.second);
            em[(size_t)k * N + kv.first] = (T)std::exp(-4.0 * kv.second);
          }
        o_ep = A.add(ep.data(), ep.size() * sizeof(T));
        o_em = A.add(em.data(), em.size() * sizeof(T));
      }
    } else if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF) {
      std::vector<T> ep((size_t)N * deg, T(1)), em((size_t)N * deg, T(1));
      for (int k = 0; k < N; ++k) {
        int c = 0;
        for (auto &kv : lists[k]) {
          ep[(size_t)k * deg + c] = (T)std::exp(4.0 * kv.second);
          em[(size_t)k * deg + c] = (T)std::exp(-4.0 * kv.second);
          ++c;
        }
      }
      o_ep = A.add(ep.data(), ep.size() * sizeof(T));
      o_em = A.add(em.data(), em.size() * sizeof(T));
    }
    o_nbr = A.add(nbr.data(), nbr.size() * 4);
    o_nbrw = A.add(nbrw.data(), nbrw.size() * sizeof(T));
    o_cnt = A.add(cnt.data(), cnt.size() * 4);
    // carried guide state: for dense or high-degree guides, and in the
    // float64 build for every guide (the per-walker rebuild, N exps, costs
    // more than 2 N values of traffic even at degree 4: the 432-site kagome
    // guide ran 39 % faster carried).  Sparse float32 guides keep the
    // rebuild: the float32 multiplicative updates drift by ~1e-7 per flip
    // between refreshes, which biased the 100-site chain's energy by 4.6
    // sigma when carried.
    h->carry = (g.dense || deg >= 16 || h->precision == GFMC_PRECISION_FP64) ? 1 : 0;
    h->carry_optional = (!g.dense && deg < 16) ? 1 : 0;   // the rebuild also works
    h->carry_pref = h->carry;
    auto pair_sum = [&](int a, int b) -> double {
      if (a == b) return 0.0;
      auto it = lists[a].find(b);
      return it == lists[a].end() ? 0.0 : it->second;
    };
    if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF) {
      std::vector<double> hh(N, 0.0);
      if (gd->h) for (int k = 0; k < N; ++k) hh[k] = gd->h[k];
      for (int k = 0; k < N; ++k) g.has_h |= (hh[k] != 0.0);
      put("gh", hh.data(), N);
      // per-edge constants of the factored edge-flip ratio: exp(-+4 Jsum_e)
      std::vector<double> ca(E > 0 ? E : 1, 1.0), cp(E > 0 ? E : 1, 1.0);
      g.uniform_c = 1;
      for (int e = 0; e < E; ++e) {
        const double js = pair_sum(md->edge_i[e], md->edge_j[e]);
        ca[e] = exp(-4.0 * js);
        cp[e] = exp(4.0 * js);
        if (ca[e] != ca[0] || cp[e] != cp[0]) g.uniform_c = 0;
      }
      g.c_anti0 = (T)ca[0];
      g.c_par0 = (T)cp[0];
      put("c_anti", ca.data(), E);
      put("c_par", cp.data(), E);
    } else {
      // per-transition summed pair weight (JastrowBoseHubbardOpCache.pair_w)
      std::vector<T> tpw(m.M, T(0));
      int t = 1;
      int blocks = (m.n_hop ? 2 : 0) + (m.n_eta ? 2 : 0);
      for (int b = 0; b < blocks; ++b)
        for (int e = 0; e < E; ++e) tpw[t++] = (T)pair_sum(md->edge_i[e], md->edge_j[e]);
      o_tpw = A.add(tpw.data(), tpw.size() * sizeof(T));
      g.beta_scale = gd->beta_tied ? (T)(-gd->beta0) : T(1);
      g.h_mode = gd->h_mode;
      g.h0 = (T)gd->h0;
      g.d_mode = gd->d_mode;
      g.d0 = (T)gd->d0;
      if (g.h_mode == 2) {
        if (!gd->h) return fail(GFMC_ERR_INVALID, "h array missing");
        put("gh", gd->h, N);
      }
      if (g.d_mode == 2) {
        if (!gd->d) return fail(GFMC_ERR_INVALID, "d array missing");
        put("gd", gd->d, N);
      }
      // the ratio's static factors (see DevGuide::slot_q, site_t)
      {
        const double bs = (double)g.beta_scale;
        std::vector<T> q(m.M, T(1));
        int o = 1;
        const int hop = m.n_hop ? 2 * E : 0, eta = m.n_eta ? 2 * E : 0;
        for (int i = 0; i < hop; ++i, ++o) q[o] = (T)std::exp(-bs * (double)tpw[o]);   // da db = -1
        for (int i = 0; i < eta; ++i, ++o) q[o] = (T)std::exp(bs * (double)tpw[o]);    // da db = +1
        o_slq = A.add(q.data(), q.size() * sizeof(T));
        const int nm = m.n_max;
        std::vector<T> st((size_t)N * (nm + 1) * 2);
        for (int k = 0; k < N; ++k) {
          const double dk = g.d_mode == 2 ? gd->d[k] : (g.d_mode == 1 ? gd->d0 : 0.0);
          const double hk = g.h_mode == 2 ? gd->h[k] : (g.h_mode == 1 ? gd->h0 : 0.0);
          for (int n = 0; n <= nm; ++n)
            for (int si = 0; si < 2; ++si) {
              const double sv = si ? 1.0 : -1.0;
              const double ds = (n + sv) * (n + sv) - (double)n * n;
              st[((size_t)k * (nm + 1) + n) * 2 + si] = (T)std::exp(-dk * ds + hk * sv);
            }
        }
        o_sit = A.add(st.data(), st.size() * sizeof(T));
      }
    }
  }

  // ---- upload
  GFMC_CUDA(cudaMalloc(&h->d_tables, A.host.size() ? A.host.size() : 256));
  GFMC_CUDA(cudaMemcpy(h->d_tables, A.host.data(), A.host.size(), cudaMemcpyHostToDevice));
  unsigned char *base = (unsigned char *)h->d_tables;
  auto ptr = [&](const char *name) -> const T * {
    auto it = off.find(name);
    return it == off.end() ? nullptr : (const T *)(base + it->second);
  };
  m.edge = E ? (const uint32_t *)(base + o_edge) : nullptr;
  m.jpm = ptr("jpm"); m.jpmpm = ptr("jpmpm"); m.jz = ptr("jz"); m.hz = ptr("hz");
  m.hx_half = ptr("hx_half");
  m.t = ptr("t"); m.eta = ptr("eta"); m.U = ptr("U"); m.mu = ptr("mu"); m.hpm = ptr("hpm");
  m.sqrt_tab = ptr("sqrt");
  g.lamp = ptr("lamp");
  if (jastrow) {
    g.nbr = (const uint32_t *)(base + o_nbr);
    g.nbr_w = (const T *)(base + o_nbrw);
    g.nbr_cnt = (const int *)(base + o_cnt);
    g.h = ptr("gh");
    g.d = ptr("gd");
    if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF) {
      g.c_anti = ptr("c_anti");
      g.c_par = ptr("c_par");
    } else {
      g.trans_pw = (const T *)(base + o_tpw);
      g.slot_q = (const T *)(base + o_slq);
      g.site_t = (const T *)(base + o_sit);
    }
    if (g.dense) g.Jd = (const T *)(base + o_jd);
    if (g.dense && g.jdig_d) g.jdig = (const int8_t *)(base + o_jdig);
    if (gk == GFMC_GUIDE_JASTROW_SPIN_HALF) {
      if (g.dense) {
        g.Ep = (const T *)(base + o_ep);
        g.Em = (const T *)(base + o_em);
        if (g.ti) {
          g.tE = (const T *)(base + o_tep);
          g.tq = (const int *)(base + o_xy);
        }
      } else {
        g.nbr_ep = (const T *)(base + o_ep);
        g.nbr_em = (const T *)(base + o_em);
      }
    }
  }
  // fast spin layout (see DevModel::fast)
  if (m.family == SPIN_HALF) {
    const bool guided_ok = gk == GFMC_GUIDE_NONE || (gk == GFMC_GUIDE_JASTROW_SPIN_HALF && g.uniform_c);
    m.fast = (m.n_hx == 0 && m.n_jpm == E && E > 0 && m.uniform_pm && (!m.has_jz || m.uniform_jz) &&
              !m.has_hz && guided_ok) ? 1 : 0;
    if (m.fast) {
      const bool gd_on = gk == GFMC_GUIDE_JASTROW_SPIN_HALF;
      m.k_anti = m.jpm0 * (gd_on ? g.c_anti0 : T(1));
      m.k_par = m.jpmpm0 * (gd_on ? g.c_par0 : T(1));
      // the min form of k_par = 0 measured faster in float32 and slower in
      // float64 than the coefficient select
      m.fast = (m.k_par == T(0) && sizeof(T) == 4) ? 1 : 2;
    }
  }
  cudaError_t e = plan_evolve<T>(m, g, m.M, &h->plan);
  if (e != cudaSuccess)
    return fail(GFMC_ERR_CUDA, "planning the evolve kernel failed: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int ensure_scratch(gfmc_handle *h, int n, int n_steps) {
  int nb = recon_tiles(n);
  if (n > h->cap_n) {
    cudaFree(h->psum); cudaFree(h->cdf); cudaFree(h->wbuf); cudaFree(h->plp);
    h->psum = h->cdf = h->wbuf = nullptr; h->plp = nullptr;
    GFMC_CUDA(cudaMalloc(&h->psum, sizeof(double) * nb));
    GFMC_CUDA(cudaMalloc(&h->plp, sizeof(int) * nb));
    GFMC_CUDA(cudaMalloc(&h->cdf, sizeof(double) * n));
    GFMC_CUDA(cudaMalloc(&h->wbuf, sizeof(double) * n));
    cudaFree(h->pE);
    h->pE = nullptr;
    h->cap_steps = 0;
    h->cap_n = n;
  }
  int nbc = recon_tiles(h->cap_n);
  if (n_steps > h->cap_steps) {
    cudaFree(h->pE); cudaFree(h->ctr); cudaFree(h->hops);
    h->pE = nullptr; h->ctr = nullptr; h->hops = nullptr;
    GFMC_CUDA(cudaMalloc(&h->pE, sizeof(double) * (size_t)nbc * n_steps));
    GFMC_CUDA(cudaMalloc(&h->ctr, sizeof(int) * n_steps));
    GFMC_CUDA(cudaMalloc(&h->hops, sizeof(unsigned long long) * n_steps));
    h->cap_steps = n_steps;
  }
  if (!h->rctr) {
    GFMC_CUDA(cudaMalloc(&h->rctr, sizeof(unsigned)));
    GFMC_CUDA(cudaMemset(h->rctr, 0, sizeof(unsigned)));
    h->rbase = 0;
    h->fused_tiles = recon_fused_max_tiles();
  }
  if (!h->pmax) {
    size_t np = (size_t)(h->plan.grid > 0 ? h->plan.grid : 1) * (h->plan.wpb > 0 ? h->plan.wpb : 1);
    if (h->rbm_on)
      np = std::max(np, (size_t)rbm_partials(h->rbm_grid, h->rbm_grid * RBF_WARPS,
                                             h->precision == GFMC_PRECISION_MIXED));
    if (h->mlp_on) np = std::max(np, (size_t)mlp_partials(h->mlp_grid, h->mlp_grid));
    GFMC_CUDA(cudaMalloc(&h->pmax, sizeof(double) * np));
  }
  if (h->carry_optional) {
    // the optional carried state (sparse guides): only when chosen at create
    // and by gfmc_carry_mode, and while its buffers take at most half the
    // free memory at the call that sizes them; otherwise the step rebuilds
    // every walker's state (the same values up to the last bits in float64)
    int want = h->carry_pref && h->carry_mode;
    if (want && n > h->cap_field) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const size_t tsz = h->precision == GFMC_PRECISION_FP64 ? 8 : 4;
        const size_t need = 2 * tsz * (size_t)n * ((size_t)h->state_len + EVAL_REC);
        if (need > free_b / 2) want = 0;
      }
    }
    if (want != h->carry) {
      h->carry = want;
      h->field_valid = 0;
      h->eval_valid = 0;
    }
  }
  if (h->carry && n > h->cap_field) {
    size_t tsz = h->precision == GFMC_PRECISION_FP64 ? sizeof(double) : sizeof(float);
    // every old buffer is released (and forgotten) before any new one is
    // allocated, so none is freed twice
    cudaFree(h->fbuf[0]); cudaFree(h->fbuf[1]);
    cudaFree(h->ebuf[0]); cudaFree(h->ebuf[1]);
    h->fbuf[0] = h->fbuf[1] = nullptr;
    h->ebuf[0] = h->ebuf[1] = nullptr;
    h->cap_field = 0;
    h->field_valid = 0;
    h->eval_valid = 0;
    GFMC_CUDA(cudaMalloc(&h->fbuf[0], tsz * (size_t)n * h->state_len));
    GFMC_CUDA(cudaMalloc(&h->fbuf[1], tsz * (size_t)n * h->state_len));
    if (!h->rbm_on && !h->mlp_on) {
      GFMC_CUDA(cudaMalloc(&h->ebuf[0], tsz * (size_t)n * EVAL_REC));
      GFMC_CUDA(cudaMalloc(&h->ebuf[1], tsz * (size_t)n * EVAL_REC));
    }
    h->cap_field = n;
    h->field_valid = 0;
    h->eval_valid = 0;
  }
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  return GFMC_OK;
}

template <typename T>
int run_steps_t(gfmc_handle *h, const DevModel<T> &m, const DevGuide<T> &g, int method,
                double step, double lam, double alw, int n_steps, const uint32_t *keys, int n,
                void *cfg, void *cfg_tmp, int32_t *parents, int parents_valid, double *log_w,
                double *e_loc, double *logG_out, double *E_out, uint64_t *hops_out,
                cudaStream_t s) {
  int rc = ensure_scratch(h, n, n_steps);
  if (rc) return rc;
  if (h->diag_out && (!h->diag_ready || h->diag_cap_n != n))
    return fail(GFMC_ERR_INVALID, "diagonal output set but gfmc_reset_diag not called for %d walkers", n);
  const int nb = recon_tiles(n);
  const int nbc = recon_tiles(h->cap_n);
  GFMC_CUDA(cudaMemsetAsync(h->ctr, 0, sizeof(int) * n_steps, s));
  unsigned long long *hops = hops_out ? (unsigned long long *)hops_out : h->hops;
  GFMC_CUDA(cudaMemsetAsync(hops, 0, sizeof(unsigned long long) * n_steps, s));
  if (h->mlp_on && method != CONT_TIME)
    return fail(GFMC_ERR_UNSUPPORTED, "the MLP guide propagates with cont_time only");
  const int n_partials = step_partials(h, n);
  void *cur = cfg, *nxt = cfg_tmp;
  for (int st = 0; st < n_steps; ++st) {
    EvolveArgs a{};
    a.method = method;
    a.step = step;
    a.lam = lam;
    a.alw = alw;
    a.key = Key{keys[4 * st + 0], keys[4 * st + 1]};
    a.n_walkers = n;
    a.parents = (st == 0 && !parents_valid) ? nullptr : parents;
    a.cfg_in = cur;
    a.cfg_out = nxt;
    a.log_w = log_w;
    a.e_loc = e_loc;
    a.hops = hops + st;
    a.work_ctr = h->ctr + st;
    a.partial_max = h->pmax;
    a.status = h->status;
    a.max_iters = h->max_iters;
    if (h->carry) {
      const bool fresh = (st == 0 && !parents_valid) || !h->field_valid || h->field_cfg != cfg ||
                         h->since_refresh >= h->refresh_every;
      a.field_in = fresh ? nullptr : h->fbuf[h->fcur];
      if (fresh && h->rbm_on && h->precision == GFMC_PRECISION_MIXED) {
        // the float32 build rebuilds theta for the whole population on the
        // tensor cores (rows indexed like cfg_in; the step reads them
        // through the parent map)
        cudaError_t eg = launch_rbm_theta(h->rbm, n, cur, nullptr, (h->N + 63) / 64,
                                          (float *)h->fbuf[h->fcur], h->status, s);
        if (eg != cudaSuccess) return fail(GFMC_ERR_CUDA, "theta GEMM: %s", cudaGetErrorString(eg));
        a.field_in = h->fbuf[h->fcur];
      } else if (fresh && !h->rbm_on && !h->mlp_on && g.dense && g.jdig) {
        // dense Jastrow couplings: the population's state as one product
        cudaError_t eg = launch_fields<T>(m, g, n, cur, (T *)h->fbuf[h->fcur], h->status, s);
        if (eg != cudaSuccess) return fail(GFMC_ERR_CUDA, "guide fields: %s", cudaGetErrorString(eg));
        a.field_in = h->fbuf[h->fcur];
      }
      a.field_out = h->fbuf[1 - h->fcur];
      if (h->ebuf[0] && method == CONT_TIME) {
        // carried fields and the last step's records: reuse its final evaluation
        a.eval_in = (!fresh && a.field_in == h->fbuf[h->fcur] && h->eval_valid) ? h->ebuf[h->fcur]
                                                                                : nullptr;
        a.eval_out = h->ebuf[1 - h->fcur];
      }
      h->eval_valid = a.eval_out != nullptr;
      h->fcur = 1 - h->fcur;
      h->field_valid = 1;
      h->field_cfg = cfg;
      h->since_refresh = fresh ? 1 : h->since_refresh + 1;
    }
    cudaError_t e = launch_step<T>(h, m, g, a, s);
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "evolve launch: %s", cudaGetErrorString(e));
    ReconArgs r{};
    r.n = n;
    r.log_w = log_w;
    r.e_loc = e_loc;
    r.partial_max = h->pmax;
    r.n_partial_max = n_partials;
    r.key = Key{keys[4 * st + 2], keys[4 * st + 3]};
    r.psum = h->psum;
    r.pE = h->pE + (size_t)st * nb;
    r.plp = h->plp;
    r.cdf = h->cdf;
    r.wbuf = h->wbuf;
    r.parents = parents;
    r.logG_out = logG_out + st;
    r.status = h->status;
    if (nb <= h->fused_tiles) {
      // one cooperative launch (all tiles resident, E_n summed in it); each
      // block adds 2 to the counter
      r.E_step = E_out ? E_out + st : nullptr;
      e = launch_reconfigure_fused(r, h->rctr, h->rbase, s);
      if (e == cudaSuccess) {
        h->rbase += 2u * (unsigned)nb;
      } else {
        // the cooperative launch was refused (nothing ran): the three
        // launches from now on; the chunk's series reduction then writes
        // every E_n (the tile partials are written on both paths)
        (void)cudaGetLastError();
        h->fused_tiles = 0;
        r.E_step = nullptr;
        e = launch_reconfigure(r, s);
      }
    } else {
      e = launch_reconfigure(r, s);
    }
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "reconfigure launch: %s", cudaGetErrorString(e));
    if (h->fw) {
      FwHook &f = *h->fw;
      double *pp = f.rec[st + 1] ? f.partial + (size_t)(st + 1) * f.nb : nullptr;
      e = launch_fw_remap(n, parents, f.v[f.cur], f.v[1 - f.cur], pp, s);
      if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "forward-walk remap: %s", cudaGetErrorString(e));
      f.cur = 1 - f.cur;
    }
    if (h->diag_out && h->diag_ready) {
      const int NW = (h->N + 63) / 64;
      e = launch_diag_step(h->diag, h->family, n, NW, h->cfg_bytes, nxt, parents, h->diag_slot,
                           h->diag_partial,
                           h->diag_out + (size_t)st * h->diag.width * h->diag.n_p, s);
      if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "diagonal step: %s", cudaGetErrorString(e));
      h->diag_slot = (h->diag_slot + 1) % (h->diag.m_max + 1);
    }
    void *t = cur; cur = nxt; nxt = t;
  }
  (void)nbc;
  if (nb > h->fused_tiles && E_out) {   // (the one-launch resampling wrote E_n itself)
    cudaError_t e = launch_series_reduce(h->pE, nb, n_steps, E_out, s);
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "series reduce: %s", cudaGetErrorString(e));
  }
  if (cur != cfg)
    GFMC_CUDA(cudaMemcpyAsync(cfg, cur, (size_t)n * h->cfg_bytes, cudaMemcpyDeviceToDevice, s));
  return GFMC_OK;
}

// One launch of the per-walker kernel in APPLY or MIN_RATE mode through
// handle h (an operator's handle): reads cfg[parents[i]], writes the moved
// configuration (cfg_out, nullable) and one float64 per walker.  Touches only
// the handle's work counter and status word, so an operator handle holds no
// population-sized scratch.
template <typename T>
int single_launch_t(gfmc_handle *h, const DevModel<T> &m, const DevGuide<T> &g, int method,
                    Key key, int n, const void *cfg, const int32_t *parents, void *cfg_out,
                    double *out, cudaStream_t s) {
  if (!h->ctr1) GFMC_CUDA(cudaMalloc(&h->ctr1, sizeof(int)));
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  GFMC_CUDA(cudaMemsetAsync(h->ctr1, 0, sizeof(int), s));
  EvolveArgs a{};
  a.method = method;
  a.key = key;
  a.n_walkers = n;
  a.parents = parents;
  a.cfg_in = cfg;
  a.cfg_out = cfg_out;
  a.e_loc = out;
  a.work_ctr = h->ctr1;
  a.status = h->status;
  a.max_iters = 1;
  cudaError_t e = launch_evolve<T>(m, g, h->plan, a, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "operator launch: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int single_launch(gfmc_handle *h, int method, Key key, int n, const void *cfg,
                  const int32_t *parents, void *cfg_out, double *out, cudaStream_t s) {
  if (h->rbm_on || h->mlp_on)
    return fail(GFMC_ERR_UNSUPPORTED, "measurement operators under a learned guide are not built");
  if (h->precision == GFMC_PRECISION_FP64)
    return single_launch_t<double>(h, h->m64, h->g64, method, key, n, cfg, parents, cfg_out, out, s);
  return single_launch_t<float>(h, h->m32, h->g32, method, key, n, cfg, parents, cfg_out, out, s);
}

int check_method(int method, double step) {
  if (method < 0 || method > 2) return fail(GFMC_ERR_INVALID, "unknown method %d", method);
  if (method != GFMC_METHOD_CONT_TIME && (step < 1.0 || step != (double)(long long)step))
    return fail(GFMC_ERR_INVALID, "discrete methods need a positive integer step");
  if (!(step > 0.0)) return fail(GFMC_ERR_INVALID, "step must be > 0");
  return GFMC_OK;
}

// The variance-loss gradient of the RBM guide over the population
// cfg[parents[i]] (float32 build): gather, theta on the tensor cores, the
// EVALUATE pass with per-slot rates, coefficients, the fused gradient kernel.
// Leaves grad_W (Hp, Np), grad_b, grad_a and (E, var) in the handle's scratch.
int rbm_gradient_t(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                   int parents_valid, const double *omega, cudaStream_t s) {
  const RbmTables &r = h->rbm;
  const int NW = (h->N + 63) / 64, n_off = h->M - 1;
  if (h->precision != GFMC_PRECISION_MIXED)
    return fail(GFMC_ERR_UNSUPPORTED, "RBM training runs in the float32 (mixed) build");
  if (r.Np > 448) return fail(GFMC_ERR_UNSUPPORTED, "RBM training supports at most 448 sites");
  if (n > h->train_cap) {
    cudaFree(h->tr_cfg); cudaFree(h->tr_theta); cudaFree(h->tr_rates); cudaFree(h->tr_rsum);
    cudaFree(h->tr_gw); cudaFree(h->tr_e); cudaFree(h->tr_recs);
    h->tr_cfg = nullptr; h->tr_theta = h->tr_rates = h->tr_rsum = h->tr_gw = nullptr;
    h->tr_e = nullptr;
    h->tr_recs = nullptr;
    h->train_cap = 0;
    GFMC_CUDA(cudaMalloc(&h->tr_cfg, sizeof(uint64_t) * (size_t)n * NW));
    GFMC_CUDA(cudaMalloc(&h->tr_theta, sizeof(float) * (size_t)n * r.Hp));
    GFMC_CUDA(cudaMalloc(&h->tr_rates, sizeof(float) * (size_t)n * (n_off > 0 ? n_off : 1)));
    GFMC_CUDA(cudaMalloc(&h->tr_rsum, sizeof(float) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->tr_gw, sizeof(float) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->tr_e, sizeof(double) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->tr_recs, 16 * (size_t)n * (size_t)(n_off + 1)));
    h->train_cap = n;
  }
  if (!h->tr_stats) {
    GFMC_CUDA(cudaMalloc(&h->tr_stats, sizeof(double) * 2));
    GFMC_CUDA(cudaMalloc(&h->tr_gW, sizeof(float) * (size_t)r.Hp * r.Np));
    GFMC_CUDA(cudaMalloc(&h->tr_gb, sizeof(float) * (size_t)r.Hp));
    GFMC_CUDA(cudaMalloc(&h->tr_ga, sizeof(float) * (size_t)r.Np));
  }
  if (!h->ctr1) GFMC_CUDA(cudaMalloc(&h->ctr1, sizeof(int)));
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  cudaError_t e = launch_gather(n, h->cfg_bytes, parents_valid ? parents : nullptr, cfg, h->tr_cfg,
                                nullptr, nullptr, nullptr, s);
  if (e == cudaSuccess) e = launch_rbm_theta(r, n, h->tr_cfg, nullptr, NW, h->tr_theta, h->status, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->ctr1, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    EvolveArgs a{};
    a.method = EVALUATE;
    a.n_walkers = n;
    a.cfg_in = h->tr_cfg;
    a.e_loc = h->tr_e;
    a.work_ctr = h->ctr1;
    a.status = h->status;
    a.max_iters = 1;
    a.field_in = h->tr_theta;
    a.rates_out = h->tr_rates;
    a.rsum_out = h->tr_rsum;
    e = launch_rbm_evolve<float>(h->m32, r, a, h->rbm_grid, s);
  }
  if (e == cudaSuccess) e = launch_train_coeff(n, h->tr_e, omega, h->tr_gw, h->tr_stats, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->tr_gW, 0, sizeof(float) * (size_t)r.Hp * r.Np, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->tr_gb, 0, sizeof(float) * (size_t)r.Hp, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->tr_ga, 0, sizeof(float) * (size_t)r.Np, s);
  if (e == cudaSuccess) {
    GradArgs g{};
    g.cfg = h->tr_cfg;
    g.NW = NW;
    g.n = n;
    g.N = h->N;
    g.Np = r.Np;
    g.Hp = r.Hp;
    g.n_off = n_off;
    g.n_hx = h->m32.n_hx;
    g.edge = h->m32.edge;
    g.WT = r.WT;
    g.theta = h->tr_theta;
    g.rates = h->tr_rates;
    g.rsum = h->tr_rsum;
    g.gw = h->tr_gw;
    g.grad_W = h->tr_gW;
    g.grad_b = h->tr_gb;
    g.grad_a = h->tr_ga;
    g.status = h->status;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = launch_rbm_grad(g, h->tr_recs, sms, s);
  }
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "RBM gradient: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

// The variance-loss gradient of the MLP guide over the population
// cfg[parents[i]] (float32 build): gather, the EVALUATE pass with per-move
// rates, coefficients, the training rows, the three tensor-core GEMMs and the
// one-hot layer.  Leaves the gradient (master-parameter order) in
// mtr_grad and (E, var) in mtr_stats.
int mlp_gradient_t(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                   int parents_valid, const double *omega, cudaStream_t s) {
  const MlpTables &t = h->mlp;
  if (t.H2 % 64)
    return fail(GFMC_ERR_UNSUPPORTED, "MLP training needs mlp_H2 a multiple of 64, got %d", t.H2);
  const int n_off = h->M - 1, rpw = n_off + 1, D = h->N * t.np1, CB = h->cfg_bytes;
  if ((size_t)D * 64 * 4 > 200 * 1024)
    return fail(GFMC_ERR_UNSUPPORTED, "MLP training supports at most 800 one-hot inputs, got %d", D);
  if (rpw < 10)
    return fail(GFMC_ERR_UNSUPPORTED, "MLP training needs at least 9 moves per configuration");
  const long long R = (long long)n * rpw, Mpad = (R + 127) / 128 * 128;
  const size_t per_row = (size_t)t.H1 * 2 * 3 + (size_t)t.H2 * 2 * 4 + (size_t)t.H1 * 4 + 4 + 16;
  if ((double)Mpad * per_row > 64e9)
    return fail(GFMC_ERR_UNSUPPORTED, "MLP training scratch for %d walkers exceeds 64 GB", n);
  const long long np = mlp_param_count(t.H1, t.H2, D);
  if (n > h->mtr_cap || Mpad > h->mtr_rows) {
    cudaFree(h->mtr_cfg); cudaFree(h->mtr_rates); cudaFree(h->mtr_rsum); cudaFree(h->mtr_gw);
    cudaFree(h->mtr_e); cudaFree(h->mtr_coef); cudaFree(h->mtr_h1); cudaFree(h->mtr_h1T);
    cudaFree(h->mtr_h1lo); cudaFree(h->mtr_rowcols); cudaFree(h->mtr_d2); cudaFree(h->mtr_d2T); cudaFree(h->mtr_d1);
    cudaFree(h->mtr_rowcols);
    h->mtr_rowcols = nullptr;
    h->mtr_cfg = nullptr; h->mtr_rates = h->mtr_rsum = h->mtr_gw = h->mtr_coef = h->mtr_d1 = nullptr;
    h->mtr_e = nullptr;
    h->mtr_h1 = h->mtr_h1lo = h->mtr_h1T = h->mtr_d2 = h->mtr_d2T = nullptr;
    h->mtr_cap = 0;
    h->mtr_rows = 0;
    GFMC_CUDA(cudaMalloc(&h->mtr_cfg, (size_t)n * CB));
    GFMC_CUDA(cudaMalloc(&h->mtr_rates, sizeof(float) * (size_t)n * (n_off > 0 ? n_off : 1)));
    GFMC_CUDA(cudaMalloc(&h->mtr_rsum, sizeof(float) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->mtr_gw, sizeof(float) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->mtr_e, sizeof(double) * (size_t)n));
    GFMC_CUDA(cudaMalloc(&h->mtr_coef, sizeof(float) * (size_t)Mpad));
    GFMC_CUDA(cudaMalloc(&h->mtr_h1, 2 * (size_t)Mpad * t.H1));
    GFMC_CUDA(cudaMalloc(&h->mtr_h1T, 2 * (size_t)Mpad * t.H1));
    GFMC_CUDA(cudaMalloc(&h->mtr_h1lo, 2 * (size_t)Mpad * t.H1));
    GFMC_CUDA(cudaMalloc(&h->mtr_d2, 4 * (size_t)Mpad * t.H2));     // hi | lo
    GFMC_CUDA(cudaMalloc(&h->mtr_d2T, 4 * (size_t)Mpad * t.H2));
    GFMC_CUDA(cudaMalloc(&h->mtr_d1, 4 * (size_t)Mpad * t.H1));
    GFMC_CUDA(cudaMalloc(&h->mtr_rowcols, sizeof(int4) * (size_t)Mpad));
    h->mtr_cap = n;
    h->mtr_rows = Mpad;
  }
  if (!h->mtr_stats) {
    GFMC_CUDA(cudaMalloc(&h->mtr_stats, sizeof(double) * 2));
    GFMC_CUDA(cudaMalloc(&h->mtr_grad, sizeof(float) * (size_t)np));
  }
  if (!h->ctr1) GFMC_CUDA(cudaMalloc(&h->ctr1, sizeof(int)));
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  cudaError_t e = launch_gather(n, CB, parents_valid ? parents : nullptr, cfg, h->mtr_cfg, nullptr,
                                nullptr, nullptr, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->ctr1, 0, sizeof(int), s);
  if (e == cudaSuccess) {
    EvolveArgs a{};
    a.method = EVALUATE;
    a.n_walkers = n;
    a.cfg_in = h->mtr_cfg;
    a.e_loc = h->mtr_e;
    a.work_ctr = h->ctr1;
    a.status = h->status;
    a.max_iters = 1;
    a.rates_out = h->mtr_rates;
    a.rsum_out = h->mtr_rsum;
    e = launch_mlp_evolve(h->m32, t, a, h->mlp_grid, s);
  }
  if (e == cudaSuccess) e = launch_train_coeff(n, h->mtr_e, omega, h->mtr_gw, h->mtr_stats, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->mtr_grad, 0, sizeof(float) * (size_t)np, s);
  if (e == cudaSuccess)
    e = launch_mlp_rows(h->m32, t, h->mtr_cfg, CB, n, Mpad, h->mtr_rates, h->mtr_rsum, h->mtr_gw,
                        h->mtr_coef, h->mtr_rowcols, h->mtr_h1, h->mtr_h1lo, h->mtr_h1T, s);
  float *gW1 = h->mtr_grad, *gb1 = gW1 + (size_t)t.H1 * D, *gW2 = gb1 + t.H1,
        *gb2 = gW2 + (size_t)t.H2 * t.H1, *gw3 = gb2 + t.H2;
  if (e == cudaSuccess) {
    MlpGemmArgs g{};
    g.mode = MLP_EPI_FWD;
    g.A = h->mtr_h1; g.lda = t.H1;
    g.B = t.W2; g.ldb = t.H1;
    g.M = (int)Mpad; g.N = t.H2; g.K = t.H1;
    g.coef = h->mtr_coef; g.b2 = t.b2; g.w3 = t.w3;
    g.d2 = h->mtr_d2; g.d2T = h->mtr_d2T; g.ldT = 2 * Mpad;
    g.g_w3 = gw3; g.g_b2 = gb2;
    g.status = h->status;
    e = launch_mlp_gemm(g, s);
  }
  if (e == cudaSuccess) {
    MlpGemmArgs g{};
    g.mode = MLP_EPI_BWD;
    g.A = h->mtr_d2; g.lda = 2 * t.H2;          // [hi | lo] against W2^T twice
    g.B = t.W2T; g.ldb = t.H2;
    g.M = (int)Mpad; g.N = t.H1; g.K = 2 * t.H2; g.kb = t.H2;
    g.h1 = h->mtr_h1; g.h1lo = h->mtr_h1lo; g.d1 = h->mtr_d1; g.g_b1 = gb1;
    g.status = h->status;
    e = launch_mlp_gemm(g, s);
  }
  if (e == cudaSuccess) {
    MlpGemmArgs g{};
    g.mode = MLP_EPI_ACC;
    g.A = h->mtr_d2T; g.lda = 2 * Mpad;         // [hi^T | lo^T] against h1^T twice
    g.B = h->mtr_h1T; g.ldb = Mpad;
    g.M = t.H2; g.N = t.H1; g.K = (int)(2 * Mpad); g.kb = (int)Mpad;
    g.C = gW2; g.ldc = t.H1;
    g.status = h->status;
    e = launch_mlp_gemm(g, s);
  }
  if (e == cudaSuccess)
    e = launch_mlp_dw1(h->m32, t, h->mtr_cfg, CB, n, h->mtr_d1, h->mtr_rowcols, gW1, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "MLP gradient: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

template <typename T>
int local_energy_t(gfmc_handle *h, const DevModel<T> &m, const DevGuide<T> &g, int n,
                   const void *cfg, const int32_t *parents, double *e_loc, cudaStream_t s,
                   double *diag_out = nullptr) {
  int rc = ensure_scratch(h, n, 1);
  if (rc) return rc;
  GFMC_CUDA(cudaMemsetAsync(h->ctr, 0, sizeof(int), s));
  EvolveArgs a{};
  a.method = EVALUATE;
  a.n_walkers = n;
  a.parents = parents;
  a.cfg_in = cfg;
  a.cfg_out = nullptr;
  a.log_w = nullptr;
  a.e_loc = e_loc;
  a.diag_out = diag_out;
  a.hops = nullptr;
  a.work_ctr = h->ctr;
  a.partial_max = nullptr;
  a.status = h->status;
  a.max_iters = 1;
  if (h->carry && !h->rbm_on && !h->mlp_on && g.dense && g.jdig) {
    // dense couplings: the carried state when it belongs to cfg, else the
    // population's state as one product into the spare carried buffer
    if (h->field_valid && h->field_cfg == cfg) {
      a.field_in = h->fbuf[h->fcur];
    } else {
      cudaError_t eg = launch_fields<T>(m, g, n, cfg, (T *)h->fbuf[1 - h->fcur], h->status, s);
      if (eg != cudaSuccess) return fail(GFMC_ERR_CUDA, "guide fields: %s", cudaGetErrorString(eg));
      a.field_in = h->fbuf[1 - h->fcur];
    }
  }
  cudaError_t e = launch_step<T>(h, m, g, a, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "local energy launch: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

}  // namespace

extern "C" {

int gfmc_create(const gfmc_model_desc *model, const gfmc_guide_desc *guide, int precision,
                gfmc_handle **out) {
  if (!model || !out) return fail(GFMC_ERR_INVALID, "null argument");
  if (model->n_sites <= 0) return fail(GFMC_ERR_INVALID, "n_sites must be positive");
  if (model->n_sites > 65535) return fail(GFMC_ERR_UNSUPPORTED, "at most 65535 sites");
  if (model->n_edges < 0 || (model->n_edges && (!model->edge_i || !model->edge_j)))
    return fail(GFMC_ERR_INVALID, "n_edges must be >= 0, with edge_i and edge_j given");
  if (precision != GFMC_PRECISION_FP64 && precision != GFMC_PRECISION_MIXED)
    return fail(GFMC_ERR_INVALID, "unknown precision %d", precision);
  gfmc_handle *h = new gfmc_handle();
  h->precision = precision;
  h->family = model->kind;
  h->N = model->n_sites;
  h->E = model->n_edges;
  h->n_max = model->n_max;
  int rc = precision == GFMC_PRECISION_FP64 ? build_tables<double>(h, model, guide, h->m64, h->g64)
                                            : build_tables<float>(h, model, guide, h->m32, h->g32);
  if (rc) {
    gfmc_destroy(h);
    return rc;
  }
  h->M = precision == GFMC_PRECISION_FP64 ? h->m64.M : h->m32.M;
  h->state_len = h->N;
  if (guide && guide->kind == GFMC_GUIDE_RBM_SPIN_HALF) {
    rc = build_rbm(h, model, guide, h->N);
    if (rc == GFMC_OK)
      h->rbm_grid = precision == GFMC_PRECISION_FP64 ? rbm_grid<double>(h->m64, h->rbm)
                                                     : rbm_grid<float>(h->m32, h->rbm);
    if (rc) {
      gfmc_destroy(h);
      return rc;
    }
  }
  if (guide && guide->kind == GFMC_GUIDE_MLP_BOSE_HUBBARD) {
    rc = build_mlp(h, guide, h->N, h->n_max);
    if (rc == GFMC_OK &&
        mlp_smem_bytes(h->mlp.H1, h->mlp.H2, h->M - 1, h->N) > (size_t)227 * 1024)
      rc = fail(GFMC_ERR_UNSUPPORTED, "MLP guide: %d moves with (%d, %d) hidden units exceed "
                "the shared memory of one SM", h->M - 1, h->mlp.H1, h->mlp.H2);
    if (rc) {
      gfmc_destroy(h);
      return rc;
    }
  }
  // float32 factors drift faster under the multiplicative updates
  h->refresh_every = precision == GFMC_PRECISION_FP64 ? 100 : 50;
  *out = h;
  g_last_error.clear();
  return GFMC_OK;
}

int gfmc_destroy(gfmc_handle *h) {
  if (!h) return GFMC_OK;
  cudaFree(h->d_tables);
  cudaFree(h->rctr);
  cudaFree(h->pmax); cudaFree(h->psum); cudaFree(h->pE); cudaFree(h->cdf); cudaFree(h->wbuf);
  cudaFree(h->plp); cudaFree(h->ctr); cudaFree(h->status); cudaFree(h->hops);
  cudaFree(h->fbuf[0]); cudaFree(h->fbuf[1]);
  cudaFree(h->ebuf[0]); cudaFree(h->ebuf[1]);
  cudaFree(h->d_ops); cudaFree(h->d_diag_tables); cudaFree(h->diag.ring_parents);
  cudaFree(h->diag.ring_vals); cudaFree(h->diag_partial);
  cudaFree(h->fw_partial); cudaFree(h->fw_logG); cudaFree(h->fw_E); cudaFree(h->ctr1);
  cudaFree(h->d_rbm);
  cudaFree(h->d_rbm_rt);
  cudaFree(h->d_rbm_ch);
  cudaFree(h->d_mlp);
  cudaFree(h->mtr_cfg); cudaFree(h->mtr_rates); cudaFree(h->mtr_rsum); cudaFree(h->mtr_gw);
  cudaFree(h->mtr_e); cudaFree(h->mtr_coef); cudaFree(h->mtr_h1); cudaFree(h->mtr_h1T);
  cudaFree(h->mtr_h1lo); cudaFree(h->mtr_d2); cudaFree(h->mtr_d2T); cudaFree(h->mtr_d1); cudaFree(h->mtr_stats);
  cudaFree(h->mtr_grad); cudaFree(h->mtr_p); cudaFree(h->mtr_m1); cudaFree(h->mtr_m2);
  cudaFree(h->tr_cfg); cudaFree(h->tr_theta); cudaFree(h->tr_rates); cudaFree(h->tr_rsum);
  cudaFree(h->tr_gw); cudaFree(h->tr_e); cudaFree(h->tr_stats); cudaFree(h->tr_gW);
  cudaFree(h->tr_gb); cudaFree(h->tr_ga); cudaFree(h->ms_W); cudaFree(h->ms_b); cudaFree(h->ms_a);
  cudaFree(h->ad_m); cudaFree(h->ad_v); cudaFree(h->tr_recs); cudaFree(h->dist_out);
  delete h;
  return GFMC_OK;
}

int gfmc_config_bytes(const gfmc_handle *h) { return h ? h->cfg_bytes : GFMC_ERR_INVALID; }
int gfmc_n_transitions(const gfmc_handle *h) { return h ? h->M : GFMC_ERR_INVALID; }

int gfmc_pack(gfmc_handle *h, int n, const double *cfg, void *packed, void *stream) {
  if (!h || n < 0 || (n && (!cfg || !packed))) return fail(GFMC_ERR_INVALID, "gfmc_pack: bad argument");
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  if (n == 0) return GFMC_OK;
  h->field_valid = 0;
  cudaError_t e = launch_pack(h->family, n, h->N, h->cfg_bytes, cfg, packed, h->n_max, h->status,
                              (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "pack: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_unpack(gfmc_handle *h, int n, const void *packed, double *cfg, void *stream) {
  if (!h || n < 0 || (n && (!cfg || !packed))) return fail(GFMC_ERR_INVALID, "gfmc_unpack: bad argument");
  if (n == 0) return GFMC_OK;
  cudaError_t e = launch_unpack(h->family, n, h->N, h->cfg_bytes, packed, cfg, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "unpack: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_run_steps(gfmc_handle *h, int method, double step, double lam, double alw, int n_steps,
                   const uint32_t *keys, int n_walkers, void *cfg, void *cfg_tmp, int32_t *parents,
                   int parents_valid, double *log_w, double *e_loc, double *logG_out,
                   double *E_out, uint64_t *hops_out, void *stream) {
  if (!h) return fail(GFMC_ERR_INVALID, "null handle");
  if (n_steps <= 0 || n_walkers <= 0) return fail(GFMC_ERR_INVALID, "n_steps and n_walkers must be positive");
  if (!keys || !cfg || !cfg_tmp || !parents || !log_w || !e_loc || !logG_out || !E_out)
    return fail(GFMC_ERR_INVALID, "gfmc_run_steps: null buffer");
  if (method < 0 || method > 2) return fail(GFMC_ERR_INVALID, "unknown method %d", method);
  if (method != GFMC_METHOD_CONT_TIME && (step < 1.0 || step != (double)(long long)step))
    return fail(GFMC_ERR_INVALID, "discrete methods need a positive integer step");
  if (!(step > 0.0)) return fail(GFMC_ERR_INVALID, "step must be > 0");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->precision == GFMC_PRECISION_FP64)
    return run_steps_t<double>(h, h->m64, h->g64, method, step, lam, alw, n_steps, keys, n_walkers,
                               cfg, cfg_tmp, parents, parents_valid, log_w, e_loc, logG_out, E_out,
                               hops_out, s);
  return run_steps_t<float>(h, h->m32, h->g32, method, step, lam, alw, n_steps, keys, n_walkers, cfg,
                            cfg_tmp, parents, parents_valid, log_w, e_loc, logG_out, E_out,
                            hops_out, s);
}

int gfmc_local_energy(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                      double *e_loc, void *stream) {
  if (!h || n <= 0 || !cfg || !e_loc) return fail(GFMC_ERR_INVALID, "gfmc_local_energy: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->precision == GFMC_PRECISION_FP64)
    return local_energy_t<double>(h, h->m64, h->g64, n, cfg, parents, e_loc, s);
  return local_energy_t<float>(h, h->m32, h->g32, n, cfg, parents, e_loc, s);
}

int gfmc_local_energy_parts(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                            double *e_loc, double *diag, void *stream) {
  if (!h || n <= 0 || !cfg || !e_loc || !diag)
    return fail(GFMC_ERR_INVALID, "gfmc_local_energy_parts: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->precision == GFMC_PRECISION_FP64)
    return local_energy_t<double>(h, h->m64, h->g64, n, cfg, parents, e_loc, s, diag);
  return local_energy_t<float>(h, h->m32, h->g32, n, cfg, parents, e_loc, s, diag);
}

int gfmc_gather(gfmc_handle *h, int n, const int32_t *parents, const void *cfg_in, void *cfg_out,
                const double *e_in, double *e_out, double *log_w, void *stream) {
  if (!h || n <= 0 || !cfg_in || !cfg_out || cfg_in == cfg_out)
    return fail(GFMC_ERR_INVALID, "gfmc_gather: bad argument");
  if (e_out && !e_in) return fail(GFMC_ERR_INVALID, "gfmc_gather: e_out given without e_in");
  cudaError_t e = launch_gather(n, h->cfg_bytes, parents, cfg_in, cfg_out, e_in, e_out, log_w,
                                (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "gather: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_windowed_energy(int n_steps, const double *logG, const double *E, int n_p, const int *p,
                         double *out, void *stream) {
  if (n_steps <= 0 || n_p <= 0 || !logG || !E || !p || !out)
    return fail(GFMC_ERR_INVALID, "gfmc_windowed_energy: bad argument");
  for (int i = 0; i < n_p; ++i)
    if (p[i] <= 0 || p[i] >= n_steps)
      return fail(GFMC_ERR_INVALID, "window p=%d must lie in [1, n_steps)", p[i]);
  cudaStream_t s = (cudaStream_t)stream;
  int *dp = nullptr;
  double *work = nullptr;
  GFMC_CUDA(cudaMalloc(&dp, sizeof(int) * n_p));
  cudaError_t e = cudaMalloc(&work, sizeof(double) * (n_steps + n_p));
  if (e != cudaSuccess) { cudaFree(dp); return fail(GFMC_ERR_CUDA, "windowed alloc: %s", cudaGetErrorString(e)); }
  e = cudaMemcpyAsync(dp, p, sizeof(int) * n_p, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_windowed(logG, E, n_steps, dp, n_p, work, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, work + n_steps, sizeof(double) * n_p, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dp);
  cudaFree(work);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "windowed energy: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_set_diag_operators(gfmc_handle *h, int n_ops, const gfmc_diag_desc *ops, int n_p,
                            const int *m_array) {
  if (!h || n_ops < 0 || (n_ops && !ops) || n_p < 1 || n_p > GFMC_DIAG_MAX_P || !m_array)
    return fail(GFMC_ERR_INVALID, "gfmc_set_diag_operators: bad argument (1 <= n_p <= %d)",
                GFMC_DIAG_MAX_P);
  for (int j = 0; j < n_p; ++j)
    if (m_array[j] < 0 || (j && m_array[j] < m_array[j - 1]))
      return fail(GFMC_ERR_INVALID, "m_array must be sorted and non-negative");
  cudaFree(h->d_ops); cudaFree(h->d_diag_tables);
  h->d_ops = nullptr; h->d_diag_tables = nullptr;
  h->diag_ready = 0;
  Arena A;
  std::vector<DiagOp> host(n_ops);
  std::vector<std::map<std::string, size_t>> offs(n_ops);
  int col = 0;
  for (int o = 0; o < n_ops; ++o) {
    const gfmc_diag_desc &d = ops[o];
    DiagOp &op = host[o];
    memset(&op, 0, sizeof(op));
    op.kind = d.kind;
    op.col = col;
    op.N = d.n_sites;
    op.E = d.n_edges;
    if (d.n_sites != h->N) return fail(GFMC_ERR_INVALID, "diagonal operator %d: n_sites %d != %d", o, d.n_sites, h->N);
    // every table a flag announces must be given (the kernels read it unchecked)
    if ((d.kind == GFMC_DIAG_SPIN_HALF &&
         (d.n_edges < 0 || (d.n_edges && (!d.edge_i || !d.edge_j)) ||
          (d.has_jz && !d.jz) || (d.has_hz && !d.hz))) ||
        (d.kind == GFMC_DIAG_BOSE_HUBBARD && ((d.has_U && !d.U) || (d.has_mu && !d.mu))))
      return fail(GFMC_ERR_INVALID, "diagonal operator %d: a table its flags announce is missing", o);
    auto addd = [&](const char *nm, const double *p, size_t cnt) {
      if (p && cnt) offs[o][nm] = A.add(p, cnt * sizeof(double));
    };
    if (d.kind == GFMC_DIAG_SPIN_HALF) {
      if (h->family != GFMC_MODEL_SPIN_HALF) return fail(GFMC_ERR_INVALID, "SpinHalf operator on bosons");
      std::vector<int> ei(d.n_edges), ej(d.n_edges);
      for (int e = 0; e < d.n_edges; ++e) {
        ei[e] = d.edge_i[e]; ej[e] = d.edge_j[e];
        if (ei[e] < 0 || ej[e] < 0 || ei[e] >= h->N || ej[e] >= h->N)
          return fail(GFMC_ERR_INVALID, "diagonal operator %d: edge out of range", o);
      }
      if (d.n_edges) {
        offs[o]["ei"] = A.add(ei.data(), ei.size() * 4);
        offs[o]["ej"] = A.add(ej.data(), ej.size() * 4);
      }
      op.has_jz = d.has_jz; op.uniform_jz = d.uniform_jz; op.has_hz = d.has_hz;
      addd("jz", d.jz, d.has_jz ? (d.uniform_jz ? 1 : d.n_edges) : 0);
      addd("hz", d.hz, d.has_hz ? d.n_sites : 0);
      col += 1;
    } else if (d.kind == GFMC_DIAG_BOSE_HUBBARD) {
      if (h->family != GFMC_MODEL_BOSE_HUBBARD) return fail(GFMC_ERR_INVALID, "BoseHubbard operator on spins");
      op.has_U = d.has_U; op.has_mu = d.has_mu;
      addd("U", d.U, d.has_U ? d.n_sites : 0);
      addd("mu", d.mu, d.has_mu ? d.n_sites : 0);
      col += 1;
    } else if (d.kind == GFMC_DIAG_SZSZ) {
      if (d.n_k < 1 || !d.cos_kr || !d.sin_kr) return fail(GFMC_ERR_INVALID, "SzSz operator %d: no wavevectors", o);
      op.n_k = d.n_k;
      op.offset = d.offset;
      addd("cos", d.cos_kr, (size_t)d.n_k * d.n_sites);
      addd("sin", d.sin_kr, (size_t)d.n_k * d.n_sites);
      col += d.n_k;
    } else {
      return fail(GFMC_ERR_UNSUPPORTED, "unknown diagonal operator kind %d", d.kind);
    }
  }
  GFMC_CUDA(cudaMalloc(&h->d_diag_tables, A.host.size() ? A.host.size() : 256));
  if (A.host.size())
    GFMC_CUDA(cudaMemcpy(h->d_diag_tables, A.host.data(), A.host.size(), cudaMemcpyHostToDevice));
  unsigned char *base = (unsigned char *)h->d_diag_tables;
  for (int o = 0; o < n_ops; ++o) {
    auto P = [&](const char *nm) -> const void * {
      auto it = offs[o].find(nm);
      return it == offs[o].end() ? nullptr : (const void *)(base + it->second);
    };
    host[o].ei = (const int *)P("ei"); host[o].ej = (const int *)P("ej");
    host[o].jz = (const double *)P("jz"); host[o].hz = (const double *)P("hz");
    host[o].U = (const double *)P("U"); host[o].mu = (const double *)P("mu");
    host[o].cos_kr = (const double *)P("cos"); host[o].sin_kr = (const double *)P("sin");
  }
  GFMC_CUDA(cudaMalloc(&h->d_ops, sizeof(DiagOp) * (n_ops ? n_ops : 1)));
  if (n_ops) GFMC_CUDA(cudaMemcpy(h->d_ops, host.data(), sizeof(DiagOp) * n_ops, cudaMemcpyHostToDevice));
  h->diag.n_ops = n_ops;
  h->diag.ops = h->d_ops;
  h->diag.width = col;
  h->diag.n_p = n_p;
  for (int j = 0; j < n_p; ++j) h->diag.m[j] = m_array[j];
  h->diag.m_max = m_array[n_p - 1];
  h->diag_cap_n = 0;   // rings sized again by gfmc_reset_diag
  return GFMC_OK;
}

int gfmc_diag_width(const gfmc_handle *h) { return h ? h->diag.width : GFMC_ERR_INVALID; }

int gfmc_reset_diag(gfmc_handle *h, int n, void *stream) {
  if (!h || n <= 0 || !h->d_ops) return fail(GFMC_ERR_INVALID, "gfmc_reset_diag: no operators set");
  cudaFree(h->diag.ring_parents); cudaFree(h->diag.ring_vals); cudaFree(h->diag_partial);
  h->diag.ring_parents = nullptr; h->diag.ring_vals = nullptr; h->diag_partial = nullptr;
  h->diag_ready = 0;   // until the rings below exist
  const size_t size = (size_t)(h->diag.m_max + 1);
  GFMC_CUDA(cudaMalloc(&h->diag.ring_parents, sizeof(int) * size * n));
  GFMC_CUDA(cudaMalloc(&h->diag.ring_vals, sizeof(double) * size * n * (h->diag.width ? h->diag.width : 1)));
  GFMC_CUDA(cudaMalloc(&h->diag_partial, sizeof(double) * (size_t)diag_walk_blocks(n) *
                                              (h->diag.width ? h->diag.width : 1) * h->diag.n_p));
  cudaError_t e = launch_diag_reset(h->diag, n, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "diag reset: %s", cudaGetErrorString(e));
  h->diag_cap_n = n;
  h->diag_slot = 0;
  h->diag_ready = 1;
  return GFMC_OK;
}

int gfmc_set_diag_output(gfmc_handle *h, double *out) {
  if (!h) return fail(GFMC_ERR_INVALID, "null handle");
  h->diag_out = out;
  return GFMC_OK;
}

int gfmc_set_max_iters(gfmc_handle *h, int max_iters) {
  if (!h || max_iters < 1) return fail(GFMC_ERR_INVALID, "max_iters must be >= 1");
  h->max_iters = max_iters;
  return GFMC_OK;
}

int gfmc_carry_mode(gfmc_handle *h, int mode, int *carrying_out) {
  if (!h || mode > 1) return fail(GFMC_ERR_INVALID, "gfmc_carry_mode: bad argument");
  if (mode >= 0 && mode != h->carry_mode) {
    h->carry_mode = mode;
    if (h->carry_optional) {
      // takes effect at the next call that sizes the buffers
      h->carry = h->carry_pref && mode;
      h->field_valid = 0;
      h->eval_valid = 0;
    }
  }
  if (carrying_out) *carrying_out = h->carry;
  return GFMC_OK;
}

int gfmc_read_status(gfmc_handle *h, int *status_out, void *stream) {
  if (!h || !status_out) return fail(GFMC_ERR_INVALID, "gfmc_read_status: bad argument");
  *status_out = 0;
  if (!h->status) return GFMC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int v = 0;
  GFMC_CUDA(cudaMemcpyAsync(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  GFMC_CUDA(cudaStreamSynchronize(s));
  GFMC_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), s));
  *status_out = v;
  return GFMC_OK;
}

int gfmc_key_schedule(const uint32_t key[2], int n_steps, uint32_t *keys_out, uint32_t key_next[2]) {
  if (!key || n_steps < 0 || (n_steps && !keys_out) || !key_next)
    return fail(GFMC_ERR_INVALID, "gfmc_key_schedule: bad argument");
  Key k{key[0], key[1]};
  for (int s = 0; s < n_steps; ++s) {
    Key nk = fold(k, 0u), rng = fold(k, 1u);
    Key k1 = fold(rng, 0u), k2 = fold(rng, 1u);
    keys_out[4 * s + 0] = k1.a; keys_out[4 * s + 1] = k1.b;
    keys_out[4 * s + 2] = k2.a; keys_out[4 * s + 3] = k2.b;
    k = nk;
  }
  key_next[0] = k.a;
  key_next[1] = k.b;
  return GFMC_OK;
}

int gfmc_rbm_theta(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                   int parents_valid, float *theta_out, void *stream) {
  if (!h || n <= 0 || !cfg || !theta_out || (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_rbm_theta: bad argument");
  if (!h->rbm_on) return fail(GFMC_ERR_INVALID, "gfmc_rbm_theta: the handle has no RBM guide");
  if (!h->status) {
    GFMC_CUDA(cudaMalloc(&h->status, sizeof(int)));
    GFMC_CUDA(cudaMemset(h->status, 0, sizeof(int)));
  }
  cudaError_t e = launch_rbm_theta(h->rbm, n, cfg, parents_valid ? parents : nullptr,
                                   (h->N + 63) / 64, theta_out, h->status, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "theta GEMM: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_rbm_gradient(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                      int parents_valid, const double *omega, float *grad_W, float *grad_b,
                      float *grad_a, double stats[2], void *stream) {
  if (!h || n <= 0 || !cfg || !stats || (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_rbm_gradient: bad argument");
  if (!h->rbm_on) return fail(GFMC_ERR_INVALID, "gfmc_rbm_gradient: the handle has no RBM guide");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = rbm_gradient_t(h, n, cfg, parents, parents_valid, omega, s);
  if (rc) return rc;
  const RbmTables &r = h->rbm;
  if (grad_W)
    GFMC_CUDA(cudaMemcpy2DAsync(grad_W, sizeof(float) * h->N, h->tr_gW, sizeof(float) * r.Np,
                                sizeof(float) * h->N, r.H, cudaMemcpyDeviceToDevice, s));
  if (grad_b)
    GFMC_CUDA(cudaMemcpyAsync(grad_b, h->tr_gb, sizeof(float) * r.H, cudaMemcpyDeviceToDevice, s));
  if (grad_a)
    GFMC_CUDA(cudaMemcpyAsync(grad_a, h->tr_ga, sizeof(float) * h->N, cudaMemcpyDeviceToDevice, s));
  GFMC_CUDA(cudaMemcpyAsync(stats, h->tr_stats, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  GFMC_CUDA(cudaStreamSynchronize(s));
  return GFMC_OK;
}

int gfmc_rbm_train_step(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                        int parents_valid, const double *omega, double lr, double stats[2],
                        void *stream) {
  if (!h || n <= 0 || !cfg || !stats || (parents_valid && !parents) || !(lr > 0.0))
    return fail(GFMC_ERR_INVALID, "gfmc_rbm_train_step: bad argument");
  if (!h->rbm_on) return fail(GFMC_ERR_INVALID, "gfmc_rbm_train_step: the handle has no RBM guide");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = rbm_gradient_t(h, n, cfg, parents, parents_valid, omega, s);
  if (rc) return rc;
  RbmTables &r = h->rbm;
  const size_t P = (size_t)r.H * h->N + r.H + h->N;
  if (!h->adam_ready) {
    // (a first call that failed part-way may have left some of them)
    cudaFree(h->ms_W); cudaFree(h->ms_b); cudaFree(h->ms_a); cudaFree(h->ad_m); cudaFree(h->ad_v);
    h->ms_W = h->ms_b = h->ms_a = h->ad_m = h->ad_v = nullptr;
    GFMC_CUDA(cudaMalloc(&h->ms_W, sizeof(float) * (size_t)r.H * h->N));
    GFMC_CUDA(cudaMalloc(&h->ms_b, sizeof(float) * r.H));
    GFMC_CUDA(cudaMalloc(&h->ms_a, sizeof(float) * h->N));
    GFMC_CUDA(cudaMalloc(&h->ad_m, sizeof(float) * P));
    GFMC_CUDA(cudaMalloc(&h->ad_v, sizeof(float) * P));
    GFMC_CUDA(cudaMemsetAsync(h->ad_m, 0, sizeof(float) * P, s));
    GFMC_CUDA(cudaMemsetAsync(h->ad_v, 0, sizeof(float) * P, s));
    cudaError_t e = launch_rbm_master_init(r, h->N, h->ms_W, h->ms_b, h->ms_a, s);
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "master init: %s", cudaGetErrorString(e));
    h->adam_step = 0;
    h->adam_ready = 1;
  }
  h->adam_step += 1;
  cudaError_t e = launch_adam(r.H, h->N, r.Hp, r.Np, h->ms_W, h->ms_b, h->ms_a, h->tr_gW, h->tr_gb,
                              h->tr_ga, h->ad_m, h->ad_v, (float)lr, 0.9f, 0.999f, 1e-8f,
                              h->adam_step, (__nv_bfloat16 *)r.WT, (__nv_bfloat16 *)r.W,
                              (float *)r.b, (float *)r.a, s);
  if (e == cudaSuccess) e = launch_rbm_derive(r, h->N, s);   // the float32 kernel's tables
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "Adam step: %s", cudaGetErrorString(e));
  // the guide changed: carried theta is stale
  h->field_valid = 0;
  GFMC_CUDA(cudaMemcpyAsync(stats, h->tr_stats, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  GFMC_CUDA(cudaStreamSynchronize(s));
  return GFMC_OK;
}

int gfmc_rbm_get_params(gfmc_handle *h, float *W, float *b, float *a) {
  if (!h || !h->rbm_on || !W || !b || !a) return fail(GFMC_ERR_INVALID, "gfmc_rbm_get_params: bad argument");
  const RbmTables &r = h->rbm;
  std::vector<uint16_t> Wt((size_t)r.Hp * r.Np);
  GFMC_CUDA(cudaMemcpy(Wt.data(), r.W, Wt.size() * 2, cudaMemcpyDeviceToHost));
  for (int hh = 0; hh < r.H; ++hh)
    for (int i = 0; i < h->N; ++i) {
      const uint32_t u = (uint32_t)Wt[(size_t)hh * r.Np + i] << 16;
      memcpy(&W[(size_t)hh * h->N + i], &u, 4);
    }
  GFMC_CUDA(cudaMemcpy(b, r.b, sizeof(float) * r.H, cudaMemcpyDeviceToHost));
  GFMC_CUDA(cudaMemcpy(a, r.a, sizeof(float) * h->N, cudaMemcpyDeviceToHost));
  return GFMC_OK;
}

long long gfmc_mlp_param_count(const gfmc_handle *h) {
  if (!h || !h->mlp_on) return GFMC_ERR_INVALID;
  return mlp_param_count(h->mlp.H1, h->mlp.H2, h->N * h->mlp.np1);
}

int gfmc_mlp_gradient(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                      int parents_valid, const double *omega, float *grad, double stats[2],
                      void *stream) {
  if (!h || n <= 0 || !cfg || !stats || (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_mlp_gradient: bad argument");
  if (!h->mlp_on) return fail(GFMC_ERR_INVALID, "gfmc_mlp_gradient: the handle has no MLP guide");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = mlp_gradient_t(h, n, cfg, parents, parents_valid, omega, s);
  if (rc) return rc;
  const long long np = mlp_param_count(h->mlp.H1, h->mlp.H2, h->N * h->mlp.np1);
  if (grad)
    GFMC_CUDA(cudaMemcpyAsync(grad, h->mtr_grad, sizeof(float) * (size_t)np,
                              cudaMemcpyDeviceToDevice, s));
  GFMC_CUDA(cudaMemcpyAsync(stats, h->mtr_stats, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  GFMC_CUDA(cudaStreamSynchronize(s));
  return GFMC_OK;
}

int gfmc_mlp_train_step(gfmc_handle *h, int n, const void *cfg, const int32_t *parents,
                        int parents_valid, const double *omega, double lr, double stats[2],
                        void *stream) {
  if (!h || n <= 0 || !cfg || !stats || (parents_valid && !parents) || !(lr > 0.0))
    return fail(GFMC_ERR_INVALID, "gfmc_mlp_train_step: bad argument");
  if (!h->mlp_on) return fail(GFMC_ERR_INVALID, "gfmc_mlp_train_step: the handle has no MLP guide");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = mlp_gradient_t(h, n, cfg, parents, parents_valid, omega, s);
  if (rc) return rc;
  const MlpTables &t = h->mlp;
  const int D = h->N * t.np1;
  const long long np = mlp_param_count(t.H1, t.H2, D);
  if (!h->mtr_ready) {
    // (a first call that failed part-way may have left some of them)
    cudaFree(h->mtr_p); cudaFree(h->mtr_m1); cudaFree(h->mtr_m2);
    h->mtr_p = h->mtr_m1 = h->mtr_m2 = nullptr;
    GFMC_CUDA(cudaMalloc(&h->mtr_p, sizeof(float) * (size_t)np));
    GFMC_CUDA(cudaMalloc(&h->mtr_m1, sizeof(float) * (size_t)np));
    GFMC_CUDA(cudaMalloc(&h->mtr_m2, sizeof(float) * (size_t)np));
    GFMC_CUDA(cudaMemsetAsync(h->mtr_m1, 0, sizeof(float) * (size_t)np, s));
    GFMC_CUDA(cudaMemsetAsync(h->mtr_m2, 0, sizeof(float) * (size_t)np, s));
    cudaError_t e = launch_mlp_master_init(t, D, h->mtr_p, s);
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "MLP master init: %s", cudaGetErrorString(e));
    h->mtr_step = 0;
    h->mtr_ready = 1;
  }
  h->mtr_step += 1;
  cudaError_t e = launch_mlp_adam(np, h->mtr_p, h->mtr_grad, h->mtr_m1, h->mtr_m2, (float)lr,
                                  h->mtr_step, s);
  if (e == cudaSuccess)
    e = launch_mlp_tables(t, D, h->mtr_p, (__nv_bfloat16 *)t.W1T, (float *)t.b1,
                          (__nv_bfloat16 *)t.W2, (__nv_bfloat16 *)t.W2T, (float *)t.b2,
                          (float *)t.w3, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "MLP Adam step: %s", cudaGetErrorString(e));
  // the guide changed: the carried z1 and log psi are stale
  h->field_valid = 0;
  GFMC_CUDA(cudaMemcpyAsync(stats, h->mtr_stats, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  GFMC_CUDA(cudaStreamSynchronize(s));
  return GFMC_OK;
}

int gfmc_mlp_get_params(gfmc_handle *h, float *params) {
  if (!h || !h->mlp_on || !params) return fail(GFMC_ERR_INVALID, "gfmc_mlp_get_params: bad argument");
  const MlpTables &t = h->mlp;
  const int D = h->N * t.np1;
  const long long np = mlp_param_count(t.H1, t.H2, D);
  float *tmp = nullptr;
  GFMC_CUDA(cudaMalloc(&tmp, sizeof(float) * (size_t)np));
  cudaError_t e = launch_mlp_master_init(t, D, tmp, 0);
  if (e == cudaSuccess) e = cudaMemcpy(params, tmp, sizeof(float) * (size_t)np, cudaMemcpyDeviceToHost);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "gfmc_mlp_get_params: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_rbm_hidden_padded(const gfmc_handle *h) {
  return (h && h->rbm_on) ? h->rbm.Hp : GFMC_ERR_INVALID;
}

// The evolve half of a step alone (gfmc_evolve, gfmc_evolve_walkers): lw_in,
// when given, seeds each walker's log weight (read at its parent); log_w may
// be the same array when there is no parent map, since the warp that owns a
// walker reads its entry before it writes it and no other warp touches it.
static int evolve_only(gfmc_handle *h, const char *name, int method, double step, double lam,
                       double alw, const uint32_t key[2], long long walker_offset, int n,
                       const void *cfg, const int32_t *parents, int parents_valid, void *cfg_out,
                       const double *lw_in, double *log_w, double *e_loc, uint64_t *hops,
                       void *stream) {
  if (!h || !key || n <= 0 || !cfg || !cfg_out || cfg == cfg_out || !log_w || !e_loc ||
      (parents_valid && !parents) || walker_offset < 0 || (lw_in == log_w && parents_valid))
    return fail(GFMC_ERR_INVALID, "%s: bad argument", name);
  int rc = check_method(method, step);
  if (rc) return rc;
  if (h->mlp_on && method != CONT_TIME)
    return fail(GFMC_ERR_UNSUPPORTED, "the MLP guide propagates with cont_time only");
  rc = ensure_scratch(h, n, 1);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  GFMC_CUDA(cudaMemsetAsync(h->ctr, 0, sizeof(int), s));
  if (hops) GFMC_CUDA(cudaMemsetAsync(hops, 0, sizeof(uint64_t), s));
  EvolveArgs a{};
  a.method = method;
  a.step = step;
  a.lam = lam;
  a.alw = alw;
  a.key = Key{key[0], key[1]};
  a.walker_offset = walker_offset;
  a.n_walkers = n;
  a.parents = parents_valid ? parents : nullptr;
  a.cfg_in = cfg;
  a.cfg_out = cfg_out;
  a.log_w = log_w;
  a.lw_in = lw_in;
  a.e_loc = e_loc;
  a.hops = (unsigned long long *)hops;
  a.work_ctr = h->ctr;
  a.status = h->status;
  a.max_iters = h->max_iters;
  h->field_valid = 0;   // carried state is not kept across a sharded step
  cudaError_t e = cudaSuccess;
  const bool dense_state = h->carry && !h->rbm_on && !h->mlp_on &&
                           (h->precision == GFMC_PRECISION_FP64 ? h->g64.dense && h->g64.jdig
                                                                : h->g32.dense && h->g32.jdig);
  if (dense_state) {
    // the guide state of cfg's rows as one product (read through the parents)
    e = h->precision == GFMC_PRECISION_FP64
            ? launch_fields<double>(h->m64, h->g64, n, cfg, (double *)h->fbuf[h->fcur], h->status, s)
            : launch_fields<float>(h->m32, h->g32, n, cfg, (float *)h->fbuf[h->fcur], h->status, s);
    a.field_in = h->fbuf[h->fcur];
  }
  if (e == cudaSuccess)
    e = h->precision == GFMC_PRECISION_FP64 ? launch_step<double>(h, h->m64, h->g64, a, s)
                                            : launch_step<float>(h, h->m32, h->g32, a, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "evolve launch: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_evolve(gfmc_handle *h, int method, double step, double lam, double alw,
                const uint32_t key[2], long long walker_offset, int n, const void *cfg,
                const int32_t *parents, int parents_valid, void *cfg_out, double *log_w,
                double *e_loc, uint64_t *hops, void *stream) {
  return evolve_only(h, "gfmc_evolve", method, step, lam, alw, key, walker_offset, n, cfg, parents,
                     parents_valid, cfg_out, nullptr, log_w, e_loc, hops, stream);
}

int gfmc_evolve_walkers(gfmc_handle *h, int method, double step, double lam, double alw,
                        const uint32_t key[2], int n, const void *cfg, void *cfg_out,
                        double *log_w, double *e_loc, uint64_t *hops, void *stream) {
  return evolve_only(h, "gfmc_evolve_walkers", method, step, lam, alw, key, 0, n, cfg, nullptr, 0,
                     cfg_out, log_w, log_w, e_loc, hops, stream);
}

static int dist_prepare(gfmc_handle *h, int n) {
  int rc = ensure_scratch(h, n, 1);
  if (rc) return rc;
  if (!h->dist_out) GFMC_CUDA(cudaMalloc(&h->dist_out, sizeof(double) * 4));
  return GFMC_OK;
}

int gfmc_dist_local_max(gfmc_handle *h, int n, const double *log_w, double *max_out,
                        void *stream) {
  if (!h || n <= 0 || !log_w || !max_out)
    return fail(GFMC_ERR_INVALID, "gfmc_dist_local_max: bad argument");
  int rc = dist_prepare(h, n);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = launch_dist_max(n, log_w, h->psum, h->dist_out, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(max_out, h->dist_out, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "dist max: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_dist_local_sums(gfmc_handle *h, int n, const double *log_w, const double *e_loc,
                         double shift, double out[3], void *stream) {
  if (!h || n <= 0 || !log_w || !e_loc || !out)
    return fail(GFMC_ERR_INVALID, "gfmc_dist_local_sums: bad argument");
  int rc = dist_prepare(h, n);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = launch_dist_sums(n, log_w, e_loc, shift, nullptr, h->psum, h->pE, h->plp,
                                   h->dist_out, s);
  double tmp[4];
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(tmp, h->dist_out, sizeof(double) * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "dist sums: %s", cudaGetErrorString(e));
  out[0] = tmp[1];
  out[1] = tmp[2];
  out[2] = tmp[3];
  return GFMC_OK;
}

int gfmc_dist_local_max_dev(gfmc_handle *h, int n, const double *log_w, double *max_out,
                            void *stream) {
  if (!h || n <= 0 || !log_w || !max_out)
    return fail(GFMC_ERR_INVALID, "gfmc_dist_local_max_dev: bad argument");
  int rc = dist_prepare(h, n);
  if (rc) return rc;
  cudaError_t e = launch_dist_max(n, log_w, h->psum, max_out, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "dist max: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_dist_local_sums_dev(gfmc_handle *h, int n, const double *log_w, const double *e_loc,
                             const double *shift, double *out, void *stream) {
  if (!h || n <= 0 || !log_w || !e_loc || !shift || !out)
    return fail(GFMC_ERR_INVALID, "gfmc_dist_local_sums_dev: bad argument");
  int rc = dist_prepare(h, n);
  if (rc) return rc;
  cudaError_t e = launch_dist_sums(n, log_w, e_loc, 0.0, shift, h->psum, h->pE, h->plp, out,
                                   (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "dist sums: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_dist_parents(gfmc_handle *h, int n, const double *log_w, double shift, double offset,
                      double S_total, double psi, long long N_total, long long slot_lo, int count,
                      int last_pos, int32_t *parents_out, void *stream) {
  if (!h || n <= 0 || !log_w || count < 0 || (count && !parents_out) || N_total <= 0 ||
      last_pos < 0 || last_pos >= n || slot_lo < 0 || slot_lo + count > N_total)
    return fail(GFMC_ERR_INVALID, "gfmc_dist_parents: bad argument");
  int rc = dist_prepare(h, n);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the tile sums of this shift (the weighted-energy partials are not used)
  cudaError_t e = launch_dist_sums(n, log_w, log_w, shift, nullptr, h->psum, h->pE, h->plp,
                                   h->dist_out, s);
  if (e == cudaSuccess)
    e = launch_dist_parents(n, log_w, shift, offset, h->psum, h->cdf, h->wbuf, psi, S_total,
                            N_total, slot_lo, count, last_pos, parents_out, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "dist parents: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_key_schedule_ex(const uint32_t key[2], int n_steps, int n_sub, uint32_t *keys_out,
                         uint32_t key_next[2]) {
  if (!key || n_steps < 0 || n_sub < 1 || (n_steps && !keys_out) || !key_next)
    return fail(GFMC_ERR_INVALID, "gfmc_key_schedule_ex: bad argument");
  Key k{key[0], key[1]};
  for (int s = 0; s < n_steps; ++s) {
    const Key nk = fold(k, 0u), rng = fold(k, 1u);
    for (int j = 0; j < n_sub; ++j) {
      const Key kj = fold(rng, (uint32_t)j);
      keys_out[2 * ((size_t)s * n_sub + j) + 0] = kj.a;
      keys_out[2 * ((size_t)s * n_sub + j) + 1] = kj.b;
    }
    k = nk;
  }
  key_next[0] = k.a;
  key_next[1] = k.b;
  return GFMC_OK;
}

int gfmc_apply_operator(gfmc_handle *op, const uint32_t key[2], int n, const void *cfg,
                        const int32_t *parents, int parents_valid, void *cfg_out, double *vals,
                        void *stream) {
  if (!op || !key || n <= 0 || !cfg || !cfg_out || !vals || cfg == cfg_out ||
      (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_apply_operator: bad argument");
  return single_launch(op, APPLY, Key{key[0], key[1]}, n, cfg, parents_valid ? parents : nullptr,
                       cfg_out, vals, (cudaStream_t)stream);
}

int gfmc_operator_min_rate(gfmc_handle *op, int n, const void *cfg, const int32_t *parents,
                           int parents_valid, double *min_out, void *stream) {
  if (!op || n <= 0 || !cfg || !min_out || (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_operator_min_rate: bad argument");
  return single_launch(op, MIN_RATE, Key{0u, 0u}, n, cfg, parents_valid ? parents : nullptr,
                       nullptr, min_out, (cudaStream_t)stream);
}

int gfmc_forward_walk(gfmc_handle *sh, gfmc_handle *op, int method, double step, double lam,
                      double alw, const uint32_t apply_key[2], const uint32_t *shadow_keys, int n,
                      const void *cfg, const int32_t *parents, int parents_valid, void *s_cfg,
                      void *s_cfg_tmp, int32_t *s_parents, double *s_log_w, double *s_e_loc,
                      double *vals, double *vals_tmp, int n_m, const int *m_array,
                      double *val_out, double *norm_out, void *stream) {
  if (!sh || !op || !apply_key || n <= 0 || !cfg || !s_cfg || !s_cfg_tmp || !s_parents ||
      !s_log_w || !s_e_loc || !vals || !vals_tmp || !m_array || !val_out || !norm_out ||
      (parents_valid && !parents))
    return fail(GFMC_ERR_INVALID, "gfmc_forward_walk: bad argument");
  if (cfg == s_cfg || cfg == s_cfg_tmp || s_cfg == s_cfg_tmp || vals == vals_tmp)
    return fail(GFMC_ERR_INVALID, "gfmc_forward_walk: the shadow buffers must be distinct from "
                                  "each other and from the main population");
  if (n_m < 1 || n_m > GFMC_FW_MAX_P)
    return fail(GFMC_ERR_INVALID, "gfmc_forward_walk: 1 <= n_m <= %d", GFMC_FW_MAX_P);
  for (int j = 0; j < n_m; ++j)
    if (m_array[j] < 0 || (j && m_array[j] < m_array[j - 1]))
      return fail(GFMC_ERR_INVALID, "m_array must be sorted and non-negative");
  if (sh->precision != op->precision || sh->family != op->family || sh->N != op->N)
    return fail(GFMC_ERR_INVALID, "operator and shadow handles differ in precision, model family "
                                  "or site count");
  const int m_max = m_array[n_m - 1];
  if (m_max > 0) {
    if (!shadow_keys) return fail(GFMC_ERR_INVALID, "gfmc_forward_walk: shadow_keys missing");
    int rc = check_method(method, step);
    if (rc) return rc;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = fw_blocks(n);
  const int rows = m_max + 1;
  if (rows > sh->fw_cap_rows || nb > sh->fw_cap_nb) {
    cudaFree(sh->fw_partial); cudaFree(sh->fw_logG); cudaFree(sh->fw_E);
    sh->fw_partial = sh->fw_logG = sh->fw_E = nullptr;
    sh->fw_cap_rows = sh->fw_cap_nb = 0;
    GFMC_CUDA(cudaMalloc(&sh->fw_partial, sizeof(double) * (size_t)rows * nb));
    GFMC_CUDA(cudaMalloc(&sh->fw_logG, sizeof(double) * rows));
    GFMC_CUDA(cudaMalloc(&sh->fw_E, sizeof(double) * rows));
    sh->fw_cap_rows = rows;
    sh->fw_cap_nb = nb;
  }
  // 1. the operator on the main population (apply_operator_one, vmapped)
  int rc = single_launch(op, APPLY, Key{apply_key[0], apply_key[1]}, n, cfg,
                         parents_valid ? parents : nullptr, s_cfg, vals, s);
  if (rc) return rc;
  // 2. depth 0: the un-propagated values
  std::vector<char> rec(rows, 0);
  for (int j = 0; j < n_m; ++j) rec[m_array[j]] = 1;
  cudaError_t e = cudaSuccess;
  if (rec[0]) {
    e = launch_fw_remap(n, nullptr, vals, nullptr, sh->fw_partial, s);
    if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "forward-walk sum: %s", cudaGetErrorString(e));
  }
  // 3. the shadow chain, the values following every parent map
  if (m_max > 0) {
    FwHook hook{{vals, vals_tmp}, 0, rec.data(), sh->fw_partial, nb};
    double *saved_diag = sh->diag_out;
    sh->diag_out = nullptr;
    sh->fw = &hook;
    rc = gfmc_run_steps(sh, method, step, lam, alw, m_max, shadow_keys, n, s_cfg, s_cfg_tmp,
                        s_parents, 0, s_log_w, s_e_loc, sh->fw_logG, sh->fw_E, nullptr, stream);
    sh->fw = nullptr;
    sh->diag_out = saved_diag;
    if (rc) return rc;
  }
  // 4. means and accumulated log norms at the recorded depths
  FwRows r{};
  r.n_m = n_m;
  for (int j = 0; j < n_m; ++j) r.m[j] = m_array[j];
  e = launch_fw_finish(sh->fw_partial, nb, n, sh->fw_logG, r, val_out, norm_out, s);
  if (e != cudaSuccess) return fail(GFMC_ERR_CUDA, "forward-walk finish: %s", cudaGetErrorString(e));
  return GFMC_OK;
}

int gfmc_threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t out[2]) {
  if (!out) return fail(GFMC_ERR_INVALID, "null output");
  threefry2x32(k0, k1, c0, c1, out[0], out[1]);
  return GFMC_OK;
}

int gfmc_last_error(char *buf, size_t len) {
  if (!buf || !len) return GFMC_ERR_INVALID;
  snprintf(buf, len, "%s", g_last_error.c_str());
  return GFMC_OK;
}

const char *gfmc_version(void) { return "gfmc_b200 0.1.0 (sm_100a)"; }

}  // extern "C"

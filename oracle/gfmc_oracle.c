/*
 * CPU oracle for the GFMC hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement, in float64, of the reference algorithm that
 * pygfmc.run executes per walker and per branching step.  It is the checker
 * the CUDA engine is compared against and the timed CPU baseline; nothing in
 * the product links or calls it.  Every function names the reference source
 * (paths relative to the PyGFMC project root) whose semantics it restates.
 *
 * Random numbers: the JAX Threefry-2x32 stream (Salmon et al., SC'11, 20
 * rounds, the Random123 rotation constants) with JAX's key semantics:
 *   split(key)[i] = fold_in(key, i) = threefry2x32(key, (0, i))
 *   uniform64(key) = bits (y0 << 32 | y1) of threefry2x32(key, (0, 0)),
 *                    top 52 bits as the mantissa of [1, 2), minus 1.
 * Pinned by the rng_key -> rng_key_next pairs of the reference's golden file
 * (tests/core/reference_data/golden_cpu.npz, 300 splits each).
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Threefry-2x32 (jax._src.prng threefry2x32 semantics)                      */
/* ------------------------------------------------------------------------- */
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

void om_threefry2x32(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1,
                     uint32_t *o0, uint32_t *o1) {
  static const int R[2][4] = {{13, 15, 26, 6}, {17, 29, 16, 24}};
  uint32_t ks[3] = {k0, k1, k0 ^ k1 ^ 0x1BD11BDAu};
  uint32_t x0 = c0 + ks[0], x1 = c1 + ks[1];
  for (int i = 0; i < 5; ++i) {
    for (int j = 0; j < 4; ++j) {
      x0 += x1; x1 = rotl32(x1, R[i & 1][j]); x1 ^= x0;
    }
    x0 += ks[(i + 1) % 3];
    x1 += ks[(i + 2) % 3] + (uint32_t)(i + 1);
  }
  *o0 = x0; *o1 = x1;
}

typedef struct { uint32_t a, b; } om_key;

static inline om_key om_fold(om_key k, uint32_t d) {
  om_key r; om_threefry2x32(k.a, k.b, 0u, d, &r.a, &r.b); return r;
}

/* jax.random.uniform(key) for float64 (jax._src.random._uniform). */
static inline double om_uniform64(om_key k) {
  uint32_t y0, y1; om_threefry2x32(k.a, k.b, 0u, 0u, &y0, &y1);
  uint64_t bits = (((uint64_t)y0 << 32) | (uint64_t)y1) >> 12;
  bits |= 0x3FF0000000000000ull;
  double f; memcpy(&f, &bits, 8);
  return f - 1.0;
}

void om_fold_in(const uint32_t key[2], uint32_t d, uint32_t out[2]) {
  om_key k = {key[0], key[1]}; om_key r = om_fold(k, d); out[0] = r.a; out[1] = r.b;
}
double om_uniform(const uint32_t key[2]) { om_key k = {key[0], key[1]}; return om_uniform64(k); }

/* ------------------------------------------------------------------------- */
/* Model and guide descriptions (filled from Python, all arrays float64).    */
/* ------------------------------------------------------------------------- */
typedef struct {
  int kind;                 /* 0 SpinHalf, 1 BoseHubbard */
  int N, n_edges;
  const int *ei, *ej;
  /* SpinHalf (hamiltonian/SpinHalf.py:70-142): per-edge couplings,
   * stored fields (h_z = -public h_z, hx_half = -public h_x / 2). */
  int n_hx, n_jpm, has_jz, uniform_jz, has_hz;
  const double *jz, *jpm, *jpmpm, *hz, *hx_half;
  /* BoseHubbard (hamiltonian/bose_hubbard.py:67-120). */
  int n_max, n_hop, n_eta, n_hpm, has_U, has_mu;
  const double *t, *eta, *U, *mu, *hpm;   /* per edge / per site (broadcast) */
} om_model;

typedef struct {
  int kind;                 /* 0 none, 1 JastrowSpinHalf, 2 JastrowBoseHubbard */
  int max_deg;
  /* JastrowSpinHalf (wavefunction/jastrow_spin_half.py): per-site partner
   * tables (N, max_deg), padding has J = 0; per-H-edge external partner
   * tables (n_edges, 2, max_deg) as JastrowOpCache (build_cache:400-459). */
  const int *site_other; const double *site_J;
  const int *edge_other; const double *edge_J;
  const double *h;          /* (N,) one-body field */
  /* JastrowBoseHubbard (wavefunction/jastrow_bose_hubbard.py): pairs with
   * per-pair neighbour-sum weights (-beta, or 1 for a tied beta), the per
   * transition summed pair weight of the cache, tied/array forms. */
  int n_pairs; const int *pair_i, *pair_j; const double *pair_wt;
  const double *trans_pw;   /* (M,) pair_w of JastrowBoseHubbardOpCache */
  int beta_tied; double beta0;
  int h_mode;  double h0;   /* 0 none, 1 tied (h0), 2 array (h) */
  int d_mode;  double d0; const double *d;
  /* RBM (no PyGFMC counterpart): log psi = sum_h log cosh(b_h + sum_i W_hi s_i) + a.s,
   * W (n_hidden, N) row-major with bfloat16-representable values. */
  int n_hidden; const double *rbm_W, *rbm_b, *rbm_a;
  /* Bose-Hubbard MLP (no PyGFMC counterpart): one-hot occupations ->
   * H1 tanh -> (bf16) -> H2 tanh -> w3 . h2 + b3; W1 (H1, N np1), W2 (H2, H1). */
  int mlp_H1, mlp_H2, mlp_np1;
  const double *mlp_W1, *mlp_b1, *mlp_W2, *mlp_b2, *mlp_w3;
  double mlp_b3;
  /* ExactGroundState (wavefunction/exact_ground_state.py:43-190) on spin-1/2:
   * log |psi_0| over the 2^N basis states, indexed over the digits of
   * SpinHalf.local_hilbert_space (1, -1) with site 0 most significant. */
  int exact_N; const double *log_amp;
} om_guide;

/* Extra scratch doubles om_rates needs for a guide (theta and theta'). */
static inline int om_guide_scratch(const om_guide *g) {
  if (g && g->kind == 3) return 2 * g->n_hidden;
  if (g && g->kind == 4) return 2 * g->mlp_H1 + 4096;
  return 0;
}

/* float64 -> nearest bfloat16 (through float32, ties to even) */
static double om_bf16(double v) {
  float f = (float)v;
  uint32_t u; memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &u, 4);
  return (double)f;
}

/* MLP log amplitude of occupations n (length N) */
static double mlp_logpsi(const om_guide *g, int N, const double *n, double *z1) {
  const int H1 = g->mlp_H1, H2 = g->mlp_H2, D = N * g->mlp_np1;
  for (int h = 0; h < H1; ++h) {
    double z = g->mlp_b1[h];
    for (int k = 0; k < N; ++k) z += g->mlp_W1[(size_t)h * D + k * g->mlp_np1 + (int)n[k]];
    z1[h] = om_bf16(tanh(z));
  }
  double lp = g->mlp_b3;
  for (int j = 0; j < H2; ++j) {
    double z = g->mlp_b2[j];
    for (int h = 0; h < H1; ++h) z += g->mlp_W2[(size_t)j * H1 + h] * z1[h];
    lp += g->mlp_w3[j] * tanh(z);
  }
  return lp;
}

/* log cosh(x) - log 2, the RBM hidden-unit term (the constant cancels in
 * every ratio). */
static inline double om_lncosh(double x) {
  double y = fabs(x);
  return y + log1p(exp(-2.0 * y)) - 0.6931471805599453;
}

/* RBM: theta = b + W x (W row-major (H, N)) and sum_h lncosh(theta_h). */
static double rbm_theta(const om_guide *g, int N, const double *x, double *theta) {
  double lcs = 0.0;
  for (int h = 0; h < g->n_hidden; ++h) {
    double t = g->rbm_b[h];
    const double *w = g->rbm_W + (size_t)h * N;
    for (int k = 0; k < N; ++k) t += w[k] * x[k];
    theta[h] = t;
    lcs += om_lncosh(t);
  }
  return lcs;
}

/* RBM log ratio psi(x')/psi(x) for flipping site i and, when j >= 0, site j:
 * theta'_h = theta_h - 2 x_i W_hi - 2 x_j W_hj. */
static double rbm_log_diff(const om_guide *g, int N, const double *x, const double *theta,
                           double lcsum, int i, int j) {
  double s = 0.0;
  for (int h = 0; h < g->n_hidden; ++h) {
    const double *w = g->rbm_W + (size_t)h * N;
    double t = theta[h] - 2.0 * x[i] * w[i];
    if (j >= 0) t -= 2.0 * x[j] * w[j];
    s += om_lncosh(t);
  }
  double d = s - lcsum - 2.0 * g->rbm_a[i] * x[i];
  if (j >= 0) d -= 2.0 * g->rbm_a[j] * x[j];
  return d;
}

static inline int om_M(const om_model *m) {
  if (m->kind == 0) return 1 + m->n_hx + m->n_jpm;
  return 1 + m->n_hop + m->n_eta + 2 * m->n_hpm;
}

/* ---- SpinHalf rates: SpinHalf.diagonal_weight:291-314, get_rates:316-369 */
static double spin_diag(const om_model *m, const double *x) {
  double d = 0.0;
  if (m->has_jz) {
    if (m->uniform_jz) {
      int na = 0;
      for (int e = 0; e < m->n_edges; ++e) na += (x[m->ei[e]] != x[m->ej[e]]);
      int np_ = m->n_edges - na;
      d = (m->jz[0] / 4.0) * (double)(np_ - na);
    } else {
      for (int e = 0; e < m->n_edges; ++e)
        d += (x[m->ei[e]] != x[m->ej[e]]) ? -m->jz[e] / 4.0 : m->jz[e] / 4.0;
    }
  }
  if (m->has_hz) {
    double s = 0.0;
    for (int k = 0; k < m->N; ++k) s += m->hz[k] * x[k];
    d = d + s / 2.0;
  }
  return d;
}

/* JastrowSpinHalf._site_log_diff:290-297 */
static double jsh_site_ld(const om_guide *g, const double *x, int k) {
  double mf = 0.0;
  for (int s = 0; s < g->max_deg; ++s)
    mf += g->site_J[k * g->max_deg + s] * x[g->site_other[k * g->max_deg + s]];
  return -2.0 * x[k] * mf - 2.0 * g->h[k] * x[k];
}

/* JastrowSpinHalf._edge_log_diff_from_cache:462-472 */
static double jsh_edge_ld(const om_guide *g, const om_model *m, const double *x, int e) {
  double mf0 = 0.0, mf1 = 0.0;
  const int D = g->max_deg;
  for (int s = 0; s < D; ++s) {
    mf0 += g->edge_J[(e * 2 + 0) * D + s] * x[g->edge_other[(e * 2 + 0) * D + s]];
    mf1 += g->edge_J[(e * 2 + 1) * D + s] * x[g->edge_other[(e * 2 + 1) * D + s]];
  }
  int i = m->ei[e], j = m->ej[e];
  double pair = x[i] * mf0 + x[j] * mf1;
  double ht = g->h[i] * x[i] + g->h[j] * x[j];
  return -2.0 * pair - 2.0 * ht;
}

/* ---- BoseHubbard: diagonal_weight:271-281, get_rates:285-393 */
static double bose_diag(const om_model *m, const double *n) {
  double out = 0.0;
  if (m->has_U) {
    double s = 0.0;
    for (int k = 0; k < m->N; ++k) s += m->U[k] * n[k] * (n[k] - 1.0);
    out = out + 0.5 * s;
  }
  if (m->has_mu) {
    double s = 0.0;
    for (int k = 0; k < m->N; ++k) s += m->mu[k] * n[k];
    out = out - s;
  }
  return out;
}

/* Site/increment of transition idx (>=1) of the BoseHubbard layout:
 * _move_blocks:412-425 and hamiltonian/_common.py two_site_move:34-72. */
static void bose_move(const om_model *m, int idx, int *sa, int *sb, int *da, int *db) {
  int off = idx - 1, E = m->n_edges;
  *sa = *sb = 0; *da = *db = 0;
  if (idx == 0) return;
  if (m->n_hop > 0) {
    if (off < E) { *sa = m->ei[off]; *sb = m->ej[off]; *da = -1; *db = +1; return; }
    if (off < 2 * E) { *sa = m->ei[off - E]; *sb = m->ej[off - E]; *da = +1; *db = -1; return; }
    off -= 2 * E;
  }
  if (m->n_eta > 0) {
    if (off < E) { *sa = m->ei[off]; *sb = m->ej[off]; *da = +1; *db = +1; return; }
    if (off < 2 * E) { *sa = m->ei[off - E]; *sb = m->ej[off - E]; *da = -1; *db = -1; return; }
    off -= 2 * E;
  }
  if (m->n_hpm > 0) {
    if (off < m->N) { *sa = *sb = off; *da = +1; *db = 0; return; }
    off -= m->N;
    *sa = *sb = off; *da = -1; *db = 0;
  }
}

/* JastrowBoseHubbard.log_diff_from_operator:253-286 (non-incremental) */
static void jbh_log_diff(const om_guide *g, const om_model *m, const double *n,
                         double *S, double *out) {
  for (int k = 0; k < m->N; ++k) S[k] = 0.0;
  for (int p = 0; p < g->n_pairs; ++p) S[g->pair_i[p]] += g->pair_wt[p] * n[g->pair_j[p]];
  for (int p = 0; p < g->n_pairs; ++p) S[g->pair_j[p]] += g->pair_wt[p] * n[g->pair_i[p]];
  int M = om_M(m);
  for (int t = 0; t < M; ++t) {
    int a, b, ia, ib;
    bose_move(m, t, &a, &b, &ia, &ib);
    double da = ia, db = ib, na = n[a], nb = n[b];
    double o = 0.0;
    if (g->d_mode) {
      double dsa = (na + da) * (na + da) - na * na, dsb = (nb + db) * (nb + db) - nb * nb;
      o = (g->d_mode == 2) ? -(g->d[a] * dsa + g->d[b] * dsb) : -g->d0 * (dsa + dsb);
    }
    if (!g->beta_tied) o = o + da * S[a] + db * S[b] + da * db * g->trans_pw[t];
    else o = o + (-g->beta0) * (da * S[a] + db * S[b] + da * db * g->trans_pw[t]);
    if (g->h_mode == 2) o = o + (g->h[a] * da + g->h[b] * db);
    else if (g->h_mode == 1) o = o + g->h0 * (da + db);
    out[t] = o;
  }
}

/* ExactGroundState.basis_index:141-147: digit 1 for a down spin (x = -1). */
static long exact_index(const double *x, int N) {
  long idx = 0;
  for (int i = 0; i < N; ++i) idx = 2 * idx + (x[i] < 0.0 ? 1 : 0);
  return idx;
}

/* evolution.transition_rates:205-261 (guide ratio folded in, masked zeros) */
static void om_rates(const om_model *m, const om_guide *g, const double *x,
                     double *r, double *scratch) {
  int M = om_M(m);
  if (m->kind == 0) {
    r[0] = spin_diag(m, x);
    for (int k = 0; k < m->n_hx; ++k) r[1 + k] = m->hx_half[k];
    for (int e = 0; e < m->n_jpm; ++e)
      r[1 + m->n_hx + e] = (x[m->ei[e]] != x[m->ej[e]]) ? m->jpm[e] : m->jpmpm[e];
    if (g && g->kind == 1) {
      for (int k = 0; k < m->n_hx; ++k)
        if (r[1 + k] != 0.0) r[1 + k] *= exp(jsh_site_ld(g, x, k));
      for (int e = 0; e < m->n_jpm; ++e) {
        double *re = &r[1 + m->n_hx + e];
        if (*re != 0.0) *re *= exp(jsh_edge_ld(g, m, x, e));
      }
    } else if (g && g->kind == 5) {
      /* log_diff_from_configs:150-190: the successor of a flip differs from x
       * in the flipped sites' digits */
      const int N = m->N;
      const long ix = exact_index(x, N);
      const double l0 = g->log_amp[ix];
      for (int k = 0; k < m->n_hx; ++k)
        if (r[1 + k] != 0.0) r[1 + k] *= exp(g->log_amp[ix ^ (1L << (N - 1 - k))] - l0);
      for (int e = 0; e < m->n_jpm; ++e) {
        double *re = &r[1 + m->n_hx + e];
        const long fl = (1L << (N - 1 - m->ei[e])) ^ (1L << (N - 1 - m->ej[e]));
        if (*re != 0.0) *re *= exp(g->log_amp[ix ^ fl] - l0);
      }
    } else if (g && g->kind == 3) {
      double *theta = scratch + M;   /* om_guide_scratch doubles past the M-slot area */
      double lcs = rbm_theta(g, m->N, x, theta);
      for (int k = 0; k < m->n_hx; ++k)
        if (r[1 + k] != 0.0) r[1 + k] *= exp(rbm_log_diff(g, m->N, x, theta, lcs, k, -1));
      for (int e = 0; e < m->n_jpm; ++e) {
        double *re = &r[1 + m->n_hx + e];
        if (*re != 0.0) *re *= exp(rbm_log_diff(g, m->N, x, theta, lcs, m->ei[e], m->ej[e]));
      }
    }
  } else {
    const double nmax = (double)m->n_max;
    r[0] = bose_diag(m, x);
    int idx = 1, E = m->n_edges;
    if (m->n_hop > 0) {
      for (int e = 0; e < E; ++e) {
        double ni = x[m->ei[e]], nj = x[m->ej[e]];
        r[idx + e] = -m->t[e] * sqrt(ni * (nj + 1.0)) * (nj < nmax ? 1.0 : 0.0);
        r[idx + E + e] = -m->t[e] * sqrt((ni + 1.0) * nj) * (ni < nmax ? 1.0 : 0.0);
      }
      idx += 2 * E;
    }
    if (m->n_eta > 0) {
      for (int e = 0; e < E; ++e) {
        double ni = x[m->ei[e]], nj = x[m->ej[e]];
        r[idx + e] = -m->eta[e] * sqrt((ni + 1.0) * (nj + 1.0)) * ((ni < nmax && nj < nmax) ? 1.0 : 0.0);
        r[idx + E + e] = -m->eta[e] * sqrt(ni * nj);
      }
      idx += 2 * E;
    }
    if (m->n_hpm > 0) {
      for (int k = 0; k < m->N; ++k)
        r[idx + k] = m->hpm[k] * sqrt(x[k] + 1.0) * (x[k] < nmax ? 1.0 : 0.0);
      idx += m->N;
      for (int k = 0; k < m->N; ++k) r[idx + k] = m->hpm[k] * sqrt(x[k]);
    }
    if (g && g->kind == 2) {
      double *ld = scratch, *S = scratch + M;
      jbh_log_diff(g, m, x, S, ld);
      for (int t = 1; t < M; ++t)
        if (r[t] != 0.0) r[t] *= exp(ld[t]);
    } else if (g && g->kind == 4) {
      double *z1 = scratch + M, *y = z1 + g->mlp_H1;
      const double lp0 = mlp_logpsi(g, m->N, x, z1);
      for (int t = 1; t < M; ++t) {
        if (r[t] == 0.0) continue;
        memcpy(y, x, sizeof(double) * m->N);
        int a, b, da, db;
        bose_move(m, t, &a, &b, &da, &db);
        y[a] += (double)da;
        y[b] += (double)db;
        r[t] *= exp(mlp_logpsi(g, m->N, y, z1) - lp0);
      }
    }
  }
}

/* generate_state: SpinHalf.py:371-405, BoseHubbard via _common.two_site_update */
static void om_apply(const om_model *m, double *x, int idx) {
  if (idx == 0) return;
  if (m->kind == 0) {
    int off = idx - 1;
    if (off < m->n_hx) { x[off] = -x[off]; return; }
    int e = off - m->n_hx, a = m->ei[e], b = m->ej[e];
    double xa = x[a], xb = x[b];
    x[a] = -xa; x[b] = -xb;
  } else {
    int a, b, da, db; bose_move(m, idx, &a, &b, &da, &db);
    x[a] += (double)da; x[b] += (double)db;
  }
}

/* evolution.sample_index:30-59 over cdf/weights of length M. */
static int om_sample_index(const double *cdf, const double *w, int M, double U) {
  double total = cdf[M - 1];
  double u = U * total, cap = nextafter(total, 0.0);
  if (cap < u) u = cap;
  int lo = 0, hi = M;                  /* searchsorted side="right" */
  while (lo < hi) { int mid = (lo + hi) >> 1; if (cdf[mid] <= u) lo = mid + 1; else hi = mid; }
  int idx = lo < M - 1 ? lo : M - 1;
  int prev = -1;
  for (int s = 0; s <= idx; ++s) if (w[s] > 0.0) prev = s;
  return prev >= 0 ? prev : idx;
}

/* ---- per-walker propagators ------------------------------------------- */
typedef struct { double *r, *cdf, *w, *scratch, *xn; } om_ws;

static double rates_sum(const double *r, int M) {
  double s = 0.0; for (int k = 0; k < M; ++k) s += r[k]; return s;
}

/* evolve_walker_cont_time:559-721 (plain path, 683-700). */
static void evolve_cont_time(const om_model *m, const om_guide *g, double beta, om_key kw,
                             double alw, double *x, double *lw, double *el, int *hops,
                             om_ws *ws) {
  int M = om_M(m), N = m->N;
  if (M == 1) {
    om_rates(m, g, x, ws->r, ws->scratch);
    double eL = ws->r[0];
    *lw = *lw - eL * beta - alw * beta; *el = eL; return;
  }
  double t = 0.0, eloc = 0.0; uint32_t it = 0; int nh = 0;
  while (t < beta) {
    om_rates(m, g, x, ws->r, ws->scratch);
    double acc = 0.0;
    for (int k = 1; k < M; ++k) { ws->w[k - 1] = -ws->r[k]; acc += ws->w[k - 1]; ws->cdf[k - 1] = acc; }
    double R = ws->cdf[M - 2];
    double eL = ws->r[0] - R;
    double U1 = om_uniform64(om_fold(kw, 2u * it));
    double psi = om_uniform64(om_fold(kw, 2u * it + 1u));
    int si = (R > 0.0) ? om_sample_index(ws->cdf, ws->w, M - 1, U1) : 0;
    double tau_raw = (R > 0.0) ? -log1p(-psi) / R : INFINITY;
    double rem = beta - t;
    double tau = tau_raw < rem ? tau_raw : rem;
    *lw = *lw - eL * tau;
    t = t + tau;
    if (tau_raw < rem) { om_apply(m, x, si + 1); ++nh; }
    eloc = rates_sum(ws->r, M);
    ++it;
  }
  (void)N;
  *lw -= alw * beta; *el = eloc; if (hops) *hops = nh;
}

/* evolve_walker_single_step:322-406 (plain path). */
static void evolve_single_step(const om_model *m, const om_guide *g, int n_bra, double lam,
                               om_key kw, double alw, double *x, double *lw, double *el,
                               int *hops, om_ws *ws) {
  int M = om_M(m), nh = 0;
  for (int s = 0; s < n_bra; ++s) {
    om_rates(m, g, x, ws->r, ws->scratch);
    double acc = 0.0;
    for (int k = 0; k < M; ++k) { acc += ws->r[k]; ws->cdf[k] = lam - acc; ws->w[k] = -ws->r[k]; }
    ws->w[0] = ws->w[0] + lam;
    double bx = ws->cdf[M - 1];
    int idx = om_sample_index(ws->cdf, ws->w, M, om_uniform64(om_fold(kw, (uint32_t)s)));
    if (idx != 0) ++nh;
    om_apply(m, x, idx);
    *lw = *lw + log(bx);
  }
  om_rates(m, g, x, ws->r, ws->scratch);
  *el = rates_sum(ws->r, M);
  *lw -= alw * n_bra;
  if (hops) *hops = nh;
}

/* evolve_walker_multi_step:409-556 (plain path). */
static void evolve_multi_step(const om_model *m, const om_guide *g, int n_bra, double lam,
                              om_key kw, double alw, double *x, double *lw, double *el,
                              int *hops, om_ws *ws) {
  int M = om_M(m), nh = 0;
  if (M == 1) {
    om_rates(m, g, x, ws->r, ws->scratch);
    double bx = lam - ws->r[0];
    *lw = *lw + n_bra * log(bx) - alw * n_bra; *el = ws->r[0]; return;
  }
  int used = 0; uint32_t it = 0;
  while (used < n_bra) {
    om_rates(m, g, x, ws->r, ws->scratch);
    double acc = 0.0;
    for (int k = 1; k < M; ++k) { ws->w[k - 1] = -ws->r[k]; acc += ws->w[k - 1]; ws->cdf[k - 1] = acc; }
    double R = ws->cdf[M - 2];
    double bx = lam - ws->r[0] + R;
    double U1 = om_uniform64(om_fold(kw, 2u * it));
    double psi = om_uniform64(om_fold(kw, 2u * it + 1u));
    int si = (R > 0.0) ? om_sample_index(ws->cdf, ws->w, M - 1, U1) : 0;
    int remaining = n_bra - used;
    double hp = R / bx;
    int can_hop = hp > 0.0;
    double log_pd = can_hop ? log1p(-hp) : -1.0;
    double hold = floor(log1p(-psi) / log_pd) + 1.0;
    double cap = (double)(remaining + 1);
    double hm = hold < cap ? hold : cap;
    int k_raw = can_hop ? (int)hm : remaining + 1;
    int k = k_raw < remaining ? k_raw : remaining;
    *lw = *lw + log(bx) * (double)k;
    used += k;
    if (k_raw <= remaining) { om_apply(m, x, si + 1); ++nh; }
    ++it;
  }
  om_rates(m, g, x, ws->r, ws->scratch);
  *el = rates_sum(ws->r, M);
  *lw -= alw * n_bra;
  if (hops) *hops = nh;
}

/* _evolve_walkers_jit:817-843: one key per walker, split(key, N_walkers).
 * method: 0 cont_time, 1 single_step, 2 multi_step. */
int om_evolve(const om_model *m, const om_guide *g, int method, double step, double lam,
              double alw, const uint32_t key[2], int n_walkers, double *cfg, double *lw,
              double *el, int *hops, int n_threads) {
  int M = om_M(m), N = m->N;
  const om_guide *gg = (g && g->kind) ? g : NULL;
  om_key k = {key[0], key[1]};
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
#pragma omp parallel
  {
    om_ws ws;
    size_t S = (size_t)(4 * M + 2 * N + 8 + om_guide_scratch(gg));
    double *buf = (double *)malloc(sizeof(double) * S);
    ws.r = buf; ws.cdf = buf + M; ws.w = buf + 2 * M; ws.scratch = buf + 3 * M; ws.xn = NULL;
#pragma omp for schedule(dynamic, 16)
    for (int w = 0; w < n_walkers; ++w) {
      om_key kw = om_fold(k, (uint32_t)w);
      double *x = cfg + (size_t)w * N;
      int *h = hops ? &hops[w] : NULL;
      if (method == 0) evolve_cont_time(m, gg, step, kw, alw, x, &lw[w], &el[w], h, &ws);
      else if (method == 1) evolve_single_step(m, gg, (int)step, lam, kw, alw, x, &lw[w], &el[w], h, &ws);
      else evolve_multi_step(m, gg, (int)step, lam, kw, alw, x, &lw[w], &el[w], h, &ws);
    }
    free(buf);
  }
  return 0;
}

/* Guide-transformed rates of every walker (the full M-vector), for tests. */
int om_rates_batch(const om_model *m, const om_guide *g, int n_walkers, const double *cfg,
                   double *rates_out) {
  int M = om_M(m), N = m->N;
  const om_guide *gg = (g && g->kind) ? g : NULL;
  double *scratch = (double *)malloc(sizeof(double) * (size_t)(M + N + 8 + om_guide_scratch(gg)));
  for (int w = 0; w < n_walkers; ++w)
    om_rates(m, gg, cfg + (size_t)w * N, rates_out + (size_t)w * M, scratch);
  free(scratch);
  return M;
}

/* estimators.estimate_average_log_branch_weight:722-751 */
double om_initial_alw(const om_model *m, const om_guide *g, int method, double lam,
                      int n_walkers, const double *cfg) {
  int M = om_M(m), N = m->N;
  const om_guide *gg = (g && g->kind) ? g : NULL;
  double *r = (double *)malloc(sizeof(double) * (size_t)(2 * M + N + 8 + om_guide_scratch(gg)));
  double s = 0.0;
  for (int w = 0; w < n_walkers; ++w) {
    om_rates(m, gg, cfg + (size_t)w * N, r, r + M);
    double e = rates_sum(r, M);
    s += (method == 0) ? -e : log(lam - e);
  }
  free(r);
  return s / n_walkers;
}

/* walkers/reconfiguration.py:9-62: logsumexp, normalised weights, E_n,
 * systematic parents (searchsorted right, capped at the last positive
 * weight), gather of configurations and local energies, log_w := 0. */
int om_reconfigure(const uint32_t key[2], int n, int N, double *cfg, double *lw, double *el,
                   int *parents, double *logG_out, double *En_out) {
  double amax = -INFINITY;
  for (int i = 0; i < n; ++i) if (lw[i] > amax) amax = lw[i];
  double s = 0.0;
  if (isfinite(amax)) for (int i = 0; i < n; ++i) s += exp(lw[i] - amax);
  double lG = isfinite(amax) ? log(s) + amax : amax;
  double *w = (double *)malloc(sizeof(double) * (size_t)n * 2);
  double *cdf = w + n;
  double En = 0.0, acc = 0.0; int last_pos = 0;
  for (int i = 0; i < n; ++i) {
    w[i] = exp(lw[i] - lG);
    En += el[i] * w[i];
    acc += w[i]; cdf[i] = acc;
    if (w[i] > 0.0) last_pos = i;
  }
  om_key k = {key[0], key[1]};
  double psi = om_uniform64(k);
  for (int i = 0; i < n; ++i) {
    double u = ((double)i + psi) / (double)n;
    int lo = 0, hi = n;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (cdf[mid] <= u) lo = mid + 1; else hi = mid; }
    parents[i] = lo < last_pos ? lo : last_pos;
  }
  double *tmp = (double *)malloc(sizeof(double) * (size_t)n * (N + 1));
  memcpy(tmp, cfg, sizeof(double) * (size_t)n * N);
  memcpy(tmp + (size_t)n * N, el, sizeof(double) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    memcpy(cfg + (size_t)i * N, tmp + (size_t)parents[i] * N, sizeof(double) * N);
    el[i] = tmp[(size_t)n * N + parents[i]];
    lw[i] = 0.0;
  }
  free(tmp); free(w);
  *logG_out = lG - log((double)n);
  *En_out = En;
  return 0;
}

/* evolution.apply_operator_one:849-888, vmapped with per-walker keys
 * fold_in(key, w) (forward_walk_operator:1008-1012): the successor drawn
 * from cdf = cumsum(rates) (slot 0 = stay), value = the rate sum, 0 and no
 * move when it is not positive; M_total == 1 keeps x and returns rates[0]. */
int om_apply_operator(const om_model *m, const om_guide *g, const uint32_t key[2], int n_walkers,
                      double *cfg, double *vals) {
  int M = om_M(m), N = m->N;
  const om_guide *gg = (g && g->kind) ? g : NULL;
  double *buf = (double *)malloc(sizeof(double) * (size_t)(3 * M + N + 8 + om_guide_scratch(gg)));
  double *r = buf, *cdf = buf + M, *scratch = buf + 2 * M;
  om_key k = {key[0], key[1]};
  for (int w = 0; w < n_walkers; ++w) {
    double *x = cfg + (size_t)w * N;
    om_rates(m, gg, x, r, scratch);
    if (M == 1) { vals[w] = r[0]; continue; }
    double acc = 0.0;
    for (int s = 0; s < M; ++s) { acc += r[s]; cdf[s] = acc; }
    double total = cdf[M - 1];
    if (total <= 0.0) { vals[w] = 0.0; continue; }
    int idx = om_sample_index(cdf, r, M, om_uniform64(om_fold(k, (uint32_t)w)));
    om_apply(m, x, idx);
    vals[w] = total;
  }
  free(buf);
  return 0;
}

/* sample_index exported for the sampler edge-case tests. */
int om_sample_index_export(const double *cdf, const double *w, int M, double U) {
  return om_sample_index(cdf, w, M, U);
}

int om_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

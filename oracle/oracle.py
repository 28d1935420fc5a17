"""CPU oracle of the GFMC hot path -- TEST INFRASTRUCTURE ONLY.

Python half of the oracle: ctypes access to ``gfmc_oracle.c`` plus numpy
restatements of the reference's host-side pieces.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, and
only as the checker; the product never imports it.

Parity of this oracle is pinned against the reference's own golden file
(``tests/golden/golden_subset.npz``, extracted from PyGFMC's
``tests/core/reference_data/golden_cpu.npz`` by ``tests/golden/make_golden.py``):
the Threefry key chains, and whole 300-step float64 runs (final
configurations exact, series and energies to rtol 1e-10).

Reference files restated here (paths inside the PyGFMC project):
  hamiltonian/SpinHalf.py            SpinHalf.create:144-288
  hamiltonian/bose_hubbard.py        BoseHubbard.create:129-267
  wavefunction/jastrow_spin_half.py  __init__:79-157, build_cache:400-459
  wavefunction/jastrow_bose_hubbard.py  _transition_tables:172, build_cache:206
  walkers/walker.py                  prepare_walkers_random:199, prepare_walkers_sz:257,
                                     _base_config_for_sum:143
  engine/driver.py                   run_gfmc:1148, _warmup:747, _warmup_stage:713,
                                     _warmup_schedule:567, _production:940
  engine/estimators.py               _energy_and_diagonal_estimates:268,
                                     _off_diagonal_estimates:308
  engine/evolution.py                apply_operator_one:849, forward_walk_operator:891
  engine/io.py                       evaluate_observables jackknife:1084-1104
"""
import ctypes
import math
import os
import subprocess
import zlib
from types import SimpleNamespace

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libgfmc_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_up = ctypes.POINTER(ctypes.c_uint32)


class _Model(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("N", ctypes.c_int), ("n_edges", ctypes.c_int),
                ("ei", _ip), ("ej", _ip),
                ("n_hx", ctypes.c_int), ("n_jpm", ctypes.c_int), ("has_jz", ctypes.c_int),
                ("uniform_jz", ctypes.c_int), ("has_hz", ctypes.c_int),
                ("jz", _dp), ("jpm", _dp), ("jpmpm", _dp), ("hz", _dp), ("hx_half", _dp),
                ("n_max", ctypes.c_int), ("n_hop", ctypes.c_int), ("n_eta", ctypes.c_int),
                ("n_hpm", ctypes.c_int), ("has_U", ctypes.c_int), ("has_mu", ctypes.c_int),
                ("t", _dp), ("eta", _dp), ("U", _dp), ("mu", _dp), ("hpm", _dp)]


class _Guide(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("max_deg", ctypes.c_int),
                ("site_other", _ip), ("site_J", _dp), ("edge_other", _ip), ("edge_J", _dp),
                ("h", _dp),
                ("n_pairs", ctypes.c_int), ("pair_i", _ip), ("pair_j", _ip), ("pair_wt", _dp),
                ("trans_pw", _dp), ("beta_tied", ctypes.c_int), ("beta0", ctypes.c_double),
                ("h_mode", ctypes.c_int), ("h0", ctypes.c_double),
                ("d_mode", ctypes.c_int), ("d0", ctypes.c_double), ("d", _dp),
                ("n_hidden", ctypes.c_int), ("rbm_W", _dp), ("rbm_b", _dp), ("rbm_a", _dp),
                ("mlp_H1", ctypes.c_int), ("mlp_H2", ctypes.c_int), ("mlp_np1", ctypes.c_int),
                ("mlp_W1", _dp), ("mlp_b1", _dp), ("mlp_W2", _dp), ("mlp_b2", _dp), ("mlp_w3", _dp),
                ("mlp_b3", ctypes.c_double), ("exact_N", ctypes.c_int), ("log_amp", _dp)]


def build():
    """Compile the C oracle (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.om_evolve.argtypes = [ctypes.POINTER(_Model), ctypes.POINTER(_Guide), ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, _up,
                                ctypes.c_int, _dp, _dp, _dp, _ip, ctypes.c_int]
        L.om_reconfigure.argtypes = [_up, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _ip, _dp, _dp]
        L.om_initial_alw.restype = ctypes.c_double
        L.om_initial_alw.argtypes = [ctypes.POINTER(_Model), ctypes.POINTER(_Guide), ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, _dp]
        L.om_rates_batch.argtypes = [ctypes.POINTER(_Model), ctypes.POINTER(_Guide), ctypes.c_int,
                                     _dp, _dp]
        L.om_threefry2x32.argtypes = [ctypes.c_uint32] * 4 + [_up, _up]
        L.om_uniform.restype = ctypes.c_double
        L.om_uniform.argtypes = [_up]
        L.om_sample_index_export.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_double]
        L.om_apply_operator.argtypes = [ctypes.POINTER(_Model), ctypes.POINTER(_Guide), _up,
                                        ctypes.c_int, _dp, _dp]
        L.om_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------------------
# Threefry key helpers (the JAX key semantics, restated)
# ----------------------------------------------------------------------------
_M32 = np.uint64(0xFFFFFFFF)


def threefry_np(k0, k1, c0, c1):
    """Vectorised Threefry-2x32 over uint32 arrays (jax._src.prng)."""
    k0 = np.asarray(k0, np.uint64); k1 = np.asarray(k1, np.uint64)
    ks = [k0, k1, (k0 ^ k1 ^ np.uint64(0x1BD11BDA))]
    x0 = (np.asarray(c0, np.uint64) + ks[0]) & _M32
    x1 = (np.asarray(c1, np.uint64) + ks[1]) & _M32
    rots = [[13, 15, 26, 6], [17, 29, 16, 24]]
    for i in range(5):
        for r in rots[i % 2]:
            x0 = (x0 + x1) & _M32
            x1 = ((x1 << np.uint64(r)) | (x1 >> np.uint64(32 - r))) & _M32
            x1 = x1 ^ x0
        x0 = (x0 + ks[(i + 1) % 3]) & _M32
        x1 = (x1 + ks[(i + 2) % 3] + np.uint64(i + 1)) & _M32
    return x0.astype(np.uint32), x1.astype(np.uint32)


def PRNGKey(seed):
    """jax.random.PRNGKey for a 32-bit seed: [0, seed]."""
    return np.array([0, int(seed) & 0xFFFFFFFF], dtype=np.uint32)


def case_key(name):
    """The golden-file case key: PRNGKey(crc32(name))."""
    return PRNGKey(zlib.crc32(name.encode()))


def fold_in(key, d):
    y0, y1 = threefry_np(key[0], key[1], 0, int(d) & 0xFFFFFFFF)
    return np.array([y0, y1], dtype=np.uint32)


def split(key, n=2):
    """split(key, n)[i] = threefry(key, (0, i)) (partitionable Threefry)."""
    i = np.arange(n, dtype=np.uint64)
    y0, y1 = threefry_np(key[0], key[1], np.zeros(n, np.uint64), i)
    return np.stack([y0, y1], axis=1)


def uniform64(key):
    y0, y1 = threefry_np(key[0], key[1], 0, 0)
    bits = ((np.uint64(y0) << np.uint64(32)) | np.uint64(y1)) >> np.uint64(12)
    return float(np.array(bits | np.uint64(0x3FF0000000000000)).view(np.float64) - 1.0)


def random_bits32(key, n):
    """jax.random.bits(key, (n,), uint32): y0 ^ y1 of threefry(key, (0, i))."""
    y0, y1 = threefry_np(key[0], key[1], np.zeros(n, np.uint64), np.arange(n, dtype=np.uint64))
    return y0 ^ y1


def random_bits64(key, n):
    y0, y1 = threefry_np(key[0], key[1], np.zeros(n, np.uint64), np.arange(n, dtype=np.uint64))
    return (y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)


def randint64(key, shape, minval, maxval):
    """jax.random.randint with int64 (x64 mode): two 64-bit draws combined
    through the multiplier 2**64 % span."""
    n = int(np.prod(shape))
    k1, k2 = split(key, 2)
    hi = random_bits64(k1, n)
    lo = random_bits64(k2, n)
    span = np.uint64(maxval - minval)
    mult = np.uint64((2 ** 32) % int(span))
    mult = np.uint64((int(mult) * int(mult)) % int(span))
    off = ((hi % span) * mult + (lo % span)) % span
    return (minval + off.astype(np.int64)).reshape(shape)


def prepare_walkers_random(n_walkers, n_sites, key, states=(-1.0, 1.0)):
    """walkers/walker.py prepare_walkers_random (x64 mode)."""
    vals = np.asarray(states, dtype=np.float64)
    idx = randint64(key, (n_walkers, n_sites), 0, vals.size)
    return vals[idx]


def base_config_for_sum(n_sites, target, states):
    """walkers/walker.py _base_config_for_sum:143-196 (greedy over increments)."""
    vals = np.asarray(states, dtype=float).ravel()
    den = next(d for d in (1, 2, 3, 4, 5, 6, 8, 10, 12)
               if np.allclose(vals * d, np.round(vals * d))
               and abs(target * d - round(target * d)) < 1e-9)
    S = np.sort(np.round(vals * den).astype(np.int64))
    Z = int(round(target * den))
    inc = S - S[0]
    D = Z - n_sites * int(S[0])
    counts = np.zeros(S.size, dtype=np.int64)
    remaining, d = n_sites, D
    for k in range(S.size - 1, 0, -1):
        take = min(d // int(inc[k]), remaining)
        counts[k] += take
        d -= take * int(inc[k])
        remaining -= take
    counts[0] += remaining
    assert d == 0
    return np.repeat(S, counts).astype(float) / den


def permutation(key, x):
    """jax.random.permutation of a 1-D array: sort-based shuffle rounds."""
    x = np.asarray(x).copy()
    rounds = int(np.ceil(3 * np.log(max(1, x.size)) / np.log(np.iinfo(np.uint32).max)))
    for _ in range(rounds):
        key, sub = split(key, 2)
        sk = random_bits32(sub, x.size)
        x = x[np.argsort(sk, kind="stable")]
    return x


def prepare_walkers_sz(n_walkers, n_sites, key, sz=0, states=(-1.0, 1.0)):
    """walkers/walker.py prepare_walkers_sz: one permutation per walker."""
    base = base_config_for_sum(n_sites, sz, states)
    keys = split(key, n_walkers)
    return np.stack([permutation(keys[w], base) for w in range(n_walkers)])


# ----------------------------------------------------------------------------
# Models and guides
# ----------------------------------------------------------------------------
def chain_edges(L):
    """hamiltonian/lattice.py chain:36-46 (periodic)."""
    e = [(i, i + 1) for i in range(L - 1)]
    if L > 2:
        e.append((L - 1, 0))
    return np.asarray(e, dtype=np.int64)


class OracleModel:
    def __init__(self):
        self.keep = []

    def _arr(self, a, dtype=np.float64):
        a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
        self.keep.append(a)
        return a

    @property
    def M(self):
        s = self.s
        if s.kind == 0:
            return 1 + s.n_hx + s.n_jpm
        return 1 + s.n_hop + s.n_eta + 2 * s.n_hpm


def spin_half(edges, J_x=0.0, J_y=0.0, J_z=0.0, h_z=None, h_x=None, N=None):
    """SpinHalf.create:144-288 restated: J_pm=(J_x+J_y)/4, J_pmpm=(J_x-J_y)/4,
    fields stored negated (h_x stored halved)."""
    edges = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    E = len(edges)
    Nmin = int(edges.max()) + 1 if E else 0
    for a in (h_z, h_x):
        if a is not None and np.ndim(a) > 0:
            Nmin = max(Nmin, len(a))
    N = Nmin if N is None else int(N)
    uniform = not any(np.ndim(v) > 0 for v in (J_x, J_y, J_z))
    jx = np.broadcast_to(np.asarray(J_x, float), (E,)) if E else np.zeros(0)
    jy = np.broadcast_to(np.asarray(J_y, float), (E,)) if E else np.zeros(0)
    jz = np.broadcast_to(np.asarray(J_z, float), (E,)) if E else np.zeros(0)
    jpm = (jx + jy) / 4.0
    jpmpm = (jx - jy) / 4.0
    m = OracleModel()
    s = _Model()
    s.kind = 0; s.N = N; s.n_edges = E
    ei = m._arr(edges[:, 0] if E else [], np.int32); ej = m._arr(edges[:, 1] if E else [], np.int32)
    s.ei = _p(ei, _ip); s.ej = _p(ej, _ip)
    if uniform:
        jz_arr = m._arr([float(J_z)]); s.uniform_jz = 1
        jz_norm = abs(float(J_z))
    else:
        jz_arr = m._arr(jz); s.uniform_jz = 0
        jz_norm = float(np.linalg.norm(jz))
    s.jz = _p(jz_arr)
    s.jpm = _p(m._arr(jpm)); s.jpmpm = _p(m._arr(jpmpm))
    s.has_jz = int(jz_norm > 0)
    s.n_jpm = E if (np.linalg.norm(jpm) > 0 or np.linalg.norm(jpmpm) > 0) else 0
    if h_z is not None:
        hz = -np.broadcast_to(np.asarray(h_z, float), (N,))
        s.hz = _p(m._arr(hz)); s.has_hz = int(np.linalg.norm(hz) > 0)
    if h_x is not None:
        hxh = -np.broadcast_to(np.asarray(h_x, float), (N,)) / 2
        s.hx_half = _p(m._arr(hxh)); s.n_hx = N if np.linalg.norm(hxh) > 0 else 0
    m.s = s
    m.N = N
    m.edges = edges
    m.kind = 0
    return m


def bose_hubbard(edges, t=0.0, eta=0.0, U=0.0, mu=0.0, h_pm=None, N=None, n_max=4):
    """BoseHubbard.create:129-267 restated (h_pm stored negated)."""
    edges = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    E = len(edges)
    Nmin = int(edges.max()) + 1 if E else 0
    for a in (U, mu, h_pm):
        if a is not None and np.ndim(a) > 0:
            Nmin = max(Nmin, len(a))
    N = Nmin if N is None else int(N)
    m = OracleModel()
    s = _Model()
    s.kind = 1; s.N = N; s.n_edges = E; s.n_max = int(n_max)
    ei = m._arr(edges[:, 0] if E else [], np.int32); ej = m._arr(edges[:, 1] if E else [], np.int32)
    s.ei = _p(ei, _ip); s.ej = _p(ej, _ip)
    tt = np.broadcast_to(np.asarray(t, float), (E,))
    ee = np.broadcast_to(np.asarray(eta, float), (E,))
    s.t = _p(m._arr(tt)); s.eta = _p(m._arr(ee))
    s.n_hop = 2 * E if np.linalg.norm(tt) > 0 else 0
    s.n_eta = 2 * E if np.linalg.norm(ee) > 0 else 0
    UU = np.broadcast_to(np.asarray(U, float), (N,))
    MU = np.broadcast_to(np.asarray(mu, float), (N,))
    s.U = _p(m._arr(UU)); s.mu = _p(m._arr(MU))
    s.has_U = int(np.linalg.norm(UU) > 0); s.has_mu = int(np.linalg.norm(MU) > 0)
    if h_pm is not None:
        hp = -np.broadcast_to(np.asarray(h_pm, float), (N,))
        s.hpm = _p(m._arr(hp)); s.n_hpm = N if np.linalg.norm(hp) > 0 else 0
    m.s = s
    m.N = N
    m.edges = edges
    m.kind = 1
    m.n_max = int(n_max)
    return m


class OracleGuide:
    def __init__(self):
        self.keep = []

    def _arr(self, a, dtype=np.float64):
        a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
        self.keep.append(a)
        return a


def no_guide():
    g = OracleGuide(); g.s = _Guide(); g.s.kind = 0
    return g


def jastrow_spin_half(N, pairs, beta, h, model):
    """JastrowSpinHalf.__init__:79-157 and build_cache:400-459 for ``model``'s
    edges (partner tables with J = -beta, the i<->j bond masked out)."""
    pairs = np.sort(np.asarray(pairs, dtype=np.int64).reshape(-1, 2), axis=1)
    P = len(pairs)
    J = -np.broadcast_to(np.asarray(beta, float), (P,))
    hh = np.zeros(N) if h is None else np.broadcast_to(np.asarray(h, float), (N,)).copy()
    lists = [[] for _ in range(N)]
    for p, (a, b) in enumerate(pairs):
        lists[a].append((int(b), p)); lists[b].append((int(a), p))
    D = max([len(l) for l in lists] + [0]) or 1
    other = -np.ones((N, D), np.int64); sJ = np.zeros((N, D))
    for k in range(N):
        for s_, (o, p) in enumerate(lists[k]):
            other[k, s_] = o; sJ[k, s_] = J[p]
    valid = other >= 0
    other_c = np.clip(other, 0, None)
    ei, ej = model.edges[:, 0], model.edges[:, 1]
    ip, jp = other_c[ei], other_c[ej]
    im = valid[ei] & ~(ip == ej[:, None]); jm = valid[ej] & ~(jp == ei[:, None])
    edge_other = np.stack([ip, jp], axis=1)
    edge_J = np.where(np.stack([im, jm], axis=1), np.stack([sJ[ei], sJ[ej]], axis=1), 0.0)
    g = OracleGuide()
    s = _Guide(); s.kind = 1; s.max_deg = D
    s.site_other = _p(g._arr(other_c, np.int32), _ip)
    s.site_J = _p(g._arr(np.where(valid, sJ, 0.0)))
    s.edge_other = _p(g._arr(edge_other, np.int32), _ip)
    s.edge_J = _p(g._arr(edge_J))
    s.h = _p(g._arr(hh))
    g.s = s
    return g


def rbm_spin_half(W, b, a):
    """RBM guide (no reference counterpart): log psi = sum_h log cosh(b_h +
    sum_i W_hi s_i) + a.s on the given (bf16-valued) parameters, float64."""
    W = np.asarray(W, np.float64); H, N = W.shape
    g = OracleModel()
    s = _Guide()
    s.kind = 3
    s.n_hidden = H
    s.rbm_W = _p(g._arr(W.ravel()))
    s.rbm_b = _p(g._arr(np.broadcast_to(np.asarray(b, np.float64), (H,))))
    s.rbm_a = _p(g._arr(np.broadcast_to(np.asarray(a, np.float64), (N,))))
    g.s = s
    return g


def mlp_bose_hubbard(W1, b1, W2, b2, w3, b3, n_max):
    """Bose-Hubbard MLP guide (no reference counterpart): one-hot occupations ->
    tanh -> bf16 -> tanh -> w3 . h2 + b3, float64 on the given (bf16-valued)
    weights."""
    W1 = np.asarray(W1, np.float64); W2 = np.asarray(W2, np.float64)
    g = OracleModel()
    s = _Guide()
    s.kind = 4
    s.mlp_H1, s.mlp_H2, s.mlp_np1 = W1.shape[0], W2.shape[0], int(n_max) + 1
    s.mlp_W1 = _p(g._arr(W1.ravel())); s.mlp_b1 = _p(g._arr(b1))
    s.mlp_W2 = _p(g._arr(W2.ravel())); s.mlp_b2 = _p(g._arr(b2)); s.mlp_w3 = _p(g._arr(w3))
    s.mlp_b3 = float(b3)
    g.s = s
    return g


def exact_spin_half(log_amp, local_hilbert_space=(1.0, -1.0)):
    """ExactGroundState on spin-1/2 (wavefunction/exact_ground_state.py:
    43-190): log |psi_0| over the 2^N positional basis states of
    local_hilbert_space (site 0 most significant), float64.  The C side
    indexes over (1, -1), so a table over (-1, 1) is stored reversed (the
    complementary index)."""
    la = np.asarray(log_amp, np.float64).ravel()
    N = int(la.size).bit_length() - 1
    if la.size != 2 ** N:
        raise ValueError(f"log_amp has {la.size} entries, not a power of two")
    vals = tuple(float(v) for v in local_hilbert_space)
    if vals == (-1.0, 1.0):
        la = la[::-1]
    elif vals != (1.0, -1.0):
        raise ValueError(f"spin-1/2 local space expected, got {vals}")
    g = OracleModel()
    s = _Guide()
    s.kind = 5
    s.exact_N = N
    s.log_amp = _p(g._arr(la))
    g.s = s
    return g


def jastrow_bose_hubbard(N, pairs, beta, model, h=None, d=None):
    """JastrowBoseHubbard (non-incremental): neighbour sums with per-pair
    weight -beta (1 for a tied beta), cache pair_w per transition
    (_transition_tables:172-197, _pair_sum:164-170)."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    P = len(pairs)
    tied = np.ndim(beta) == 0
    wt = np.ones(P) if tied else -np.asarray(beta, float)
    g = OracleGuide()
    s = _Guide(); s.kind = 2
    s.n_pairs = P
    s.pair_i = _p(g._arr(pairs[:, 0], np.int32), _ip)
    s.pair_j = _p(g._arr(pairs[:, 1], np.int32), _ip)
    s.pair_wt = _p(g._arr(wt))
    s.beta_tied = int(tied); s.beta0 = float(beta) if tied else 0.0
    # per-transition sites of the BoseHubbard layout
    E = model.s.n_edges
    a, b = [0], [0]
    blocks = (2 if model.s.n_hop else 0) + (2 if model.s.n_eta else 0)
    for _ in range(blocks):
        a += list(model.edges[:, 0]); b += list(model.edges[:, 1])
    if model.s.n_hpm:
        a += list(range(N)) * 2; b += list(range(N)) * 2
    a = np.asarray(a); b = np.asarray(b)
    key = np.minimum(pairs[:, 0], pairs[:, 1]) * N + np.maximum(pairs[:, 0], pairs[:, 1])
    tk = np.minimum(a, b) * N + np.maximum(a, b)
    pw = np.array([wt[key == k].sum() for k in tk])
    s.trans_pw = _p(g._arr(pw))
    if h is None:
        s.h_mode = 0
    elif np.ndim(h) == 0:
        s.h_mode = 1; s.h0 = float(h)
    else:
        s.h_mode = 2; s.h = _p(g._arr(np.asarray(h, float)))
    if d is None:
        s.d_mode = 0
    elif np.ndim(d) == 0:
        s.d_mode = 1; s.d0 = float(d)
    else:
        s.d_mode = 2; s.d = _p(g._arr(np.asarray(d, float)))
    g.s = s
    assert E == len(model.edges)
    return g


# ----------------------------------------------------------------------------
# Batch primitives
# ----------------------------------------------------------------------------
_METHODS = {"cont_time": 0, "single_step": 1, "multi_step": 2}


def evolve(model, guide, method, step, lam, alw, key, cfg, lw, el, n_threads=0):
    """One evolve_walkers call, in place on float64 arrays; returns hops."""
    key = np.ascontiguousarray(key, dtype=np.uint32)
    n = cfg.shape[0]
    hops = np.zeros(n, np.int32)
    lib().om_evolve(ctypes.byref(model.s), ctypes.byref(guide.s), _METHODS[method],
                    float(step), float(lam if lam is not None else 0.0), float(alw),
                    _p(key, _up), n, _p(cfg), _p(lw), _p(el), _p(hops, _ip), int(n_threads))
    return hops


def reconfigure(key, cfg, lw, el):
    """walkers/reconfiguration.py:27-62 in place; returns (parents, logG, En)."""
    key = np.ascontiguousarray(key, dtype=np.uint32)
    n, N = cfg.shape
    par = np.zeros(n, np.int32)
    lG = ctypes.c_double(); En = ctypes.c_double()
    lib().om_reconfigure(_p(key, _up), n, N, _p(cfg), _p(lw), _p(el), _p(par, _ip),
                         ctypes.byref(lG), ctypes.byref(En))
    return par, lG.value, En.value


def rates(model, guide, cfg):
    cfg = np.ascontiguousarray(cfg, dtype=np.float64)
    out = np.zeros((cfg.shape[0], model.M))
    lib().om_rates_batch(ctypes.byref(model.s), ctypes.byref(guide.s), cfg.shape[0],
                         _p(cfg), _p(out))
    return out


def initial_alw(model, guide, method, lam, cfg):
    cfg = np.ascontiguousarray(cfg, dtype=np.float64)
    return lib().om_initial_alw(ctypes.byref(model.s), ctypes.byref(guide.s),
                                _METHODS[method], float(lam if lam is not None else 0.0),
                                cfg.shape[0], _p(cfg))


def apply_operator(model, guide, key, cfg):
    """apply_operator_one over the walkers (per-walker keys fold_in(key, w)),
    in place on cfg; returns the operator values."""
    key = np.ascontiguousarray(key, dtype=np.uint32)
    vals = np.zeros(cfg.shape[0])
    lib().om_apply_operator(ctypes.byref(model.s), ctypes.byref(guide.s), _p(key, _up),
                            cfg.shape[0], _p(cfg), _p(vals))
    return vals


def forward_walk(cfg, op_model, op_guide, model, guide, method, step, lam, alw, apply_key,
                 shadow_key, m_array, n_threads=0):
    """engine/evolution.py forward_walk_operator:891-1101 restated: apply
    the operator, then max(m_array) shadow steps of the main model from the
    applied walkers (zero log weights) under the key recurrence started at
    shadow_key; the values follow each parent map.  Returns (val, log_norm)
    at the depths m_array (row m = 0: the plain mean, norm 0)."""
    x = np.array(cfg, dtype=np.float64, copy=True)
    n = x.shape[0]
    v = apply_operator(op_model, op_guide, apply_key, x)
    lw = np.zeros(n); el = np.zeros(n)
    m_max = max(m_array)
    fw = [float(np.mean(v))]
    nrm = [0.0]
    acc = 0.0
    key = np.asarray(shadow_key, np.uint32)
    for _ in range(m_max):
        key, r = split(key, 2)
        evolve(model, guide, method, step, lam, alw, fold_in(r, 0), x, lw, el, n_threads)
        par, lG, _ = reconfigure(fold_in(r, 1), x, lw, el)
        v = v[par]
        acc = acc + lG
        fw.append(float(np.mean(v)))
        nrm.append(acc)
    return np.array([fw[m] for m in m_array]), np.array([nrm[m] for m in m_array])


def off_diagonal_estimates(p_array, m_array, log_weights, fw, nrm, steps, m_max_common=0):
    """engine/estimators.py _off_diagonal_estimates:308-355 restated for one
    operator: fw, nrm (n_rows, n_p) at main-chain steps `steps`."""
    L = np.concatenate([[0.0], np.cumsum(np.asarray(log_weights, float))])
    n = len(log_weights)
    steps = np.asarray(steps)
    out = {}
    for j, (p, m) in enumerate(zip(sorted(p_array), m_array)):
        sel = (steps >= p + max(0, m_max_common - m)) & (steps < n - m)
        i = steps[sel] - p
        num_l = L[p + 1 + i] - L[p - m + 1 + i] + np.asarray(nrm)[sel, j]
        den_l = L[p + m + 1 + i] - L[p - m + 1 + i]
        sh = max(np.max(num_l[np.isfinite(num_l)]), np.max(den_l))
        out[p] = float(np.sum(np.exp(num_l - sh) * np.asarray(fw)[sel, j])) / \
            float(np.sum(np.exp(den_l - sh)))
    return out


def sample_index(cdf, w, U):
    cdf = np.ascontiguousarray(cdf, np.float64); w = np.ascontiguousarray(w, np.float64)
    return lib().om_sample_index_export(_p(cdf), _p(w), len(cdf), float(U))


def _logsumexp(a):
    a = np.asarray(a, float)
    m = np.max(a)
    if not np.isfinite(m):
        return m
    return math.log(np.sum(np.exp(a - m))) + m


def warmup_schedule(method, step_f, warmup_steps):
    """engine/driver.py _warmup_schedule:567-584."""
    if warmup_steps <= 0:
        return []
    base, extra = divmod(warmup_steps, 4)
    counts = [base + (i < extra) for i in range(4)]
    if method == "cont_time":
        sizes = [step_f / 8.0, step_f / 4.0, step_f / 2.0, step_f]
    else:
        nb = int(step_f)
        sizes = [float(max(1, nb // 8)), float(max(1, nb // 4)), float(max(1, nb // 2)), float(nb)]
    return [(s, c) for s, c in zip(sizes, counts) if c > 0]


def run(cfg, n_steps, model, step_size, guide, p_array, method="cont_time", rng_key=None,
        lam=None, warmup_steps=1000, avg_log_weight=None, n_threads=0, off_diag_operators=None):
    """engine/driver.py run_gfmc restated for the main chain (warm-up ramp
    on the aux side-streams, then the production key recurrence
    key, rng = split(key); k1, k2 = fold_in(rng, 0), fold_in(rng, 1)).
    off_diag_operators: list of (name, op_model, op_guide) measured by
    forward walking after every production step (stride 1), apply keys
    fold_in(fold_in(rng, 2), i) and the shadow started from the next key.
    Returns a namespace with the final walkers, alw, raw series, energies."""
    cfg = np.array(cfg, dtype=np.float64, copy=True)
    n = cfg.shape[0]
    lw = np.zeros(n); el = np.zeros(n)
    rng_key = np.asarray(rng_key, np.uint32)
    aux_root = fold_in(rng_key, 9000)
    step_f = float(step_size)
    alw_pinned = avg_log_weight is not None
    alw = avg_log_weight if alw_pinned else initial_alw(model, guide, method, lam, cfg)
    for step_, n_w in warmup_schedule(method, step_f, warmup_steps):
        sub = fold_in(fold_in(aux_root, n_w), int(step_ * 1000))
        remaining = n_w
        lgs = []
        while remaining > 0:
            mm = min(50, remaining)
            sub, k = split(sub, 2)
            for r in split(k, mm):
                k1, k2 = split(r, 2)
                evolve(model, guide, method, step_, lam, alw, k1, cfg, lw, el, n_threads)
                _, lG, _ = reconfigure(k2, cfg, lw, el)
                lgs.append(lG)
            remaining -= mm
        measured = alw + (_logsumexp(lgs) - math.log(n_w)) / step_
        if not alw_pinned:
            alw = measured
    key = rng_key.copy()
    LG = np.zeros(n_steps); E = np.zeros(n_steps); hops = np.zeros(n_steps)
    parents = np.zeros((n_steps, n), np.int32)
    ops = list(off_diag_operators or [])
    m_array = [p // 2 for p in sorted(set(int(p) for p in p_array))]
    off = {nm: np.zeros((n_steps, len(m_array))) for nm, _, _ in ops}
    off_norm = {nm: np.zeros((n_steps, len(m_array))) for nm, _, _ in ops}
    for s_ in range(n_steps):
        key, r = split(key, 2)
        k1, k2 = fold_in(r, 0), fold_in(r, 1)
        h = evolve(model, guide, method, step_size, lam, alw, k1, cfg, lw, el, n_threads)
        par, LG[s_], E[s_] = reconfigure(k2, cfg, lw, el)
        parents[s_] = par
        hops[s_] = h.mean()
        if ops:
            k3 = fold_in(r, 2)
            for i, (nm, om, og) in enumerate(ops):
                off[nm][s_], off_norm[nm][s_] = forward_walk(
                    cfg, om, og, model, guide, method, step_size, lam, alw, fold_in(k3, i), key,
                    m_array, n_threads)
    energy = windowed_energy(p_array, LG, E)
    return SimpleNamespace(config=cfg, log_weight=lw, e_loc=el, alw=alw, log_weights=LG,
                           energy_series=E, energy=energy, rng_key_next=key, parents=parents,
                           hops=hops, off_diag=off, off_diag_norm=off_norm, m_array=m_array)


def windowed_energy(p_array, log_weights, E):
    """engine/estimators.py _energy_and_diagonal_estimates:268-305 (energy)."""
    L = np.cumsum(np.asarray(log_weights, float))
    E = np.asarray(E, float)
    out = {}
    for p in sorted(set(int(p) for p in p_array)):
        lg = L[p:] - L[:-p]
        G = np.exp(lg - np.max(lg))
        out[p] = float(np.sum(G * E[p:])) / float(np.sum(G))
    return out


def jackknife_energy(p_array, log_weights, E, n_blocks):
    """engine/io.py:1084-1104: leave-one-block-out replicas of the windowed
    energy; err = sqrt((nb-1)/nb * sum (x_b - mean)^2)."""
    n = len(E)
    blen = n // n_blocks
    usable = blen * n_blocks
    lw = np.asarray(log_weights)[:usable]; EE = np.asarray(E)[:usable]
    grid = sorted(set(int(p) for p in p_array))
    reps = []
    for b in range(n_blocks):
        m = np.ones(usable, bool); m[b * blen:(b + 1) * blen] = False
        e = windowed_energy(grid, lw[m], EE[m])
        reps.append([e[p] for p in grid])
    arr = np.asarray(reps)
    c = arr - arr.mean(axis=0, keepdims=True)
    err = np.sqrt((n_blocks - 1) / n_blocks * np.sum(c ** 2, axis=0))
    return windowed_energy(grid, lw, EE), dict(zip(grid, err))

"""The drop-in boundary for guides: objects carrying exactly the attribute set
PyGFMC's own Jastrow guides store are lowered like this package's classes.

JAX is absent here, so PyGFMC's classes cannot be imported; the stand-ins
below hold the same attributes with the same meaning and the same dtype
rounding as ``wavefunction/jastrow_spin_half.py:79-186`` (``site_other``,
``site_valid_mask``, ``_pair_site``, ``_pair_slot``, ``_site_pair``, ``_J``,
``_h``, ``dtype``, ``N``; properties ``site_J``, ``h``, ``beta``) and
``wavefunction/jastrow_bose_hubbard.py:97-125`` (``pair_i``, ``pair_j``,
``key_order``, ``sorted_keys``, ``_beta``, ``_h``, ``_d``, ``incremental``;
properties ``beta``, ``h``, ``d``), built by code of their own.  Nothing else
of this package's classes is visible to the engine through them.
"""
import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200 import engine as E
from oracle_guides import oracle_guide


class RefShapedJastrowSpinHalf:
    """PyGFMC's JastrowSpinHalf attribute set (numpy arrays in place of jnp)."""

    def __init__(self, N, pairs, beta, h=None, dtype=np.float32):
        pairs = np.sort(np.asarray(pairs, np.int32).reshape(-1, 2), axis=1)
        dt = np.dtype(dtype)
        table = {k: [] for k in range(N)}
        self._pair_site = pairs[:, 0].copy()
        self._pair_slot = np.array([0] * len(pairs), np.int32)
        for p, (a, b) in enumerate(pairs):
            self._pair_slot[p] = len(table[a])
            table[a].append((b, p))
            table[b].append((a, p))
        width = max([len(v) for v in table.values()] + [1])
        self.site_other = np.zeros((N, width), np.int32)
        self._site_pair = np.zeros((N, width), np.int32)
        self.site_valid_mask = np.zeros((N, width), bool)
        for k, lst in table.items():
            for c, (o, p) in enumerate(lst):
                self.site_other[k, c], self._site_pair[k, c], self.site_valid_mask[k, c] = o, p, True
        self.N, self.dtype = int(N), dt
        self._J = (np.asarray(-float(beta), dt) if np.ndim(beta) == 0
                   else (-np.asarray(beta, np.float64)).astype(dt))
        self._h = (None if h is None else np.asarray(float(h), dt) if np.ndim(h) == 0
                   else np.asarray(h, np.float64).astype(dt))

    @property
    def site_J(self):
        J = self._J if self._J.ndim == 0 else self._J[self._site_pair]
        return np.where(self.site_valid_mask, J, 0).astype(self.dtype)

    @property
    def h(self):
        return np.zeros(self.N, self.dtype) if self._h is None else np.broadcast_to(self._h, (self.N,))

    @property
    def beta(self):
        return -np.broadcast_to(self._J, self._pair_site.shape)

    def log_psi(self, config):
        x = np.asarray(config, np.float64)
        other = self.site_other
        pair = 0.5 * (self.site_J.astype(np.float64) * x[..., :, None] * x[..., other]).sum((-2, -1))
        return pair + (self.h.astype(np.float64) * x).sum(-1)


class RefShapedJastrowBoseHubbard:
    """PyGFMC's JastrowBoseHubbard attribute set (numpy arrays in place of jnp)."""

    def __init__(self, N, pairs, beta, h=None, d=None, dtype=np.float32, incremental=False):
        pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
        self.N, self.dtype, self.incremental = int(N), np.dtype(dtype), bool(incremental)
        self.pair_i = pairs[:, 0].astype(np.int32)
        self.pair_j = pairs[:, 1].astype(np.int32)
        keys = pairs.min(1) * N + pairs.max(1)
        self.key_order = np.argsort(keys, kind="stable").astype(np.int32)
        self.sorted_keys = keys[self.key_order].astype(np.int32)

        def par(v):
            if v is None:
                return None
            return np.asarray(float(v) if np.ndim(v) == 0 else np.asarray(v, np.float64), self.dtype)
        self._beta, self._h, self._d = par(beta), par(h), par(d)

    @property
    def beta(self):
        return np.broadcast_to(self._beta, self.pair_i.shape).astype(self.dtype)

    @property
    def h(self):
        return np.zeros(self.N, self.dtype) if self._h is None else np.broadcast_to(self._h, (self.N,))

    @property
    def d(self):
        return np.zeros(self.N, self.dtype) if self._d is None else np.broadcast_to(self._d, (self.N,))

    def log_psi(self, config):
        n = np.asarray(config, np.float64)
        out = -(self.d.astype(np.float64) * n * n).sum(-1)
        out -= (self.beta.astype(np.float64) * n[..., self.pair_i] * n[..., self.pair_j]).sum(-1)
        return out + (self.h.astype(np.float64) * n).sum(-1)


def _pairs_longrange(L):
    lat = P.square(L)
    pairs = np.array([(i, j) for i in range(L * L) for j in range(i + 1, L * L)])
    d = np.abs(lat.extras["positions"][pairs[:, 0]] - lat.extras["positions"][pairs[:, 1]])
    d = np.minimum(d, L - d)
    return lat, pairs, 0.3 / np.sqrt((d ** 2).sum(1))


def test_jastrow_parameters_are_rounded_to_the_guide_dtype():
    """jastrow_spin_half.py:95,145-153 and jastrow_bose_hubbard.py _param:36-45:
    a float32 guide holds its couplings and fields rounded to float32; a
    float64 guide holds them exactly."""
    e = P.chain(6).edges
    G = P.JastrowSpinHalf(6, e, beta=0.3, h=0.05)
    assert G.tied_beta and G._J.dtype == np.float32
    assert np.all(G.beta == np.float32(0.3)) and np.all(G.h == np.float32(0.05))
    assert float(G.beta[0]) != 0.3
    G64 = P.JastrowSpinHalf(6, e, beta=0.3, h=0.05, dtype=np.float64)
    assert np.all(G64.beta == 0.3) and np.all(G64.h == 0.05)
    b = np.linspace(0.1, 0.2, 6)
    Ga = P.JastrowSpinHalf(6, e, beta=b)
    assert not Ga.tied_beta and np.array_equal(Ga.beta, b.astype(np.float32)) and Ga._h is None
    GB = P.JastrowBoseHubbard(6, e, beta=0.05, h=None, d=np.linspace(0.1, 0.3, 6))
    assert np.ndim(GB._beta) == 0 and GB._beta.dtype == np.float32 and GB._h is None
    assert np.array_equal(GB.d, np.linspace(0.1, 0.3, 6).astype(np.float32))


@pytest.mark.parametrize("tied", [True, False])
def test_reference_shaped_spin_jastrow_lowers_like_ours(tied):
    """The engine reads the same pairs (constructor order), couplings and
    fields from the PyGFMC-shaped object as from this package's class."""
    lat, pairs, beta = _pairs_longrange(4)
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(pairs))
    pairs = pairs[perm][:, ::-1] if not tied else pairs   # any order, either orientation
    beta = 0.3 if tied else beta[perm]
    h = None if tied else rng.uniform(-0.1, 0.1, 16)
    ref = RefShapedJastrowSpinHalf(16, pairs, beta, h)
    ours = P.JastrowSpinHalf(16, pairs, beta, h)
    E.require_guide_protocol(ref)
    a, b = E.spin_jastrow_tables(ref), E.spin_jastrow_tables(ours)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.array_equal(a[0], np.sort(pairs, axis=1))
    np.testing.assert_array_equal(a[1], -np.broadcast_to(np.float32(beta) if tied else
                                                         beta.astype(np.float32), (len(pairs),)))
    H = P.SpinHalf.create(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    x = P.prepare_walkers_sz(3, 16, P.PRNGKey(2), sz=0).config
    np.testing.assert_allclose(ref.log_psi(x), ours.log_psi(x), rtol=1e-12)
    for kind, G in (("ref", ref), ("ours", ours)):
        keep = E._Keep()
        d = E.guide_desc(G, H, keep)
        assert d.kind == P._lib.GUIDE_JASTROW_SPIN_HALF and d.n_pairs == len(pairs), kind
        assert [d.pair_i[k] for k in range(4)] == list(a[0][:4, 0])
        assert [d.pair_w[k] for k in range(4)] == list(a[1][:4])


def test_reference_shaped_bose_jastrow_lowers_like_ours():
    e = P.chain(8).edges
    B = P.BoseHubbard.create(e, t=1.0, U=2.0, n_max=3, dtype=np.float64)
    for beta, h, d in ((0.05, 0.1, 0.3), (np.linspace(0.01, 0.08, 8), None, np.linspace(0.1, 0.2, 8))):
        descs = []
        for G in (RefShapedJastrowBoseHubbard(8, e, beta, h, d), P.JastrowBoseHubbard(8, e, beta, h, d)):
            E.require_guide_protocol(G)
            keep = E._Keep()
            g = E.guide_desc(G, B, keep)
            assert g.kind == P._lib.GUIDE_JASTROW_BOSE_HUBBARD
            descs.append((g.beta_tied, g.beta0, [g.pair_w[k] for k in range(8)], g.h_mode, g.h0,
                          g.d_mode, g.d0, [g.d[k] for k in range(8)] if g.d_mode == 2 else None))
        assert descs[0] == descs[1]
        if np.ndim(beta) == 0:
            assert descs[0][1] == float(np.float32(beta))


def test_guides_without_the_attribute_set_are_refused():
    class Opaque:
        def log_psi(self, x):
            return 0.0
    with pytest.raises(TypeError, match="no device implementation"):
        E.require_guide_protocol(Opaque())
    with pytest.raises(TypeError, match="must implement"):
        E.require_guide_protocol(object())
    ref = RefShapedJastrowSpinHalf(6, P.chain(6).edges, 0.3)
    H8 = P.SpinHalf.create(P.chain(8).edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    with pytest.raises(ValueError, match="N=6 for 8 sites"):
        E.guide_desc(ref, H8, E._Keep())
    B = P.BoseHubbard.create(P.chain(6).edges, t=1.0, n_max=2)
    with pytest.raises(TypeError, match="SpinHalf transition layout"):
        E.guide_desc(ref, B, E._Keep())


@pytest.mark.gpu
def test_reference_shaped_guides_run_like_the_oracle(oracle):
    """run() with the PyGFMC-shaped float32 guides (spin chain with a field,
    Bose-Hubbard chain) reproduces the oracle built with the same
    float32-rounded couplings: identical final walkers, series to 1e-10."""
    O = oracle
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)
    G = RefShapedJastrowSpinHalf(16, e, beta=0.3, h=0.05)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2)
    w = P.prepare_walkers_sz(256, 16, P.PRNGKey(0), sz=0)
    eb = P.chain(10).edges
    B = P.BoseHubbard.create(eb, t=1.0, U=2.5, mu=0.3, n_max=3, dtype=np.float64)
    GB = RefShapedJastrowBoseHubbard(10, eb, beta=np.linspace(0.02, 0.11, 10), d=0.3)
    mb = O.bose_hubbard(eb, t=1.0, U=2.5, mu=0.3, n_max=3)
    wb = P.prepare_walkers_sz(256, 10, P.PRNGKey(4), sz=10, states=(0.0, 1.0, 2.0, 3.0))
    for Hm, Gm, om, ww in ((H, G, m, w), (B, GB, mb, wb)):
        g = oracle_guide(O, Gm, om)
        key = P.PRNGKey(1)
        walkers, energy, _, stats, raw = P.run(ww, 40, Hm, 0.1, Gm, [4], rng_key=key, warmup_steps=8,
                                               verbosity=0)
        r = O.run(ww.config, 40, om, 0.1, g, [4], rng_key=key, warmup_steps=8)
        assert np.array_equal(walkers.config, r.config)
        np.testing.assert_allclose(raw["log_weights"], r.log_weights, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(raw["energy"], r.energy_series, rtol=1e-10, atol=1e-12)

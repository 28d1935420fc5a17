"""Saving and loading the Jastrow guides (wavefunction/jastrow_spin_half.py
save / load / from_jax:192-286, jastrow_bose_hubbard.py save / load:290-316):
every parameter comes back in the form it was given (tied, per pair / site,
absent), the pairs in constructor order, so log_psi and the tables the engine
lowers are unchanged; a load bound to a larger Hamiltonian pads the field;
extra attributes are stored.  npz containers (h5py is absent).  Host only."""
import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.engine import spin_jastrow_tables

E8 = P.chain(8).edges
PAIRS8 = [(0, 3), (1, 2), (5, 1), (2, 7), (6, 4)]       # one pair given as (high, low)


@pytest.mark.parametrize("beta,h", [(0.3, None), (np.linspace(0.1, 0.5, 5), 0.07),
                                    (np.linspace(0.1, 0.5, 5), np.linspace(-0.2, 0.2, 8))])
def test_spin_jastrow_round_trip(tmp_path, beta, h):
    g = P.JastrowSpinHalf(8, PAIRS8, beta=beta, h=h, dtype=np.float64)
    path = str(tmp_path / "j.npz")
    g.save(path, E_vmc=-3.5, note="x")
    with np.load(path) as z:
        assert float(z["jastrow_spin_half/attrs/E_vmc"]) == -3.5
    g2 = P.JastrowSpinHalf.load(path, dtype=np.float64)
    assert g2.N == 8 and np.array_equal(g2.pairs, g.pairs)
    assert np.ndim(g2._J) == np.ndim(g._J) and (g2._h is None) == (g._h is None)
    if g._h is not None:
        assert np.ndim(g2._h) == np.ndim(g._h)
    x = np.random.default_rng(0).choice([-1.0, 1.0], size=(32, 8))
    np.testing.assert_array_equal(g2.log_psi(x), g.log_psi(x))
    for a, b in zip(spin_jastrow_tables(g2), spin_jastrow_tables(g)):
        np.testing.assert_array_equal(a, b)


def test_spin_jastrow_load_onto_a_larger_system(tmp_path):
    g = P.JastrowSpinHalf(6, P.chain(6).edges, beta=0.2, h=np.linspace(0.1, 0.6, 6), dtype=np.float64)
    path = str(tmp_path / "j.npz")
    g.save(path)
    H = P.SpinHalf.create(P.chain(10).edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    g2 = P.JastrowSpinHalf.load(path, hamiltonian=H, dtype=np.float64)
    assert g2.N == 10
    np.testing.assert_array_equal(g2.h[:6], g.h)
    np.testing.assert_array_equal(g2.h[6:], 0.0)
    assert np.array_equal(g2.pairs, g.pairs)
    with pytest.raises(KeyError):
        P.JastrowSpinHalf.load(path, group="other")


def test_spin_jastrow_from_stored_arrays():
    g = P.JastrowSpinHalf(8, PAIRS8, beta=np.linspace(0.1, 0.5, 5), h=0.05, dtype=np.float64)
    g2 = P.JastrowSpinHalf.from_jax(g.dtype, g.N, g.site_other, g._J, g.site_valid_mask, g._h,
                                    g._pair_site, g._pair_slot, g._site_pair)
    x = np.random.default_rng(1).choice([-1.0, 1.0], size=(16, 8))
    np.testing.assert_array_equal(g2.log_psi(x), g.log_psi(x))
    np.testing.assert_array_equal(g2.beta, g.beta)
    np.testing.assert_array_equal(g2.site_J, g.site_J)


@pytest.mark.parametrize("kw", [dict(beta=0.21), dict(beta=0.21, h=0.13, d=0.37),
                                dict(beta=np.linspace(-0.1, 0.3, 8), h=np.linspace(-0.2, 0.2, 8),
                                     d=np.linspace(0.1, 0.5, 8)),
                                dict(beta=0.15, d=np.linspace(0.1, 0.5, 8), incremental=True)])
def test_bose_jastrow_round_trip(tmp_path, kw):
    g = P.JastrowBoseHubbard(8, E8, dtype=np.float64, **kw)
    path = str(tmp_path / "b.npz")
    g.save(path, tag=3)
    g2 = P.JastrowBoseHubbard.load(path, dtype=np.float64)
    assert g2.N == 8 and g2.incremental == g.incremental
    np.testing.assert_array_equal(g2.pair_i, g.pair_i)
    np.testing.assert_array_equal(g2.pair_j, g.pair_j)
    for name in ("_beta", "_h", "_d"):
        a, b = getattr(g2, name), getattr(g, name)
        assert (a is None) == (b is None)
        if a is not None:
            assert np.ndim(a) == np.ndim(b)
            np.testing.assert_array_equal(a, b)
    x = np.random.default_rng(2).integers(0, 3, (16, 8)).astype(np.float64)
    np.testing.assert_array_equal(g2.log_psi(x), g.log_psi(x))

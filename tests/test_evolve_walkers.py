"""engine.evolve_walkers and engine.estimate_average_log_branch_weight, the
per-step functions of PyGFMC's engine (engine/evolution.py:761-843,
engine/estimators.py:722-751), on the device: their argument checks (host,
before any device work); one evolution with non-zero incoming log weights
against the oracle, which accumulates onto them in place as PyGFMC does
(identical configurations, log weights and local energies to 1e-12), for the
Jastrow and RBM guides under the three propagators; the seed's effect in the
float32 and MLP kernels (the incoming log weight shifts the result and
changes nothing else); and the production loop of PyGFMC's
tests/core/test_walker_io.py:17-30 (evolve_walkers, then reconfiguration)
against the oracle's."""
import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.engine import estimate_average_log_branch_weight, evolve_walkers
from pygfmc_b200.walkers import Walker, reconfiguration

METHODS = [("cont_time", 0.15, None), ("single_step", 3, 12.0), ("multi_step", 4, 12.0)]


def _ring(N=8):
    return P.SpinHalf.create(P.chain(N).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)


def _seeded(cfg, seed):
    rng = np.random.default_rng(seed)
    n = len(cfg)
    return Walker(config=np.array(cfg, copy=True), log_weight=rng.normal(0.0, 2.0, n),
                  e_loc=np.zeros(n))


def test_arguments_are_checked_before_any_device_work():
    H = _ring()
    w = P.prepare_walkers_random(16, 8, P.PRNGKey(0))
    key = P.PRNGKey(1)
    with pytest.raises(ValueError):
        evolve_walkers(w, H, -0.1, None, "cont_time", key, 0.0)              # beta must be positive
    with pytest.raises(ValueError):
        evolve_walkers(w, H, 2.5, None, "single_step", key, 0.0, lam=5.0)    # n_bra an integer
    with pytest.raises(ValueError, match="lam"):
        evolve_walkers(w, H, 3, None, "single_step", key, 0.0)
    with pytest.raises(ValueError, match="return_rates"):
        evolve_walkers(w, H, 0.1, None, "cont_time", key, 0.0, return_rates=True)
    with pytest.raises(ValueError, match="log_weight, e_loc"):
        evolve_walkers(w._replace(e_loc=w.e_loc[:3]), H, 0.1, None, "cont_time", key, 0.0)
    with pytest.raises(ValueError, match="lam"):
        estimate_average_log_branch_weight(w, H, None, method="multi_step")
    with pytest.raises(ValueError, match="precision"):
        evolve_walkers(w, H, 0.1, None, "cont_time", key, 0.0, precision="fp16")
    with pytest.raises(TypeError):
        evolve_walkers(w, object(), 0.1, None, "cont_time", key, 0.0)       # not an operator
    assert {"evolve_walkers", "estimate_average_log_branch_weight"} <= set(P.engine.__all__)


def _compare(O, m, g, method, step, lam, alw, key, w, out, name):
    c = np.array(w.config, dtype=np.float64, copy=True)
    lw = np.array(w.log_weight, dtype=np.float64, copy=True)
    el = np.zeros(len(c))
    O.evolve(m, g, method, step, lam, alw, key, c, lw, el)
    assert np.array_equal(out.config, c), f"{name}: configurations differ"
    np.testing.assert_allclose(out.log_weight, lw, rtol=1e-12, atol=1e-12, err_msg=name)
    np.testing.assert_allclose(out.e_loc, el, rtol=1e-12, atol=1e-12, err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("method,step,lam", METHODS)
def test_jastrow_systems_match_the_oracle(oracle, method, step, lam):
    from test_gpu_parity import _systems
    for name, H, G, m, g, cfg in _systems(P, oracle):
        w = _seeded(cfg, 5)
        key = P.PRNGKey(91)
        out = evolve_walkers(w, H, step, G, method, key, -1.3, lam=lam)
        _compare(oracle, m, g, method, step, lam, -1.3, key, w, out, name)


@pytest.mark.gpu
@pytest.mark.parametrize("method,step,lam", METHODS)
def test_rbm_systems_match_the_oracle(oracle, method, step, lam):
    from test_rbm import _rbm_systems
    for name, H, G, m, g, cfg in _rbm_systems(P, oracle):
        lam_ = 40.0 if lam is not None and name.startswith("chain64") else lam
        w = _seeded(cfg, 6)
        key = P.PRNGKey(92)
        out = evolve_walkers(w, H, step, G, method, key, -1.1, lam=lam_)
        _compare(oracle, m, g, method, step, lam_, -1.1, key, w, out, name)


def _shift_only(w, H, G, method, step, lam, precision):
    """The incoming log weight seeds the accumulation and changes nothing
    else: same configurations and local energies as from zero weights, log
    weights shifted by the seed (to the rounding of one addition)."""
    key = P.PRNGKey(93)
    zero = w._replace(log_weight=np.zeros_like(w.log_weight))
    a = evolve_walkers(w, H, step, G, method, key, -0.7, lam=lam, precision=precision)
    b = evolve_walkers(zero, H, step, G, method, key, -0.7, lam=lam, precision=precision)
    np.testing.assert_array_equal(a.config, b.config)
    np.testing.assert_array_equal(a.e_loc, b.e_loc)
    np.testing.assert_allclose(a.log_weight, b.log_weight + w.log_weight, rtol=1e-13, atol=1e-12)
    assert not np.array_equal(a.log_weight, b.log_weight)


@pytest.mark.gpu
@pytest.mark.parametrize("method,step,lam", METHODS)
def test_seed_in_the_float32_kernels(oracle, method, step, lam):
    from test_gpu_parity import _systems
    from test_rbm import _rbm_systems
    cases = [s for s in _systems(P, oracle) if s[0] in ("square4_longrange", "bose12_jastrow")]
    cases += [s for s in _rbm_systems(P, oracle) if s[0] == "square4_h64"]
    for name, H, G, m, g, cfg in cases:
        _shift_only(_seeded(cfg, 7), H, G, method, step, lam, "mixed")


@pytest.mark.gpu
def test_seed_in_the_mlp_kernel(oracle):
    from test_mlp import _mlp_systems
    for name, H, G, m, g, cfg in _mlp_systems(oracle):
        _shift_only(_seeded(cfg, 8), H, G, "cont_time", 0.1, None, "mixed")


@pytest.mark.gpu
def test_production_loop_matches_the_oracle(oracle):
    """PyGFMC's own production loop (tests/core/test_walker_io.py:17-30):
    key, k1, k2 = split(key, 3); evolve_walkers(..., k1, ...);
    reconfiguration(..., k2), six times; the oracle's loop on the same keys
    gives the same walkers."""
    O = oracle
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, -1.0, -1 / 3, 0.0, h_z=0.0, h_x=0.7, dtype=np.float64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1 / 3, J_z=0.0, h_z=0.0, h_x=0.7)
    w = P.prepare_walkers_random(256, 16, P.PRNGKey(7))
    lam = 0.1
    alw = estimate_average_log_branch_weight(w, H, None, method="single_step", lam=lam)
    el0 = np.array([O.rates(m, O.no_guide(), w.config[i:i + 1])[0].sum() for i in range(4)])
    assert np.isfinite(alw) and np.all(lam - el0 > 0)
    c = np.array(w.config, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    key = P.PRNGKey(3)
    for _ in range(6):
        ks = P.random.split(key, 3)
        key, k1, k2 = ks[0], ks[1], ks[2]
        w = evolve_walkers(w, H, 10, None, "single_step", k1, alw, lam=lam)
        w, lg, E, idx = reconfiguration(w, k2)
        O.evolve(m, O.no_guide(), "single_step", 10, lam, alw, k1, c, lw, el)
        par, lG, En = O.reconfigure(k2, c, lw, el)
        np.testing.assert_array_equal(idx, par)
        np.testing.assert_array_equal(w.config, c)
        np.testing.assert_allclose([lg, E], [lG, En], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("method,lam", [("cont_time", None), ("single_step", 12.0)])
def test_average_log_branch_weight(oracle, method, lam):
    from test_gpu_parity import _systems
    name, H, G, m, g, cfg = [s for s in _systems(P, oracle) if s[0] == "square4_longrange"][0]
    w = Walker(config=cfg, log_weight=np.zeros(len(cfg)), e_loc=np.zeros(len(cfg)))
    got = estimate_average_log_branch_weight(w, H, G, method=method, lam=lam)
    e = oracle.rates(m, g, np.asarray(cfg, np.float64)).sum(axis=1)
    want = np.mean(-e) if method == "cont_time" else np.mean(np.log(lam - e))
    assert got == pytest.approx(float(want), rel=1e-12, abs=1e-12)

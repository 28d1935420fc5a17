"""Bit-level parity at the benchmark workloads' own shapes (float64 build,
through the C ABI), with populations reduced to a size the oracle finishes
in seconds:

* C0  Heisenberg chain L = 100, nearest-neighbour Jastrow beta = 0.3
  (2 configuration words), tau = 0.2;
* C1  16 x 16 Heisenberg torus, long-range Jastrow v(r) = 0.3 / r on all
  32640 pairs (4 words; the translation-invariant factor table, the guide
  state of the whole population as one int8 tensor-core product, the
  carried fields and the carried evaluation record), tau = 0.05;
* C3  Bose-Hubbard ring L = 64, 64 bosons, n_max = 4, t = 1, U = 3,
  Gutzwiller + density Jastrow (64-byte occupation rows), tau = 0.02;
* C4  kagome 12 x 12 x 3 = 432 sites, 864 bonds, nearest-neighbour Jastrow
  (7 words), tau = 0.02;
* C2  the 16 x 16 torus with an RBM guide of 512 hidden units.

One step of every propagator gives the oracle's configurations, moves and
parents exactly, with log weights, local energies, log G and E_n within
1e-12 relative (engine/evolution.py:322-721, walkers/reconfiguration.py:9-62).
Chained runs of 110 steps cross the engine's refresh of its carried guide
state (rebuilt from scratch after 100 steps in the float64 build): every
step's log G and E_n stay within 1e-12 of the oracle's fresh evaluation and
the final population and parent map are identical.

The guides keep their couplings rounded to float32 (their default dtype, as
in PyGFMC); the oracle is built from those stored values.
"""
import ctypes

import numpy as np
import pytest

import pygfmc_b200 as P
from oracle_guides import oracle_guide

pytestmark = pytest.mark.gpu

HEIS = dict(J_x=-1.0, J_y=-1.0, J_z=1.0)


def _longrange_pairs(L):
    lat = P.square(L)
    pairs = np.stack(np.triu_indices(L * L, 1), axis=1)
    d = np.abs(lat.extras["positions"][pairs[:, 0]] - lat.extras["positions"][pairs[:, 1]])
    d = np.minimum(d, L - d)
    return lat, pairs, 0.3 / np.sqrt((d ** 2).sum(1))


def config_system(name, O, n):
    """(engine H, engine guide, oracle model, oracle guide, configurations,
    tau, lam for the discrete propagators)."""
    if name == "C0_chain100":
        e = P.chain(100).edges
        H = P.SpinHalf.create(e, dtype=np.float64, **HEIS)
        G = P.JastrowSpinHalf(100, e, beta=0.3)
        m = O.spin_half(e, **HEIS)
        cfg = P.prepare_walkers_sz(n, 100, P.PRNGKey(100), sz=0).config
        return H, G, m, oracle_guide(O, G, m), cfg, 0.2, 26.0
    if name == "C1_square16_longrange":
        lat, pairs, beta = _longrange_pairs(16)
        H = P.SpinHalf.create(lat.edges, dtype=np.float64, **HEIS)
        G = P.JastrowSpinHalf(256, pairs, beta=beta)
        m = O.spin_half(lat.edges, **HEIS)
        cfg = P.prepare_walkers_sz(n, 256, P.PRNGKey(101), sz=0).config
        return H, G, m, oracle_guide(O, G, m), cfg, 0.05, 130.0
    if name == "C3_bose_ring64":
        e = P.chain(64).edges
        H = P.BoseHubbard.create(e, t=1.0, U=3.0, n_max=4, dtype=np.float64)
        G = P.JastrowBoseHubbard(64, e, beta=0.05, d=0.3)
        m = O.bose_hubbard(e, t=1.0, U=3.0, n_max=4)
        cfg = P.prepare_walkers_occupations(n, 64, 64, 4, P.PRNGKey(103)).config
        return H, G, m, oracle_guide(O, G, m), cfg, 0.02, 300.0
    if name == "C4_kagome12":
        lat = P.kagome(12, 12)
        H = P.SpinHalf.create(lat.edges, dtype=np.float64, **HEIS)
        G = P.JastrowSpinHalf(lat.N, lat.edges, beta=0.3)
        m = O.spin_half(lat.edges, **HEIS)
        cfg = P.prepare_walkers_sz(n, lat.N, P.PRNGKey(104), sz=0).config
        return H, G, m, oracle_guide(O, G, m), cfg, 0.02, 220.0
    raise KeyError(name)


CONFIGS = {"C0_chain100": 1024, "C1_square16_longrange": 1024, "C3_bose_ring64": 1024,
           "C4_kagome12": 512}


def _raw_cfg(eng):
    import torch
    out = torch.empty((eng.n, eng.N), dtype=torch.float64, device=eng.device)
    P._lib.check(eng.L.gfmc_unpack(eng.h, eng.n, ctypes.c_void_p(eng.cfg.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), eng._stream()), "gfmc_unpack")
    return out.cpu().numpy()


def _compare_step(eng, O, m, g, method, step, lam, alw, key, c, lw, el, lg, En, tag):
    """The oracle's evolve + reconfiguration of (c, lw, el) with the step's
    key pair against the engine state after its step (pre-gather
    configurations, weights, local energies, parents, log G, E_n)."""
    O.evolve(m, g, method, step, lam, alw, key[:2], c, lw, el)
    assert np.array_equal(_raw_cfg(eng), c), f"{tag}: configurations differ"
    np.testing.assert_allclose(eng.log_w.cpu().numpy(), lw, rtol=1e-12, atol=1e-12, err_msg=tag)
    np.testing.assert_allclose(eng.e_loc.cpu().numpy(), el, rtol=1e-12, atol=1e-12, err_msg=tag)
    par, lG, E = O.reconfigure(key[2:], c, lw, el)
    assert np.array_equal(eng.parents.cpu().numpy(), par), f"{tag}: parents differ"
    np.testing.assert_allclose(lg, lG, rtol=1e-12, atol=1e-13, err_msg=tag)
    np.testing.assert_allclose(En, E, rtol=1e-12, atol=1e-12, err_msg=tag)


@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("method", ["cont_time", "single_step", "multi_step"])
def test_one_step_at_config_shape(oracle, name, method):
    import torch
    O = oracle
    P._lib.load()
    H, G, m, g, cfg, tau, lam = config_system(name, O, CONFIGS[name])
    step = tau if method == "cont_time" else (3 if method == "single_step" else 4)
    lam = None if method == "cont_time" else lam
    eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
    eng.load(cfg)
    alw = float((-eng.local_energy()).mean().item()) if method == "cont_time" else \
        float(np.log(lam - eng.local_energy().cpu().numpy()).mean())
    keys, _ = P.engine.key_schedule(P.PRNGKey(7), 1)
    lg = torch.empty(1, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    eng.steps(method, step, lam, alw, keys, lg, En)
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    _compare_step(eng, O, m, g, method, step, lam, alw, keys[0], c, lw, el, lg.item(), En.item(),
                  f"{name} {method}")
    assert eng.status() == 0


@pytest.mark.parametrize("name", list(CONFIGS))
def test_chained_steps_across_the_refresh(oracle, name):
    """110 chained cont_time steps in one gfmc_run_steps call: the carried
    guide state (fields through the parent map, the carried evaluation
    record) and its rebuild after 100 steps against the oracle, which
    evaluates every rate afresh."""
    import torch
    O = oracle
    P._lib.load()
    n_steps = 110
    H, G, m, g, cfg, tau, _ = config_system(name, O, CONFIGS[name])
    eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
    eng.load(cfg)
    alw = float((-eng.local_energy()).mean().item())
    keys, _ = P.engine.key_schedule(P.PRNGKey(8), n_steps)
    lg = torch.empty(n_steps, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    eng.steps("cont_time", tau, None, alw, keys, lg, En)
    lg, En = lg.cpu().numpy(), En.cpu().numpy()
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    LG = np.zeros(n_steps); EE = np.zeros(n_steps)
    for s in range(n_steps - 1):
        O.evolve(m, g, "cont_time", tau, None, alw, keys[s, :2], c, lw, el)
        _, LG[s], EE[s] = O.reconfigure(keys[s, 2:], c, lw, el)
    np.testing.assert_allclose(lg[:-1], LG[:-1], rtol=1e-12, atol=1e-13, err_msg=name)
    np.testing.assert_allclose(En[:-1], EE[:-1], rtol=1e-12, atol=1e-12, err_msg=name)
    _compare_step(eng, O, m, g, "cont_time", tau, None, alw, keys[-1], c, lw, el, lg[-1], En[-1],
                  f"{name} step {n_steps}")
    assert eng.status() == 0


def _rbm_c2(O, n):
    lat = P.square(16)
    H = P.SpinHalf.create(lat.edges, dtype=np.float64, **HEIS)
    G = P.RBMSpinHalf(256, 512, seed=0, sigma=0.01)
    m = O.spin_half(lat.edges, **HEIS)
    cfg = P.prepare_walkers_sz(n, 256, P.PRNGKey(102), sz=0).config
    return H, G, m, O.rbm_spin_half(G.W, G.b, G.a), cfg


@pytest.mark.parametrize("method,step,lam", [("cont_time", 0.05, None), ("single_step", 3, 130.0)])
def test_rbm_one_step_at_c2_shape(oracle, method, step, lam):
    """The RBM guide at the C2 shape (256 visible, 512 hidden, bf16 weights
    N(0, 0.01^2)), float64 build: one step equals the oracle's."""
    import torch
    O = oracle
    P._lib.load()
    H, G, m, g, cfg = _rbm_c2(O, 256)
    eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
    eng.load(cfg)
    alw = float((-eng.local_energy()).mean().item()) if lam is None else \
        float(np.log(lam - eng.local_energy().cpu().numpy()).mean())
    keys, _ = P.engine.key_schedule(P.PRNGKey(9), 1)
    lg = torch.empty(1, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    eng.steps(method, step, lam, alw, keys, lg, En)
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    _compare_step(eng, O, m, g, method, step, lam, alw, keys[0], c, lw, el, lg.item(), En.item(),
                  f"rbm C2 {method}")
    assert eng.status() == 0


def test_rbm_chained_steps_at_c2_shape(oracle):
    """55 chained cont_time steps of the C2-shaped RBM (theta carried through
    the parent maps and rebuilt after 50 steps) against the oracle."""
    import torch
    O = oracle
    P._lib.load()
    n_steps = 55
    H, G, m, g, cfg = _rbm_c2(O, 128)
    eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
    eng.load(cfg)
    alw = float((-eng.local_energy()).mean().item())
    keys, _ = P.engine.key_schedule(P.PRNGKey(10), n_steps)
    lg = torch.empty(n_steps, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    eng.steps("cont_time", 0.05, None, alw, keys, lg, En)
    lg, En = lg.cpu().numpy(), En.cpu().numpy()
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    for s in range(n_steps - 1):
        O.evolve(m, g, "cont_time", 0.05, None, alw, keys[s, :2], c, lw, el)
        _, lG, E = O.reconfigure(keys[s, 2:], c, lw, el)
        np.testing.assert_allclose(lg[s], lG, rtol=1e-12, atol=1e-13, err_msg=f"step {s}")
        np.testing.assert_allclose(En[s], E, rtol=1e-12, atol=1e-12, err_msg=f"step {s}")
    _compare_step(eng, O, m, g, "cont_time", 0.05, None, alw, keys[-1], c, lw, el, lg[-1], En[-1],
                  f"rbm C2 step {n_steps}")

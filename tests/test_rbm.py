"""RBM guide: host class (bf16 rounding, ratios), the oracle's RBM rates, and
the device step kernel against the oracle (float64 build: identical moves
and parents, weights to 1e-12; mixed build: local energies to float32
accuracy; a long run agrees with exact diagonalisation)."""
import ctypes

import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.wavefunction import round_bf16


def test_round_bf16_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-30, 65504.0, np.inf], np.float32)
    r = round_bf16(x)
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1
    assert r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] - x[3]) <= 2.0 ** -8 * 4 and np.isinf(r[6])
    rng = np.random.default_rng(0)
    v = rng.normal(0, 0.01, 10000).astype(np.float32)
    rv = round_bf16(v)
    assert np.all(np.abs(rv - v) <= np.abs(v) * 2.0 ** -8 + 1e-45)


def test_rbm_host_ratios_and_validation():
    e = P.chain(8).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-0.7, J_z=1.0, h_x=0.2, dtype=np.float64)
    G = P.RBMSpinHalf(8, 12, seed=1, sigma=0.4, b=0.1, a=np.linspace(-0.2, 0.2, 8))
    x = P.prepare_walkers_random(1, 8, P.PRNGKey(3)).config[0]
    ld = G.log_diff_from_operator(x, H)
    y = x.copy(); y[2] = -y[2]
    assert np.isclose(ld[1 + 2], G.log_psi(y) - G.log_psi(x))
    y = x.copy(); y[[3, 4]] = -y[[3, 4]]
    assert np.isclose(ld[1 + 8 + 3], G.log_psi(y) - G.log_psi(x))
    assert np.all((G.W.view(np.uint32) & 0xFFFF) == 0)
    with pytest.raises(ValueError):
        P.RBMSpinHalf(8, 0)
    with pytest.raises(ValueError):
        P.RBMSpinHalf(8, 4, W=np.zeros((3, 8)))


def test_oracle_rbm_rates_match_host(oracle):
    O = oracle
    e = P.chain(10).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-0.8, J_z=1.0, h_x=0.3, dtype=np.float64)
    m = O.spin_half(e, J_x=-1.0, J_y=-0.8, J_z=1.0, h_x=0.3)
    G = P.RBMSpinHalf(10, 24, seed=3, sigma=0.3, b=np.linspace(-0.2, 0.2, 24),
                      a=np.linspace(0.1, -0.1, 10))
    g = O.rbm_spin_half(G.W, G.b, G.a)
    cfg = P.prepare_walkers_random(6, 10, P.PRNGKey(2)).config
    r = O.rates(m, g, cfg)
    r0 = O.rates(m, O.no_guide(), cfg)
    for w in range(len(cfg)):
        ld = G.log_diff_from_operator(cfg[w], H)
        ref = np.where(r0[w] != 0, r0[w] * np.exp(ld), 0.0)
        ref[0] = r0[w][0]
        np.testing.assert_allclose(r[w], ref, rtol=1e-12, atol=1e-15)


def _rbm_systems(P, O):
    out = []
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3, dtype=np.float64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3)
    G = P.RBMSpinHalf(16, 40, seed=5, sigma=0.2, b=0.05, a=0.02)
    cfg = P.prepare_walkers_random(384, 16, P.PRNGKey(31)).config
    out.append(("chain16_hx_h40", H, G, m, O.rbm_spin_half(G.W, G.b, G.a), cfg))
    sq = P.square(4)
    Hs = P.SpinHalf.create(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    ms = O.spin_half(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    Gs = P.RBMSpinHalf(16, 64, seed=6, sigma=0.1)
    cfgs = P.prepare_walkers_sz(384, 16, P.PRNGKey(32), sz=0).config
    out.append(("square4_h64", Hs, Gs, ms, O.rbm_spin_half(Gs.W, Gs.b, Gs.a), cfgs))
    e64 = P.chain(64).edges
    rng = np.random.default_rng(4)
    jx = -rng.uniform(0.5, 1.5, 64)
    jy = jx + rng.uniform(0.0, 0.2, 64)
    Hg = P.SpinHalf.create(e64, J_x=jx, J_y=jy, J_z=1.0, h_z=0.2, dtype=np.float64)
    mg = O.spin_half(e64, J_x=jx, J_y=jy, J_z=1.0, h_z=0.2)
    Gg = P.RBMSpinHalf(64, 300, seed=7, sigma=0.05, b=rng.normal(0, 0.1, 300),
                       a=rng.normal(0, 0.05, 64))
    cfgg = P.prepare_walkers_random(256, 64, P.PRNGKey(33)).config
    out.append(("chain64_xyz_h300", Hg, Gg, mg, O.rbm_spin_half(Gg.W, Gg.b, Gg.a), cfgg))
    return out


def _unpack(eng, torch):
    out = torch.empty((eng.n, eng.N), dtype=torch.float64, device=eng.device)
    eng.L.gfmc_unpack(eng.h, eng.n, ctypes.c_void_p(eng.cfg.data_ptr()),
                      ctypes.c_void_p(out.data_ptr()), eng._stream())
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("method,step,lam", [("cont_time", 0.15, None), ("single_step", 3, 12.0),
                                             ("multi_step", 4, 12.0)])
def test_rbm_one_step_parity_with_oracle(oracle, method, step, lam):
    import torch
    O = oracle
    P._lib.load()
    for name, H, G, m, g, cfg in _rbm_systems(P, O):
        if lam is not None and name.startswith("chain64"):
            lam = 40.0
        eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
        eng.load(cfg)
        keys, _ = P.engine.key_schedule(P.PRNGKey(78), 1)
        lg = torch.empty(1, dtype=torch.float64, device=eng.device)
        En = torch.empty_like(lg)
        alw = -1.1
        eng.steps(method, step, lam, alw, keys, lg, En)
        c_gpu = _unpack(eng, torch)
        lw_gpu, el_gpu = eng.log_w.cpu().numpy(), eng.e_loc.cpu().numpy()
        par_gpu = eng.parents.cpu().numpy()
        c = np.array(cfg, dtype=np.float64, copy=True)
        lw = np.zeros(len(c)); el = np.zeros(len(c))
        O.evolve(m, g, method, step, lam, alw, keys[0, :2], c, lw, el)
        assert np.array_equal(c_gpu, c), f"{name}: configurations differ"
        np.testing.assert_allclose(lw_gpu, lw, rtol=1e-12, atol=1e-12, err_msg=name)
        np.testing.assert_allclose(el_gpu, el, rtol=1e-12, atol=1e-12, err_msg=name)
        par, lG, E = O.reconfigure(keys[0, 2:], c, lw, el)
        assert np.array_equal(par_gpu, par), f"{name}: parents differ"
        np.testing.assert_allclose(lg.item(), lG, rtol=1e-12, atol=1e-13, err_msg=name)


@pytest.mark.gpu
def test_rbm_local_energy_both_precisions(oracle):
    """e_L through gfmc_local_energy: float64 to 1e-12, the mixed build
    (float32 theta, rates; fast exp/log) to 2e-5 relative of the scale."""
    O = oracle
    P._lib.load()
    for name, H, G, m, g, cfg in _rbm_systems(P, O):
        ref = O.rates(m, g, cfg).sum(axis=1)
        for prec, tol in (("fp64", 1e-12), ("mixed", 2e-5)):
            eng = P.GFMCEngine(H, G, cfg.shape[0], precision=prec)
            eng.load(cfg)
            el = eng.local_energy().cpu().numpy()
            scale = np.abs(O.rates(m, g, cfg)).sum(axis=1)
            assert np.all(np.abs(el - ref) <= tol * scale + 1e-12), (name, prec)


@pytest.mark.gpu
def test_rbm_chained_run_matches_oracle(oracle):
    """40 production steps through run(): theta carried through the parent
    maps on the device, recomputed from scratch in the oracle."""
    O = oracle
    name, H, G, m, g, cfg = _rbm_systems(P, O)[1]
    key = P.PRNGKey(9)
    _, _, _, stats, raw = P.run(P.Walker(cfg, np.zeros(len(cfg)), np.zeros(len(cfg))), 40, H, 0.1, G,
                                [4], rng_key=key, warmup_steps=8, verbosity=0)
    r = O.run(cfg, 40, m, 0.1, g, [4], rng_key=key, warmup_steps=8)
    np.testing.assert_allclose(raw["log_weights"], r.log_weights, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw["energy"], r.energy_series, rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
def test_rbm_mixed_run_matches_exact_energy():
    """A float32 RBM-guided run of the periodic 16-site Heisenberg chain gives
    the exact ground-state energy within its error bar."""
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.RBMSpinHalf(16, 32, seed=2, sigma=0.05)
    w = P.prepare_walkers_sz(2048, 16, P.PRNGKey(0), sz=0)
    _, E, _, st, raw = P.run(w, 1500, H, 0.1, G, [8, 32], rng_key=P.PRNGKey(1), warmup_steps=200,
                             verbosity=0, precision="mixed")
    Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 15)
    assert abs(Ej[32] / 16 - (-0.4463935)) < max(5e-3, 4 * err[32] / 16)


@pytest.mark.gpu
@pytest.mark.parametrize("N,H,n", [(16, 40, 300), (256, 512, 1024), (100, 700, 257),
                                   (256, 512, 65613), (100, 700, 37893), (432, 432, 20011),
                                   (600, 256, 3001)])
def test_rbm_theta_gemm_on_tensor_cores(N, H, n):
    """theta = b + W s from the tcgen05 kernel (bf16 inputs, f32 accumulation)
    equals the float64 product of the same bf16 weights to float32 rounding;
    padded hidden units are exactly zero; the parent map is honoured.  The
    two large populations give every CTA several tiles in two and three
    passes, with the per-pass rotation of the tile assignment (513 and 297
    tiles over the SMs); the 432-site case takes passes of 128 hidden
    columns over 7 site chunks, the 600-site case 10 site chunks (spin words
    loaded per chunk past the eighth)."""
    import torch
    P._lib.load()
    e = P.chain(N).edges
    Hm = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.RBMSpinHalf(N, H, seed=N + H, sigma=0.05, b=np.linspace(-0.3, 0.3, H))
    cfg = P.prepare_walkers_random(n, N, P.PRNGKey(H)).config
    eng = P.GFMCEngine(Hm, G, n, precision="mixed")
    eng.load(cfg)
    th = eng.rbm_theta().cpu().numpy()
    ref = G.theta(cfg)
    assert th.shape[1] % 256 == 0 and th.shape[1] >= H
    np.testing.assert_allclose(th[:, :H], ref, rtol=0, atol=2e-6 * np.sqrt(N))
    assert np.all(th[:, H:] == 0.0)
    # through a parent map
    par = torch.as_tensor(np.random.default_rng(1).integers(0, n, n).astype(np.int32), device=eng.device)
    eng.parents.copy_(par)
    eng.parents_valid = 1
    th2 = eng.rbm_theta().cpu().numpy()
    np.testing.assert_allclose(th2[:, :H], ref[par.cpu().numpy()], rtol=0, atol=2e-6 * np.sqrt(N))
    assert eng.status() == 0

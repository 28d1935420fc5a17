"""Parity of the CUDA engine (called through its C ABI) with the oracle and
with PyGFMC's golden runs.  Float64 build: bit-identical configurations,
moves and parents; weights, local energies and series within 1e-12 relative
for one step (1e-10 over whole runs, the golden file's tolerance)."""
import ctypes

import numpy as np
import pytest

from golden_cases import (CASES, engine_diag_ops, engine_off_ops, engine_system, method_of,
                          oracle_off_ops, oracle_system)
from oracle_guides import oracle_guide

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def P():
    import pygfmc_b200 as P
    P._lib.load()
    return P


@pytest.mark.parametrize("name", CASES)
def test_engine_reproduces_golden_run(P, golden, name):
    H, w, g, dt, lam = engine_system(P, name)
    method = method_of(name)
    step = dt if method == "cont_time" else 2
    key = golden[name + "/stats/parameters/rng_key"]
    walkers, energy, obs, stats, raw = P.run(
        w, 300, H, step, g, [2, 4], method=method, rng_key=key,
        lam=None if method == "cont_time" else lam, warmup_steps=8, verbosity=0,
        diag_operators=engine_diag_ops(P, name), off_diag_operators=engine_off_ops(P, name))
    p = name + "/"
    for on in engine_off_ops(P, name):
        np.testing.assert_allclose(raw["off_diag"][on], golden[p + f"raw/off_diag/{on}"], rtol=1e-10,
                                   atol=1e-12, err_msg=on)
        np.testing.assert_allclose(raw["off_diag_norm"][on], golden[p + f"raw/off_diag_norm/{on}"],
                                   rtol=1e-10, atol=1e-12, err_msg=on)
    assert np.array_equal(raw["off_diag_steps"], np.arange(300))
    for nm in list(engine_diag_ops(P, name)) + list(engine_off_ops(P, name)):
        for pp in (2, 4):
            np.testing.assert_allclose(obs[nm][pp], golden[p + f"obs/{nm}/{pp}"], rtol=1e-10,
                                       atol=1e-12, err_msg=f"{nm} p={pp}")
    for dn in engine_diag_ops(P, name):
        np.testing.assert_allclose(raw["diag"][dn], golden[p + f"raw/diag/{dn}"], rtol=1e-10,
                                   atol=1e-12, err_msg=dn)
        np.testing.assert_allclose(raw["additional_diag"][dn], golden[p + f"raw/additional_diag/{dn}"],
                                   rtol=1e-10, atol=1e-12, err_msg=dn)
    assert np.array_equal(walkers.config, golden[p + "config"].astype(np.float64))
    np.testing.assert_allclose(raw["log_weights"], golden[p + "raw/log_weights"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw["energy"], golden[p + "raw/energy"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(walkers.e_loc, golden[p + "e_loc"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(stats["avg_log_weight"], golden[p + "stats/avg_log_weight"], rtol=1e-10)
    for pp in (2, 4):
        np.testing.assert_allclose(energy[pp], golden[p + f"energy/{pp}"], rtol=1e-10, atol=1e-12)
    assert np.array_equal(stats["parameters/rng_key_next"], golden[p + "stats/parameters/rng_key_next"])
    # the end-of-run statistics pass (engine/estimators.py statistics:1139)
    np.testing.assert_allclose(stats["offspring_k0"], golden[p + "stats/offspring_k0"], rtol=0, atol=1e-12)
    if method == "cont_time":
        np.testing.assert_allclose(stats["hops_per_step_mean"], golden[p + "stats/hops_per_step_mean"],
                                   rtol=2e-6)


def _systems(P, O):
    """(name, engine H, engine guide, oracle model, oracle guide, configs, step, lam)."""
    out = []
    e = P.chain(32).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3, dtype=np.float64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3)
    cfg = P.prepare_walkers_random(512, 32, P.PRNGKey(11)).config
    out.append(("chain32_hx_none", H, None, m, O.no_guide(), cfg))
    G = P.JastrowSpinHalf(32, e, beta=0.3, h=0.05)
    out.append(("chain32_hx_jastrow", H, G, m, oracle_guide(O, G, m), cfg))
    sq = P.square(4)
    Hs = P.SpinHalf.create(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    ms = O.spin_half(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    pairs = np.array([(i, j) for i in range(16) for j in range(i + 1, 16)])
    pos = sq.extras["positions"]
    d = pos[pairs[:, 0]] - pos[pairs[:, 1]]
    d = np.abs(d); d = np.minimum(d, 4 - d); r = np.sqrt((d ** 2).sum(1))
    beta = 0.3 / r
    Gs = P.JastrowSpinHalf(16, pairs, beta=beta)
    cfgs = P.prepare_walkers_sz(512, 16, P.PRNGKey(12), sz=0).config
    out.append(("square4_longrange", Hs, Gs, ms, oracle_guide(O, Gs, ms), cfgs))
    # dense couplings without translation invariance, with a field
    rng = np.random.default_rng(21)
    bd = rng.uniform(0.05, 0.4, len(pairs))
    hd = rng.uniform(-0.1, 0.1, 16)
    Gd = P.JastrowSpinHalf(16, pairs, beta=bd, h=hd)
    out.append(("square4_dense_random", Hs, Gd, ms, oracle_guide(O, Gd, ms), cfgs))
    # non-uniform couplings and both fields (general spin path)
    e12 = P.chain(12).edges
    jx = -rng.uniform(0.5, 1.5, 12)
    jy = jx + rng.uniform(0.0, 0.2, 12)     # J_pmpm = (J_x - J_y) / 4 <= 0
    jz = rng.uniform(0.5, 1.5, 12)
    Hg = P.SpinHalf.create(e12, J_x=jx, J_y=jy, J_z=jz, h_z=0.3, h_x=0.2, dtype=np.float64)
    mg = O.spin_half(e12, J_x=jx, J_y=jy, J_z=jz, h_z=0.3, h_x=0.2)
    Gg = P.JastrowSpinHalf(12, e12, beta=0.2, h=0.03)
    cfgg = P.prepare_walkers_random(512, 12, P.PRNGKey(14)).config
    out.append(("chain12_xyz_fields", Hg, Gg, mg, oracle_guide(O, Gg, mg), cfgg))
    eb = P.chain(12).edges
    B = P.BoseHubbard.create(eb, t=1.0, eta=0.2, U=3.0, mu=0.4, h_pm=0.1, n_max=3, dtype=np.float64)
    mb = O.bose_hubbard(eb, t=1.0, eta=0.2, U=3.0, mu=0.4, h_pm=0.1, n_max=3)
    betas = np.linspace(0.02, 0.2, 12)
    GB = P.JastrowBoseHubbard(12, eb, beta=betas, h=0.1, d=np.linspace(0.1, 0.3, 12))
    gb = oracle_guide(O, GB, mb)
    occ = P.prepare_walkers_sz(512, 12, P.PRNGKey(13), sz=12, states=(0.0, 1.0, 2.0, 3.0)).config
    out.append(("bose12_jastrow", B, GB, mb, gb, occ))
    GBt = P.JastrowBoseHubbard(12, eb, beta=0.1, d=0.2)
    gbt = oracle_guide(O, GBt, mb)
    out.append(("bose12_jastrow_tied", B, GBt, mb, gbt, occ))
    # all-pairs density Jastrow: the dense path (population fields as one product)
    pb = np.array([(i, j) for i in range(12) for j in range(i + 1, 12)])
    bpd = rng.uniform(0.01, 0.1, len(pb))
    GBd = P.JastrowBoseHubbard(12, pb, beta=bpd, d=0.2)
    gbd = oracle_guide(O, GBd, mb)
    out.append(("bose12_jastrow_dense", B, GBd, mb, gbd, occ))
    # translation-invariant long-range couplings on a 6 x 6 torus (36 sites:
    # two lanes' strides per row, a displacement table wider than one warp)
    s6 = P.square(6)
    H6 = P.SpinHalf.create(s6.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    m6 = O.spin_half(s6.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    p6 = np.array([(i, j) for i in range(36) for j in range(i + 1, 36)])
    d6 = np.abs(s6.extras["positions"][p6[:, 0]] - s6.extras["positions"][p6[:, 1]])
    d6 = np.minimum(d6, 6 - d6)
    b6 = 0.25 / np.sqrt((d6 ** 2).sum(1))
    G6 = P.JastrowSpinHalf(36, p6, beta=b6)
    cfg6 = P.prepare_walkers_sz(512, 36, P.PRNGKey(15), sz=0).config
    out.append(("square6_longrange", H6, G6, m6, oracle_guide(O, G6, m6), cfg6))
    return out


def _raw_cfg(eng, torch):
    out = torch.empty((eng.n, eng.N), dtype=torch.float64, device=eng.device)
    eng.L.gfmc_unpack(eng.h, eng.n, ctypes.c_void_p(eng.cfg.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      eng._stream())
    return out.cpu().numpy()


@pytest.mark.parametrize("method,step,lam", [("cont_time", 0.15, None), ("single_step", 3, 12.0),
                                             ("multi_step", 4, 12.0)])
def test_one_step_parity_with_oracle(P, oracle, method, step, lam):
    import torch
    O = oracle
    for name, H, G, m, g, cfg in _systems(P, O):
        eng = P.GFMCEngine(H, G, cfg.shape[0], precision="fp64")
        eng.load(cfg)
        key = P.PRNGKey(77)
        keys, _ = P.engine.key_schedule(key, 1)
        lg = torch.empty(1, dtype=torch.float64, device=eng.device)
        En = torch.empty(1, dtype=torch.float64, device=eng.device)
        alw = -1.3
        eng.steps(method, step, lam, alw, keys, lg, En)
        c_gpu = _raw_cfg(eng, torch)
        lw_gpu = eng.log_w.cpu().numpy(); el_gpu = eng.e_loc.cpu().numpy()
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
        np.testing.assert_allclose(En.item(), E, rtol=1e-12, atol=1e-12, err_msg=name)


def test_trajectory_parity_with_oracle(P, oracle):
    """60 chained production steps of the long-range Jastrow on the 4x4 torus:
    the final population is identical and the series agree to 1e-10."""
    O = oracle
    name, H, G, m, g, cfg = _systems(P, O)[2]
    key = P.PRNGKey(5)
    _, _, _, stats, raw = P.run(P.Walker(cfg, np.zeros(len(cfg)), np.zeros(len(cfg))), 60, H, 0.1, G,
                                [4], rng_key=key, warmup_steps=8, verbosity=0)
    r = O.run(cfg, 60, m, 0.1, g, [4], rng_key=key, warmup_steps=8)
    np.testing.assert_allclose(raw["log_weights"], r.log_weights, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw["energy"], r.energy_series, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(stats["avg_log_weight"], r.alw, rtol=1e-10)


def test_mixed_precision_agrees_with_fp64(P):
    """The mixed build (float32 rates/ratios, float64 accumulators) gives the
    fp64 build's energy within the combined jackknife error."""
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(16, e, beta=0.3)
    w = P.prepare_walkers_sz(2048, 16, P.PRNGKey(0), sz=0)
    res = {}
    for prec in ("fp64", "mixed"):
        _, E, _, st, raw = P.run(w, 2000, H, 0.1, G, [8, 32], rng_key=P.PRNGKey(1), warmup_steps=200,
                                 verbosity=0, precision=prec)
        Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 20)
        res[prec] = (Ej[32], err[32])
    (a, ea), (b, eb) = res["fp64"], res["mixed"]
    assert abs(a - b) < 4 * np.hypot(ea, eb) + 1e-6, res
    # exact ground state of the periodic 16-site Heisenberg chain
    assert abs(a / 16 - (-0.4463935)) < 5e-3


def test_mixed_precision_dense_guide_agrees_with_fp64(P):
    """The long-range (all-pairs) Jastrow on the 4x4 torus, whose fresh guide
    state is built for the whole population as one product: the float32 and
    float64 builds agree with each other and with the exact ground state."""
    sq = P.square(4)
    H = P.SpinHalf.create(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    pairs = np.array([(i, j) for i in range(16) for j in range(i + 1, 16)])
    pos = sq.extras["positions"]
    d = np.abs(pos[pairs[:, 0]] - pos[pairs[:, 1]])
    d = np.minimum(d, 4 - d)
    G = P.JastrowSpinHalf(16, pairs, beta=0.3 / np.sqrt((d ** 2).sum(1)))
    w = P.prepare_walkers_sz(2048, 16, P.PRNGKey(0), sz=0)
    res = {}
    for prec in ("fp64", "mixed"):
        _, E, _, st, raw = P.run(w, 1500, H, 0.1, G, [8, 32], rng_key=P.PRNGKey(1), warmup_steps=200,
                                 verbosity=0, precision=prec)
        Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 20)
        res[prec] = (Ej[32], err[32])
    (a, ea), (b, eb) = res["fp64"], res["mixed"]
    assert abs(a - b) < 4 * np.hypot(ea, eb) + 1e-6, res
    assert abs(a - (-11.228483)) < max(4 * ea, 2e-3 * 11.228483), res


def test_hop_cap_is_reported_not_hung(P):
    """A step so long that every walker exceeds the iteration cap returns
    with a status error instead of spinning."""
    e = P.chain(8).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    w = P.prepare_walkers_sz(32, 8, P.PRNGKey(0), sz=0)
    with pytest.raises(P._lib.GFMCError, match="iteration cap"):
        P.run(w, 4, H, 500.0, None, [2], rng_key=P.PRNGKey(1), warmup_steps=4, verbosity=0,
              max_hops_per_step=64)


@pytest.mark.parametrize("n", [100_000, 310_000])
def test_resampling_at_scale_matches_oracle(P, oracle, n):
    """One cont_time step of 100 k walkers (the resampling as one cooperative
    launch, E_n summed inside it) and of 310 k walkers (more tiles than can be
    resident at once on a B200: the three-launch path and the series
    reduction) on the 16-site Heisenberg chain with a nearest-neighbour
    Jastrow guide: identical configurations and parents, log G and E_n to
    1e-12, against the oracle's evolve and reconfiguration."""
    import torch
    O = oracle
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(16, e, beta=0.3)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0)
    g = oracle_guide(O, G, m)
    cfg = P.prepare_walkers_sz(n, 16, P.PRNGKey(21), sz=0).config
    eng = P.GFMCEngine(H, G, n, precision="fp64")
    eng.load(cfg)
    keys, _ = P.engine.key_schedule(P.PRNGKey(22), 1)
    lg = torch.empty(1, dtype=torch.float64, device=eng.device)
    En = torch.empty(1, dtype=torch.float64, device=eng.device)
    alw = 0.45
    eng.steps("cont_time", 0.2, None, alw, keys, lg, En)
    c_gpu = _raw_cfg(eng, torch)
    par_gpu = eng.parents.cpu().numpy()
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(n); el = np.zeros(n)
    O.evolve(m, g, "cont_time", 0.2, None, alw, keys[0, :2], c, lw, el)
    assert np.array_equal(c_gpu, c), "configurations differ"
    par, lG, E = O.reconfigure(keys[0, 2:], c, lw, el)
    assert np.array_equal(par_gpu, par), "parents differ"
    np.testing.assert_allclose(lg.item(), lG, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(En.item(), E, rtol=1e-12, atol=1e-12)
    assert eng.status() == 0

"""Off-diagonal forward walking on the device against the oracle, through
the C ABI: the operator application alone (successor configurations exact,
values to 1e-13), the positivity probe's minimum rate, and whole forward
walks (applied operator + shadow chain keyed by a main chain's future keys)
at several depths, on systems larger than the golden ones."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F64 = np.float64


@pytest.fixture(scope="module")
def P():
    import pygfmc_b200 as P
    P._lib.load()
    return P


def _spin_case(P, O):
    e = P.chain(32).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3, dtype=F64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3)
    G = P.JastrowSpinHalf(32, e, beta=0.3, h=0.05, dtype=F64)
    g = O.jastrow_spin_half(32, e, 0.3, 0.05, m)
    ops = {
        "spsm": (P.SpinHalf.create(e, J_x=2.0, J_y=2.0, sign_check=False, dtype=F64),
                 O.spin_half(e, J_x=2.0, J_y=2.0)),
        "sx": (P.SpinHalf.create(e, h_x=-1.0, sign_check=False, dtype=F64), O.spin_half(e, h_x=-1.0)),
        "xx": (P.SpinHalf.create(np.asarray(e, np.int32), J_x=np.full(len(e), 1.5), J_y=np.zeros(len(e)),
                                 N=32, sign_check=False, dtype=F64),
               O.spin_half(e, J_x=np.full(len(e), 1.5), J_y=np.zeros(len(e)), N=32)),
        "zz": (P.SpinHalf.create(e, J_z=1.0, dtype=F64), O.spin_half(e, J_z=1.0)),
    }
    cfg = P.prepare_walkers_random(512, 32, P.PRNGKey(21)).config
    og = {k: O.jastrow_spin_half(32, e, 0.3, 0.05, om) for k, (_, om) in ops.items()}
    return H, G, m, g, ops, og, cfg


def _bose_case(P, O):
    e = P.chain(12).edges
    H = P.BoseHubbard.create(e, t=1.0, eta=0.2, U=2.0, mu=0.5, h_pm=0.1, n_max=3, dtype=F64)
    m = O.bose_hubbard(e, t=1.0, eta=0.2, U=2.0, mu=0.5, h_pm=0.1, n_max=3)
    G = P.JastrowBoseHubbard(12, e, beta=0.1, h=0.05, d=0.2, dtype=F64)
    g = O.jastrow_bose_hubbard(12, e, 0.1, m, h=0.05, d=0.2)
    ops = {
        "hop": (P.BoseHubbard.create(e, t=-1.0, n_max=3, sign_check=False, dtype=F64),
                O.bose_hubbard(e, t=-1.0, n_max=3)),
        "pair": (P.BoseHubbard.create(e, eta=-0.3, n_max=3, sign_check=False, dtype=F64),
                 O.bose_hubbard(e, eta=-0.3, n_max=3)),
    }
    cfg = P.prepare_walkers_sz(384, 12, P.PRNGKey(22), sz=12, states=(0.0, 1.0, 2.0, 3.0)).config
    og = {k: O.jastrow_bose_hubbard(12, e, 0.1, om, h=0.05, d=0.2) for k, (_, om) in ops.items()}
    return H, G, m, g, ops, og, cfg


CASES = {"spin": _spin_case, "bose": _bose_case}


def _unpack(P, eng, packed):
    import torch
    out = torch.empty((eng.n, eng.N), dtype=torch.float64, device=eng.device)
    P._lib.check(eng.L.gfmc_unpack(eng.h, eng.n, eng._ptr(packed), eng._ptr(out), eng._stream()),
                 "gfmc_unpack")
    return out.cpu().numpy()


@pytest.mark.parametrize("case", list(CASES))
def test_apply_operator_and_min_rate_match_oracle(P, oracle, case):
    H, G, m, g, ops, og, cfg = CASES[case](P, oracle)
    from pygfmc_b200.engine import GFMCEngine, OperatorHandle
    eng = GFMCEngine(H, G, cfg.shape[0])
    eng.load(cfg)
    for i, (nm, (op, om)) in enumerate(ops.items()):
        oh = OperatorHandle(op, G, "fp64")
        key = oracle.fold_in(oracle.case_key("apply " + nm), i)
        cfg_out, vals = oh.apply(eng, key)
        x = np.array(cfg, dtype=F64, copy=True)
        ref_vals = oracle.apply_operator(om, og[nm], key, x)
        assert np.array_equal(_unpack(P, eng, cfg_out), x), nm
        np.testing.assert_allclose(vals.cpu().numpy(), ref_vals, rtol=1e-13, atol=1e-14, err_msg=nm)
        mins = oh.min_rates(eng, cfg.shape[0])
        np.testing.assert_allclose(mins, oracle.rates(om, og[nm], cfg).min(axis=1), rtol=1e-13,
                                   atol=1e-14, err_msg=nm)


@pytest.mark.parametrize("case,method", [("spin", "cont_time"), ("spin", "single_step"),
                                         ("bose", "multi_step"), ("bose", "cont_time")])
def test_forward_walk_matches_oracle(P, oracle, case, method):
    import torch
    H, G, m, g, ops, og, cfg = CASES[case](P, oracle)
    from pygfmc_b200.engine import GFMCEngine, OperatorHandle, key_schedule
    n = cfg.shape[0]
    step, lam = (0.15, None) if method == "cont_time" else (2, 12.0 if case == "spin" else 80.0)
    alw = oracle.initial_alw(m, g, method, lam, cfg)
    eng = GFMCEngine(H, G, n)
    eng.load(cfg)
    shadow = GFMCEngine(H, G, n)
    m_array = [0, 1, 3, 6]
    shadow_key = oracle.case_key(f"shadow {case} {method}")
    sk, _ = key_schedule(shadow_key, max(m_array))
    for i, (nm, (op, om)) in enumerate(ops.items()):
        oh = OperatorHandle(op, G, "fp64")
        apply_key = oracle.fold_in(oracle.case_key("fw apply"), i)
        val = torch.empty(len(m_array), dtype=torch.float64, device=eng.device)
        nrm = torch.empty_like(val)
        # twice: the shadow handle's scratch and carried state are reused
        for _ in range(2):
            shadow.forward_walk(oh, eng, method, step, lam, alw, apply_key, sk, m_array, val, nrm)
            rv, rn = oracle.forward_walk(cfg, om, og[nm], m, g, method, step, lam, alw, apply_key,
                                         shadow_key, m_array)
            np.testing.assert_allclose(val.cpu().numpy(), rv, rtol=1e-12, atol=1e-13, err_msg=nm)
            np.testing.assert_allclose(nrm.cpu().numpy(), rn, rtol=1e-12, atol=1e-13, err_msg=nm)


def test_forward_walk_through_the_main_handle(P, oracle):
    """The shadow may run through the main chain's own handle: the main chain
    then continues exactly as without the walk (its carried guide state is
    rebuilt), here on a dense long-range guide that carries state."""
    import torch
    from pygfmc_b200.engine import GFMCEngine, OperatorHandle, key_schedule
    sq = P.square(4)
    H = P.SpinHalf.create(sq.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=F64)
    pairs = np.array([(i, j) for i in range(16) for j in range(i + 1, 16)])
    beta = 0.3 / (1.0 + np.arange(len(pairs)) % 5)
    G = P.JastrowSpinHalf(16, pairs, beta=beta, dtype=F64)
    op = P.SpinHalf.create(sq.edges, J_x=2.0, J_y=2.0, sign_check=False, dtype=F64)
    cfg = P.prepare_walkers_sz(256, 16, P.PRNGKey(4)).config
    keys, _ = key_schedule(oracle.case_key("main"), 12)
    runs = []
    for walk in (False, True):
        eng = GFMCEngine(H, G, 256)
        eng.load(cfg)
        oh = OperatorHandle(op, G, "fp64")
        lg = torch.empty(12, dtype=torch.float64, device=eng.device)
        E = torch.empty_like(lg)
        eng.steps("cont_time", 0.1, None, 0.3, keys[:6], lg[:6], E[:6])
        if walk:
            v = torch.empty(2, dtype=torch.float64, device=eng.device)
            nrm = torch.empty_like(v)
            sbuf = GFMCEngine(H, G, 256)   # shadow population buffers
            vals = torch.empty(256, dtype=torch.float64, device=eng.device)
            vals_tmp = torch.empty_like(vals)
            P._lib.check(eng.L.gfmc_forward_walk(
                eng.h, oh.h, 0, 0.1, 0.0, 0.3,
                np.array([3, 4], np.uint32).ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                np.ascontiguousarray(keys[6:10]).ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                256, eng._ptr(eng.cfg), eng._ptr(eng.parents), 1, sbuf._ptr(sbuf.cfg),
                sbuf._ptr(sbuf.cfg_tmp), sbuf._ptr(sbuf.parents), sbuf._ptr(sbuf.log_w),
                sbuf._ptr(sbuf.e_loc), sbuf._ptr(vals), sbuf._ptr(vals_tmp), 2,
                np.array([2, 4], np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                eng._ptr(v), eng._ptr(nrm), eng._stream()), "gfmc_forward_walk")
        eng.steps("cont_time", 0.1, None, 0.3, keys[6:], lg[6:], E[6:])
        runs.append((lg.cpu().numpy(), E.cpu().numpy(), eng.population()[0].cpu().numpy()))
    np.testing.assert_allclose(runs[1][0], runs[0][0], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(runs[1][1], runs[0][1], rtol=1e-12, atol=1e-13)
    assert np.array_equal(runs[1][2], runs[0][2])


def test_structure_factor_operator_through_run(P, oracle):
    """A StructureFactor operator (one slot per pair, weights 1 + cos(k.dr))
    measured by off-diagonal forward walking through run(): the raw rows and
    the pure estimates equal the oracle's run with the same operator."""
    O = oracle
    L = 10
    e = P.chain(L).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=F64)
    G = P.JastrowSpinHalf(L, e, beta=0.3, dtype=F64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0)
    g = O.jastrow_spin_half(L, e, 0.3, None, m)
    pos = np.arange(L, dtype=F64)[:, None]
    sf = P.hamiltonian.StructureFactor(pos, [2 * np.pi * 3 / L], "SpSm+SpSp", dtype=F64)
    jpm, jpp = np.asarray(sf.J_pm, F64), np.asarray(sf.J_pmpm, F64)
    om = O.spin_half(np.stack([sf.edge_i, sf.edge_j], axis=1), J_x=2 * (jpm + jpp),
                     J_y=2 * (jpm - jpp), J_z=0.0, N=L)
    og = O.jastrow_spin_half(L, e, 0.3, None, om)
    w = P.prepare_walkers_sz(128, L, P.PRNGKey(8), sz=0)
    key = P.PRNGKey(9)
    _, _, obs, _, raw = P.run(w, 30, H, 0.1, G, [2, 4], rng_key=key, warmup_steps=8, verbosity=0,
                              off_diag_operators={"sf": sf})
    r = O.run(w.config, 30, m, 0.1, g, [2, 4], rng_key=key, warmup_steps=8,
              off_diag_operators=[("sf", om, og)])
    np.testing.assert_allclose(raw["off_diag"]["sf"], r.off_diag["sf"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw["off_diag_norm"]["sf"], r.off_diag_norm["sf"], rtol=1e-10,
                               atol=1e-12)
    ref = O.off_diagonal_estimates([2, 4], r.m_array, r.log_weights, r.off_diag["sf"],
                                   r.off_diag_norm["sf"], np.arange(30))
    for p in (2, 4):
        np.testing.assert_allclose(obs["sf"][p], ref[p], rtol=1e-10)

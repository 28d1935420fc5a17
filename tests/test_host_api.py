"""Host-side API: constructors and validation mirror PyGFMC, the walker
initialisers draw PyGFMC's walkers, and the lattices are the reference's."""
import itertools

import numpy as np
import pytest

import pygfmc_b200 as P
from oracle_guides import oracle_guide


def test_spinhalf_create_conventions_and_errors():
    H = P.SpinHalf.create(P.chain(6).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.4)
    assert H.M_total == 1 + 6 + 6 and H.n_hx == 6 and H.n_jpm == 6
    assert float(H.J_pm[0]) == -0.5 and float(H.J_pmpm[0]) == 0.0
    assert np.allclose(H.h_x_half, -0.2)
    with pytest.raises(ValueError, match="J_pmpm"):
        P.SpinHalf.create([(0, 1)], J_x=1.0, J_y=-1.0)
    with pytest.raises(ValueError, match="J_pm"):
        P.SpinHalf.create([(0, 1)], J_x=1.0, J_y=1.0)
    with pytest.raises(ValueError, match="h_x"):
        P.SpinHalf.create([(0, 1)], J_x=-1.0, J_y=-1.0, h_x=-0.3)
    with pytest.raises(ValueError, match="self-edges"):
        P.SpinHalf.create([(1, 1)], J_x=-1.0, J_y=-1.0)
    S = P.SpinHalf.create([(0, 1)], J_x=1.0, J_y=1.0, sign_check=False)
    assert S.M_total == 2


def test_bose_hubbard_create_conventions_and_errors():
    H = P.BoseHubbard.create(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2)
    assert H.M_total == 1 + 12 + 12 + 12
    assert np.allclose(H.h_pm, -0.2)
    with pytest.raises(ValueError, match="t must"):
        P.BoseHubbard.create([(0, 1)], t=-1.0)
    with pytest.raises(ValueError, match="n_max"):
        P.BoseHubbard.create([(0, 1)], t=1.0, n_max=0)


def test_host_rates_match_oracle(oracle):
    e = P.chain(8).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5, h_z=0.1, dtype=np.float64)
    m = oracle.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5, h_z=0.1)
    cfg = P.prepare_walkers_random(16, 8, P.PRNGKey(3)).config
    r_or = oracle.rates(m, oracle.no_guide(), cfg)
    for w in range(16):
        np.testing.assert_allclose(H.get_rates(cfg[w])[0], r_or[w], rtol=1e-14, atol=1e-15)
    B = P.BoseHubbard.create(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2,
                             dtype=np.float64)
    mb = oracle.bose_hubbard(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2)
    occ = P.prepare_walkers_sz(16, 6, P.PRNGKey(4), sz=6, states=(0.0, 1.0, 2.0)).config
    r_or = oracle.rates(mb, oracle.no_guide(), occ)
    for w in range(16):
        np.testing.assert_allclose(B.get_rates(occ[w])[0], r_or[w], rtol=1e-14, atol=1e-15)


def test_guide_ratios_match_log_psi_differences(oracle):
    """tests/core/test_guides.py:145 idea: the oracle's ratio tables equal
    log_psi differences of the guide objects."""
    e = P.chain(8).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5)
    G = P.JastrowSpinHalf(8, e, beta=0.3, h=0.05)
    m = oracle.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5)
    g = oracle_guide(oracle, G, m)
    cfg = P.prepare_walkers_random(8, 8, P.PRNGKey(5)).config
    guided = oracle.rates(m, g, cfg)
    bare = oracle.rates(m, oracle.no_guide(), cfg)
    for w in range(8):
        ld = G.log_diff_from_operator(cfg[w], H)
        expect = bare[w] * np.exp(np.where(bare[w] == 0, 0, ld))
        np.testing.assert_allclose(guided[w], expect, rtol=1e-12, atol=1e-14)
    B = P.BoseHubbard.create(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2)
    GB = P.JastrowBoseHubbard(6, P.chain(6).edges, beta=[0.05, 0.1, 0.02, 0.3, 0.07, 0.01],
                              h=0.1, d=np.linspace(0.1, 0.4, 6))
    mb = oracle.bose_hubbard(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2)
    gb = oracle_guide(oracle, GB, mb)
    occ = P.prepare_walkers_sz(8, 6, P.PRNGKey(6), sz=6, states=(0.0, 1.0, 2.0)).config
    guided = oracle.rates(mb, gb, occ)
    bare = oracle.rates(mb, oracle.no_guide(), occ)
    for w in range(8):
        ld = GB.log_diff_from_operator(occ[w], B)
        expect = bare[w] * np.exp(np.where(bare[w] == 0, 0, ld))
        np.testing.assert_allclose(guided[w], expect, rtol=1e-12, atol=1e-14)


def test_walker_initialisers_match_oracle(oracle):
    k = oracle.case_key("spinhalf walkers")
    assert np.array_equal(P.prepare_walkers_random(64, 8, k).config, oracle.prepare_walkers_random(64, 8, k))
    k = oracle.case_key("bose walkers")
    a = P.prepare_walkers_sz(64, 6, k, sz=6, states=(0.0, 1.0, 2.0)).config
    assert np.array_equal(a, oracle.prepare_walkers_sz(64, 6, k, sz=6, states=(0.0, 1.0, 2.0)))
    w = P.prepare_walkers_sz(128, 100, P.PRNGKey(0), sz=0)
    assert np.all(w.config.sum(1) == 0) and w.config.dtype == np.float64
    occ = P.prepare_walkers_occupations(64, 16, 16, 4, P.PRNGKey(1)).config
    assert np.all(occ.sum(1) == 16) and occ.max() <= 4 and occ.min() >= 0


def test_lattices():
    assert P.chain(100).edges[-1] == (99, 0) and len(P.chain(100).edges) == 100
    sq = P.square(16)
    assert sq.N == 256 and len(sq.edges) == 512
    kg = P.kagome(12, 12)
    assert kg.N == 432 and len(kg.edges) == 864
    deg = np.bincount(np.asarray(kg.edges).ravel(), minlength=432)
    assert np.all(deg == 4)


def _pairs_at(pos, d, torus=None):
    """Every (i < j) pair at distance d, with the minimum image over the torus
    translations when given (brute force over all pairs)."""
    disp = pos[None, :, :] - pos[:, None, :]
    if torus is not None:
        shifts = np.array(list(itertools.product((-1, 0, 1), repeat=3))) @ torus
        dist = np.min(np.linalg.norm(disp[:, :, None, :] + shifts[None, None], axis=-1), axis=-1)
    else:
        dist = np.linalg.norm(disp, axis=-1)
    i, j = np.nonzero(np.triu(np.isclose(dist, d, atol=1e-9), 1))
    return sorted(zip(i.tolist(), j.tolist()))


@pytest.mark.parametrize("dims,periodic", [((2, 2, 2), True), ((3, 3, 3), True), ((3, 2, 4), True),
                                           ((2, 3, 2), False), ((1, 1, 1), False)])
def test_pyrochlore(dims, periodic):
    """hamiltonian/lattice.py pyrochlore:49-183: N = 4 nx ny nz, 3N bonds and
    coordination 6 when periodic, cell index z + nz y + nz ny x, bonds as
    sorted (i < j) pairs; the bond set equals a brute-force search for pairs
    at the nearest-neighbour distance 1/(2 sqrt 2) (minimum image on the
    torus; every cell size here has a unique minimum image except 2, where
    the search over images still finds exactly the lattice's bonds)."""
    lat = P.hamiltonian.pyrochlore(*dims, periodic=periodic)
    nx, ny, nz = dims
    assert lat.N == 4 * nx * ny * nz and lat.edges == sorted(lat.edges)
    assert all(i < j for i, j in lat.edges)
    pos = lat.extras["positions"]
    prim = lat.extras["primitive_vectors"]
    if nz > 1:
        np.testing.assert_allclose(pos[4 * 1], prim[2])                # cell (0, 0, 1): z fastest
    if ny > 1:
        np.testing.assert_allclose(pos[4 * nz], prim[1])               # cell (0, 1, 0)
    nn = 1.0 / (2.0 * np.sqrt(2.0))
    want = _pairs_at(pos, nn, lat.extras["torus"] if periodic else None)
    assert lat.edges == want
    for c in range(lat.N // 4):                                        # each cell's up tetrahedron
        for a, b in itertools.combinations(range(4 * c, 4 * c + 4), 2):
            assert (a, b) in set(lat.edges)
    if periodic:
        assert len(lat.edges) == 3 * lat.N
        assert np.all(np.bincount(np.asarray(lat.edges).ravel(), minlength=lat.N) == 6)
    else:
        assert len(lat.edges) == len(_pairs_at(pos, nn))


@pytest.mark.parametrize("name,fn,args,periodic", [
    ("pyrochlore_2x2x2", "pyrochlore", (2, 2, 2), True), ("pyrochlore_3x2x4", "pyrochlore", (3, 2, 4), True),
    ("pyrochlore_4x4x4", "pyrochlore", (4, 4, 4), True),
    ("pyrochlore_2x3x2_open", "pyrochlore", (2, 3, 2), False),
    ("pyrochlore_1x1x1_open", "pyrochlore", (1, 1, 1), False),
    ("kagome_12x12", "kagome", (12, 12), True), ("kagome_3x2_open", "kagome", (3, 2), False),
    ("chain_100", "chain", (100,), True), ("chain_7_open", "chain", (7,), False)])
def test_lattices_match_the_reference_fixture(name, fn, args, periodic):
    """Edge lists (in order) and positions equal those of PyGFMC's own
    hamiltonian/lattice.py on the same arguments (tests/golden/lattices.npz,
    written by tests/golden/make_lattice_golden.py from that file)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "lattices.npz"))
    lat = getattr(P.hamiltonian, fn)(*args, periodic=periodic)
    assert lat.N == int(z[f"{name}/N"])
    assert lat.edges == [tuple(e) for e in z[f"{name}/edges"].tolist()]
    if f"{name}/positions" in z.files:
        np.testing.assert_allclose(lat.extras["positions"], z[f"{name}/positions"], rtol=0, atol=1e-14)
    if f"{name}/hexagons" in z.files:                  # kagome: one loop per cell, CCW from angle 0
        np.testing.assert_array_equal(lat.extras["hexagons"], z[f"{name}/hexagons"])
        np.testing.assert_allclose(lat.extras["hexagon_centers"], z[f"{name}/hexagon_centers"],
                                   rtol=0, atol=1e-14)


def test_protocol_classes():
    """PyGFMC's top-level Operator / DiagonalOperator / Guide (protocols.py:25-143)
    exist with the same member names, and this package's objects have the
    members the protocols require."""
    import typing
    for cls, members in ((P.Operator, ("M_total", "get_rates", "generate_state", "move")),
                         (P.DiagonalOperator, ("diagonal_weight",)),
                         (P.Guide, ("log_diff_from_operator", "log_diff_from_configs", "log_psi",
                                    "build_cache", "incremental", "init_state", "update_state"))):
        assert typing.Protocol in cls.__mro__
        for m in members:
            assert hasattr(cls, m) or m in cls.__annotations__, (cls.__name__, m)
    H = P.SpinHalf.create(P.chain(6).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    assert all(hasattr(H, m) for m in ("M_total", "get_rates", "generate_state", "diagonal_weight"))
    for g in (P.JastrowSpinHalf(6, P.chain(6).edges, beta=0.3), P.ExactGroundState(H)):
        assert any(hasattr(g, m) for m in ("log_diff_from_operator", "log_diff_from_configs", "log_psi"))


def test_pyrochlore_rejects_single_cell_tori():
    for dims in ((1, 2, 2), (2, 1, 2), (2, 2, 1)):
        with pytest.raises(ValueError, match=">= 2"):
            P.hamiltonian.pyrochlore(*dims)
    with pytest.raises(ValueError, match="at least one cell"):
        P.hamiltonian.pyrochlore(0, 2, 2, periodic=False)


def test_run_validation_errors_before_any_work():
    w = P.prepare_walkers_sz(8, 6, P.PRNGKey(0))
    H = P.SpinHalf.create(P.chain(6).edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    with pytest.raises(ValueError, match="step_size must be > 0"):
        P.run(w, 10, H, -0.1, None, [2])
    with pytest.raises(ValueError, match="integer step_size"):
        P.run(w, 10, H, 0.5, None, [2], method="single_step", lam=4.0)
    with pytest.raises(ValueError, match="needs the GFMC shift"):
        P.run(w, 10, H, 2, None, [2], method="single_step")
    with pytest.raises(ValueError, match="n_steps"):
        P.run(w, 0, H, 0.1, None, [2])
    with pytest.raises(ValueError, match="p_array"):
        P.run(w, 10, H, 0.1, None, [])
    with pytest.raises(ValueError, match="smaller than n_steps"):
        P.run(w, 10, H, 0.1, None, [10], rng_key=P.PRNGKey(1))
    with pytest.raises(ValueError, match="warmup_steps=0 needs"):
        P.run(w, 10, H, 0.1, None, [2], warmup_steps=0, rng_key=P.PRNGKey(1))
    with pytest.raises(TypeError):
        P.run(w, 10, object(), 0.1, None, [2], rng_key=P.PRNGKey(1))
    # off-diagonal operators: name collisions, odd p, too short a run,
    # an empty equal-window band (engine/driver.py:1444-1466, 478-551)
    op = P.SpinHalf.create(P.chain(6).edges, J_x=2.0, J_y=2.0, sign_check=False)
    with pytest.raises(ValueError, match="share name"):
        P.run(w, 40, H, 0.1, None, [2], diag_operators={"a": H}, off_diag_operators={"a": op},
              rng_key=P.PRNGKey(1))
    with pytest.raises(ValueError, match="divisible by 2"):
        P.run(w, 40, H, 0.1, None, [2, 3], off_diag_operators={"a": op}, rng_key=P.PRNGKey(1))
    with pytest.raises(ValueError, match="n_steps > 1.5"):
        P.run(w, 12, H, 0.1, None, [8], off_diag_operators={"a": op}, rng_key=P.PRNGKey(1))
    with pytest.raises(ValueError, match="equal off-diagonal windows"):
        P.run(w, 14, H, 0.1, None, [8], off_diag_operators={"a": op}, rng_key=P.PRNGKey(1),
              return_raw=False, off_diag_stride=7)


def test_measurement_plan_grid():
    """Stride grid, equal-window band and offset (engine/driver.py:478-564)."""
    from pygfmc_b200.engine import measured_steps, measurement_plan
    pl = measurement_plan(100, [2, 8], 2, 1, True)
    assert not pl.gate_off_diag and pl.off_diag_offset == 0
    assert np.array_equal(measured_steps(100, pl), np.arange(100))
    pl = measurement_plan(100, [2, 8], 2, 3, True)
    assert pl.gate_off_diag and np.array_equal(measured_steps(100, pl), np.arange(2, 100, 3))
    pl = measurement_plan(100, [2, 8], 2, 3, False)
    assert pl.equal_windows and pl.off_diag_offset == 8
    assert np.array_equal(measured_steps(100, pl), np.arange(8, 96, 3))


@pytest.mark.parametrize("name", ["spinhalf_jastrow_cont_time", "bose_none_single_step",
                                  "spinhalf_none_multi_step", "bose_jastrow_cont_time"])
def test_estimators_reproduce_golden_observables(golden, name):
    """The host estimators on the golden raw series give the golden obs:
    diagonal and off-diagonal windows both restricted to i >= max(m)."""
    from pygfmc_b200.estimators import diagonal_estimates, off_diagonal_estimates
    p = name + "/"
    lw = golden[p + "raw/log_weights"]
    diag = {k.split("/")[-1]: golden[k] for k in golden.files if k.startswith(p + "raw/diag/")}
    off = {k.split("/")[-1]: golden[k] for k in golden.files if k.startswith(p + "raw/off_diag/")}
    norm = {nm: golden[p + f"raw/off_diag_norm/{nm}"] for nm in off}
    assert diag and off
    obs = diagonal_estimates([2, 4], lw, diag, 2)
    obs.update(off_diagonal_estimates([2, 4], [1, 2], lw, off, norm, np.arange(len(lw)), 2))
    for nm in list(diag) + list(off):
        for pp in (2, 4):
            np.testing.assert_allclose(obs[nm][pp], golden[p + f"obs/{nm}/{pp}"], rtol=1e-10,
                                       atol=1e-12, err_msg=f"{nm} p={pp}")


_N4 = 4


def _run_table():
    """(label, overrides, exception, message) in the form of the reference's
    validation table (tests/core/test_validation_messages.py:62-96, engine
    part); each must raise before any device work (none is possible on a CPU
    host)."""
    XX = P.SpinHalf.create(P.chain(_N4).edges, J_x=-1.0, J_y=-1.0, sign_check=False)

    class NoRatios:
        pass

    rows = [(f"nonfinite step {v}", dict(step_size=v), ValueError, "step_size must be finite")
            for v in (np.nan, np.inf, -np.inf)]
    rows += [(f"nonfinite shift {m} {v}", dict(method=m, step_size=2, lam=v), ValueError,
              "lam must be finite") for m in ("single_step", "multi_step")
             for v in (np.nan, np.inf, -np.inf)]
    rows += [
        ("zero walkers", dict(walkers=P.prepare_walkers_from_configs(np.zeros((0, _N4)))),
         ValueError, "At least one walker is required"),
        ("step_size zero", dict(step_size=0.0), ValueError, "step_size must be > 0"),
        ("step_size negative", dict(step_size=-1.0), ValueError, "step_size must be > 0"),
        ("non-integer discrete step", dict(step_size=2.5, method="multi_step", lam=3.0), ValueError,
         "method='multi_step' requires an integer step_size"),
        ("hamiltonian without get_rates", dict(hamiltonian=type("Bare", (), {"M_total": 2})()),
         TypeError, "hamiltonian 'Bare' is missing required attribute(s) get_rates"),
        ("off-diagonal operator without get_rates",
         dict(off_diag_operators={"bad": type("Bare", (), {"M_total": 1})()}), TypeError,
         "off-diagonal operator 'bad' 'Bare' is missing required attribute(s) get_rates"),
        ("guide without ratio routines", dict(guide=NoRatios()), TypeError,
         "Guide 'NoRatios' must implement at least one of log_diff_from_operator"),
        ("batch size not dividing the walkers", dict(off_diag_batch_size=3), ValueError,
         "off_diag_batch_size=3 must divide N_walkers=8"),
        ("max(p) not below n_steps", dict(n_steps=8, p_array=[8]), ValueError,
         "every p value must be smaller than n_steps: got n_steps=8 and max(p)=8"),
        ("off-diagonal run too short", dict(n_steps=10, p_array=[8], off_diag_operators={"xx": XX}),
         ValueError, "off-diagonal operators need n_steps > 1.5*max(p)"),
        ("equal windows hold no stride step",
         dict(n_steps=13, p_array=[8], off_diag_stride=4, return_raw=False,
              off_diag_operators={"xx": XX}),
         ValueError, "measure only the steps 8..8 (n_steps=13"),
        ("odd p with an off-diagonal operator", dict(p_array=[3], off_diag_operators={"xx": XX}),
         ValueError, "All p values must be divisible by 2 when off_diag_operators have "
                     "off-diagonal elements (M_total > 1); got [3]"),
    ]
    return rows


@pytest.mark.parametrize("row", range(len(_run_table())))
def test_run_messages_match_the_reference_table(row):
    import re
    label, overrides, exc, message = _run_table()[row]
    kw = dict(walkers=P.prepare_walkers_sz(8, _N4, P.PRNGKey(0), sz=0), n_steps=20,
              hamiltonian=P.SpinHalf.create(P.chain(_N4).edges, J_x=-1.0, J_y=-1.0, J_z=1.0),
              step_size=0.1, guide=None, p_array=[2], rng_key=P.PRNGKey(1), warmup_steps=8,
              verbosity=0)
    kw.update(overrides)
    with pytest.raises(exc, match=re.escape(message)):
        P.run(**kw)


def test_require_lam_contract():
    """engine/evolution.py require_lam:724-741: cont_time takes no shift
    (any lam is dropped), the discrete methods need a finite one."""
    from pygfmc_b200.engine import require_lam
    assert require_lam("cont_time", None) is None
    assert require_lam("cont_time", 5.0) is None
    assert require_lam("multi_step", 4) == 4.0 and isinstance(require_lam("single_step", 4.5), float)
    for m in ("single_step", "multi_step"):
        with pytest.raises(ValueError, match="needs the GFMC shift"):
            require_lam(m, None)
    with pytest.raises(ValueError, match="Unknown method"):
        require_lam("exact", 1.0)


def test_lam_stays_a_keyword():
    """lam comes after rng_key: a shift placed positionally after the
    Hamiltonian lands in the step_size slot and the call is rejected
    (engine/multi_gpu.py run:822)."""
    w = P.prepare_walkers_sz(64, 8, P.PRNGKey(0), sz=0)
    H = P.SpinHalf.create(P.chain(8).edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    with pytest.raises(TypeError, match="got multiple values for argument 'step_size'"):
        P.run(w, 30, H, 4.0, step_size=2, guide=None, p_array=[2], method="multi_step",
              rng_key=P.PRNGKey(0), verbosity=0)


@pytest.mark.parametrize("model", ["SpinHalf", "BoseHubbard"])
@pytest.mark.parametrize("edges", [[0, 1], [[0, 1, 2]], [[-1, 0]], [[0, 1.5]], [[0, np.nan]],
                                   [[0, np.inf]], np.empty((0, 3)), [[0, 2**63]]],
                         ids=["flat", "three-column", "negative", "fractional", "nan", "inf",
                              "empty-three-column", "overflow"])
def test_models_reject_invalid_edges(model, edges):
    """Invalid connectivity raises instead of changing the Hamiltonian
    (hamiltonian/_common.py edges_array; the reference's
    tests/core/test_hamiltonian_fixes.py:23-31 cases)."""
    with pytest.raises(ValueError, match="edge"):
        getattr(P, model).create(edges, N=3)


@pytest.mark.parametrize("edges", [[], np.empty((0, 2)), [[0., 1.]],
                                   np.array([[0, 1]], dtype=np.uint64)])
def test_valid_edge_inputs_are_kept(edges):
    H = P.SpinHalf.create(edges, N=3)
    assert np.asarray(H.edges).shape == (len(edges), 2)


def test_spinhalf_sign_checks_name_the_remedy():
    """A wrong-sign J_pmpm or J_pm raises with the fix in the message, per
    edge too; the caller-side J_x <-> J_y swap is accepted; sign_check=False
    builds measurement operators as given (hamiltonian/SpinHalf.py create)."""
    edges = P.chain(8).edges
    with pytest.raises(ValueError, match="sign-problem-free"):
        P.SpinHalf.create(edges, J_x=-0.3, J_y=-1.1, J_z=0.5, h_x=0.7)
    with pytest.raises(ValueError, match="swap"):
        P.SpinHalf.create(edges, J_x=-0.3, J_y=-1.1, J_z=0.5)
    with pytest.raises(ValueError, match="J_pm"):
        P.SpinHalf.create(edges, J_x=1.0, J_y=1.0, J_z=0.5)
    Jx, Jy = -np.ones(len(edges)), -np.ones(len(edges))
    Jx[3] = -0.2
    with pytest.raises(ValueError, match="Offending edges"):
        P.SpinHalf.create(edges, J_x=Jx, J_y=Jy, J_z=0.5)
    ok = P.SpinHalf.create(edges, J_x=-1.1, J_y=-0.3, J_z=0.5, h_x=0.7)
    assert float(np.ravel(ok.J_pmpm)[0]) == pytest.approx(-0.2)
    assert float(np.ravel(ok.J_pm)[0]) == pytest.approx(-0.35)
    meas = P.SpinHalf.create(edges, J_x=-0.3, J_y=-1.1, J_z=0.5, sign_check=False)
    assert float(np.ravel(meas.J_pmpm)[0]) == pytest.approx(0.2)


def test_structure_factor_factory():
    """hamiltonian/SpinHalf.py StructureFactor:464-628: one slot per pair of
    nonzero weight 1 + cos(k.dr), J_x = 2 (a + b) W, J_y = 2 (a - b) W per
    channel, the diagonal channel warns, unreachable channels are named."""
    import warnings
    L = 8
    pos = np.arange(L, dtype=float)[:, None]
    k = [np.pi / 2]
    ops = {ch: P.hamiltonian.StructureFactor(pos, k, ch, dtype=np.float64)
           for ch in ("SpSm", "SpSp", "spsm + spsp")}
    iu = np.triu_indices(L, 1)
    W = 1.0 + np.cos((pos[iu[0]] - pos[iu[1]]) @ np.asarray(k))
    keep = W > 1e-12
    assert len(ops["SpSm"].edge_i) == keep.sum() < len(W)        # cos = -1 pairs dropped
    np.testing.assert_allclose(ops["SpSm"].J_pm, W[keep], rtol=1e-15)     # (J_x + J_y) / 4 = a W
    np.testing.assert_allclose(ops["SpSm"].J_pmpm, 0.0, atol=0)
    np.testing.assert_allclose(ops["SpSp"].J_pm, 0.0, atol=1e-15)
    np.testing.assert_allclose(ops["SpSp"].J_pmpm, W[keep], rtol=1e-15)
    np.testing.assert_allclose(ops["spsm + spsp"].J_pm, W[keep], rtol=1e-15)
    np.testing.assert_allclose(ops["spsm + spsp"].J_pmpm, W[keep], rtol=1e-15)
    assert ops["SpSm"].M_total == 1 + keep.sum()
    # rates of a measurement operator are non-negative
    x = P.prepare_walkers_random(1, L, P.PRNGKey(1)).config[0]
    assert np.all(ops["spsm + spsp"].get_rates(x)[0][1:] >= 0)
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        zz = P.hamiltonian.StructureFactor(pos, k, "SzSz", dtype=np.float64)
    assert any("DIAGONAL" in str(r.message) for r in rec) and zz.M_total == 1
    np.testing.assert_allclose(zz.J_z, 2.0 * W[keep], rtol=1e-15)
    for bad, msg in (("YY", "SpSm minus SpSp"), ("zz", "spelled 'SzSz'"), ("S.S", "separately")):
        with pytest.raises(ValueError, match=msg):
            P.hamiltonian.StructureFactor(pos, k, bad)
    with pytest.raises(ValueError, match="ONE wavevector"):
        P.hamiltonian.StructureFactor(pos, [[0.1], [0.2]])
    with pytest.raises(ValueError, match="zone boundary"):
        P.hamiltonian.StructureFactor(np.array([[0.0], [1.0]]), [np.pi])


def test_is_valid_k():
    """hamiltonian/observables.py is_valid_k:14-65 (the pins of PyGFMC's
    tests/core/test_structure_factor_operator.py:190-202): k . L_j / 2 pi an
    integer for every periodic vector; a bool for one wavevector, an array for
    a stack; and only a valid k leaves SzSzStructureFactor unchanged when the
    positions move to other periodic images."""
    is_valid_k = P.hamiltonian.is_valid_k
    L = np.array([[4.0, 0.0], [2.0, 2.0 * np.sqrt(3.0)]])       # a triangular torus
    ks = 2 * np.pi * np.array([[0, 0], [1, 0], [0, 1], [3, -2]]) @ np.linalg.inv(L).T
    got = is_valid_k(ks, L)
    assert isinstance(got, np.ndarray) and got.dtype == bool and got.all()
    assert is_valid_k(ks[1], L) is True
    assert is_valid_k(0.5 * ks[1], L) is False
    assert is_valid_k(ks[3] + 1e-7, L) is True                    # float32-built k pass
    np.testing.assert_array_equal(is_valid_k(np.vstack([ks[2], 0.5 * ks[2]]), L), [True, False])
    np.testing.assert_array_equal(is_valid_k(2 * np.pi * np.arange(3)[:, None] / 8, [[8.0]]),
                                  [True, True, True])
    assert is_valid_k([1.0], [[8.0]]) is False
    with pytest.raises(ValueError, match=r"\(d, d\)"):
        is_valid_k(ks, L[:1])
    with pytest.raises(ValueError, match="k_vectors must be"):
        is_valid_k(np.zeros(3), L)
    # image independence of the structure factor exactly for valid k
    rng = np.random.default_rng(5)
    N = 6
    pos = rng.normal(size=(N, 2))
    shifted = pos + rng.integers(-2, 3, size=(N, 2)) @ L
    x = rng.choice([1.0, -1.0], size=(16, N))
    for k, same in ((ks[3], True), (1.3 * ks[3], False)):
        a = P.hamiltonian.SzSzStructureFactor(pos, k[None], dtype=np.float64).diagonal_weight(x)
        b = P.hamiltonian.SzSzStructureFactor(shifted, k[None], dtype=np.float64).diagonal_weight(x)
        assert (np.max(np.abs(a - b)) < 1e-9) == same


def test_three_ratio_routines_agree():
    """tests/core/test_guides.py:144-165: log_diff_from_operator,
    log_diff_from_configs and log_psi give the same log-ratios, each called
    as PyGFMC's engine calls them (the optional cache argument passed)."""
    e = P.chain(8).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.4, dtype=np.float64)
    guides = [P.JastrowSpinHalf(8, e, beta=0.3, h=0.05, dtype=np.float64),
              P.RBMSpinHalf(8, 12, seed=1, sigma=0.3), P.ExactGroundState(H, dtype=np.float64)]
    rng = np.random.default_rng(3)
    for g in guides:
        cache = g.build_cache(H) if hasattr(g, "build_cache") else None
        for _ in range(3):
            x = rng.choice([-1.0, 1.0], size=8)
            _, succ = H.get_rates(x, return_configs=True)
            from_cfg = np.asarray(g.log_diff_from_configs(x, succ, None), np.float64)
            if hasattr(g, "log_diff_from_operator"):
                from_op = np.asarray(g.log_diff_from_operator(x, H, cache), np.float64)
                np.testing.assert_allclose(from_op[1:], from_cfg[1:], rtol=0, atol=1e-10,
                                           err_msg=type(g).__name__)
            if hasattr(g, "log_psi"):
                base = g.log_psi(x, None)
                want = np.array([g.log_psi(c, None) - base for c in succ])
                np.testing.assert_allclose(from_cfg[1:], want[1:], rtol=0, atol=1e-10,
                                           err_msg=type(g).__name__)

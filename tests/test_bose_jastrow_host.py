"""JastrowBoseHubbard's ratios on the host and in the oracle, over every block
of the Bose-Hubbard transition layout (hopping, pair creation and
annihilation, single-site terms) and every parameter form (tied, per pair /
per site, absent), with guide pairs that differ from the bonds and repeat one
pair -- the cases of PyGFMC's tests/core/test_jastrow_bose_hubbard.py:19-66:
``log_diff_from_operator`` equals log_psi differences over the successors
``get_rates`` returns, and the oracle's guided rates (what the device is
checked against) are the bare rates times exp of those ratios.  Also the
operators' ``move`` and ``diagonal_weight`` against ``generate_state`` and
``get_rates`` (tests/core/test_get_rates_all_classes.py).  Host only."""
import itertools

import numpy as np
import pytest

import pygfmc_b200 as P
from oracle_guides import oracle_guide

L = 9
EDGES = np.asarray(P.chain(L).edges)
PAIRS = np.concatenate([EDGES, [[0, 4], [2, 7], [1, 2]]])      # (1, 2) twice
_rng = np.random.default_rng(3)
MODELS = {
    "hopping": dict(t=1.0, U=2.0, n_max=2),
    "hopping+pairs": dict(t=1.0, eta=0.25, U=4.0, mu=1.0, n_max=3),
    "pairs+h_pm": dict(eta=0.3, h_pm=0.2, U=1.0, n_max=3, N=L),
    "all": dict(t=1.0, eta=0.2, h_pm=0.1, U=3.0, mu=0.5, n_max=2, N=L),
}
FORMS = {
    "tied beta, h, d": dict(beta=0.21, h=0.13, d=0.37),
    "tied beta only": dict(beta=0.21),
    "per pair / per site": dict(beta=_rng.uniform(-0.2, 0.4, len(PAIRS)),
                                h=_rng.uniform(-0.3, 0.3, L), d=_rng.uniform(0.1, 0.6, L)),
    "tied beta, per site d, no h": dict(beta=0.15, d=_rng.uniform(0.1, 0.6, L)),
}


def _guide(form):
    return P.JastrowBoseHubbard(L, PAIRS, dtype=np.float64, **FORMS[form])


@pytest.mark.parametrize("name,form", list(itertools.product(MODELS, FORMS)))
def test_ratio_equals_log_psi_differences(name, form):
    H = P.BoseHubbard.create(EDGES, dtype=np.float64, **MODELS[name])
    G = _guide(form)
    x = np.random.default_rng(0).integers(0, int(H.n_max) + 1, (40, L)).astype(np.float64)
    for c in x:
        fast = np.asarray(G.log_diff_from_operator(c, H), np.float64)
        rates, succ = H.get_rates(c, return_configs=True)
        assert fast.shape == (H.M_total,)
        ref = np.array([G.log_psi(s) for s in succ]) - G.log_psi(c)
        live = np.asarray(rates) != 0          # the moves that exist from c
        np.testing.assert_allclose(fast[live], ref[live], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name,form", list(itertools.product(MODELS, FORMS)))
def test_oracle_guided_rates(oracle, name, form):
    H = P.BoseHubbard.create(EDGES, dtype=np.float64, **MODELS[name])
    G = _guide(form)
    kw = {k: v for k, v in MODELS[name].items() if k != "N"}
    m = oracle.bose_hubbard(EDGES, **kw)
    g = oracle_guide(oracle, G, m)
    x = np.random.default_rng(1).integers(0, int(H.n_max) + 1, (16, L)).astype(np.float64)
    guided, bare = oracle.rates(m, g, x), oracle.rates(m, oracle.no_guide(), x)
    for w in range(len(x)):
        ld = np.asarray(G.log_diff_from_operator(x[w], H), np.float64)
        expect = bare[w] * np.exp(np.where(bare[w] == 0, 0.0, ld))
        np.testing.assert_allclose(guided[w], expect, rtol=1e-12, atol=1e-14, err_msg=f"{name} {form}")


def test_move_reproduces_generate_state():
    """hamiltonian/bose_hubbard.py move:427-435 (PyGFMC's
    tests/core/test_get_rates_all_classes.py:154-177): adding ``deltas`` at
    ``sites`` gives ``generate_state`` for every transition."""
    ring = np.asarray([[i, (i + 1) % 6] for i in range(6)])
    H = P.BoseHubbard.create(ring, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, N=6, n_max=2,
                             dtype=np.float64)
    rng = np.random.default_rng(0)
    for _ in range(3):
        x = rng.choice(np.asarray(H.local_hilbert_space), size=H.N)
        for idx in range(H.M_total):
            sites, deltas = H.move(x, idx)
            assert sites.shape == (2,) and deltas.shape == (2,)
            y = np.array(x, copy=True)
            y[sites[0]] += deltas[0]
            y[sites[1]] += deltas[1]
            np.testing.assert_array_equal(y, H.generate_state(x, idx))
    with pytest.raises(ValueError):
        H.move(x, H.M_total)


def test_diagonal_weight_is_the_first_rate():
    """tests/core/test_get_rates_all_classes.py:110-125 on the all-parameters
    models: ``diagonal_weight`` equals slot 0 of ``get_rates`` on random
    configurations, and the diagonal is not constant."""
    rng = np.random.default_rng(0)
    pairs = [(i, j) for i in range(6) for j in range(i + 1, 6)]
    n = len(pairs)
    jx = -rng.uniform(0.6, 1.2, n)
    S = P.SpinHalf.create(pairs, J_x=jx, J_y=jx + rng.uniform(0.05, 0.4, n), J_z=rng.uniform(-1, 1, n),
                          h_z=-rng.uniform(-1, 1, 6), h_x=rng.uniform(0.1, 0.6, 6), dtype=np.float64)
    rng = np.random.default_rng(2)
    B = P.BoseHubbard.create(pairs, t=rng.uniform(0.2, 1.0, n), eta=rng.uniform(0.2, 1.0, n), U=1.3,
                             mu=-0.4, n_max=2, dtype=np.float64)
    for H in (S, B):
        vals = np.asarray(H.local_hilbert_space)
        x = np.random.default_rng(1234).choice(vals, size=(512, H.N))
        fast = np.asarray(H.diagonal_weight(x), np.float64)
        slow = np.array([H.get_rates(c)[0][0] for c in x])
        assert np.ptp(slow) > 0
        np.testing.assert_allclose(fast, slow, rtol=0, atol=1e-12)


@pytest.mark.parametrize("form", FORMS)
def test_incremental_state_follows_the_moves(form):
    """tests/core/test_jastrow_bose_hubbard.py:69-90: the neighbour sums
    updated through 200 random moves (``BoseHubbard.move``) equal a rebuild to
    rounding, and the ratios with that state equal the plain ones."""
    H = P.BoseHubbard.create(EDGES, dtype=np.float64, **MODELS["all"])
    G = P.JastrowBoseHubbard(L, PAIRS, dtype=np.float64, incremental=True, **FORMS[form])
    rng = np.random.default_rng(5)
    x = rng.integers(0, int(H.n_max) + 1, L).astype(np.float64)
    state = G.init_state(x)
    for _ in range(200):
        idx = int(rng.integers(0, H.M_total))
        sites, deltas = H.move(x, idx)
        state = G.update_state(state, x, sites, deltas)
        x = H.generate_state(x, idx)
    np.testing.assert_allclose(state, G.init_state(x), rtol=0, atol=1e-12)
    np.testing.assert_array_equal(G.log_diff_from_operator(x, H, state=state),
                                  G.log_diff_from_operator(x, H))


def test_incremental_update_without_pairs_is_a_no_op():
    H = P.BoseHubbard.create(EDGES, dtype=np.float64, **MODELS["all"])
    G = P.JastrowBoseHubbard(L, np.zeros((0, 2), dtype=np.int64), beta=0.3, d=0.2, incremental=True)
    x = np.random.default_rng(1).integers(0, int(H.n_max) + 1, L).astype(np.float64)
    state = G.init_state(x)
    assert state.shape == (L,) and not np.any(state)
    sites, deltas = H.move(x, 1)
    np.testing.assert_array_equal(G.update_state(state, x, sites, deltas), state)


def test_a_wrong_coupling_is_detected():
    """Non-vacuity of the ratio checks: the opposite beta disagrees."""
    H = P.BoseHubbard.create(EDGES, dtype=np.float64, **MODELS["all"])
    good = P.JastrowBoseHubbard(L, PAIRS, beta=0.21, h=0.13, d=0.37, dtype=np.float64)
    bad = P.JastrowBoseHubbard(L, PAIRS, beta=-0.21, h=0.13, d=0.37, dtype=np.float64)
    x = np.array([2, 0, 1, 1, 2, 0, 1, 2, 1], dtype=np.float64)
    rates, succ = H.get_rates(x, return_configs=True)
    ref = np.array([good.log_psi(s) for s in succ]) - good.log_psi(x)
    assert np.max(np.abs(bad.log_diff_from_operator(x, H) - ref)) > 0.1


def test_parameters_keep_their_form_and_bad_shapes_raise():
    """tests/core/test_jastrow_bose_hubbard.py:115-135: tied parameters stay
    0-d, per-pair / per-site ones stay arrays, an absent h reads as zeros;
    wrong lengths and a missing beta raise."""
    g = P.JastrowBoseHubbard(L, PAIRS, beta=0.5)
    assert np.ndim(g._beta) == 0 and g._h is None and g._d is None
    g = P.JastrowBoseHubbard(L, PAIRS, beta=0.1, h=0.2, d=0.5)
    assert (np.ndim(g._beta), np.ndim(g._h), np.ndim(g._d)) == (0, 0, 0)
    g = P.JastrowBoseHubbard(L, PAIRS, **FORMS["per pair / per site"])
    assert (g._beta.shape, g._h.shape, g._d.shape) == ((len(PAIRS),), (L,), (L,))
    g = P.JastrowBoseHubbard(L, PAIRS, beta=0.1, d=0.5)
    assert g._h is None and np.all(g.h == 0.0)
    assert np.allclose(g.beta, 0.1) and g.beta.shape == (len(PAIRS),)
    with pytest.raises(ValueError):
        P.JastrowBoseHubbard(L, PAIRS, beta=0.1, d=np.ones(L + 1))
    with pytest.raises(ValueError):
        P.JastrowBoseHubbard(L, PAIRS, beta=np.ones(L))
    with pytest.raises(ValueError):
        P.JastrowBoseHubbard(L, PAIRS, beta=None)

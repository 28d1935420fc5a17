"""Contracts of the reference's own statistical and estimator tests, restated
for this engine:

* guided GFMC within 0.02 per site of exact diagonalisation under every
  method, on the 6-site XXZ ring with a transverse field and the 6-site
  Bose-Hubbard chain (tests/core/test_guides.py:127-142,
  tests/core/test_guided_methods.py:25-56), which also makes the three
  methods agree with each other (tests/core/test_method_equivalence.py);
* the statistics() invariants: offspring fractions sum to 1, ESS(m = 0) = N
  and non-increasing in m (tests/core/test_statistics_contract.py:62-88);
* the blocked jackknife with two blocks is the half-chain split
  (tests/core/test_io_hdf5.py:724).

The exact energies come from the Hamiltonian rebuilt from the model's own
get_rates over every configuration (tests/core/rates.py:115 does the same),
cross-checked against an independent Kronecker-product construction."""
import itertools

import numpy as np
import pytest

import pygfmc_b200 as P


def _matrix_from_rates(H, states):
    """H[x', x] from get_rates(x) over the listed states (rows = states)."""
    index = {tuple(s): i for i, s in enumerate(states)}
    M = np.zeros((len(states), len(states)))
    for i, x in enumerate(states):
        rates, succ = H.get_rates(x, return_configs=True)
        M[i, i] += rates[0]
        for r, y in zip(rates[1:], succ[1:]):
            if r != 0:
                M[index[tuple(y)], i] += r
    return M


def _xxz_ring(h_x=0.4):
    return P.SpinHalf.create(P.chain(6).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=h_x,
                             dtype=np.float64)


def _spin_states(N):
    return np.array(list(itertools.product((-1.0, 1.0), repeat=N)))


def _kron_xxz(N, jx, jy, jz, hx):
    """sum_e (jx Sx Sx + jy Sy Sy + jz Sz Sz) - hx sum Sx on the periodic ring,
    basis |s_0 .. s_{N-1}>, s = -1 first (spin down = first basis vector)."""
    sx = np.array([[0, 0.5], [0.5, 0]])
    sy = np.array([[0, 0.5j], [-0.5j, 0]])
    sz = np.diag([-0.5, 0.5])

    def site(op, k):
        out = np.ones((1, 1), dtype=complex)
        for j in range(N):
            out = np.kron(out, op if j == k else np.eye(2))
        return out

    Hm = np.zeros((2 ** N, 2 ** N), dtype=complex)
    for i in range(N):
        j = (i + 1) % N
        Hm += jx * site(sx, i) @ site(sx, j) + jy * site(sy, i) @ site(sy, j) + jz * site(sz, i) @ site(sz, j)
        Hm -= hx * site(sx, i)
    return Hm


def test_exact_energies_from_rates_match_kronecker_construction():
    H = _xxz_ring()
    M = _matrix_from_rates(H, _spin_states(6))
    K = _kron_xxz(6, -1.0, -1.0, 1.0, 0.4)
    assert np.allclose(M, K.real) and np.allclose(K.imag, 0.0)


def _systems():
    Hs = _xxz_ring()
    Es = float(np.linalg.eigvalsh(_matrix_from_rates(Hs, _spin_states(6)))[0])
    Gs = P.JastrowSpinHalf(6, P.chain(6).edges, beta=0.3)
    ws = P.prepare_walkers_random(512, 6, P.PRNGKey(0))
    Hb = P.BoseHubbard.create(P.chain(6).edges, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2,
                              dtype=np.float64)
    states_b = np.array(list(itertools.product((0.0, 1.0, 2.0), repeat=6)))
    Eb = float(np.linalg.eigvalsh(_matrix_from_rates(Hb, states_b))[0])
    Gb = P.JastrowBoseHubbard(6, P.chain(6).edges, beta=0.05, h=0.1, d=0.3)
    wb = P.prepare_walkers_random(512, 6, P.PRNGKey(1), states=(0.0, 1.0, 2.0))
    # lam above every diagonal element (spin: 6 J_z / 4; Bose: U n(n-1)/2 per site)
    return [("xxz6_hx", Hs, Gs, ws, Es, 3.0), ("bose6", Hb, Gb, wb, Eb, 8.0)]


@pytest.mark.gpu
@pytest.mark.parametrize("method,step", [("cont_time", 0.1), ("single_step", 2), ("multi_step", 4)])
def test_guided_gfmc_matches_exact_diagonalisation(method, step):
    for name, H, G, w, E0, lam in _systems():
        _, E, _, st, raw = P.run(w, 800, H, step, G, [4, 16], method=method,
                                 lam=None if method == "cont_time" else lam,
                                 rng_key=P.PRNGKey(3), warmup_steps=100, verbosity=0)
        Ej, err = P.estimators.jackknife_energy([16], raw["log_weights"], raw["energy"], 10)
        assert abs(Ej[16] - E0) / 6 < 0.02, (name, method, Ej[16], err[16], E0)


@pytest.mark.gpu
def test_statistics_contract():
    name, H, G, w, E0, lam = _systems()[0]
    m_array = [0, 1, 2, 4, 8]
    _, st = P.statistics(w, H, 0.1, G, "cont_time", P.PRNGKey(5), M=8, quiet=True, m_array=m_array)
    k = sorted(key for key in st if key.startswith("offspring_k"))
    total = sum(np.asarray(st[key]) for key in k)
    np.testing.assert_allclose(total, 1.0, rtol=0, atol=1e-12)
    ess = np.asarray(st["effective_sample_size"])
    assert ess[0] == len(w.config)
    assert np.all(np.diff(ess) <= 1e-9) and np.all(ess > 0)
    frac = np.asarray(st["ancestor_fraction"])
    assert frac[0] == 1.0 and np.all(np.diff(frac) <= 1e-12)
    np.testing.assert_allclose(st["survival_rate"], 1.0 - np.asarray(st["offspring_k0"]))


def test_jackknife_two_blocks_is_the_half_chain_split():
    rng = np.random.default_rng(7)
    n = 400
    lw = rng.normal(0.0, 0.05, n)
    E = -3.0 + rng.normal(0.0, 0.2, n)
    p = [2, 8]
    est, err = P.estimators.jackknife_energy(p, lw, E, 2)
    h = n // 2
    first = P.estimators.windowed_energy_host(p, lw[:h], E[:h])
    second = P.estimators.windowed_energy_host(p, lw[h:], E[h:])
    full = P.estimators.windowed_energy_host(p, lw, E)
    for q in p:
        # the two leave-one-out replicas are the two halves
        assert err[q] == pytest.approx(abs(first[q] - second[q]) / 2, rel=1e-12)
        assert est[q] == pytest.approx(full[q], rel=1e-14)

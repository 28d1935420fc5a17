"""Exact diagonalisation and the exact-amplitude guide on the host and in the
oracle (hamiltonian/exact.py:212-375, wavefunction/exact_ground_state.py:
43-256; the properties of PyGFMC's tests/core/test_exact_ground_state.py):
the protocol-built spectrum against a Kronecker-product construction, the
basis index as a bijection, log-ratios against the ground-state vector, the
local energy E0 on every supported configuration (host rates and the C
oracle's rates), save / load, and the lowering to the C ABI -- this package's
guide and a stand-in with the reference's attribute set indexed over (-1, 1)."""
import itertools

import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200 import _lib
from pygfmc_b200.engine import _Keep, exact_amplitude_table, guide_desc
from test_contracts import _kron_xxz


def _ring(h_x=0.0, N=6):
    return P.SpinHalf.create(P.chain(N).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=h_x,
                             dtype=np.float64)


def _all(N, values):
    return np.array(list(itertools.product(values, repeat=N)), dtype=np.float64)


def test_spectrum_matches_kronecker_construction():
    H = _ring(h_x=0.4)
    E, _, _, psi = P.exact_diagonalization(H, (-1.0, 1.0), number_of_states=3, return_states=True)
    w, v = np.linalg.eigh(_kron_xxz(6, -1.0, -1.0, 1.0, 0.4))
    np.testing.assert_allclose(E, w[:3], atol=1e-12)
    # (-1, 1) is the Kronecker basis order (spin down first); the default
    # (1, -1) order is its complement, i.e. the reversed vector
    np.testing.assert_allclose(np.abs(psi[:, 0]), np.abs(v[:, 0]), atol=1e-10)
    _, _, _, psi_d = P.exact_diagonalization(H, return_states=True)
    np.testing.assert_allclose(np.abs(psi_d[:, 0]), np.abs(v[::-1, 0]), atol=1e-10)


def test_sparse_solver_and_observables():
    H = _ring(N=12)
    E_sparse, dobs, oobs = P.exact_diagonalization(H, diag_operators={"Hd": H},
                                                   off_diag_operators={"H": H}, number_of_states=2)
    assert 2 ** 12 > 2048   # the Lanczos branch
    E_dense = np.linalg.eigvalsh(_dense(H, 12))[:2]
    np.testing.assert_allclose(E_sparse, E_dense, atol=1e-9)
    np.testing.assert_allclose(oobs["H"], E_sparse, atol=1e-9)   # <psi|H|psi> = E
    assert dobs["Hd"].shape == (2,)
    # the diagonal part's expectation: sum |psi|^2 H_xx
    _, _, _, psi = P.exact_diagonalization(H, return_states=True)
    cfg, _ = P.hamiltonian._basis((1.0, -1.0), 12)
    hd = np.array([H.diagonal_weight(x) for x in cfg])
    np.testing.assert_allclose(dobs["Hd"][0], (psi[:, 0] ** 2 * hd).sum(), atol=1e-9)


def _dense(H, N):
    cfg, powers = P.hamiltonian._basis((1.0, -1.0), N)
    return P.hamiltonian._protocol_matrix(H, cfg, (1.0, -1.0), powers).toarray()


def test_bose_hubbard_spectrum():
    B = P.BoseHubbard.create(P.chain(3).edges, t=1.0, U=2.0, mu=0.5, h_pm=0.1, eta=0.2, n_max=2,
                             dtype=np.float64)
    E, _, _ = P.exact_diagonalization(B)
    M = _dense_any(B, 3, (0.0, 1.0, 2.0))
    assert np.allclose(M, M.T)
    np.testing.assert_allclose(E[0], np.linalg.eigvalsh(M)[0], atol=1e-12)


def _dense_any(op, N, values):
    states = _all(N, values)
    index = {tuple(s): i for i, s in enumerate(states)}
    M = np.zeros((len(states), len(states)))
    for i, x in enumerate(states):
        rates, succ = op.get_rates(x, return_configs=True)
        for r, y in zip(rates, succ):
            if r != 0:
                M[index[tuple(y)], i] += r
    return M


def test_exact_diagonalization_rejects_bad_arguments():
    H = _ring()
    with pytest.raises(ValueError, match="differs from the values"):
        P.exact_diagonalization(H, (0.0, 1.0))
    with pytest.raises(ValueError, match="distinct"):
        P.exact_diagonalization(H, (1.0, 1.0))
    with pytest.raises(ValueError, match="number_of_states"):
        P.exact_diagonalization(H, number_of_states=65)
    with pytest.raises(ValueError, match="limit"):
        P.exact_diagonalization(_ring(N=25))
    with pytest.raises(ValueError, match="Hamiltonian reports N=6"):
        P.exact_diagonalization(H, N=7)


class _ThreeStateStandIn:
    """A three-state operator's reported sizes (spin 1 on three sites)."""
    N, d, M_total = 3, 3, 1


def test_exact_diagonalization_messages_of_the_reference():
    """The validation pins of PyGFMC's tests/core/test_exact_diagonalization.py
    :95-113, in its order: too few values, a basis above the limit (checked
    before the site count), state counts outside [1, dim], an N or a local
    dimension contradicting the operator."""
    h = P.SpinHalf.create(P.chain(4).edges, -1.0, -1.0, 1.0, dtype=np.float64)
    with pytest.raises(ValueError, match="at least two values"):
        P.exact_diagonalization(h, (1,), 4)
    with pytest.raises(ValueError, match="exceeds the"):
        P.exact_diagonalization(h, (-1, 1), 40)
    with pytest.raises(ValueError, match="number_of_states"):
        P.exact_diagonalization(h, (-1, 1), 4, number_of_states=0)
    with pytest.raises(ValueError, match="number_of_states"):
        P.exact_diagonalization(h, (-1, 1), 4, number_of_states=17)     # dim = 16
    with pytest.raises(ValueError, match="Hamiltonian reports N"):
        P.exact_diagonalization(h, (-1, 1), 5)
    with pytest.raises(ValueError, match="local dimension"):
        P.exact_diagonalization(_ThreeStateStandIn(), (-1, 1), 3)
    # the allocation estimate (basis, matrix triplets, dense solve) is checked
    # before anything is built
    old = P.hamiltonian._ED_MAX_BYTES
    try:
        P.hamiltonian._ED_MAX_BYTES = 2 ** 20
        with pytest.raises(ValueError, match="GiB"):
            P.exact_diagonalization(_ring(N=12))
    finally:
        P.hamiltonian._ED_MAX_BYTES = old


class _FlipSiteZero:
    """A two-site spin-1/2 operator with one transition, site 0 flipped (or set
    to ``target``), of amplitude ``up`` from a down spin and ``down`` from an
    up spin; only the rate protocol."""
    M_total, N, local_hilbert_space = 2, 2, (-1.0, 1.0)

    def __init__(self, up, down, target=None):
        self.up, self.down, self.target = up, down, target

    def generate_state(self, x, k):
        y = np.array(x, dtype=np.float64, copy=True)
        if k == 1:
            y[0] = -y[0] if self.target is None else self.target
        return y

    def get_rates(self, x, return_configs=False):
        x = np.asarray(x, dtype=np.float64)
        rates = np.array([0.0, self.down if x[0] > 0 else self.up])
        succ = np.stack([x, self.generate_state(x, 1)]) if return_configs else None
        return rates, succ


def test_protocol_operators_are_checked_as_the_reference_does():
    """PyGFMC's tests/core/test_exact_ground_state.py:220-235: a transition of
    nonzero amplitude out of the basis and an asymmetric matrix are refused;
    the symmetric flip has the ground energy -1."""
    with pytest.raises(ValueError, match="leads outside the supplied local_hilbert_space"):
        P.exact_diagonalization(_FlipSiteZero(-1.0, -1.0, target=2.0))
    with pytest.raises(ValueError, match="not Hermitian"):
        P.exact_diagonalization(_FlipSiteZero(-1.0, -2.0))
    E = P.exact_diagonalization(_FlipSiteZero(-1.0, -1.0))[0]
    np.testing.assert_allclose(E[0], -1.0, atol=1e-12)
    H = P.SpinHalf.create(np.zeros((0, 2), dtype=np.int64), h_z=1.0, N=2, dtype=np.float64)
    e_ref = P.exact_diagonalization(H)[0][0]
    assert P.exact_diagonalization(H, local_hilbert_space=(-1.0, 1.0))[0][0] == e_ref
    with pytest.raises(ValueError, match="differs from the values"):
        P.exact_diagonalization(H, local_hilbert_space=(0.5, -0.5))
    with pytest.raises(ValueError, match="distinct finite"):
        P.exact_diagonalization(H, local_hilbert_space=(1.0, np.nan))


class _OneConfigDiagonal:
    """A diagonal operator that accepts one configuration at a time (a batch
    would fail its shape check), vector-valued like a structure factor."""

    def __init__(self, sf):
        self.sf = sf

    def diagonal_weight(self, x):
        x = np.asarray(x)
        assert x.ndim == 1
        return self.sf.diagonal_weight(x)


def test_vector_valued_diagonal_observables():
    """A structure factor over several wavevectors gives (k, n_k) expectations
    (hamiltonian/exact.py:366-369): sum_x |psi_k(x)|^2 S(q; x) for each q, the
    same through the whole-basis and the per-configuration evaluation."""
    N = 8
    H = _ring(h_x=0.3, N=N)
    q = 2 * np.pi * np.arange(N)[:, None] / N
    sf = P.hamiltonian.SzSzStructureFactor(np.arange(N, dtype=np.float64)[:, None], q, dtype=np.float64)
    E, dobs, _, psi = P.exact_diagonalization(
        H, diag_operators={"sf": sf, "sf1": _OneConfigDiagonal(sf), "H": H},
        number_of_states=2, return_states=True)
    assert dobs["sf"].shape == (2, N) and dobs["H"].shape == (2,)
    cfg, _ = P.hamiltonian._basis((1.0, -1.0), N)
    direct = np.array([[np.sum(psi[:, k] ** 2 * np.array([sf.diagonal_weight(x)[j] for x in cfg]))
                        for j in range(N)] for k in range(2)])
    np.testing.assert_allclose(dobs["sf"], direct, rtol=0, atol=1e-12)
    np.testing.assert_allclose(dobs["sf1"], dobs["sf"], rtol=0, atol=1e-12)
    # S(q) is a pair sum over i < j, and sum_q cos(q (r_i - r_j)) = 0 for
    # i != j over the N wavevectors of the ring: the q-sum vanishes
    np.testing.assert_allclose(dobs["sf"].sum(axis=1), 0.0, atol=1e-10)


def test_lanczos_solves_are_reproducible():
    """Two solves of one 4096-state matrix in one process agree bit for bit
    (a fixed Lanczos start vector), so two ExactGroundState guides built from
    one Hamiltonian are the same guide."""
    H = _ring(N=12)
    E1, _, _, v1 = P.exact_diagonalization(H, number_of_states=2, return_states=True)
    E2, _, _, v2 = P.exact_diagonalization(H, number_of_states=2, return_states=True)
    np.testing.assert_array_equal(E1, E2)
    np.testing.assert_array_equal(v1, v2)


@pytest.mark.parametrize("values", [(1.0, -1.0), (-1.0, 1.0)])
def test_basis_index_is_a_bijection(values):
    g = P.ExactGroundState(_ring(), local_hilbert_space=values, dtype=np.float64)
    idx = g.basis_index(_all(6, values))
    assert sorted(idx.tolist()) == list(range(64))
    np.testing.assert_array_equal(idx, np.arange(64))   # itertools order = positional order


def test_log_diff_matches_the_ground_state_vector():
    H = _ring(h_x=0.3)
    g = P.ExactGroundState(H, dtype=np.float64)
    _, _, _, psi = P.exact_diagonalization(H, return_states=True)
    la = np.log(np.maximum(np.abs(psi[:, 0]), 1e-30))
    rng = np.random.default_rng(0)
    for x in rng.choice([-1.0, 1.0], size=(5, 6)):
        ld = g.log_diff_from_configs(x)
        assert ld[0] == 0.0
        for k in range(1, H.M_total):
            y = H.generate_state(x, k)
            assert ld[k] == pytest.approx(la[g.basis_index(y)] - la[g.basis_index(x)], abs=1e-12)
        _, succ = H.get_rates(x, return_configs=True)
        np.testing.assert_allclose(g.log_diff_from_configs(x, succ)[1:], ld[1:], atol=0)


def _host_local_energy(H, g, x):
    rates, succ = H.get_rates(x, return_configs=True)
    ld = g.log_diff_from_configs(x, succ).astype(np.float64)
    r = rates * np.exp(np.where(rates == 0, 0.0, ld))
    return r.sum()


@pytest.mark.parametrize("h_x,dtype,tol", [(0.0, np.float64, 1e-10), (0.3, np.float64, 1e-10),
                                           (0.3, np.float32, 2e-5)])
def test_local_energy_is_E0_on_the_support(h_x, dtype, tol):
    """exact_ground_state tests:85-103: the guided rates sum to E0 wherever
    psi_0 does not vanish (for h_x = 0 the Sz = 0 sector: the exact
    wavefunction has nodes elsewhere)."""
    H = _ring(h_x=h_x)
    g = P.ExactGroundState(H, dtype=dtype)
    _, _, _, psi = P.exact_diagonalization(H, return_states=True)
    cfg = _all(6, (1.0, -1.0))
    support = np.abs(psi[:, 0]) > 1e-10
    if h_x == 0.0:
        assert not support.all() and np.array_equal(support, cfg.sum(1) == 0)
    e = np.array([_host_local_energy(H, g, x) for x in cfg[support]])
    np.testing.assert_allclose(e, g.E0, rtol=0, atol=tol)


def test_oracle_exact_guide_gives_E0(oracle):
    """The oracle's restatement (gfmc_oracle.c, kind 5) over both index
    orders: local energy E0 on every Sz = 0 configuration of the 10-site ring,
    and on every configuration with a transverse field."""
    O = oracle
    for h_x in (0.0, 0.25):
        H = P.SpinHalf.create(P.chain(10).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=h_x,
                              dtype=np.float64)
        m = O.spin_half(P.chain(10).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=h_x)
        cfg = _all(10, (1.0, -1.0))
        if h_x == 0.0:
            cfg = cfg[cfg.sum(1) == 0]
        for values in ((1.0, -1.0), (-1.0, 1.0)):
            g = P.ExactGroundState(H, local_hilbert_space=values, dtype=np.float64)
            r = O.rates(m, O.exact_spin_half(g.log_amp, values), cfg)
            np.testing.assert_allclose(r.sum(axis=1), g.E0, rtol=0, atol=1e-10)


def test_mixed_sign_vector_warns():
    """A Hamiltonian with a sign problem: the guide uses |psi_0| and says so."""
    H = P.SpinHalf.create(P.chain(3).edges, J_x=1.0, J_y=1.0, J_z=1.0, dtype=np.float64,
                          sign_check=False)
    with pytest.warns(UserWarning, match="sign"):
        P.ExactGroundState(H, dtype=np.float64)


def test_constructor_validation():
    H = _ring()
    with pytest.raises(ValueError, match="entries"):
        P.ExactGroundState(H, log_amp=np.zeros(10))
    g = P.ExactGroundState(H, log_amp=np.zeros(64))
    assert np.isnan(g.E0) and g.log_amp.dtype == np.float32

    class NoSpace:
        N, M_total = 2, 2
    with pytest.raises(ValueError, match="local_hilbert_space"):
        P.ExactGroundState(NoSpace(), log_amp=np.zeros(4))


def test_save_load_round_trip(tmp_path):
    H = _ring()
    g = P.ExactGroundState(H)
    path = str(tmp_path / "egs.npz")
    g.save(path, note="run 1")
    g2 = P.ExactGroundState.load(path, H)
    np.testing.assert_array_equal(g2.log_amp, g.log_amp)
    assert g2.E0 == g.E0 and g2.local_hilbert_space == g.local_hilbert_space
    x = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])
    np.testing.assert_array_equal(g2.log_diff_from_configs(x), g.log_diff_from_configs(x))
    with np.load(path) as z:
        assert str(z["exact_ground_state/attrs/family"]) == "SpinHalf"
        assert int(z["exact_ground_state/attrs/N"]) == 6
        assert str(z["exact_ground_state/attrs/note"]) == "run 1"
    B = P.BoseHubbard.create(P.chain(6).edges, t=1.0, U=2.0, n_max=1, dtype=np.float64)
    with pytest.raises(ValueError, match="family"):
        P.ExactGroundState.load(path, B)
    with pytest.raises(ValueError, match="N=6"):
        P.ExactGroundState.load(path, _ring(N=8))


class RefShapedExactGuide:
    """The attributes PyGFMC's ExactGroundState stores (exact_ground_state.py:
    72-139), indexed over (-1, 1), with the reference's method names."""

    def __init__(self, log_amp, N):
        self.local_hilbert_space = (-1.0, 1.0)
        self.N = N
        self._powers = tuple(2 ** k for k in range(N - 1, -1, -1))
        self.log_amp = np.asarray(log_amp, np.float32)
        self.E0 = float("nan")
        self.dtype = np.float32
        self.M_total = 0
        self.hamiltonian = None

    def basis_index(self, config):
        return (np.asarray(config) > 0).astype(np.int64) @ np.asarray(self._powers)

    def log_diff_from_configs(self, config, new_configs=None, cache=None):
        raise NotImplementedError


def test_lowering_to_the_c_abi():
    H = _ring(h_x=0.3)
    g = P.ExactGroundState(H, dtype=np.float32)
    keep = _Keep()
    d = guide_desc(g, H, keep)
    assert d.kind == _lib.GUIDE_EXACT_SPIN_HALF == 5 and d.exact_n_sites == 6
    tab = np.ctypeslib.as_array(d.exact_log_amp, shape=(64,))
    np.testing.assert_array_equal(tab, g.log_amp.astype(np.float64))
    # the same amplitudes indexed over (-1, 1) lower to the same table
    g2 = P.ExactGroundState(H, local_hilbert_space=(-1.0, 1.0), dtype=np.float32)
    np.testing.assert_array_equal(exact_amplitude_table(g2), tab)
    ref = RefShapedExactGuide(g2.log_amp, 6)
    np.testing.assert_array_equal(exact_amplitude_table(ref), tab)
    assert guide_desc(ref, H, keep).kind == 5
    P.engine.require_guide_protocol(ref)
    B = P.BoseHubbard.create(P.chain(6).edges, t=1.0, U=2.0, n_max=1, dtype=np.float64)
    with pytest.raises(TypeError, match="SpinHalf"):
        guide_desc(g, B, keep)
    with pytest.raises(ValueError, match="2\\*\\*26"):
        guide_desc(RefShapedExactGuide(np.zeros(4), 27), _ring(N=27), keep)
    with pytest.raises(ValueError, match="sites"):
        guide_desc(g, _ring(N=8), keep)


class _ProtocolOnly:
    """Forwards just the Hamiltonian protocol (the generic matrix build)."""

    def __init__(self, op):
        self.op = op
        self.N, self.M_total, self.local_hilbert_space = op.N, op.M_total, op.local_hilbert_space

    def get_rates(self, config, return_configs=False):
        return self.op.get_rates(config, return_configs=return_configs)

    def generate_state(self, config, idx):
        return self.op.generate_state(config, idx)

    def diagonal_weight(self, config):
        return self.op.diagonal_weight(config)


@pytest.mark.parametrize("case", ["spin_fields", "spin_reversed", "bose", "bose_permuted"])
def test_vectorised_matrix_equals_the_protocol_build(case):
    """This package's operators take a vectorised matrix build; it equals the
    per-configuration build from get_rates: off-diagonal elements exactly, the
    diagonal to rounding (numpy sums diagonal_weight over a batch in another
    order than over one configuration)."""
    rng = np.random.default_rng(11)
    if case.startswith("spin"):
        e = P.chain(8).edges
        jx = -rng.uniform(0.5, 1.5, 8)
        op = P.SpinHalf.create(e, J_x=jx, J_y=jx + rng.uniform(0, 0.2, 8), J_z=rng.uniform(0.5, 1.5, 8),
                               h_z=0.3, h_x=0.2, dtype=np.float64)
        values = (1.0, -1.0) if case == "spin_fields" else (-1.0, 1.0)
    else:
        op = P.BoseHubbard.create(P.chain(4).edges, t=1.0, U=2.0, mu=0.5, h_pm=0.1, eta=0.2, n_max=2,
                                  dtype=np.float64)
        values = (0.0, 1.0, 2.0) if case == "bose" else (2.0, 0.0, 1.0)
    cfg, powers = P.hamiltonian._basis(values, op.N)
    fast = P.hamiltonian._batch_matrix(op, cfg, values, powers).toarray()
    slow = P.hamiltonian._protocol_matrix(_ProtocolOnly(op), cfg, values, powers).toarray()
    off = ~np.eye(len(fast), dtype=bool)
    np.testing.assert_array_equal(fast[off], slow[off])
    np.testing.assert_allclose(np.diag(fast), np.diag(slow), rtol=1e-14, atol=1e-15)
    E_fast, _, _ = P.exact_diagonalization(op, values)
    E_slow, _, _ = P.exact_diagonalization(_ProtocolOnly(op), values)
    np.testing.assert_allclose(E_fast, E_slow, atol=1e-12)


def test_bose_hubbard_exact_guide_on_the_host():
    """The host guide on a Bose-Hubbard chain (exact_ground_state tests:
    85-103, their bose_hubbard case): the guided rates sum to E0 on every
    configuration of the support, over both the default digit order and a
    permuted local space; the device lowering refuses it (spin-1/2 only)."""
    B = P.BoseHubbard.create(P.chain(3).edges, t=1.0, U=2.0, mu=0.5, h_pm=0.1, eta=0.2, n_max=2,
                             dtype=np.float64)
    for values in ((0.0, 1.0, 2.0), (2.0, 0.0, 1.0)):
        g = P.ExactGroundState(B, local_hilbert_space=values, dtype=np.float64)
        cfg = _all(3, values)
        psi = np.exp(g.log_amp[g.basis_index(cfg)])
        support = psi > 1e-10
        assert support.any()
        e = np.array([_host_local_energy(B, g, x) for x in cfg[support]])
        np.testing.assert_allclose(e, g.E0, rtol=0, atol=1e-10)
    with pytest.raises(TypeError, match="SpinHalf"):
        guide_desc(g, B, _Keep())


def test_lowering_refuses_a_non_spin_local_space():
    """A guide indexed over occupations (0, 1) is not a spin-1/2 table: the
    lowering refuses it rather than reading it with the wrong digit order."""
    ref = RefShapedExactGuide(np.zeros(64), 6)
    ref.local_hilbert_space = (0.0, 1.0)
    with pytest.raises(TypeError, match="spin-1/2"):
        exact_amplitude_table(ref)
    with pytest.raises(TypeError, match="spin-1/2"):
        guide_desc(ref, _ring(), _Keep())

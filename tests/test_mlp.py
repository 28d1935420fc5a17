"""MLP guide for Bose-Hubbard occupations (no PyGFMC counterpart): the host
class against the oracle's float64 restatement, the C-ABI lowering, and the
tcgen05 step kernel (float32 with bf16 first-layer activations) against the
oracle's local energies; a guided cont_time run against exact
diagonalisation."""
import functools

import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200 import _lib
from pygfmc_b200.engine import _Keep, guide_desc

BH = dict(t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2)


def _bh(L, n_max, **kw):
    p = dict(BH, **kw)
    return P.BoseHubbard.create(P.chain(L).edges, n_max=n_max, dtype=np.float64, **p)


def _oracle_bh(O, L, n_max, **kw):
    p = dict(BH, **kw)
    return O.bose_hubbard(P.chain(L).edges, n_max=n_max, **p)


def _oracle_mlp(O, G):
    return O.mlp_bose_hubbard(G.W1, G.b1, G.W2, G.b2, G.w3, G.b3, G.n_max)


def _occupations(n, L, n_max, seed):
    return np.random.default_rng(seed).integers(0, n_max + 1, (n, L)).astype(np.float64)


def test_mlp_host_validation_and_rounding():
    G = P.MLPBoseHubbard(6, 2, hidden=(64, 32), seed=1, sigma=0.3, b1=0.1, b2=-0.1, b3=0.5)
    for W in (G.W1, G.W2, G.w3):
        assert np.all((W.view(np.uint32) & 0xFFFF) == 0)
    assert G.W1.shape == (64, 18) and G.W2.shape == (32, 64) and G.w3.shape == (32,)
    x = _occupations(5, 6, 2, 0)
    lp = G.log_psi(x)
    assert lp.shape == (5,) and np.allclose(lp[2], G.log_psi(x[2]))
    for bad in ((64, 8), (96, 32), (64, 272)):
        with pytest.raises(ValueError):
            P.MLPBoseHubbard(6, 2, hidden=bad)
    with pytest.raises(ValueError):
        P.MLPBoseHubbard(6, 2, hidden=(64, 32), W1=np.zeros((64, 17)))


def test_oracle_mlp_rates_match_host(oracle):
    """Guided rates r_x'x = H_x'x psi(x') / psi(x) of the oracle (C, float64)
    equal the host class's log-amplitude differences on the unguided rates."""
    O = oracle
    L, n_max = 6, 2
    m = _oracle_bh(O, L, n_max)
    G = P.MLPBoseHubbard(L, n_max, hidden=(64, 32), seed=3, sigma=0.3, b1=0.05, b2=-0.05, b3=0.2)
    g = _oracle_mlp(O, G)
    cfg = _occupations(8, L, n_max, 4)
    r = O.rates(m, g, cfg)
    r0 = O.rates(m, O.no_guide(), cfg)
    H = _bh(L, n_max)
    for w in range(len(cfg)):
        x = cfg[w]
        nz = np.flatnonzero(r0[w][1:] != 0)
        succ = _successors(H, x)[nz]
        ld = G.log_psi(succ) - G.log_psi(x)
        np.testing.assert_allclose(r[w][1:][nz], r0[w][1:][nz] * np.exp(ld), rtol=1e-12, atol=1e-15)
        assert np.all(r[w][1:][r0[w][1:] == 0] == 0)
        assert r[w][0] == r0[w][0]


def _successors(H, x):
    """Configurations after each off-diagonal move of the BoseHubbard layout
    (hop forward/backward, pair up/down per edge, b+ / b- per site),
    whatever their rate."""
    ei, ej = np.asarray(H.edge_i), np.asarray(H.edge_j)
    out = []
    if H.n_hop_off:
        for da, db in ((-1, 1), (1, -1)):
            for a, b in zip(ei, ej):
                y = x.copy(); y[a] += da; y[b] += db; out.append(y)
    if H.n_eta_off:
        for da, db in ((1, 1), (-1, -1)):
            for a, b in zip(ei, ej):
                y = x.copy(); y[a] += da; y[b] += db; out.append(y)
    if H.n_hpm_off:
        for d in (1, -1):
            for k in range(len(x)):
                y = x.copy(); y[k] += d; out.append(y)
    return np.clip(np.asarray(out), 0, H.n_max)


def test_mlp_lowering():
    L, n_max = 8, 3
    G = P.MLPBoseHubbard(L, n_max, hidden=(128, 48), seed=2, b3=-0.25)
    keep = _Keep()
    g = guide_desc(G, _bh(L, n_max), keep)
    assert g.kind == _lib.GUIDE_MLP_BOSE_HUBBARD and (g.mlp_H1, g.mlp_H2) == (128, 48)
    assert g.mlp_W1[0] == G.W1[0, 0] and g.mlp_W2[47 * 128 + 5] == G.W2[47, 5]
    assert g.mlp_b3 == pytest.approx(-0.25)
    with pytest.raises(TypeError):
        guide_desc(G, P.SpinHalf.create(P.chain(L).edges, J_x=-1.0, J_y=-1.0, J_z=1.0), keep)
    with pytest.raises(ValueError):
        guide_desc(G, _bh(L, 2), keep)


def _ed_hamiltonian(L, n_max, t, eta, U, mu, h_pm):
    """The truncated Bose-Hubbard chain (periodic) as a dense matrix,
    H = -t sum (b_i+ b_j + h.c.) - eta sum (b_i+ b_j+ + h.c.)
        - h_pm sum (b_k + b_k+) + U/2 sum n (n - 1) - mu sum n,
    built from Kronecker products of the single-site operators (site 0 the
    most significant digit of the basis index)."""
    d = n_max + 1
    b = np.diag(np.sqrt(np.arange(1, d, dtype=np.float64)), 1)
    n = b.T @ b

    def site(op, k):
        out = np.ones((1, 1))
        for j in range(L):
            out = np.kron(out, op if j == k else np.eye(d))
        return out

    B = [site(b, k) for k in range(L)]
    Nk = [site(n, k) for k in range(L)]
    one = np.eye(d ** L)
    H = np.zeros((d ** L, d ** L))
    for i in range(L):
        j = (i + 1) % L
        H -= t * (B[i].T @ B[j] + B[j].T @ B[i])
        H -= eta * (B[i].T @ B[j].T + B[i] @ B[j])
    for k in range(L):
        H -= h_pm * (B[k] + B[k].T)
        H += 0.5 * U * Nk[k] @ (Nk[k] - one) - mu * Nk[k]
    return H


@functools.lru_cache(maxsize=None)
def _exact_ground_energy(L, n_max, t, eta, U, mu, h_pm):
    return float(np.linalg.eigvalsh(_ed_hamiltonian(L, n_max, t, eta, U, mu, h_pm))[0])


def test_exact_diagonalisation_matches_the_oracle_rates(oracle):
    """The ED Hamiltonian and the oracle's transition layout describe the same
    operator: the oracle's rates reproduce H psi for a random vector."""
    O = oracle
    L, n_max = 4, 2
    m = _oracle_bh(O, L, n_max)
    H = _bh(L, n_max)
    d = n_max + 1
    states = np.array(np.unravel_index(np.arange(d ** L), (d,) * L)).T.astype(np.float64)
    psi = np.random.default_rng(0).normal(size=d ** L)
    index = {tuple(s): i for i, s in enumerate(states)}
    r0 = O.rates(m, O.no_guide(), states)
    Hpsi = np.zeros(d ** L)
    for i, x in enumerate(states):
        succ = _successors(H, x)
        Hpsi[i] = r0[i][0] * psi[i] + sum(v * psi[index[tuple(y)]] for v, y in zip(r0[i][1:], succ)
                                            if v != 0)
    np.testing.assert_allclose(Hpsi, _ed_hamiltonian(L, n_max, **BH) @ psi, rtol=1e-12, atol=1e-12)


# ---- device ---------------------------------------------------------------

def _mlp_systems(O):
    out = []
    for (L, n_max, hidden, sigma, n) in ((6, 2, (64, 32), 0.3, 300), (16, 3, (256, 256), 0.1, 200),
                                          (32, 4, (192, 48), 0.08, 150), (64, 2, (128, 128), 0.05, 160)):
        H = _bh(L, n_max)
        m = _oracle_bh(O, L, n_max)
        rng = np.random.default_rng(L)
        G = P.MLPBoseHubbard(L, n_max, hidden=hidden, seed=L, sigma=sigma,
                             b1=rng.normal(0, 0.1, hidden[0]), b2=rng.normal(0, 0.1, hidden[1]),
                             b3=0.3)
        out.append((f"L{L}_nmax{n_max}_h{hidden[0]}x{hidden[1]}", H, G, m, _oracle_mlp(O, G),
                    _occupations(n, L, n_max, 7 * L)))
    return out


@pytest.mark.gpu
def test_mlp_local_energy_matches_oracle(oracle):
    """e_L through gfmc_local_energy (tcgen05 second layer over the 128-move
    tiles) against the float64 oracle, relative to the rate scale sum |r| per
    walker.  The first layer's tanh is the hardware approximation (relative
    error up to 2^-11) and its output is rounded to bf16 (step 2^-8), so about
    one activation in eight near a rounding boundary lands one bf16 unit away
    from the oracle's: most walkers carry a few such units.  Measured on these
    systems: median 5e-7 .. 7e-6, at most 10 % of walkers above 1e-4, maximum
    1.5e-3.  Asserted: median 3e-5, at most 30 % above 1e-4, 1e-4 on average,
    every walker within 2e-3."""
    O = oracle
    P._lib.load()
    for name, H, G, m, g, cfg in _mlp_systems(O):
        r = O.rates(m, g, cfg)
        ref = r.sum(axis=1)
        scale = np.abs(r).sum(axis=1)
        eng = P.GFMCEngine(H, G, cfg.shape[0], precision="mixed")
        eng.load(cfg)
        el = eng.local_energy().cpu().numpy()
        err = np.abs(el - ref) / scale
        assert np.all(err <= 2e-3), (name, err.max())
        assert err.mean() <= 1e-4, (name, err.mean())
        assert np.median(err) <= 3e-5, (name, np.median(err))
        assert (err > 1e-4).mean() <= 0.3, (name, (err > 1e-4).mean())
        assert eng.status() == 0, name


@pytest.mark.gpu
def test_mlp_carried_state_matches_the_oracle(oracle):
    """60 cont_time steps with z1 and log psi carried through the parent maps
    (rebuilt every 50 steps): the local energies the last step wrote for its
    configurations agree with the oracle's fresh evaluation of them."""
    import ctypes
    import torch
    O = oracle
    P._lib.load()
    name, H, G, m, g, cfg = _mlp_systems(O)[1]
    n = cfg.shape[0]
    eng = P.GFMCEngine(H, G, n, precision="mixed")
    eng.load(cfg)
    keys, _ = P.engine.key_schedule(P.PRNGKey(5), 60)
    lg = torch.empty(60, dtype=torch.float64, device=eng.device)
    alw = float((-eng.local_energy()).mean().item())
    eng.steps("cont_time", 0.1, None, alw, keys, lg, torch.empty_like(lg))
    out = torch.empty((n, eng.N), dtype=torch.float64, device=eng.device)
    eng.L.gfmc_unpack(eng.h, n, ctypes.c_void_p(eng.cfg.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                      eng._stream())
    c = out.cpu().numpy()
    r = O.rates(m, g, c)
    err = np.abs(eng.e_loc.cpu().numpy() - r.sum(axis=1)) / np.abs(r).sum(axis=1)
    assert np.all(err <= 2e-3) and err.mean() <= 1e-4, (err.max(), err.mean())
    assert eng.status() == 0


@pytest.mark.gpu
def test_mlp_requires_the_float32_build_and_cont_time():
    P._lib.load()
    H = _bh(6, 2)
    G = P.MLPBoseHubbard(6, 2, hidden=(64, 32))
    with pytest.raises(P._lib.GFMCError, match="float32"):
        P.GFMCEngine(H, G, 16, precision="fp64")
    eng = P.GFMCEngine(H, G, 16, precision="mixed")
    eng.load(_occupations(16, 6, 2, 1))
    import torch
    keys, _ = P.engine.key_schedule(P.PRNGKey(1), 1)
    lg = torch.empty(1, dtype=torch.float64, device=eng.device)
    with pytest.raises(P._lib.GFMCError, match="cont_time"):
        eng.steps("single_step", 2, 10.0, 0.0, keys, lg, torch.empty_like(lg))


@pytest.mark.gpu
def test_mlp_guided_run_matches_exact_energy():
    """A float32 MLP-guided cont_time run of the 6-site Bose-Hubbard chain
    (hopping, pair terms, h_pm; n_max = 2) gives the exact ground-state
    energy within its error bar."""
    L, n_max = 6, 2
    H = _bh(L, n_max)
    G = P.MLPBoseHubbard(L, n_max, hidden=(64, 32), seed=5, sigma=0.1)
    w = P.prepare_walkers_random(2048, L, P.PRNGKey(0), states=(0.0, 1.0, 2.0))
    _, E, _, st, raw = P.run(w, 1500, H, 0.1, G, [8, 32], rng_key=P.PRNGKey(1), warmup_steps=200,
                             verbosity=0)
    Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 15)
    E0 = _exact_ground_energy(L, n_max, **BH)
    assert abs(Ej[32] - E0) < max(3e-3 * abs(E0), 4 * err[32]), (Ej[32], err[32], E0)


# ---- trainer ----------------------------------------------------------------

def test_mlp_oracle_gradient_matches_finite_differences():
    """The float64 autograd statement of the variance loss (without the bf16
    rounding of h1, which makes the loss piecewise constant in W1, b1)."""
    from oracle import learned
    H = _bh(6, 2)
    G = P.MLPBoseHubbard(6, 2, hidden=(64, 64), seed=3, sigma=0.3, b1=0.05, b2=-0.05, b3=0.2)
    x = _occupations(10, 6, 2, 1)
    base = {"W1": G.W1, "b1": G.b1, "W2": G.W2, "b2": G.b2, "w3": G.w3}
    base = {k: np.asarray(v, np.float64) for k, v in base.items()}
    order = ("W1", "b1", "W2", "b2", "w3")
    _, _, g = learned.mlp_variance_loss_and_grads(H, *[base[k] for k in order], G.b3, x,
                                                  round_h1=False)
    eps = 1e-6
    for name, idx in (("W1", (1, 5)), ("W1", (7, 0)), ("b1", (4,)), ("W2", (2, 7)), ("b2", (5,)),
                      ("w3", (3,))):
        p = {k: v.copy() for k, v in base.items()}
        q = {k: v.copy() for k, v in base.items()}
        p[name][idx] += eps
        q[name][idx] -= eps
        Lp = learned.mlp_variance_loss_and_grads(H, *[p[k] for k in order], G.b3, x, round_h1=False)[1]
        Lq = learned.mlp_variance_loss_and_grads(H, *[q[k] for k in order], G.b3, x, round_h1=False)[1]
        fd = (Lp - Lq) / (2 * eps)
        assert abs(fd - g[name][idx]) < 1e-6 * max(1.0, abs(fd)), (name, idx, fd, g[name][idx])


def _trainer_systems():
    out = []
    for (L, n_max, hidden, sigma, n, kw) in ((6, 2, (64, 64), 0.2, 96, {}),
                                             (16, 3, (128, 128), 0.1, 128, {"eta": 0.0}),
                                             (64, 4, (256, 256), 0.05, 48, {"eta": 0.0, "h_pm": None,
                                                                            "mu": 0.0, "U": 3.0})):
        H = _bh(L, n_max, **kw)
        rng = np.random.default_rng(L + 1)
        G = P.MLPBoseHubbard(L, n_max, hidden=hidden, seed=L, sigma=sigma,
                             b1=rng.normal(0, 0.1, hidden[0]), b2=rng.normal(0, 0.1, hidden[1]))
        x = _occupations(n, L, n_max, 3 * L)
        out.append((f"L{L}_h{hidden[0]}", H, G, x))
    return out


@pytest.mark.gpu
def test_mlp_device_gradient_matches_oracle():
    """gfmc_mlp_gradient (second layer forward, its backward and dW2 on the
    tensor cores, one-hot first layer accumulated) against float64 autograd
    with the same straight-through bf16 rounding: E and L to float32
    accuracy, each gradient block to 3e-2 in relative norm."""
    from oracle import learned
    P._lib.load()
    for name, H, G, x in _trainer_systems():
        eng = P.GFMCEngine(H, G, x.shape[0], precision="mixed")
        eng.load(x)
        grads, (E, L) = eng.mlp_gradient()
        rE, rL, rg = learned.mlp_variance_loss_and_grads(H, G.W1, G.b1, G.W2, G.b2, G.w3, G.b3, x)
        assert abs(E - rE) < 1e-4 * abs(rE) + 1e-6 and abs(L - rL) < 3e-3 * rL + 1e-6, (name, E, rE, L, rL)
        for k, ref in rg.items():
            got = grads[k].cpu().numpy().astype(np.float64)
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err < 3e-2, (name, k, err)
        assert eng.status() == 0, name


@pytest.mark.gpu
def test_mlp_training_lowers_variance_and_keeps_the_exact_energy():
    """6-site Bose-Hubbard chain: training on GFMC walkers lowers the
    local-energy variance well below the untrained guide's, and a production
    run with the trained guide gives the exact ground-state energy within its
    error bar."""
    P._lib.load()
    L, n_max = 6, 2
    H = _bh(L, n_max)
    G0 = P.MLPBoseHubbard(L, n_max, hidden=(64, 64), seed=0, sigma=0.01)
    w = P.prepare_walkers_random(1024, L, P.PRNGKey(0), states=(0.0, 1.0, 2.0))
    trained, hist = P.learn.train_mlp_guide(w, H, G0, n_iterations=150, steps_per_iteration=4,
                                            step_size=0.1, lr=3e-3, rng_key=P.PRNGKey(1),
                                            warmup_steps=50, verbosity=0)
    v0, v1 = hist["variance"][:5].mean(), hist["variance"][-10:].mean()
    assert not hist["collapsed"]
    assert v1 < 0.5 * v0, (v0, v1)
    _, E, _, st, raw = P.run(P.prepare_walkers_random(2048, L, P.PRNGKey(5), states=(0.0, 1.0, 2.0)),
                             1500, H, 0.1, trained, [8, 32], rng_key=P.PRNGKey(6), warmup_steps=200,
                             verbosity=0)
    Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 15)
    E0 = _exact_ground_energy(L, n_max, **BH)
    assert abs(Ej[32] - E0) < max(4 * err[32], 3e-3 * abs(E0)), (Ej[32], err[32], E0)

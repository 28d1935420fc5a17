"""The oracle is pinned on PyGFMC's own golden runs (float64, jax 0.9.2):
key chains, walker initialisers, and whole 300-step trajectories."""
import numpy as np
import pytest

from golden_cases import CASES, method_of, oracle_off_ops, oracle_system


def test_threefry_key_chain_kats(golden, oracle):
    """rng_key -> rng_key_next after n_steps splits, for every golden case."""
    names = sorted({k.split("/")[0] for k in golden.files if k.endswith("stats/parameters/rng_key")})
    assert len(names) >= 40
    for name in names:
        key = golden[f"{name}/stats/parameters/rng_key"]
        nxt = golden[f"{name}/stats/parameters/rng_key_next"]
        n = int(golden[f"{name}/stats/parameters/n_steps"])
        k = key.copy()
        for _ in range(n):
            k = oracle.split(k, 2)[0]
        assert np.array_equal(k, nxt), name
        assert np.array_equal(key, oracle.case_key(name)), name


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden_run(golden, oracle, name):
    m, cfg, g, dt, lam = oracle_system(oracle, name)
    method = method_of(name)
    step = dt if method == "cont_time" else 2
    r = oracle.run(cfg, 300, m, step, g, [2, 4], method=method, rng_key=oracle.case_key(name),
                   lam=None if method == "cont_time" else lam, warmup_steps=8)
    p = name + "/"
    assert np.array_equal(r.config, golden[p + "config"].astype(np.float64))
    np.testing.assert_allclose(r.log_weights, golden[p + "raw/log_weights"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r.energy_series, golden[p + "raw/energy"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r.e_loc, golden[p + "e_loc"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(r.alw, golden[p + "stats/avg_log_weight"], rtol=1e-10, atol=1e-12)
    for pp in (2, 4):
        np.testing.assert_allclose(r.energy[pp], golden[p + f"energy/{pp}"], rtol=1e-10, atol=1e-12)
    assert np.array_equal(r.rng_key_next, golden[p + "stats/parameters/rng_key_next"])


@pytest.mark.parametrize("name", [c for c in CASES if c.endswith(("cont_time", "single_step"))]
                         + ["bose_jastrow_multi_step"])
def test_oracle_off_diagonal_forward_walk_golden(golden, oracle, name):
    """Forward-walking rows of every off-diagonal operator (operator applied
    after each step's reconfiguration, shadow chain on the main chain's future
    keys) against raw['off_diag'] / raw['off_diag_norm'] of the golden run."""
    m, cfg, g, dt, lam = oracle_system(oracle, name)
    method = method_of(name)
    step = dt if method == "cont_time" else 2
    ops = oracle_off_ops(oracle, name)
    r = oracle.run(cfg, 300, m, step, g, [2, 4], method=method, rng_key=oracle.case_key(name),
                   lam=None if method == "cont_time" else lam, warmup_steps=8,
                   off_diag_operators=ops)
    p = name + "/"
    for nm, _, _ in ops:
        np.testing.assert_allclose(r.off_diag[nm], golden[p + f"raw/off_diag/{nm}"],
                                   rtol=1e-10, atol=1e-12, err_msg=nm)
        np.testing.assert_allclose(r.off_diag_norm[nm], golden[p + f"raw/off_diag_norm/{nm}"],
                                   rtol=1e-10, atol=1e-12, err_msg=nm)
        # the pure estimate, windows restricted to i >= max(m) as with the
        # diagonal operators of the same call
        est = oracle.off_diagonal_estimates([2, 4], r.m_array, r.log_weights, r.off_diag[nm],
                                            r.off_diag_norm[nm], np.arange(300), max(r.m_array))
        for pp in (2, 4):
            np.testing.assert_allclose(est[pp], golden[p + f"obs/{nm}/{pp}"], rtol=1e-10, atol=1e-12)


def test_sample_index_edge_cases(oracle):
    """PyGFMC tests/core/test_sampler.py:20-47 restated: a zero-weight slot is
    never drawn (noisy cdf across it), trailing zeros are unreachable, and
    draws are proportional."""
    w = np.array([1.0, 0.0, 1.0]); noisy = np.array([1.0, 1.5, 2.0])
    idx = [oracle.sample_index(noisy, w, u) for u in np.linspace(0, 1, 4097)[:-1]]
    assert set(idx) <= {0, 2} and np.mean(np.array(idx) == 0) > 0.6
    w = np.array([0.0, 2.0, 0.0, 0.0]); cdf = np.array([0.0, 2.0, 2.0000002, 2.0000005])
    assert {oracle.sample_index(cdf, w, u) for u in np.linspace(0, 1, 4097)[:-1]} == {1}
    w = np.array([1.0, 0.0, 3.0])
    idx = np.array([oracle.sample_index(np.cumsum(w), w, u) for u in (np.arange(20000) + 0.5) / 20000])
    assert set(np.unique(idx)) <= {0, 2} and abs(np.mean(idx == 2) - 0.75) < 0.02
    # u rounding up to the total must stay inside the array
    assert oracle.sample_index(np.array([1.0, 2.0]), np.array([1.0, 1.0]), 1.0 - 1e-17) == 1


def test_reconfiguration_invariants(oracle):
    """Systematic resampling: parents non-decreasing, zero weights never
    chosen, offspring counts within floor/ceil of N w_i."""
    rng = np.random.default_rng(3)
    n = 257
    lw = rng.normal(size=n)
    lw[[5, 17, 200]] = -np.inf
    cfg = np.arange(n, dtype=np.float64)[:, None] * np.ones((1, 3))
    el = rng.normal(size=n)
    par, lG, En = oracle.reconfigure(np.array([1, 2], np.uint32), cfg.copy(), lw.copy(), el.copy())
    assert np.all(np.diff(par) >= 0)
    assert not set(par.tolist()) & {5, 17, 200}
    w = np.exp(lw - lw[np.isfinite(lw)].max()); w /= w.sum()
    counts = np.bincount(par, minlength=n)
    assert np.all(counts >= np.floor(n * w) - 1) and np.all(counts <= np.ceil(n * w) + 1)
    assert np.isclose(En, np.sum(w * el))

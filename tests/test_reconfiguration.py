"""walkers.reconfiguration, the standalone systematic resampling of PyGFMC's
walkers/reconfiguration.py:27-62 on the device: its argument checks (host,
before any device work), and on the GPU the parents, log G - log N and E_n
against the oracle's restatement on the same weights and key (identical
parents, scalars to 1e-12) from one walker to the 131072 limit, the dead-walker
pins of PyGFMC's tests/core/test_walker_io.py:61-76, and the dtypes of the
returned population."""
import os
import re

import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.walkers import RECONFIGURATION_MAX_WALKERS, Walker, reconfiguration

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _population(n, N, seed, spread=3.0, dead=0.0, dtype=np.float64):
    rng = np.random.default_rng(seed)
    lw = rng.normal(0.0, spread, n)
    if dead:
        lw[rng.random(n) < dead] = -np.inf
    return Walker(config=rng.choice([1.0, -1.0], size=(n, N)).astype(dtype),
                  log_weight=lw.astype(dtype), e_loc=rng.normal(-0.4, 0.2, n).astype(dtype))


def test_limit_is_the_header_limit():
    with open(os.path.join(ROOT, "include", "gfmc_b200.h")) as f:
        m = re.search(r"#define\s+GFMC_NOALLOC_MAX_WALKERS\s+(\d+)", f.read())
    assert m and int(m.group(1)) == RECONFIGURATION_MAX_WALKERS
    assert "reconfiguration" in P.walkers.__all__


def test_arguments_are_checked_before_any_device_work():
    w = _population(8, 4, 0)
    key = P.PRNGKey(0)
    with pytest.raises(ValueError, match="shape"):
        reconfiguration(w._replace(e_loc=w.e_loc[:5]), key)
    with pytest.raises(ValueError, match="shape"):
        reconfiguration(w._replace(config=w.config[:7]), key)
    with pytest.raises(ValueError, match="shape"):
        reconfiguration(w._replace(log_weight=w.log_weight[:, None]), key)
    with pytest.raises(ValueError, match="at least one walker"):
        reconfiguration(Walker(np.zeros((0, 4)), np.zeros(0), np.zeros(0)), key)
    big = RECONFIGURATION_MAX_WALKERS + 1
    with pytest.raises(ValueError, match="at most 131072"):
        reconfiguration(Walker(np.zeros((big, 1)), np.zeros(big), np.zeros(big)), key)


def test_fails_loudly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(P._lib.GFMCError, match="no CPU fallback"):
        reconfiguration(_population(8, 4, 0), P.PRNGKey(0))


@pytest.mark.gpu
@pytest.mark.parametrize("n,N,dead", [(1, 3, 0.0), (7, 5, 0.0), (1000, 16, 0.3), (3001, 33, 0.0),
                                      (131072, 8, 0.1)])
def test_matches_the_oracle(oracle, n, N, dead):
    w = _population(n, N, n + N, dead=dead)
    for seed in (1, 2):
        key = P.PRNGKey(seed)
        new, lg, E, idx = reconfiguration(w, key)
        par, lG, En = oracle.reconfigure(key, np.array(w.config, dtype=np.float64),
                                         np.array(w.log_weight), np.array(w.e_loc))
        np.testing.assert_array_equal(idx, par)
        np.testing.assert_allclose(lg, lG, rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(E, En, rtol=1e-12, atol=1e-13)
        np.testing.assert_array_equal(new.config, w.config[par])
        np.testing.assert_array_equal(new.e_loc, w.e_loc[par])
        assert np.all(new.log_weight == 0.0) and new.log_weight.dtype == w.log_weight.dtype
        assert np.all(np.isfinite(w.log_weight[idx]))          # no dead walker is a parent
        assert np.all(np.diff(idx) >= 0)                       # systematic parents are sorted


@pytest.mark.gpu
def test_dead_walkers_are_never_parents():
    """A -inf log weight is a walker of zero weight: with weights (0, 1, 0)
    every new walker descends from walker 1, for every offset
    (tests/core/test_walker_io.py:71-76); leading and trailing dead walkers
    are skipped at either end of the cumulative sum."""
    w = Walker(config=np.array([[1.0], [-1.0], [1.0]]), log_weight=np.array([-np.inf, 0.0, -np.inf]),
               e_loc=np.zeros(3))
    for seed in range(20):
        _, lg, _, idx = reconfiguration(w, P.PRNGKey(seed))
        assert idx.tolist() == [1, 1, 1]
        assert lg == pytest.approx(-np.log(3.0), abs=1e-15)
    lw = np.array([-np.inf, -np.inf, 0.0, 0.3, -0.2, -np.inf, -np.inf])
    w = Walker(config=np.arange(7.0)[:, None], log_weight=lw, e_loc=np.arange(7.0))
    for seed in range(20):
        new, _, E, idx = reconfiguration(w, P.PRNGKey(seed))
        assert set(idx.tolist()) <= {2, 3, 4}
        wts = np.exp(lw - lw[np.isfinite(lw)].max())
        assert E == pytest.approx(float((wts * w.e_loc).sum() / wts.sum()), rel=1e-14)
        np.testing.assert_array_equal(new.config[:, 0], idx.astype(np.float64))


@pytest.mark.gpu
def test_float32_walkers_and_compact_configs(oracle):
    """Float32 weights are resampled with the float64 cumulative sum of their
    values (the precision rule of the engine's resampling); the returned
    population keeps the input's dtypes, int8 configurations included."""
    w = _population(2500, 12, 9, dtype=np.float32)
    w = w._replace(config=w.config.astype(np.int8))
    new, lg, E, idx = reconfiguration(w, P.PRNGKey(4))
    par, lG, En = oracle.reconfigure(P.PRNGKey(4), w.config.astype(np.float64),
                                     w.log_weight.astype(np.float64), w.e_loc.astype(np.float64))
    np.testing.assert_array_equal(idx, par)
    np.testing.assert_allclose([lg, E], [lG, En], rtol=1e-12, atol=1e-13)
    assert new.config.dtype == np.int8 and new.log_weight.dtype == np.float32
    assert new.e_loc.dtype == np.float32

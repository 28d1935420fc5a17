"""Walker initialisers and checkpoints against the contracts of PyGFMC's own
tests (tests/core/test_walker_init.py:19-100 and
tests/core/test_walker_checkpoint_dtypes.py:23-60): the random and
fixed-sum initialisers draw only from the given local values and hit the
requested sum exactly for every walker or refuse; configuration dtypes follow
the values; checkpoints store integer-valued configurations as int8 and any
other encoding as given, and load back exactly.  Host only."""
import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.walkers import (Walker, prepare_walkers_from_configs, prepare_walkers_random,
                                 prepare_walkers_sz)

LADDERS = [(-1, 1), (-0.5, 0.5), (-1, 0, 1), (0, 1, 2)]


def test_random_walkers_are_independent_coin_flips():
    w = prepare_walkers_random(256, 12, P.PRNGKey(3))
    assert w.config.shape == (256, 12)
    assert set(np.unique(w.config).tolist()) == {-1.0, 1.0}
    assert np.std(w.config.sum(axis=1)) > 0.5          # the magnetisation varies
    assert np.all(w.log_weight == 0.0) and np.all(w.e_loc == 0.0)


@pytest.mark.parametrize("states", LADDERS)
def test_random_walkers_use_every_value_and_no_other(states):
    w = prepare_walkers_random(512, 10, P.PRNGKey(7), states=states)
    seen = set(np.unique(w.config).tolist())
    assert seen == {float(v) for v in states}


@pytest.mark.parametrize("states,sz", [((-1, 1), 4), ((-1, 1), 0), ((-0.5, 0.5), 2.0),
                                       ((-0.5, 0.5), -3.0), ((-1, 0, 1), 3), ((-1, 0, 1), -7),
                                       ((0, 1, 2), 10), ((0, 1, 2), 0)])
def test_fixed_sum_walkers_hit_the_sum_exactly(states, sz):
    w = prepare_walkers_sz(128, 10, P.PRNGKey(11), sz=sz, states=states)
    assert w.config.shape == (128, 10)
    assert set(np.unique(w.config).tolist()) <= {float(v) for v in states}
    np.testing.assert_allclose(w.config.sum(axis=1), sz, rtol=0, atol=1e-12)


@pytest.mark.parametrize("states,sz", [((-1, 1), 3), ((-1, 1), 99), ((0, 1, 2), -1),
                                       ((-0.5, 0.5), 0.25)])
def test_unreachable_sums_are_refused(states, sz):
    """Parity, above and below the range, off the half-integer ladder."""
    with pytest.raises(ValueError):
        prepare_walkers_sz(4, 10, P.PRNGKey(13), sz=sz, states=states)


@pytest.mark.parametrize("init", ["random", "sz"])
def test_configuration_dtype_follows_the_values(init):
    for states, kind in (((-1, 0, 1), "i"), ((-0.5, 0.5), "f")):
        if init == "random":
            w = prepare_walkers_random(16, 8, P.PRNGKey(17), states=states)
        else:
            w = prepare_walkers_sz(16, 8, P.PRNGKey(17), sz=2 if kind == "i" else 1.0, states=states)
        assert w.config.dtype.kind == kind, (states, w.config.dtype)
        assert w.log_weight.dtype.kind == "f" and w.e_loc.dtype.kind == "f"
        assert set(np.unique(w.config).tolist()) <= set(states)


def test_given_configurations_are_kept():
    cfg = np.random.default_rng(0).choice([-1, 1], size=(64, 10)).astype(np.int8)
    w = prepare_walkers_from_configs(cfg)
    assert w.config.dtype == np.int8
    np.testing.assert_array_equal(w.config, cfg)
    assert w.log_weight.shape == w.e_loc.shape == (64,)
    assert np.all(w.log_weight == 0.0) and np.all(w.e_loc == 0.0)
    for shape in ((10,), (4, 5, 2)):
        with pytest.raises(ValueError, match="N_walkers, N_sites"):
            prepare_walkers_from_configs(np.ones(shape))


@pytest.mark.parametrize("states,sz,stored", [((-1.0, 1.0), 0, np.int8), ((-1.0, 0.0, 1.0), 1, np.int8),
                                              ((0.0, 1.0, 2.0), 8, np.int8),
                                              ((-0.5, 0.5), 1.0, np.float64),
                                              ((-1.5, -0.5, 0.5, 1.5), 2.0, np.float64)])
def test_checkpoint_compacts_only_when_lossless(tmp_path, states, sz, stored):
    """Integer-valued configurations are stored as int8, half-integer ones as
    given; everything loads back exactly, with the key and the attributes."""
    w0 = prepare_walkers_sz(32, 8, P.PRNGKey(0), sz=sz, states=states)
    w = Walker(config=w0.config, log_weight=np.linspace(-1, 1, 32), e_loc=np.arange(32.0))
    path = str(tmp_path / "w.npz")
    key = P.PRNGKey(7)
    w.save(path, rng_key=key, avg_log_weight=0.25, note="x")
    with np.load(path) as z:
        assert z["walkers/config"].dtype == stored
        assert float(z["walkers/attrs/avg_log_weight"]) == 0.25
        assert str(z["walkers/attrs/note"]) == "x"
    loaded, key2, alw = Walker.load(path)
    np.testing.assert_array_equal(loaded.config, w.config)
    np.testing.assert_array_equal(loaded.log_weight, w.log_weight)
    np.testing.assert_array_equal(loaded.e_loc, w.e_loc)
    np.testing.assert_array_equal(key2, key)
    assert float(alw) == 0.25


def test_checkpoint_without_key_or_shift(tmp_path):
    w = prepare_walkers_sz(8, 6, P.PRNGKey(1), sz=0)
    path = str(tmp_path / "w.npz")
    w.save(path)
    loaded, key, alw = Walker.load(path)
    assert key is None and alw is None
    assert loaded.log_weight.dtype == np.float64 == loaded.config.dtype   # the x64 default
    narrow, _, _ = Walker.load(path, dtype=np.float32, config_dtype=np.int8)
    assert narrow.log_weight.dtype == np.float32 and narrow.config.dtype == np.int8
    np.testing.assert_array_equal(narrow.config, w.config.astype(np.int8))

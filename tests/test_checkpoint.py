"""Checkpoint and resume: Walker.save / Walker.load (walkers/walker.py:66-140)
and a chain continued from a checkpoint with the returned key and average
log weight.  As PyGFMC's tests/core/test_io_hdf5.py _walk_in_pieces:407
checks, a run walked in pieces through checkpoints equals the contiguous run:
bit for bit without a guide (no state is carried between steps beyond the
walkers); with a guide whose state the engine carries between steps, the
continuation rebuilds that state, so the pieces agree with the contiguous
run in their configurations exactly and in their series to 1e-12."""
import os

import numpy as np
import pytest

import pygfmc_b200 as P


def test_walker_checkpoint_round_trip(tmp_path):
    w = P.prepare_walkers_sz(50, 12, P.PRNGKey(0), sz=0)
    w = P.Walker(w.config, np.linspace(-1, 1, 50), np.linspace(-5, -4, 50))
    path = str(tmp_path / "ck.h5")
    w.save(path, rng_key=P.PRNGKey(7), avg_log_weight=1.5, steps_done=300)
    assert os.path.exists(path)
    with np.load(path) as z:
        assert z["walkers/config"].dtype == np.int8          # +-1 stored compactly
        assert int(z["walkers/attrs/steps_done"]) == 300
    w2, key, alw = P.Walker.load(path)
    assert w2.config.dtype == np.float64 and np.array_equal(w2.config, w.config)
    assert np.array_equal(w2.log_weight, w.log_weight) and np.array_equal(w2.e_loc, w.e_loc)
    assert np.array_equal(key, P.PRNGKey(7)) and alw == 1.5
    # occupations, another group, float32 weights, no key or average
    occ = P.prepare_walkers_occupations(20, 10, 10, 4, P.PRNGKey(1))
    occ.save(path, group="bosons")
    w3, key3, alw3 = P.Walker.load(path, group="bosons", dtype=np.float32)
    assert key3 is None and alw3 is None
    assert w3.log_weight.dtype == np.float32 and np.array_equal(w3.config, occ.config)
    # values that are not small integers stay as they are
    half = P.Walker(np.full((3, 4), 0.5), np.zeros(3), np.zeros(3))
    half.save(path)
    with np.load(path) as z:
        assert z["walkers/config"].dtype == np.float64
    with pytest.raises(KeyError):
        P.Walker.load(path, group="absent")
    with pytest.raises(ValueError):
        w.save(path, avg_log_weight=np.zeros(2))


def _walk_in_pieces(tmp_path, pieces, H, G, method, step, lam, w0, tag):
    """sum(pieces) production steps as len(pieces) runs, each continued from
    the checkpoint of the one before (walkers, rng_key_next,
    avg_log_weight; warmup_steps=0)."""
    path = str(tmp_path / f"{tag}.npz")
    lw, E = [], []
    w, key, alw = w0, P.PRNGKey(7), 0.7 if method == "cont_time" else 3.4
    for n in pieces:
        w, _, _, st, raw = P.run(w, n, H, step, G, [4], method=method, lam=lam, rng_key=key,
                                 warmup_steps=0, avg_log_weight=alw, verbosity=0)
        lw.append(raw["log_weights"])
        E.append(raw["energy"])
        w.save(path, rng_key=st["parameters/rng_key_next"], avg_log_weight=st["avg_log_weight"])
        w, key, alw = P.Walker.load(path)
    return w, np.concatenate(lw), np.concatenate(E)


@pytest.mark.gpu
@pytest.mark.parametrize("method,step,lam", [("cont_time", 0.1, None), ("single_step", 2, 9.0)])
@pytest.mark.parametrize("guided", [False, True])
def test_split_run_matches_contiguous(tmp_path, method, step, lam, guided):
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.3, dtype=np.float64)
    G = P.JastrowSpinHalf(16, e, beta=0.3) if guided else None
    w0 = P.prepare_walkers_sz(256, 16, P.PRNGKey(2), sz=0)
    runs = {name: _walk_in_pieces(tmp_path, pieces, H, G, method, step, lam, w0, name)
            for name, pieces in (("contiguous", [120]), ("four_equal", [30, 30, 30, 30]),
                                 ("three_unequal", [20, 70, 30]))}
    wr, lwr, Er = runs["contiguous"]
    for name in ("four_equal", "three_unequal"):
        w, lw, E = runs[name]
        assert np.array_equal(w.config, wr.config), name
        if guided:
            np.testing.assert_allclose(lw, lwr, rtol=1e-12, atol=1e-13, err_msg=name)
            np.testing.assert_allclose(E, Er, rtol=1e-12, atol=1e-12, err_msg=name)
            np.testing.assert_allclose(w.e_loc, wr.e_loc, rtol=1e-12, atol=1e-12, err_msg=name)
        else:
            assert np.array_equal(lw, lwr) and np.array_equal(E, Er), name
            assert np.array_equal(w.e_loc, wr.e_loc), name

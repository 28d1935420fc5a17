"""The GFMC shift lam through run() on the device: continuous time ignores
it bit for bit and records what was passed (NaN for none); a discrete
method records it and a different shift gives a different chain (the
contract of engine/evolution.py require_lam:724-741 and the run
parameters of engine/driver.py:1334-1389)."""
import numpy as np
import pytest

import pygfmc_b200 as P

pytestmark = pytest.mark.gpu


def _system():
    H = P.SpinHalf.create(P.chain(8).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(H.N, H.edges, beta=0.3)
    return H, G


def _walkers():
    return P.prepare_walkers_sz(64, 8, P.PRNGKey(0), sz=0)


def test_cont_time_ignores_lam_bit_for_bit():
    H, G = _system()
    outs = {lam: P.run(_walkers(), 30, H, 0.2, G, [2, 4], lam=lam, rng_key=P.PRNGKey(2),
                       warmup_steps=8, verbosity=0) for lam in (None, 5.0, -3.0)}
    ref = outs[None]
    for lam, out in outs.items():
        assert np.array_equal(np.asarray(out[0].config), np.asarray(ref[0].config)), lam
        assert np.array_equal(np.asarray(out[4]["energy"]), np.asarray(ref[4]["energy"])), lam
        assert np.array_equal(np.asarray(out[4]["log_weights"]), np.asarray(ref[4]["log_weights"])), lam
        stored = float(out[3]["parameters/lam"])
        assert np.isnan(stored) if lam is None else stored == lam


def test_discrete_lam_is_recorded_and_changes_the_chain():
    H, G = _system()
    a = P.run(_walkers(), 30, H, 2, G, [2], method="multi_step", lam=4.0, rng_key=P.PRNGKey(3),
              warmup_steps=8, verbosity=0)
    b = P.run(_walkers(), 30, H, 2, G, [2], method="multi_step", lam=6.0, rng_key=P.PRNGKey(3),
              warmup_steps=8, verbosity=0)
    assert float(a[3]["parameters/lam"]) == 4.0 and float(b[3]["parameters/lam"]) == 6.0
    assert not np.array_equal(np.asarray(a[4]["energy"]), np.asarray(b[4]["energy"]))

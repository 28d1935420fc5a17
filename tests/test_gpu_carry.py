"""The optional carried guide state of sparse Jastrow guides (gfmc_carry_mode):
carried through the parent maps (the float64 build's default) or rebuilt per
walker every step (mode 0, and what the engine falls back to when the
buffers do not fit in half the free device memory).  Both follow the oracle,
which evaluates every rate afresh: identical configurations and parents,
log G and E_n within 1e-12 relative, including a switch between the two in
the middle of a run; run() records which one ran."""
import numpy as np
import pytest

import pygfmc_b200 as P
from oracle_guides import oracle_guide

pytestmark = pytest.mark.gpu


def _oracle_chain(O, m, g, cfg, keys, tau, alw):
    c = np.array(cfg, dtype=np.float64, copy=True)
    lw = np.zeros(len(c)); el = np.zeros(len(c))
    LG, EE = [], []
    for k in keys:
        O.evolve(m, g, "cont_time", tau, None, alw, k[:2], c, lw, el)
        _, lG, E = O.reconfigure(k[2:], c, lw, el)
        LG.append(lG); EE.append(E)
    return c, np.array(LG), np.array(EE)


@pytest.mark.parametrize("modes", [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
def test_carried_and_rebuilt_guide_state_follow_the_oracle(oracle, modes):
    import torch
    O = oracle
    P._lib.load()
    e = P.chain(32).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)
    G = P.JastrowSpinHalf(32, e, beta=0.3, h=0.05)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2)
    g = oracle_guide(O, G, m)
    n, tau, alw = 600, 0.1, 0.9
    cfg = P.prepare_walkers_sz(n, 32, P.PRNGKey(5), sz=0).config
    eng = P.GFMCEngine(H, G, n, precision="fp64")
    eng.load(cfg)
    keys, _ = P.engine.key_schedule(P.PRNGKey(6), 45)
    lg = torch.empty(15, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    LG, EE = [], []
    for part, mode in enumerate(modes):
        eng.carry_mode(mode)
        eng.steps("cont_time", tau, None, alw, keys[15 * part:15 * (part + 1)], lg, En)
        assert eng.carry_mode() == bool(mode)
        LG.append(lg.cpu().numpy().copy()); EE.append(En.cpu().numpy().copy())
    c, LGo, EEo = _oracle_chain(O, m, g, cfg, keys, tau, alw)
    np.testing.assert_allclose(np.concatenate(LG), LGo, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(np.concatenate(EE), EEo, rtol=1e-12, atol=1e-12)
    cfg_d, _ = eng.population()
    assert np.array_equal(cfg_d.cpu().numpy(), c)
    assert eng.status() == 0


def test_run_records_whether_the_guide_state_was_carried():
    P._lib.load()
    e = P.chain(16).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(16, e, beta=0.3)
    w = P.prepare_walkers_sz(128, 16, P.PRNGKey(0), sz=0)
    for prec, carried in (("fp64", 1), ("mixed", 0)):
        _, _, _, st, _ = P.run(w, 10, H, 0.1, G, [2], rng_key=P.PRNGKey(1), warmup_steps=4,
                               verbosity=0, precision=prec)
        assert st["guide_state_carried"] == carried, prec

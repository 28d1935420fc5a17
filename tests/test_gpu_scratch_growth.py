"""A handle whose population grows from call to call (the C ABI takes the
walker count per call): its resampling scratch and its carried guide-state
buffers (fields and evaluation records) are released and reallocated twice.
A step of a fresh population on that handle then matches the same step on a
new handle: configurations and parents bit for bit, log G and E_n within
1e-12 relative."""
import numpy as np
import pytest

import pygfmc_b200 as P

pytestmark = pytest.mark.gpu


def _system():
    L = 6
    lat = P.square(L)
    pairs = np.array([(i, j) for i in range(L * L) for j in range(i + 1, L * L)])
    d = np.abs(lat.extras["positions"][pairs[:, 0]] - lat.extras["positions"][pairs[:, 1]])
    d = np.minimum(d, L - d)
    H = P.SpinHalf.create(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(lat.N, pairs, beta=0.25 / np.sqrt((d ** 2).sum(1)))
    return lat.N, H, G


def test_growing_population_reallocates_cleanly():
    import torch
    P._lib.load()
    N, H, G = _system()
    n = 3000
    w = P.prepare_walkers_sz(n, N, P.PRNGKey(0), sz=0)
    keys, _ = P.engine.key_schedule(P.PRNGKey(1), 3)

    # the new handle, sized for the whole population from its first call
    b = P.GFMCEngine(H, G, n, precision="fp64")
    b.load(w.config)
    cfg0 = b.cfg.clone()
    alw = float((-b.local_energy()).mean().item())
    logG_b = torch.empty(3, dtype=torch.float64, device=b.device)
    E_b = torch.empty_like(logG_b)
    b.steps("cont_time", 0.1, None, alw, keys, logG_b, E_b)
    assert b.status() == 0

    # the growing handle: 1000, then 2000, then 3000 walkers of the same buffers
    a = P.GFMCEngine(H, G, n, precision="fp64")
    a.load(w.config)
    assert torch.equal(a.cfg, cfg0)
    logG = torch.empty_like(logG_b)
    E = torch.empty_like(logG_b)
    for k in (1000, 2000):
        a.n = k
        a.parents_valid = 0
        a.steps("cont_time", 0.1, None, alw, keys, logG, E)
    a.n = n
    a.cfg.copy_(cfg0)
    a.parents_valid = 0
    a.steps("cont_time", 0.1, None, alw, keys, logG, E)
    assert a.status() == 0

    torch.cuda.synchronize()
    assert torch.equal(a.cfg, b.cfg)
    assert torch.equal(a.parents, b.parents)
    np.testing.assert_allclose(logG.cpu().numpy(), logG_b.cpu().numpy(), rtol=1e-12, atol=0)
    np.testing.assert_allclose(E.cpu().numpy(), E_b.cpu().numpy(), rtol=1e-12, atol=0)

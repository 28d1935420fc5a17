"""End-to-end energies of the benchmark workloads' plain (Jastrow-guided)
runs: the 100-site Heisenberg chain (the reference's quick-start shape)
against the Bethe-ansatz energy of the periodic chain, and the float32
build against the float64 build on the 64-site Bose-Hubbard ring."""
import numpy as np
import pytest

import pygfmc_b200 as P

pytestmark = pytest.mark.gpu

# Ground-state energy per site of the periodic spin-1/2 Heisenberg chain with
# L = 100 (Bethe ansatz).
E_BETHE_L100 = -0.4432296


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_quickstart_chain_matches_bethe_ansatz(prec):
    """L = 100, J_x = J_y = -1, J_z = 1 (Marshall frame), nearest-neighbour
    Jastrow beta = 0.3, 1024 walkers from random Sz = 0 strings, tau = 0.2,
    2000 warm-up + 3000 steps, p = [4, 16, 64, 128]."""
    e = P.chain(100).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    G = P.JastrowSpinHalf(100, e, beta=0.3)
    w = P.prepare_walkers_sz(1024, 100, P.PRNGKey(0), sz=0)
    _, E, _, st, raw = P.run(w, 3000, H, 0.2, G, [4, 16, 64, 128], rng_key=P.PRNGKey(1),
                             warmup_steps=2000, verbosity=0, precision=prec)
    Ej, err = P.estimators.jackknife_energy([128], raw["log_weights"], raw["energy"], 20)
    e_site, s_site = Ej[128] / 100, err[128] / 100
    # population-control bias of 1024 walkers is well below 1e-4 per site here
    assert abs(e_site - E_BETHE_L100) < max(4 * s_site, 1e-4), (e_site, s_site)


def test_bose_ring_builds_agree():
    """64-site Bose-Hubbard ring, 64 bosons, n_max = 4, t = 1, U = 3, with the
    Gutzwiller + density-Jastrow guide; 4096 walkers drawn uniformly with
    sum n = 64, tau = 0.02: the float32 build's energy agrees with the
    float64 build's within the combined error."""
    e = P.chain(64).edges
    H = P.BoseHubbard.create(e, t=1.0, U=3.0, n_max=4, dtype=np.float64)
    G = P.JastrowBoseHubbard(64, e, beta=0.05, d=0.3)
    w = P.prepare_walkers_occupations(4096, 64, 64, 4, P.PRNGKey(0))
    res = {}
    for prec in ("fp64", "mixed"):
        _, E, _, st, raw = P.run(w, 3000, H, 0.02, G, [16, 64], rng_key=P.PRNGKey(1),
                                 warmup_steps=1000, verbosity=0, precision=prec)
        Ej, err = P.estimators.jackknife_energy([64], raw["log_weights"], raw["energy"], 20)
        res[prec] = (Ej[64], err[64])
    (a, ea), (b, eb) = res["fp64"], res["mixed"]
    assert abs(a - b) < 4 * np.hypot(ea, eb), res
    assert -2.0 < a / 64 < 0.0, res

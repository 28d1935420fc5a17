"""The population guide state for dense Jastrow couplings (one product
F = X J for all walkers at once, csrc/fields.cu) through gfmc_local_energy on
fresh populations, against the oracle's local energies
(JastrowSpinHalf / JastrowBoseHubbard log-ratios, jastrow_spin_half.py:290-353,
jastrow_bose_hubbard.py:172-286): the 16 x 16 all-pairs Jastrow of the
benchmark workload, a 6 x 6 torus (N off the kernel's 16-site chunks and
128-site tiles), a 300-site random dense guide with a field (three site
tiles), and a 1040-site dense Bose guide (configurations too large to stage
per block; its digit rows too wide for the persistent kernel, so the
one-tile-per-CTA kernel runs).  The 20011-walker population gives the
persistent kernel's CTAs several walker tiles each.  Walker counts are not multiples of the 64-walker tile.  Float64
build within 1e-12 of the rate scale; float32 build within 3e-4 (float32
fields summed over up to 1040 partners in the exponent)."""
import numpy as np
import pytest

import pygfmc_b200 as P
from oracle_guides import oracle_guide

pytestmark = pytest.mark.gpu


def _torus_longrange(L, amp):
    lat = P.square(L)
    pairs = np.array([(i, j) for i in range(L * L) for j in range(i + 1, L * L)])
    d = np.abs(lat.extras["positions"][pairs[:, 0]] - lat.extras["positions"][pairs[:, 1]])
    d = np.minimum(d, L - d)
    return lat, pairs, amp / np.sqrt((d ** 2).sum(1))


def _spin_cases(O):
    out = []
    for L, amp, n in ((16, 0.3, 1000), (6, 0.25, 77), (16, 0.3, 20011)):
        lat, pairs, beta = _torus_longrange(L, amp)
        H = P.SpinHalf.create(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
        m = O.spin_half(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
        G = P.JastrowSpinHalf(lat.N, pairs, beta=beta)
        g = oracle_guide(O, G, m)
        cfg = P.prepare_walkers_sz(n, lat.N, P.PRNGKey(L), sz=0).config
        out.append((f"square{L}_longrange_{n}", H, G, m, g, cfg))
    N = 300
    rng = np.random.default_rng(3)
    e = P.chain(N).edges
    pairs = np.array([(i, j) for i in range(N) for j in range(i + 1, N)])
    beta = rng.uniform(-0.02, 0.05, len(pairs))
    h = rng.uniform(-0.1, 0.1, N)
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0)
    G = P.JastrowSpinHalf(N, pairs, beta=beta, h=h)
    g = oracle_guide(O, G, m)
    cfg = P.prepare_walkers_random(130, N, P.PRNGKey(4)).config
    out.append(("chain300_dense_random_field", H, G, m, g, cfg))
    return out


def _bose_case(O):
    N = 1040
    e = P.chain(N).edges
    rng = np.random.default_rng(5)
    pairs = np.array([(i, j) for i in range(N) for j in range(i + 1, N)])
    beta = rng.uniform(0.0, 2e-4, len(pairs))
    H = P.BoseHubbard.create(e, t=1.0, U=3.0, mu=0.2, n_max=2, dtype=np.float64)
    m = O.bose_hubbard(e, t=1.0, U=3.0, mu=0.2, n_max=2)
    G = P.JastrowBoseHubbard(N, pairs, beta=beta, d=0.2)
    g = oracle_guide(O, G, m)
    cfg = rng.integers(0, 3, (70, N)).astype(np.float64)
    return ("chain1040_bose_dense", H, G, m, g, cfg)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 3e-4)])
def test_population_guide_state_matches_oracle(oracle, prec, tol):
    O = oracle
    P._lib.load()
    for name, H, G, m, g, cfg in _spin_cases(O) + [_bose_case(O)]:
        eng = P.GFMCEngine(H, G, cfg.shape[0], precision=prec)
        eng.load(cfg)
        el = eng.local_energy().cpu().numpy()
        r = O.rates(m, g, np.asarray(cfg, dtype=np.float64))
        err = np.abs(el - r.sum(axis=1)) / np.abs(r).sum(axis=1)
        assert err.max() <= tol, (name, prec, err.max())
        assert eng.status() == 0, name

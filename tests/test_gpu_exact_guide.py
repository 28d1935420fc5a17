"""The exact-amplitude guide on the device (GFMC_GUIDE_EXACT_SPIN_HALF): the
zero-variance pins of PyGFMC's tests/core/test_exact_ground_state.py
(:85-103 the local energy E0 on the whole support, :105-118 the run's energy
on E0, :121-148 the forward-walked off-diagonal estimate exact and flat in
p), one-step parity with the oracle under the three propagators, and a guide
with the reference's attribute set running unchanged."""
import itertools

import numpy as np
import pytest

import pygfmc_b200 as P
from test_exact_guide import RefShapedExactGuide
from test_gpu_parity import _raw_cfg

pytestmark = pytest.mark.gpu


def _all(N):
    return np.array(list(itertools.product((1.0, -1.0), repeat=N)), dtype=np.float64)


def _ring(N, h_x=0.0):
    return P.SpinHalf.create(P.chain(N).edges, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=h_x,
                             dtype=np.float64)


@pytest.mark.parametrize("precision,dtype,tol", [("fp64", np.float64, 1e-10),
                                                 ("mixed", np.float32, 1e-4)])
@pytest.mark.parametrize("h_x", [0.0, 0.25])
def test_device_local_energy_is_E0_on_the_support(precision, dtype, tol, h_x):
    P._lib.load()
    H = _ring(10, h_x)
    G = P.ExactGroundState(H, dtype=dtype)
    cfg = _all(10)
    if h_x == 0.0:
        cfg = cfg[cfg.sum(1) == 0]          # the support of psi_0
    eng = P.GFMCEngine(H, G, len(cfg), precision=precision)
    eng.load(cfg)
    el = eng.local_energy().cpu().numpy()
    np.testing.assert_allclose(el, G.E0, rtol=0, atol=tol)
    assert eng.status() == 0


def _general_chain12():
    rng = np.random.default_rng(31)
    e = P.chain(12).edges
    jx = -rng.uniform(0.5, 1.5, 12)
    jy = jx + rng.uniform(0.0, 0.2, 12)
    jz = rng.uniform(0.5, 1.5, 12)
    kw = dict(J_x=jx, J_y=jy, J_z=jz, h_z=0.3, h_x=0.2)
    return e, kw


@pytest.mark.parametrize("method,step,lam", [("cont_time", 0.15, None), ("single_step", 3, 12.0),
                                             ("multi_step", 4, 12.0)])
def test_one_step_parity_with_oracle(oracle, method, step, lam):
    """Non-uniform XYZ couplings with both fields (the general spin path) and
    the Heisenberg ring: identical configurations and parents, weights,
    local energies, log G and E_n within 1e-12."""
    import torch
    O = oracle
    P._lib.load()
    e, kw = _general_chain12()
    systems = [(P.SpinHalf.create(e, dtype=np.float64, **kw), O.spin_half(e, **kw),
                P.prepare_walkers_random(512, 12, P.PRNGKey(3)).config),
               (_ring(12), O.spin_half(P.chain(12).edges, J_x=-1.0, J_y=-1.0, J_z=1.0),
                P.prepare_walkers_sz(512, 12, P.PRNGKey(4), sz=0).config)]
    for H, m, cfg in systems:
        G = P.ExactGroundState(H, dtype=np.float64)
        g = O.exact_spin_half(G.log_amp, G.local_hilbert_space)
        eng = P.GFMCEngine(H, G, len(cfg), precision="fp64")
        eng.load(cfg)
        keys, _ = P.engine.key_schedule(P.PRNGKey(78), 1)
        lg = torch.empty(1, dtype=torch.float64, device=eng.device)
        En = torch.empty(1, dtype=torch.float64, device=eng.device)
        alw = 4.0
        eng.steps(method, step, lam, alw, keys, lg, En)
        c = np.array(cfg, dtype=np.float64, copy=True)
        lw = np.zeros(len(c)); el = np.zeros(len(c))
        O.evolve(m, g, method, step, lam, alw, keys[0, :2], c, lw, el)
        assert np.array_equal(_raw_cfg(eng, torch), c)
        np.testing.assert_allclose(eng.log_w.cpu().numpy(), lw, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(eng.e_loc.cpu().numpy(), el, rtol=1e-12, atol=1e-12)
        # zero variance, to the accuracy of the Lanczos vector's small amplitudes
        np.testing.assert_allclose(el, G.E0, rtol=0, atol=1e-8)
        par, lG, E = O.reconfigure(keys[0, 2:], c, lw, el)
        assert np.array_equal(eng.parents.cpu().numpy(), par)
        np.testing.assert_allclose(lg.item(), lG, rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(En.item(), E, rtol=1e-12, atol=1e-12)
        assert eng.status() == 0


@pytest.mark.parametrize("method,step,lam", [("single_step", 8, 2.5), ("cont_time", 0.5, None),
                                             ("multi_step", 8, 2.5)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_zero_variance_run(method, step, lam, precision, tol):
    """With psi_T = psi_0 the energy of every window is E0: PyGFMC asks for
    1e-4 per site with its float32 guide; the float64 build holds 1e-10."""
    lat = P.chain(6)
    H = _ring(6)
    G = P.ExactGroundState(H, dtype=np.float64 if precision == "fp64" else np.float32)
    w = P.prepare_walkers_sz(128, lat.N, P.PRNGKey(0), sz=0)
    wf, res, _, _, raw = P.run(w, 300, H, step, G, [8, 16], method=method, lam=lam,
                               rng_key=P.PRNGKey(1), verbosity=0, warmup_steps=100,
                               precision=precision)
    assert set(res) == {8, 16}
    for p, energy in res.items():
        assert abs(energy - G.E0) / lat.N < min(1e-4, tol), (p, energy, G.E0)
    np.testing.assert_allclose(raw["energy"], G.E0, rtol=0, atol=6 * tol)
    np.testing.assert_allclose(wf.e_loc, G.E0, rtol=0, atol=6 * tol)


def test_forward_walked_off_diagonal_is_exact_at_every_p():
    """<S+S- + h.c.> on bond 0 of the 6-site ring, forward-walked with the
    exact guide: within 1e-2 of psi_0^T O psi_0 at every p and flat in p
    (a wrong window offset or shadow normalisation would drift)."""
    lat = P.chain(6)
    H = _ring(6)
    G = P.ExactGroundState(H, dtype=np.float64)
    n_e = len(lat.edges)
    one = np.zeros(n_e); one[0] = 1.0
    spm = P.SpinHalf.create(list(lat.edges), J_x=2 * one, J_y=2 * one, J_z=np.zeros(n_e),
                            sign_check=False, dtype=np.float64)
    _, _, oobs = P.exact_diagonalization(H, off_diag_operators={"spm": spm})
    exact = float(oobs["spm"][0])
    w = P.prepare_walkers_sz(2048, lat.N, P.PRNGKey(0), sz=0)
    _, _, obs, _, _ = P.run(w, 1500, H, 1, G, [2, 4, 8, 16], method="single_step",
                            lam=n_e / 4 + 1.0, rng_key=P.PRNGKey(1), off_diag_operators={"spm": spm},
                            verbosity=0, warmup_steps=100)
    got = {p: float(np.ravel(v)[0]) for p, v in obs["spm"].items()}
    for p, val in got.items():
        assert abs(val - exact) < 1e-2, (p, val, exact)
    assert max(got.values()) - min(got.values()) < 5e-3, got


def test_reference_shaped_guide_runs_unchanged():
    """A guide with PyGFMC's attribute set, indexed over (-1, 1), gives the
    run of this package's guide with the same float32 amplitudes bit for
    bit."""
    H = _ring(8, 0.2)
    G = P.ExactGroundState(H)
    ref = RefShapedExactGuide(G.log_amp[::-1], 8)     # the same amplitudes over (-1, 1)
    w = P.prepare_walkers_random(256, 8, P.PRNGKey(2))
    runs = [P.run(w, 40, H, 0.1, g, [4], rng_key=P.PRNGKey(3), warmup_steps=10, verbosity=0)
            for g in (G, ref)]
    np.testing.assert_array_equal(runs[0][4]["energy"], runs[1][4]["energy"])
    np.testing.assert_array_equal(runs[0][0].config, runs[1][0].config)
    assert abs(runs[0][1][4] - G.E0) < 1e-4 * 8

"""estimators.evaluate_observables, PyGFMC's re-estimation of the energy and
the observables from a run's raw series with blocked-jackknife errors
(engine/io.py evaluate_observables:921-1149), on the golden raw series of
PyGFMC's own runs: the point estimates are the golden energies and
observables; the energy errors are those of jackknife_energy; the observable
errors are the scatter of replicas built independently (a deleted block's
off-diagonal rows dropped, the rest renumbered into the shortened chain);
trailing steps are trimmed from every series with a warning (the case of
PyGFMC's tests/core/test_review_regressions.py:229-250); another grid
re-windows the energy alone; and a hand-built raw with dense arrays gives the
same as the named form.  Host only."""
import warnings

import numpy as np
import pytest

import pygfmc_b200 as P
from pygfmc_b200.estimators import (diagonal_estimates, evaluate_observables, jackknife_energy,
                                    off_diagonal_estimates, windowed_energy_host)

CASES = ["spinhalf_jastrow_cont_time", "bose_none_single_step", "spinhalf_none_multi_step",
         "bose_jastrow_cont_time"]


def _raw(golden, name):
    p = name + "/"
    lw = golden[p + "raw/log_weights"]
    diag = {k.split("/")[-1]: golden[k] for k in golden.files if k.startswith(p + "raw/diag/")}
    off = {k.split("/")[-1]: golden[k] for k in golden.files if k.startswith(p + "raw/off_diag/")}
    norm = {nm: golden[p + f"raw/off_diag_norm/{nm}"] for nm in off}
    return dict(log_weights=lw, energy=golden[p + "raw/energy"], diag=diag, off_diag=off,
                off_diag_norm=norm, off_diag_steps=np.arange(len(lw)), p_array=[2, 4], m_array=[1, 2])


@pytest.mark.parametrize("name", CASES)
def test_point_estimates_are_the_golden_ones(golden, name):
    E, obs = evaluate_observables(_raw(golden, name))
    for pp in (2, 4):
        np.testing.assert_allclose(E[pp], golden[f"{name}/energy/{pp}"], rtol=1e-10, atol=1e-12)
        for nm in obs:
            np.testing.assert_allclose(obs[nm][pp], golden[f"{name}/obs/{nm}/{pp}"], rtol=1e-10,
                                       atol=1e-12, err_msg=f"{nm} p={pp}")


@pytest.mark.parametrize("name", CASES)
def test_jackknife_errors(golden, name):
    raw = _raw(golden, name)
    nb = 20
    E, obs, Eerr, oerr = evaluate_observables(raw, n_blocks=nb)
    E2, err2 = jackknife_energy([2, 4], raw["log_weights"], raw["energy"], nb)
    assert E == E2
    np.testing.assert_allclose([Eerr[p] for p in (2, 4)], [err2[p] for p in (2, 4)], rtol=1e-13)
    # the replicas rebuilt here: survivors concatenated, off-diagonal rows
    # (one per step) renumbered 0 .. n - blen - 1, windows from max(m) = 2
    lw, En = raw["log_weights"], raw["energy"]
    n = len(lw)
    blen = n // nb
    reps = []
    for b in range(nb):
        keep = np.r_[0:b * blen, (b + 1) * blen:n]
        o = diagonal_estimates([2, 4], lw[keep], {k: v[keep] for k, v in raw["diag"].items()}, 2)
        o.update(off_diagonal_estimates([2, 4], [1, 2], lw[keep],
                                        {k: v[keep] for k, v in raw["off_diag"].items()},
                                        {k: v[keep] for k, v in raw["off_diag_norm"].items()},
                                        np.arange(len(keep)), 2))
        reps.append(o)
    for nm in obs:
        for pp in (2, 4):
            x = np.array([r[nm][pp] for r in reps])        # (nb,) or (nb, components)
            want = np.sqrt((nb - 1) / nb * np.sum((x - x.mean(axis=0)) ** 2, axis=0))
            np.testing.assert_allclose(oerr[nm][pp], want, rtol=1e-12, err_msg=f"{nm} p={pp}")
            assert np.all(np.asarray(oerr[nm][pp]) > 0)


def _same(a, b):
    """Equal nested estimates (dicts of floats or arrays)."""
    if isinstance(a, dict):
        return a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
    return np.array_equal(np.asarray(a), np.asarray(b))


def test_trailing_samples_are_trimmed_from_every_series():
    steps = np.arange(0, 41, 2)
    raw = {"energy": np.arange(41.0), "log_weights": np.zeros(41), "p_array": [2], "m_array": [1],
           "diag": {"z": np.arange(41.0)[:, None]}, "off_diag": {"x": steps[:, None] * 1.0},
           "off_diag_norm": {"x": np.zeros((len(steps), 1))}, "off_diag_steps": steps}
    trimmed = {**raw, "energy": raw["energy"][:40], "log_weights": np.zeros(40),
               "diag": {"z": raw["diag"]["z"][:40]}, "off_diag": {"x": raw["off_diag"]["x"][:-1]},
               "off_diag_norm": {"x": raw["off_diag_norm"]["x"][:-1]}, "off_diag_steps": steps[:-1]}
    with pytest.warns(UserWarning, match="Discarding 1 trailing"):
        got = evaluate_observables(raw, n_blocks=20)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")            # the few-blocks advice
        want = evaluate_observables(trimmed, n_blocks=20)
        as_float = evaluate_observables({**trimmed, "off_diag_steps": steps[:-1].astype(float)},
                                        n_blocks=20)
    for a, b in ((got, want), (as_float, want)):
        assert a[0] == b[0] and a[2] == b[2]
        for nm in ("z", "x"):
            assert a[1][nm] == b[1][nm] and a[3][nm] == b[3][nm]


def test_another_grid_rewindows_the_energy_only(golden):
    raw = _raw(golden, CASES[0])
    E, obs = evaluate_observables(raw, p_array=[3, 6])
    assert E == windowed_energy_host([3, 6], raw["log_weights"], raw["energy"])
    _, obs_stored = evaluate_observables(raw)
    assert _same(obs, obs_stored) and all(set(v) == {2, 4} for v in obs.values())
    E, _, Eerr, _ = evaluate_observables(raw, p_array=[3, 6], n_blocks=20)
    assert set(Eerr) == {3, 6} and all(v > 0 for v in Eerr.values())


def test_dense_arrays_and_positional_names(golden):
    raw = _raw(golden, CASES[0])
    raw["diag"] = {k: v for k, v in raw["diag"].items() if v.ndim == 2}   # scalar operators
    dn, on = list(raw["diag"]), list(raw["off_diag"])
    dense = {**raw, "diag": np.stack([raw["diag"][k] for k in dn], axis=1),
             "off_diag": np.stack([raw["off_diag"][k] for k in on], axis=1),
             "off_diag_norm": np.stack([raw["off_diag_norm"][k] for k in on], axis=1)}
    dense.pop("p_array")
    E, obs = evaluate_observables(dense, p_array=[2, 4])
    E0, obs0 = evaluate_observables(raw)
    assert E == E0
    for i, k in enumerate(dn):
        assert _same(obs[f"diag_{i}"], obs0[k])
    for i, k in enumerate(on):
        assert _same(obs[f"off_diag_{i}"], obs0[k])


def test_arguments(golden):
    raw = _raw(golden, CASES[0])
    with pytest.raises(ValueError, match="no 'energy'"):
        evaluate_observables({k: v for k, v in raw.items() if k != "energy"})
    with pytest.raises(ValueError, match="no 'log_weights'"):
        evaluate_observables({k: v for k, v in raw.items() if k != "log_weights"})
    with pytest.raises(ValueError, match="no p grid"):
        evaluate_observables({k: v for k, v in raw.items() if k != "p_array"})
    with pytest.raises(ValueError, match="window"):
        evaluate_observables({**raw, "p_array": [2, 4, 8]})
    with pytest.raises(ValueError, match="off_diag_steps"):
        evaluate_observables({**raw, "off_diag_steps": None})
    with pytest.raises(ValueError, match="integer-valued"):
        evaluate_observables({**raw, "off_diag_steps": np.arange(300) + 0.5})
    with pytest.raises(ValueError, match="increasing"):
        evaluate_observables({**raw, "off_diag_steps": np.arange(300)[::-1].copy()})
    with pytest.raises(ValueError, match="at least 2 usable blocks"):
        evaluate_observables(raw, n_blocks=1)
    with pytest.warns(UserWarning, match="few"):
        evaluate_observables(raw, n_blocks=10)
    assert P.evaluate_observables is evaluate_observables


@pytest.mark.parametrize("trim", [0, 4])
def test_off_diagonal_windows_on_an_irregular_grid(trim):
    """tests/core/test_estimator_window_reuse.py:8-33: rows measured at
    irregular main-chain steps, three operators, three windows; each estimate
    equals the explicit sum over usable rows of bra x exp(norm) x value over
    the sum of bra x ket (bra: the m weights before the row's step, ket: the
    m after), rows with k < p + max(0, trim - m) or k >= n - m left out."""
    rng = np.random.default_rng(19)
    n, windows = 40, [2, 4, 8]
    steps = np.array([0, 2, 3, 6, 9, 10, 15, 18, 24, 31, 35, 39])
    names = ["first", "second", "third"]
    lw = rng.normal(0, 0.1, n)
    values = rng.normal(size=(len(steps), len(names), len(windows)))
    norms = rng.normal(0, 0.1, values.shape)
    got = off_diagonal_estimates(windows, [p // 2 for p in windows], lw,
                                 {nm: values[:, i] for i, nm in enumerate(names)},
                                 {nm: norms[:, i] for i, nm in enumerate(names)}, steps, trim)
    for j, p in enumerate(windows):
        m = p // 2
        for i, nm in enumerate(names):
            num = den = 0.0
            for row, k in enumerate(steps):
                if k < p + max(0, trim - m) or k >= n - m:
                    continue
                bra = np.exp(lw[k - m + 1:k + 1].sum())
                ket = np.exp(lw[k + 1:k + m + 1].sum())
                num += bra * np.exp(norms[row, i, j]) * values[row, i, j]
                den += bra * ket
            assert got[nm][p] == pytest.approx(num / den, abs=1e-14)

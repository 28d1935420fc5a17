"""Host-side estimator helpers (numpy, float64).

The per-step series come from the device; what is cheap and inherently
serial on the series stays on the host, as in PyGFMC:
``validated_p_array`` (engine/estimators.py:30-42), the windowed energy for
progress lines (:268-305; the final estimate runs on the device),
``autocorrelation`` (:71-117), and the blocked jackknife of
``evaluate_observables`` (engine/io.py:1084-1104).
"""
import warnings
from collections.abc import Mapping

import numpy as np

__all__ = ["validated_p_array", "windowed_energy_host", "diagonal_estimates",
           "off_diagonal_estimates", "autocorrelation",
           "autocorrelation_stats", "jackknife_energy", "evaluate_observables"]


def validated_p_array(p_array):
    if p_array is None or len(p_array) == 0:
        raise ValueError("p_array must contain at least one positive window size.")
    out = []
    for p in p_array:
        pi = int(p)
        if float(pi) != float(p):
            raise ValueError(f"p_array values must be integers, got {p!r}.")
        if pi <= 0:
            raise ValueError(f"p_array values must be > 0, got {pi}.")
        out.append(pi)
    return sorted(set(out))


def windowed_energy_host(p_array, log_weights, E):
    """E_p = sum_i G_p(i) E(i+p) / sum_i G_p(i), G_p from windowed log weights."""
    L = np.cumsum(np.asarray(log_weights, dtype=np.float64))
    E = np.asarray(E, dtype=np.float64)
    out = {}
    for p in validated_p_array(p_array):
        if p >= len(L):
            continue
        lg = L[p:] - L[:-p]
        G = np.exp(lg - np.max(lg))
        out[p] = float(np.sum(G * E[p:])) / float(np.sum(G))
    return out


def diagonal_estimates(p_array, log_weights, diag_by_name, m_max_common=0):
    """Ancestry-traced diagonal estimates (engine/estimators.py:287-303):
    <D>_p = sum_i G_p(i) D(i+p) / sum_i G_p(i) over the window starts
    i >= m_max_common; D(t) = raw['diag'][name][t, ..., j]."""
    L = np.cumsum(np.asarray(log_weights, dtype=np.float64))
    out = {name: {} for name in diag_by_name}
    for j, p in enumerate(validated_p_array(p_array)):
        lg = (L[p:] - L[:-p])[m_max_common:]
        G = np.exp(lg - np.max(lg))
        gs = float(np.sum(G))
        for name, arr in diag_by_name.items():
            a = np.asarray(arr, dtype=np.float64)
            if a.ndim == 2:
                out[name][p] = float(np.sum(G * a[:, j][p:][m_max_common:])) / gs
            else:
                out[name][p] = np.sum(G[:, None] * a[:, :, j][p:][m_max_common:], axis=0) / gs
    return out


def off_diagonal_estimates(p_array, m_array, log_weights, off_diag, off_diag_norm, off_diag_steps,
                           m_max_common=0):
    """Forward-walking pure estimates {name: {p: value}} of the off-diagonal
    operators (engine/estimators.py _off_diagonal_estimates:308-355).

    A row measured at main-chain step k = p + i carries the mean operator
    value after m = p // 2 shadow steps and the shadow's log weight product;
    with L the cumulative main-chain log weights (L[0] = 0),
        numerator   sum_k exp(L[k+1] - L[k-m+1] + norm_k) val_k
        denominator sum_k exp(L[k+m+1] - L[k-m+1]),
    both shifted by one common maximum before exponentiating, over the rows
    with p + max(0, m_max_common - m) <= k < n - m."""
    lw = np.asarray(log_weights, dtype=np.float64)
    n = len(lw)
    L = np.concatenate([[0.0], np.cumsum(lw)])
    k_all = np.asarray(off_diag_steps, dtype=np.int64)
    names = list(off_diag)
    vals = {nm: np.asarray(off_diag[nm], dtype=np.float64) for nm in names}
    norms = {nm: np.asarray(off_diag_norm[nm], dtype=np.float64) for nm in names}
    for nm in names:
        if not (np.all(np.isfinite(vals[nm])) and np.all(np.isfinite(norms[nm]))):
            raise ValueError("off_diag_np and off_diag_norm_np must contain only finite values.")
    out = {nm: {} for nm in names}
    for j, (p, m) in enumerate(zip(validated_p_array(p_array), m_array)):
        if n - m - p <= 0:
            raise ValueError(f"Insufficient samples for off-diagonal windows [{p}]; each requires "
                             "n_samples > p + m.")
        lo, hi = np.searchsorted(k_all, [p + max(0, m_max_common - m), n - m])
        i = k_all[lo:hi] - p
        if len(i) == 0:
            raise ValueError(f"No stored off-diagonal measurement is usable for p={p}, m={m}.")
        log_num = L[p + 1 + i] - L[p - m + 1 + i]
        log_den = L[p + m + 1 + i] - L[p - m + 1 + i]
        for nm in names:
            lt = log_num + norms[nm][lo:hi, j]
            fin = np.isfinite(lt)
            shift = max(np.max(lt[fin]), np.max(log_den)) if fin.any() else np.max(log_den)
            num = float(np.sum(np.exp(lt - shift) * vals[nm][lo:hi, j]))
            den = float(np.sum(np.exp(log_den - shift)))
            out[nm][p] = num / den
    return out


def autocorrelation(series, c=5.0):
    """Integrated autocorrelation time with the self-consistent window
    (FFT autocovariance; window M >= c (0.5 + sum |rho|))."""
    if not np.isfinite(c) or c <= 0:
        raise ValueError("c must be finite and positive.")
    x = np.asarray(series, dtype=float).ravel()
    n = x.size
    if n < 16 or not np.all(np.isfinite(x)):
        return float("nan"), 0
    d = x - x.mean()
    acov0 = float(d @ d) / n
    if acov0 <= 0.0:
        return float("nan"), 0
    m = 1 << (2 * n - 1).bit_length()
    f = np.fft.rfft(d, m)
    acov = np.fft.irfft(f * np.conj(f), m)[:n].real / np.arange(n, 0, -1)
    rho = acov / acov[0]
    run = 0.5 + np.cumsum(rho[1:])
    M = np.arange(1, run.size + 1)
    env = 0.5 + np.cumsum(np.abs(rho[1:]))
    hit = np.flatnonzero(M >= c * env)
    if hit.size == 0:
        return float("nan"), 0
    i = int(hit[0])
    if run[i] <= 0 or not np.isfinite(run[i]):
        return float("nan"), int(M[i])
    return float(run[i]), int(M[i])


def _series_tau(arr, scale=1):
    a = np.asarray(arr)
    if a.ndim == 1:
        a = a[:, None]
    trailing = a.shape[1:]
    flat = a.reshape(a.shape[0], -1)
    return np.array([autocorrelation(flat[:, j])[0] * scale for j in range(flat.shape[1])],
                    dtype=float).reshape(trailing)


def autocorrelation_stats(E_np, log_weights_np, diag_np=None, off_diag_np=None, off_diag_stride=1):
    """engine/estimators.py autocorrelation_stats:172-226."""
    out = {"autocorrelation/energy_estimator": autocorrelation(E_np)[0],
           "autocorrelation/log_weights": autocorrelation(log_weights_np)[0]}
    for name, arr in (diag_np or {}).items():
        out[f"autocorrelation/diag/{name}"] = _series_tau(arr)
    for name, arr in (off_diag_np or {}).items():
        out[f"autocorrelation/off_diag/{name}"] = _series_tau(arr, scale=int(off_diag_stride))
    return out


def jackknife_energy(p_array, log_weights, E, n_blocks):
    """Blocked jackknife of the windowed energy: leave-one-block-out replicas
    (the survivors concatenated), err = sqrt((nb-1)/nb sum (x_b - mean)^2)."""
    n = len(E)
    blen = n // n_blocks
    if n_blocks < 2 or blen < 1:
        raise ValueError(f"n_blocks={n_blocks} over {n} steps leaves {blen} steps per block; "
                         "a jackknife needs at least 2 usable blocks.")
    usable = blen * n_blocks
    lw = np.asarray(log_weights, dtype=np.float64)[:usable]
    EE = np.asarray(E, dtype=np.float64)[:usable]
    grid = validated_p_array(p_array)
    reps = []
    for b in range(n_blocks):
        mask = np.ones(usable, dtype=bool)
        mask[b * blen:(b + 1) * blen] = False
        est = windowed_energy_host(grid, lw[mask], EE[mask])
        reps.append([est[p] for p in grid])
    arr = np.asarray(reps)
    c = arr - arr.mean(axis=0, keepdims=True)
    err = np.sqrt((n_blocks - 1) / n_blocks * np.sum(c ** 2, axis=0))
    return windowed_energy_host(grid, lw, EE), dict(zip(grid, err.tolist()))


def _series_by_name(series, names, kind):
    """A raw dict's operator series as name -> float64 array: a mapping as it
    is, a dense (rows, operators, windows) array split along its operator
    axis under ``names`` or positional ``<kind>_k`` names."""
    if series is None:
        return None
    if isinstance(series, Mapping):
        return {k: np.asarray(v, dtype=np.float64) for k, v in series.items()} or None
    a = np.asarray(series, dtype=np.float64)
    if a.ndim != 3:
        raise ValueError(f"raw['{kind}'] as one array must have shape (rows, operators, windows); "
                         f"got {a.shape}")
    names = list(names) if names else [f"{kind}_{k}" for k in range(a.shape[1])]
    if len(names) != a.shape[1]:
        raise ValueError(f"raw['{kind}'] holds {a.shape[1]} operators but {len(names)} names")
    return {nm: a[:, k] for k, nm in enumerate(names)}


def _estimate_all(grid, m_array, lw, E, diag, off, off_norm, off_steps):
    """The energy and the observables at ``grid`` from the series, as a run
    computes them: with both kinds of operator every observable's windows
    start at i >= max(m_array) (engine/estimators.py:596-619); the energy's
    windows are not trimmed."""
    energy = windowed_energy_host(grid, lw, E)
    m_common = max(m_array) if (diag and off) else 0
    obs = diagonal_estimates(grid, lw, diag, m_common) if diag else {}
    if off:
        obs.update(off_diagonal_estimates(grid, m_array, lw, off, off_norm, off_steps, m_common))
    return energy, obs


def _jackknife_spread(values, n_blocks):
    """sqrt((nb-1)/nb sum (x_b - mean)^2) over the leave-one-out replicas."""
    arr = np.asarray(values, dtype=np.float64)
    c = arr - arr.mean(axis=0, keepdims=True)
    return np.sqrt((n_blocks - 1) / n_blocks * np.sum(c ** 2, axis=0))


def evaluate_observables(raw, p_array=None, n_blocks=None):
    """The energy and the observables re-estimated from a ``raw`` dict
    (engine/io.py evaluate_observables:921-1149): ``(energy, obs)``, or
    ``(energy, obs, energy_err, obs_err)`` with blocked-jackknife errors when
    ``n_blocks`` is given.

    The operator series sit on the grid the run measured them at
    (``raw['p_array']``, or ``p_array`` for a hand-built ``raw`` without
    one); another ``p_array`` re-windows the energy alone and leaves the
    observables at the stored grid.  The jackknife deletes each of
    ``n_blocks`` contiguous blocks in turn and recomputes the whole estimator
    on the concatenated rest, so an off-diagonal row is dropped with its
    block and the others are renumbered into the shortened chain; trailing
    steps that do not fill a block are discarded, with a warning, from the
    point estimates and the errors alike; fewer than 20 blocks draw a
    warning (the error on the error is then comparable to the error)."""
    E, lw = raw.get("energy"), raw.get("log_weights")
    if E is None:
        raise ValueError("raw holds no 'energy' series, so nothing can be re-estimated; pass the "
                         "raw dict run() returns with return_raw=True.")
    if lw is None:
        raise ValueError("raw holds no 'log_weights' series; the windowed estimator needs the "
                         "per-step branch weights.")
    E, lw = np.asarray(E, dtype=np.float64), np.asarray(lw, dtype=np.float64)
    stored = raw.get("p_array", p_array)
    if stored is None:
        raise ValueError("no p grid available: raw carries no 'p_array' and none was passed; pass "
                         "p_array=... (the grid the run measured the operators at).")
    stored_p = validated_p_array(np.asarray(stored).ravel())
    diag = _series_by_name(raw.get("diag"), raw.get("diag_operators"), "diag")
    off = _series_by_name(raw.get("off_diag"), raw.get("off_diag_operators"), "off_diag")
    off_norm = _series_by_name(raw.get("off_diag_norm"), list(off) if off else None, "off_diag_norm")
    for kind, group in (("diag", diag), ("off_diag", off), ("off_diag_norm", off_norm)):
        for nm, a in (group or {}).items():
            if a.shape[-1] != len(stored_p):
                raise ValueError(f"raw['{kind}']['{nm}'] has {a.shape[-1]} window(s) on its last axis "
                                 f"but the grid it is said to be on, {stored_p}, has {len(stored_p)}; "
                                 "set raw['p_array'] to the grid the run measured at.")
    n = len(E)
    off_steps = None
    if off:
        if raw.get("off_diag_steps") is None or off_norm is None:
            raise ValueError("off_diag_steps and off_diag_norm are required whenever off_diag is "
                             "supplied.")
        steps_in = np.asarray(raw["off_diag_steps"])
        if steps_in.dtype.kind == "f" and not np.array_equal(steps_in, np.rint(steps_in)):
            raise ValueError("off_diag_steps must be integer-valued main-chain steps.")
        off_steps = steps_in.astype(np.int64)
        rows = {len(v) for v in off.values()} | {len(v) for v in off_norm.values()}
        if rows != {len(off_steps)} or np.any(np.diff(off_steps) <= 0) or \
                (len(off_steps) and (off_steps[0] < 0 or off_steps[-1] >= n)):
            raise ValueError("off_diag_steps must hold one increasing main-chain step in [0, n_steps) "
                             "per off-diagonal row.")
    m_array = list(raw["m_array"]) if raw.get("m_array") is not None else [p // 2 for p in stored_p]
    if n_blocks is not None:
        nb = int(n_blocks)
        if nb != n_blocks:
            raise ValueError(f"n_blocks must be an integer, got {n_blocks!r}")
        blen = n // nb
        if nb < 2 or blen < 1:
            raise ValueError(f"n_blocks={n_blocks} over {n} steps leaves {blen} steps per block; a "
                             "jackknife needs at least 2 usable blocks.")
        usable = blen * nb
        if usable != n:
            warnings.warn(f"Discarding {n - usable} trailing samples for equal jackknife blocks; the "
                          "point estimates and the errors both use the retained samples.",
                          stacklevel=2)
            E, lw = E[:usable], lw[:usable]
            if diag:
                diag = {k: v[:usable] for k, v in diag.items()}
            if off:
                keep = off_steps < usable
                off = {k: v[keep] for k, v in off.items()}
                off_norm = {k: v[keep] for k, v in off_norm.items()}
                off_steps = off_steps[keep]
            n = usable
    e_stored, obs = _estimate_all(stored_p, m_array, lw, E, diag, off, off_norm, off_steps)
    same_grid = p_array is None or validated_p_array(p_array) == stored_p
    grid = stored_p if same_grid else validated_p_array(p_array)
    e_out = e_stored if same_grid else windowed_energy_host(grid, lw, E)
    if n_blocks is None:
        return e_out, obs
    if nb < 20:
        warnings.warn(f"n_blocks={nb} is few: the error on the error is then comparable to the "
                      "error itself; ~20 or more is advisable.", stacklevel=2)
    if n - blen <= max(grid):
        raise ValueError(f"a jackknife replica keeps {n - blen} steps, not more than the largest "
                         f"window p={max(grid)}; use fewer blocks or a longer chain.")
    masks = []
    for b in range(nb):
        m = np.ones(n, dtype=bool)
        m[b * blen:(b + 1) * blen] = False
        masks.append(m)
    obs_err, e_reps = {}, None
    if obs:
        reps = []
        for m in masks:
            rows = steps_r = None
            if off:
                new_pos = np.cumsum(m) - 1           # a kept step's index in the replica
                rows = m[off_steps]
                steps_r = new_pos[off_steps[rows]]
            reps.append(_estimate_all(
                stored_p, m_array, lw[m], E[m],
                {k: v[m] for k, v in diag.items()} if diag else None,
                {k: v[rows] for k, v in off.items()} if off else None,
                {k: v[rows] for k, v in off_norm.items()} if off else None, steps_r))
        for nm in obs:
            obs_err[nm] = {}
            for p in stored_p:
                err = _jackknife_spread([np.asarray(r[1][nm][p], dtype=np.float64) for r in reps], nb)
                obs_err[nm][p] = float(err) if np.ndim(err) == 0 else err
        if same_grid:
            e_reps = [[r[0][p] for p in grid] for r in reps]
    if e_reps is None:
        e_reps = []
        for m in masks:
            est = windowed_energy_host(grid, lw[m], E[m])
            e_reps.append([est[p] for p in grid])
    energy_err = dict(zip(grid, _jackknife_spread(e_reps, nb).tolist()))
    return e_out, obs, energy_err, obs_err

"""Branching-step diagnostics on the device population, with PyGFMC's
``statistics`` signature and keys (engine/estimators.py statistics:1139-1362).

The steps run in the CUDA engine with the reference's key derivation
(evolve with fold_in(key, 3 t + 1), resampling with fold_in(key, 3 t + 2),
the per-walker probe draws with fold_in(fold_in(key, 3 t), walker)), so the
trajectory -- and every diagnostic that depends on it -- is the reference's.
The host keeps what the reference keeps on the host: unique counts and the
population overlap (from the packed configurations), the offspring and
ancestor bookkeeping (bincounts of the parent maps).
"""
import numpy as np

from . import random as _rnd
from .engine import GFMCEngine, _validated_int, require_lam

__all__ = ["statistics"]

_OFFSPRING_BINS = 4


def _validated_m_array(m_array):
    out = []
    for m in ([] if m_array is None else list(m_array)):
        mi = int(m)
        if float(mi) != float(m):
            raise ValueError(f"m_array values must be integers, got {m!r}.")
        out.append(mi)
    out = sorted(set(out))
    if any(m < 0 for m in out):
        raise ValueError(f"m_array values must be nonnegative, got {out}.")
    return out


def _row_keys(packed):
    a = np.ascontiguousarray(packed)
    return a.view(np.dtype((np.void, a.shape[1]))).ravel()


def _uniforms(key, n):
    """jax.random.uniform(fold_in(key, w)) for w < n (float64)."""
    key = _rnd.as_key(key)
    y0, y1 = _rnd.threefry2x32(key[0], key[1], np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32))
    k0, k1 = y0.astype(np.uint32), y1.astype(np.uint32)
    z0, z1 = _rnd.threefry2x32(k0, k1, np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    bits = ((z0.astype(np.uint64) << np.uint64(32)) | z1.astype(np.uint64)) >> np.uint64(12)
    bits |= np.uint64(0x3FF0000000000000)
    return bits.view(np.float64) - 1.0


def statistics(walkers, hamiltonian, step_size, guide, method, rng_key, avg_log_weight=None,
               lam=None, M=10, quiet=False, m_array=None, cache=None, precision=None,
               _engine=None):
    """Diagnostic branching steps from ``walkers`` (see the module docstring;
    the signature of engine/estimators.py statistics:1139-1143, ``cache``
    accepted and not needed, since the device builds its own tables).
    Returns ``(walkers_after, stats)`` with the reference's keys:
    n_unique_pre/post, unique_fraction, diag_min/max, changed_rate,
    overlap_rate, H_diag_max/min_observed, escape_rate_* / hops_per_step_* /
    hold_time_* (cont_time) or p_d_* / hold_steps_* (discrete methods),
    offspring_k0..3 and offspring_k4plus, survival_rate, and with m_array
    ancestor_m / ancestor_fraction / effective_sample_size /
    ancestor_correlation."""
    config = np.asarray(walkers.config)
    n = int(config.shape[0])
    if n <= 0:
        raise ValueError("statistics requires at least one walker.")
    M = _validated_int("M", M, 1)
    lam = require_lam(method, lam)
    m_sorted = _validated_m_array(m_array)
    n_total = max(M, m_sorted[-1]) if m_sorted else M
    if precision is None:
        lw = getattr(walkers, "log_weight", None)
        precision = "mixed" if getattr(lw, "dtype", np.float64) == np.float32 else "fp64"
    eng = _engine if _engine is not None else GFMCEngine(hamiltonian, guide, n, precision=precision)
    eng.load(config)
    torch = eng.torch
    e0_d, d0_d = eng.local_energy_parts()
    e0 = e0_d.cpu().numpy()
    if avg_log_weight is None:
        avg_log_weight = float(np.mean(-e0)) if method == "cont_time" else float(np.mean(np.log(lam - e0)))
    key = _rnd.as_key(rng_key)
    k_max = _OFFSPRING_BINS
    packed0 = eng.packed_population()
    keys0 = _row_keys(packed0)
    uniq0 = np.unique(keys0)
    h = {k: [] for k in ("n_unique_pre", "n_unique_post", "diag_min", "diag_max", "s_min", "s_max",
                         "s_mean", "k_mean", "k_max", "changed", "overlap")}
    offspring = np.zeros((n_total, k_max + 1))
    frac = np.zeros(n_total)
    ess = np.zeros(n_total)
    corr = np.zeros(n_total)
    anc = np.arange(n)
    lg = torch.empty(1, dtype=torch.float64, device=eng.device)
    En = torch.empty_like(lg)
    for t in range(n_total):
        if t < M:
            h["n_unique_pre"].append(int(np.unique(_row_keys(eng.packed_population())).size))
            e_d, d_d = eng.local_energy_parts()
            e, d = e_d.cpu().numpy(), d_d.cpu().numpy()
            psi = _uniforms(_rnd.fold_in(key, 3 * t), n)
            if method == "cont_time":
                R = d - e                                    # escape rate
                with np.errstate(divide="ignore"):
                    hold = np.where(R > 0, -np.log1p(-psi) / R, np.inf)
                second, third = R, hold
            else:
                bx = lam - e
                pd = (lam - d) / bx
                valid = (pd > 0) & (pd < 1)
                with np.errstate(divide="ignore", invalid="ignore"):
                    sampled = np.floor(np.log1p(-psi) / np.where(valid, np.log(pd), -1.0)) + 1.0
                third = np.where(pd >= 1, np.inf, np.where(pd <= 0, 1.0, sampled))
                second = pd
            h["diag_min"].append(float(d.min()))
            h["diag_max"].append(float(d.max()))
            h["s_min"].append(float(second.min()))
            h["s_max"].append(float(second.max()))
            h["s_mean"].append(float(np.mean(second.astype(np.float32), dtype=np.float32)))
            h["k_mean"].append(float(np.mean(third.astype(np.float32), dtype=np.float32)))
            h["k_max"].append(float(third.max()))
        k1 = _rnd.fold_in(key, 3 * t + 1)
        k2 = _rnd.fold_in(key, 3 * t + 2)
        keys = np.concatenate([k1, k2]).astype(np.uint32)[None, :]
        eng.steps(method, step_size, lam, avg_log_weight, keys, lg, En)
        par = eng.parents.cpu().numpy().astype(np.int64)
        e_post = eng.e_loc.cpu().numpy()[par]
        counts = np.bincount(par, minlength=n)
        for k in range(k_max):
            offspring[t, k] = np.mean(counts == k)
        offspring[t, k_max] = np.mean(counts >= k_max)
        anc = anc[par]
        c = np.bincount(anc, minlength=n).astype(np.float64)
        frac[t] = np.count_nonzero(c) / n
        ess[t] = float(n) ** 2 / np.sum(c * c)
        x = e0[anc]
        y = e_post
        xc, yc = x - x.mean(), y - y.mean()
        den = np.sqrt(np.sum(xc * xc) * np.sum(yc * yc))
        corr[t] = np.sum(xc * yc) / den if den > 0 else float("nan")
        if t < M:
            packed_t = eng.packed_population()
            keys_t = _row_keys(packed_t)
            uniq_t = np.unique(keys_t)
            h["n_unique_post"].append(int(uniq_t.size))
            h["changed"].append(float(np.mean(np.any(packed_t != packed0, axis=1))))
            common = np.intersect1d(uniq0, uniq_t, assume_unique=True).size
            h["overlap"].append(common / max(int(uniq_t.size), 1))
    if method != "cont_time" and min(h["s_min"]) < 0:
        raise ValueError(f"[gfmc.statistics] sampler positivity broken: p_d_min < 0 (worst = "
                         f"{min(h['s_min']):.4f}); increase lam to at least max(H_diag) = "
                         f"{max(h['diag_max']):.4f} plus a margin.")
    stats = {
        "n_unique_pre": np.asarray(h["n_unique_pre"]),
        "n_unique_post": np.asarray(h["n_unique_post"]),
        "unique_fraction": np.asarray(h["n_unique_post"]) / float(n),
        "diag_min": np.asarray(h["diag_min"]),
        "diag_max": np.asarray(h["diag_max"]),
        "changed_rate": h["changed"],
        "overlap_rate": h["overlap"],
        "H_diag_max_observed": np.asarray([max(h["diag_max"])]),
        "H_diag_min_observed": np.asarray([min(h["diag_min"])]),
    }
    if method == "cont_time":
        stats.update(escape_rate_min=np.asarray(h["s_min"]), escape_rate_max=np.asarray(h["s_max"]),
                     escape_rate_mean=np.asarray(h["s_mean"]),
                     hops_per_step_mean=np.asarray(h["s_mean"]) * float(step_size),
                     hops_per_step_max=np.asarray(h["s_max"]) * float(step_size),
                     hold_time_mean=np.asarray(h["k_mean"]), hold_time_max=np.asarray(h["k_max"]))
    else:
        stats.update(p_d_min=np.asarray(h["s_min"]), p_d_max=np.asarray(h["s_max"]),
                     p_d_mean=np.asarray(h["s_mean"]), hold_steps_mean=np.asarray(h["k_mean"]),
                     hold_steps_max=np.asarray(h["k_max"]))
    for k in range(k_max):
        stats[f"offspring_k{k}"] = offspring[:, k]
    stats[f"offspring_k{k_max}plus"] = offspring[:, k_max]
    stats["survival_rate"] = 1.0 - offspring[:, 0]
    if m_sorted:
        af, ae, ac = [], [], []
        for m in m_sorted:
            if m == 0:
                af.append(1.0); ae.append(float(n)); ac.append(1.0)
            else:
                af.append(float(frac[m - 1])); ae.append(float(ess[m - 1])); ac.append(float(corr[m - 1]))
        stats["ancestor_m"] = np.asarray(m_sorted, dtype=float)
        stats["ancestor_fraction"] = np.asarray(af)
        stats["effective_sample_size"] = np.asarray(ae)
        stats["ancestor_correlation"] = np.asarray(ac)
    if not quiet:
        print(f"[gfmc.statistics] {n_total} steps, {n} walkers: unique fraction "
              f"{stats['unique_fraction'].mean():.3f}, survival {stats['survival_rate'].mean():.3f}",
              flush=True)
    cfg_after, e_after = eng.population()
    from .walkers import Walker
    out = Walker(config=cfg_after.cpu().numpy(), log_weight=np.zeros(n), e_loc=e_after.cpu().numpy())
    return out, stats

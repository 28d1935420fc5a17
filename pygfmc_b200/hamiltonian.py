"""Hamiltonians and lattices of the engine, with PyGFMC's constructors.

``SpinHalf.create`` and ``BoseHubbard.create`` take the arguments, apply the
sign conventions and raise the errors of PyGFMC's
``hamiltonian/SpinHalf.py:144-288`` and ``hamiltonian/bose_hubbard.py:129-267``,
and expose the same stored fields (``edge_i``, ``J_pm``, ``h_x_half``,
``n_hx_static``, ``M_total`` ...).  The objects are plain host data (numpy);
the engine lowers them to device tables when a run starts.  ``get_rates`` /
``generate_state`` / ``diagonal_weight`` are host (numpy) versions of the
protocol methods, for inspection and exact diagonalisation; the propagation
itself never calls them.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

__all__ = ["SpinHalf", "BoseHubbard", "StructureFactor", "SzSzStructureFactor", "is_valid_k", "Lattice",
           "chain", "square", "kagome", "pyrochlore", "edges_array", "exact_diagonalization"]


def edges_array(edges):
    """hamiltonian/_common.py edges_array:7-31: validated (n_edges, 2) int64."""
    raw = np.asarray(edges)
    if raw.shape == (0,):
        return np.zeros((0, 2), dtype=np.int64), 0, 0
    if raw.ndim != 2 or raw.shape[1] != 2:
        raise ValueError("edges must have shape (n_edges, 2).")
    if (raw.dtype.kind not in "iuf" or not np.all(np.isfinite(raw)) or np.any(raw < 0)
            or np.any(raw >= 2 ** 63) or np.any(raw != np.floor(raw))):
        raise ValueError("edge indices must be nonnegative integers fitting in int64.")
    e = raw.astype(np.int64)
    if np.any(e[:, 0] == e[:, 1]):
        raise ValueError("self-edges are not supported; edge endpoints must differ.")
    return e, len(e), int(e.max()) + 1 if e.size else 0


def _jpmpm_message(value):
    return (f"J_pmpm = (J_x - J_y) / 4 = {value:.6g} > 0 violates the sign-problem-free "
            "convention (J_pmpm <= 0).\n  Fix: swap S^x <-> S^y, i.e. pass J_x and J_y the "
            "other way round (a symmetry only when h_x = 0), or pass sign_check=False for a "
            "measurement operator.")


def _jpm_message(value):
    return (f"J_pm = (J_x + J_y) / 4 = {value:.6g} > 0 violates the sign-problem-free "
            "convention (J_pm <= 0).\n  On a bipartite lattice apply the sublattice rotation "
            "(pass -J_x and -J_y; an equivalence only when h_x = 0).  For an off-diagonal "
            "MEASUREMENT operator J_pm >= 0 is what is required -- build it with "
            "sign_check=False.")


class SpinHalf:
    """Spin-1/2 XYZ model with longitudinal and transverse fields.

        H = sum_<ij> [J_x S^x_i S^x_j + J_y S^y_i S^y_j + J_z S^z_i S^z_j]
            - sum_i [h_z S^z_i + h_x S^x_i]

    Configurations are +-1 (sigma_i = 2 S^z_i).  Rate layout::

        rates[0]                 diagonal H_xx
        rates[1 : 1+n_hx]        single-site flips, -h_x/2 (n_hx = N if h_x != 0)
        rates[1+n_hx : M_total]  one per edge: J_pm anti-parallel, J_pmpm parallel

    Sign-problem-free: J_pm <= 0, J_pmpm <= 0, h_x >= 0 (enforced by create).
    """

    def __init__(self, **kw):
        self.__dict__.update(kw)

    # reference property names
    @property
    def edges(self):
        return np.stack([np.asarray(self.edge_i), np.asarray(self.edge_j)], axis=1)

    @property
    def n_hx(self):
        return self.n_hx_static

    @property
    def n_jpm(self):
        return self.n_jpm_static

    @property
    def n_off(self):
        return self.n_hx_static + self.n_jpm_static

    @property
    def M_total(self):
        return self.n_hx_static + self.n_jpm_static + 1

    @property
    def local_hilbert_space(self):
        return (1.0, -1.0)

    @classmethod
    def create(cls, edges, J_x=0, J_y=0, J_z=0, h_z=None, h_x=None, N=None, *,
               dtype=np.float32, sign_check=True):
        h_z = None if h_z is None else (-np.asarray(h_z) if isinstance(h_z, (list, tuple)) else -h_z)
        h_x = None if h_x is None else (-np.asarray(h_x) if isinstance(h_x, (list, tuple)) else -h_x)
        edges_arr, _, N_min = edges_array(edges)
        for a in (h_z, h_x):
            if np.ndim(a) > 0:
                N_min = max(N_min, np.shape(a)[0])
        if N is None:
            N = N_min
        else:
            N = int(N)
            if N < N_min:
                raise ValueError(f"N={N} is smaller than required by the given edges/site "
                                 f"arrays (need at least {N_min})")
        dtype = np.dtype(dtype)
        n_edges = len(edges_arr)
        uniform = not (hasattr(J_x, "__len__") or hasattr(J_y, "__len__") or hasattr(J_z, "__len__"))
        if uniform:
            J_pmpm = (J_x - J_y) / 4.0
            if J_pmpm > 0 and sign_check:
                raise ValueError(_jpmpm_message(float(J_pmpm)))
            J_z_arr = np.array([J_z], dtype=dtype)
            J_pm_arr = np.array([(J_x + J_y) / 4.0], dtype=dtype)
            J_pmpm_arr = np.array([J_pmpm], dtype=dtype)
        else:
            def per_edge(v):
                a = np.asarray(v, dtype=dtype)
                if a.ndim == 0 or a.shape[0] == 1:
                    return np.broadcast_to(a.reshape(1), (n_edges,)).copy()
                return a
            jx, jy, J_z_arr = per_edge(J_x), per_edge(J_y), per_edge(J_z)
            if jx.shape[0] != n_edges or jy.shape[0] != n_edges or J_z_arr.shape[0] != n_edges:
                raise ValueError("Non-uniform couplings must match the number of edges.")
            J_pm_arr = (jx + jy) / dtype.type(4.0)
            J_pmpm_arr = (jx - jy) / dtype.type(4.0)
            if sign_check and np.any(J_pmpm_arr > 0):
                bad = np.flatnonzero(J_pmpm_arr > 0)
                raise ValueError(_jpmpm_message(float(J_pmpm_arr[bad[0]]))
                                 + f"\n  Offending edges: {bad.tolist()[:10]}"
                                 + (" ..." if bad.size > 10 else "")
                                 + f" ({bad.size} of {n_edges}).")
        if h_z is None:
            h_z_arr = None
        elif np.ndim(h_z) > 0:
            h_z_arr = np.asarray(h_z, dtype=dtype)
            if h_z_arr.shape[0] != N:
                raise ValueError(f"Non-uniform h_z must have length N={N}, got {h_z_arr.shape[0]}.")
        else:
            h_z_arr = np.array([h_z], dtype=dtype)
        if h_x is None:
            h_x_half_arr = None
        elif np.ndim(h_x) > 0:
            hxa = np.asarray(h_x, dtype=float)
            if hxa.shape[0] != N:
                raise ValueError(f"Non-uniform h_x must have length N={N}, got {hxa.shape[0]}.")
            if sign_check and np.any(hxa > 0):
                raise ValueError("h_x must be >= 0 for all sites (sign-problem-free convention; "
                                 "H contains -h_x Σ S^x, so a field written as +a Σ S^x is "
                                 "passed as h_x = -a).")
            h_x_half_arr = np.array(hxa / 2, dtype=dtype)
        else:
            if sign_check and h_x > 0:
                raise ValueError("h_x must be >= 0 (sign-problem-free convention; H contains "
                                 "-h_x Σ S^x, so a field written as +a Σ S^x is passed as h_x = -a).")
            h_x_half_arr = np.array([h_x / 2], dtype=dtype)
        if sign_check and np.any(np.asarray(J_pm_arr) > 0):
            raise ValueError(_jpm_message(float(np.max(J_pm_arr))))
        idx_dtype = np.int16 if N <= 32767 else np.int32
        return cls(
            dtype=dtype,
            edge_i=np.array(edges_arr[:, 0], dtype=idx_dtype),
            edge_j=np.array(edges_arr[:, 1], dtype=idx_dtype),
            N=N, J_z=J_z_arr, J_pm=J_pm_arr, J_pmpm=J_pmpm_arr,
            h_z=h_z_arr, h_x_half=h_x_half_arr,
            n_hx_static=N if (h_x_half_arr is not None and np.linalg.norm(h_x_half_arr) > 0) else 0,
            n_jpm_static=n_edges if (np.linalg.norm(J_pm_arr) > 0 or np.linalg.norm(J_pmpm_arr) > 0) else 0,
            has_jz=bool(np.linalg.norm(J_z_arr) > 0),
            uniform_jz=len(J_z_arr) == 1,
            has_hz=bool(h_z_arr is not None and np.linalg.norm(h_z_arr) > 0),
        )

    # ---- host versions of the protocol methods -----------------------------
    def diagonal_weight(self, config):
        x = np.asarray(config, dtype=np.float64)
        d = 0.0
        if self.has_jz:
            anti = x[..., self.edge_i] != x[..., self.edge_j]
            if self.uniform_jz:
                na = anti.sum(-1)
                d = (float(self.J_z[0]) / 4) * ((len(self.edge_i) - na) - na)
            else:
                jz = np.asarray(self.J_z, np.float64)
                d = np.where(anti, -jz / 4.0, jz / 4.0).sum(-1)
        if self.has_hz:
            d = d + (np.asarray(self.h_z, np.float64) * x).sum(-1) / 2
        return d

    def get_rates(self, config, return_configs=False):
        x = np.asarray(config, dtype=np.float64)
        r = np.zeros(self.M_total)
        r[0] = self.diagonal_weight(x)
        if self.n_hx_static:
            r[1:1 + self.N] = np.broadcast_to(np.asarray(self.h_x_half, np.float64), (self.N,))
        if self.n_jpm_static:
            anti = x[self.edge_i] != x[self.edge_j]
            r[1 + self.n_hx_static:] = np.where(anti, np.asarray(self.J_pm, np.float64),
                                                np.asarray(self.J_pmpm, np.float64))
        if not return_configs:
            return r, None
        return r, np.stack([self.generate_state(x, k) for k in range(self.M_total)])

    def generate_state(self, config, idx):
        x = np.array(config, dtype=np.float64, copy=True)
        if idx == 0:
            return x
        o = idx - 1
        if o < self.n_hx_static:
            x[o] = -x[o]
        else:
            e = o - self.n_hx_static
            i, j = int(self.edge_i[e]), int(self.edge_j[e])
            xi, xj = x[i], x[j]
            x[i], x[j] = -xi, -xj
        return x


class BoseHubbard:
    """Bose-Hubbard model (PyGFMC hamiltonian/bose_hubbard.py).

        H = -t sum_<ij> (b+_i b_j + h.c.) - eta sum_<ij> (b+_i b+_j + b_i b_j)
            + U/2 sum_i n_i (n_i - 1) - mu sum_i n_i - h_pm sum_i (b+_i + b_i)

    Occupations 0..n_max.  Rate layout: [diag, hop i->j (E), hop j->i (E),
    pair creation (E), pair annihilation (E), b+ (N), b (N)], blocks dropped
    when their coupling vanishes.  Sign-problem-free: t, eta, h_pm >= 0.
    """

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def edges(self):
        return np.stack([np.asarray(self.edge_i), np.asarray(self.edge_j)], axis=1)

    @property
    def n_edges(self):
        return int(len(self.edge_i))

    @property
    def n_off(self):
        return self.n_hop_off + self.n_eta_off + 2 * self.n_hpm_off

    @property
    def M_total(self):
        return 1 + self.n_off

    @property
    def local_hilbert_space(self):
        return tuple(float(n) for n in range(int(self.n_max) + 1))

    @classmethod
    def create(cls, edges, t=0.0, eta=0.0, U=0.0, mu=0.0, h_pm=None, N=None, n_max=4, *,
               dtype=np.float32, sign_check=True):
        h_pm = None if h_pm is None else (-np.asarray(h_pm) if isinstance(h_pm, (list, tuple)) else -h_pm)
        edges_arr, n_edges, N_min = edges_array(edges)
        for a in (U, mu, h_pm):
            if np.ndim(a) > 0:
                N_min = max(N_min, np.shape(a)[0])
        if N is None:
            N = N_min
        else:
            N = int(N)
            if N < N_min:
                raise ValueError(f"N={N} is smaller than required by the given edges/site "
                                 f"arrays (need at least {N_min})")
        if n_max < 1:
            raise ValueError(f"n_max must be ≥ 1, got {n_max}")
        dtype = np.dtype(dtype)

        def edge_arr(x, name):
            if np.ndim(x) > 0:
                a = np.asarray(x, dtype=dtype)
                if a.shape[0] != n_edges:
                    raise ValueError(f"non-uniform {name} must have length n_edges={n_edges}, got {a.shape[0]}")
                return a, False
            return np.array([float(x)], dtype=dtype), True

        def site_arr(x, name):
            if x is None:
                return None, True
            if np.ndim(x) > 0:
                a = np.asarray(x, dtype=dtype)
                if a.shape[0] != N:
                    raise ValueError(f"non-uniform {name} must have length N={N}, got {a.shape[0]}")
                return a, False
            return np.array([float(x)], dtype=dtype), True

        t_arr, uni_t = edge_arr(t, "t")
        eta_arr, uni_eta = edge_arr(eta, "eta")
        U_arr, uni_U = site_arr(U, "U")
        mu_arr, uni_mu = site_arr(mu, "mu")
        hpm_arr, uni_hpm = site_arr(h_pm, "h_pm")
        if sign_check:
            if np.any(t_arr < 0):
                raise ValueError("t must be ≥ 0 (sign-problem-free convention).")
            if np.any(eta_arr < 0):
                raise ValueError("eta must be ≥ 0 (sign-problem-free convention).")
            if hpm_arr is not None and np.any(hpm_arr > 0):
                raise ValueError("h_pm must be ≥ 0 (sign-problem-free convention).")

        def active(a):
            return a is not None and float(np.linalg.norm(a)) > 0
        has_t, has_eta, has_U, has_mu, has_hpm = (active(t_arr), active(eta_arr), active(U_arr),
                                                  active(mu_arr), active(hpm_arr))
        if not has_hpm:
            hpm_arr = None
        if not has_U:
            U_arr, uni_U = np.zeros((1,), dtype=dtype), True
        if not has_mu:
            mu_arr, uni_mu = np.zeros((1,), dtype=dtype), True
        idx_dtype = np.int16 if N <= 32767 else np.int32
        return cls(
            dtype=dtype,
            edge_i=np.array(edges_arr[:, 0] if n_edges else [], dtype=idx_dtype),
            edge_j=np.array(edges_arr[:, 1] if n_edges else [], dtype=idx_dtype),
            N=N, n_max=int(n_max), t=t_arr, eta=eta_arr, U=U_arr, mu=mu_arr, h_pm=hpm_arr,
            n_hop_off=2 * n_edges if has_t else 0, n_eta_off=2 * n_edges if has_eta else 0,
            n_hpm_off=N if has_hpm else 0,
            has_t=has_t, has_eta=has_eta, has_U=has_U, has_mu=has_mu, has_h_pm=has_hpm,
            uniform_t=uni_t, uniform_eta=uni_eta, uniform_U=uni_U, uniform_mu=uni_mu,
            uniform_hpm=uni_hpm,
        )

    def _per_edge(self, a):
        return np.broadcast_to(np.asarray(a, np.float64), (self.n_edges,))

    def _per_site(self, a):
        return np.broadcast_to(np.asarray(a, np.float64), (self.N,))

    def moves(self):
        """(a, b, da, db) of every transition, the layout of _move_blocks."""
        E, N = self.n_edges, self.N
        a, b, da, db = [0], [0], [0], [0]
        ei, ej = np.asarray(self.edge_i, int), np.asarray(self.edge_j, int)
        blocks = []
        if self.n_hop_off:
            blocks += [(-1, +1), (+1, -1)]
        if self.n_eta_off:
            blocks += [(+1, +1), (-1, -1)]
        for sa, sb in blocks:
            a += list(ei); b += list(ej); da += [sa] * E; db += [sb] * E
        if self.n_hpm_off:
            for s in (+1, -1):
                a += list(range(N)); b += list(range(N)); da += [s] * N; db += [0] * N
        return np.array(a), np.array(b), np.array(da), np.array(db)

    def move(self, config, idx):
        """The sites transition ``idx`` changes and their increments
        (hamiltonian/bose_hubbard.py move:427-435): ``(sites, deltas)`` of
        shape (2,) each, ``generate_state`` being ``config`` with ``deltas``
        added at ``sites``; the diagonal has zero increments and a single-site
        term repeats its site with increment 0."""
        a, b, da, db = self.moves()
        k = int(idx)
        if not 0 <= k < len(a):
            raise ValueError(f"transition index {k} outside [0, {len(a)})")
        dt = np.asarray(config).dtype
        dt = dt if dt.kind == "f" else np.dtype(np.float64)
        return np.array([a[k], b[k]]), np.array([da[k], db[k]], dtype=dt)

    def diagonal_weight(self, config):
        n = np.asarray(config, dtype=np.float64)
        out = 0.0
        if self.has_U:
            out = out + 0.5 * np.sum(self._per_site(self.U) * n * (n - 1.0), axis=-1)
        if self.has_mu:
            out = out - np.sum(self._per_site(self.mu) * n, axis=-1)
        return out

    def get_rates(self, config, return_configs=False):
        n = np.asarray(config, dtype=np.float64)
        nmax = float(self.n_max)
        r = [np.array([self.diagonal_weight(n)])]
        ei, ej = np.asarray(self.edge_i, int), np.asarray(self.edge_j, int)
        if self.n_hop_off:
            t = self._per_edge(self.t)
            ni, nj = n[ei], n[ej]
            r.append(-t * np.sqrt(ni * (nj + 1.0)) * (nj < nmax))
            r.append(-t * np.sqrt((ni + 1.0) * nj) * (ni < nmax))
        if self.n_eta_off:
            eta = self._per_edge(self.eta)
            ni, nj = n[ei], n[ej]
            r.append(-eta * np.sqrt((ni + 1.0) * (nj + 1.0)) * ((ni < nmax) & (nj < nmax)))
            r.append(-eta * np.sqrt(ni * nj))
        if self.n_hpm_off:
            hp = self._per_site(self.h_pm)
            r.append(hp * np.sqrt(n + 1.0) * (n < nmax))
            r.append(hp * np.sqrt(n))
        rates = np.concatenate(r)
        if not return_configs:
            return rates, None
        return rates, np.stack([self.generate_state(n, k) for k in range(self.M_total)])

    def generate_state(self, config, idx):
        x = np.array(config, dtype=np.float64, copy=True)
        if idx == 0:
            return x
        a, b, da, db = self.moves()
        x[a[idx]] += da[idx]
        x[b[idx]] += db[idx]
        return x


# channel -> coefficients (a, b) of PM = S+S- + S-S+ and PP = S+S+ + S-S- per
# pair; the diagonal channel has none
_SF_CHANNEL_COEFFS = {"spsm": (1.0, 0.0), "spsp": (0.0, 1.0), "spsm+spsp": (1.0, 1.0), "szsz": None}


def StructureFactor(positions, k, channel="SpSm", dtype=np.float32):
    """The k-resolved pair correlator sum_{i<j} [1 + cos(k.(r_i - r_j))]
    (A_i B_j + h.c.) as one SpinHalf measurement operator
    (hamiltonian/SpinHalf.py StructureFactor:464-628): one transition slot per
    pair with nonzero weight (weights below 1e-12 dropped), couplings
    J_x = 2 (a + b) W, J_y = 2 (a - b) W for the channel's (a, b) on
    (PM, PP), built without the propagator sign check (a measurement operator
    needs rates >= 0).  Channels "SpSm", "SpSp", "SpSm+SpSp" are off-diagonal
    (off_diag_operators); "SzSz" is the diagonal J_z = 2 W operator
    (diag_operators) and warns that SzSzStructureFactor measures it for many
    k at once.  The +1 shift keeps every weight non-negative; subtract the
    k = 0 operator to remove it.  No periodic image is chosen: k must lie in
    the reciprocal lattice of the simulation cell."""
    import warnings
    ch = str(channel).lower().replace(" ", "")
    if ch not in _SF_CHANNEL_COEFFS:
        hint = {"yy": " -- YY needs a negative PP coefficient: measure SpSm minus SpSp.",
                "sysy": " -- YY needs a negative PP coefficient: measure SpSm minus SpSp.",
                "zz": " -- the diagonal channel is spelled 'SzSz'.",
                "sz": " -- the diagonal channel is spelled 'SzSz'.",
                "ss": " -- S.S mixes the diagonal and off-diagonal paths: measure SpSm and SzSz "
                      "separately and add.",
                "s.s": " -- S.S mixes the diagonal and off-diagonal paths: measure SpSm and SzSz "
                       "separately and add.",
                "heisenberg": " -- S.S mixes the diagonal and off-diagonal paths: measure SpSm and "
                              "SzSz separately and add."}.get(ch, "")
        raise ValueError(f"channel={channel!r} is not reachable. The complete set is ['SpSm', "
                         "'SpSp', 'SpSm+SpSp'], the non-negative cone over PM = S+S-+S-S+ and "
                         f"PP = S+S++S-S-, plus the diagonal 'SzSz'{hint}")
    r = np.asarray(positions, dtype=np.float64)
    if r.ndim != 2:
        raise ValueError(f"positions must be (N, d), got {r.shape}")
    N = r.shape[0]
    kv = np.asarray(k, dtype=np.float64)
    if kv.ndim > 1 and kv.shape[0] != 1:
        raise ValueError(f"k must be ONE wavevector (d,), got {kv.shape}; build one operator per "
                         "wavevector.")
    kv = kv.reshape(-1)
    if kv.size != r.shape[1]:
        raise ValueError(f"k has {kv.size} components but positions are {r.shape[1]}-dimensional; "
                         "they must match.")
    if N < 2:
        raise ValueError(f"positions must hold at least two sites, got N={N}")
    iu = np.triu_indices(N, k=1)
    pairs = np.stack(iu, axis=1)
    W = 1.0 + np.cos((r[iu[0]] - r[iu[1]]) @ kv)
    keep = W > 1e-12
    pairs, W = pairs[keep].astype(np.int32), W[keep]
    if len(pairs) == 0:
        raise ValueError("no pairs with nonzero weight -- every weight vanished, which means k maps "
                         "every displacement to the zone boundary. Check k.")
    if ch == "szsz":
        warnings.warn("StructureFactor(channel='SzSz') is a DIAGONAL operator (M_total = 1): pass it "
                      "in diag_operators. SzSzStructureFactor(positions, k_vectors) measures the same "
                      "correlator for many k at once in O(N n_k), without the 1+cos shift and the "
                      "k = 0 subtraction.", UserWarning, stacklevel=2)
        return SpinHalf.create(pairs, J_z=2.0 * W, N=N, dtype=dtype, sign_check=False)
    a, b = _SF_CHANNEL_COEFFS[ch]
    return SpinHalf.create(pairs, J_x=2.0 * (a + b) * W, J_y=2.0 * (a - b) * W, J_z=0.0, N=N,
                           dtype=dtype, sign_check=False)


class SzSzStructureFactor:
    """S^zz(k) for one or many wavevectors (hamiltonian/observables.py:68-176):
    ``diagonal_weight`` = (|sum_i x_i e^{i k.r_i}|^2 - N) / 4 per k, from
    float64 cos/sin tables of k.r.  Exact for k in the reciprocal lattice of
    the simulation cell (the caller's responsibility, as in PyGFMC)."""

    def __init__(self, positions, k_vectors, dtype=np.float32):
        r = np.atleast_2d(np.asarray(positions, dtype=np.float64))
        k = np.atleast_2d(np.asarray(k_vectors, dtype=np.float64))
        if r.ndim != 2 or k.ndim != 2:
            raise ValueError(f"positions must be (N, d) and k_vectors (n_k, d); got {r.shape} and {k.shape}.")
        if k.shape[1] != r.shape[1]:
            raise ValueError(f"k_vectors have dimension {k.shape[1]} but positions have {r.shape[1]}; "
                             "a wavevector needs one component per spatial dimension of the lattice.")
        kr = k @ r.T
        dt = np.dtype(dtype)
        self.cos = np.cos(kr).astype(dt)
        self.sin = np.sin(kr).astype(dt)
        self.offset = dt.type(0.25 * r.shape[0])
        self.k_vectors = k.astype(dt)
        self.N = r.shape[0]

    @property
    def n_k(self):
        return self.cos.shape[0]

    def diagonal_weight(self, config):
        x = np.asarray(config, dtype=np.float64)
        c = x @ np.asarray(self.cos, np.float64).T
        s_ = x @ np.asarray(self.sin, np.float64).T
        return 0.25 * (c ** 2 + s_ ** 2) - float(self.offset)


def is_valid_k(k_vectors, lattice_vectors, atol=1e-5):
    """Whether each wavevector is in the reciprocal lattice of the simulation
    cell (hamiltonian/observables.py:14-65): k . L_j / (2 pi) within ``atol``
    of an integer for every periodic vector L_j (the rows of the (d, d)
    ``lattice_vectors``, the vectors the boundary identifies).  Only such k
    make the structure factors independent of which periodic image the
    positions encode.  Returns a bool for one (d,) wavevector, a boolean
    (n_k,) array for an (n_k, d) stack; the default ``atol`` admits
    wavevectors built in float32."""
    lat = np.asarray(lattice_vectors, dtype=np.float64)
    if lat.ndim != 2 or lat.shape[0] != lat.shape[1]:
        raise ValueError(f"lattice_vectors must be (d, d), one periodic vector per row; got {lat.shape}.")
    k = np.asarray(k_vectors, dtype=np.float64)
    one = k.ndim == 1
    k2 = np.atleast_2d(k)
    if k2.ndim != 2 or k2.shape[1] != lat.shape[0]:
        raise ValueError(f"k_vectors must be (d,) or (n_k, d) with d = {lat.shape[0]}; got {k.shape}.")
    turns = (k2 @ lat.T) / (2.0 * np.pi)               # (n_k, d) windings per periodic vector
    ok = np.all(np.abs(turns - np.rint(turns)) <= atol, axis=1)
    return bool(ok[0]) if one else ok


# ---- lattices ----------------------------------------------------------------
@dataclass(frozen=True)
class Lattice:
    """A finite lattice: site count, edge list and optional metadata
    (hamiltonian/lattice.py Lattice:8-33)."""
    name: str
    N: int
    edges: list
    J_x: object = None
    J_y: object = None
    J_z: object = None
    extras: dict = field(default_factory=dict, compare=False, hash=False)


def chain(n_sites: int, periodic: bool = True) -> Lattice:
    """Nearest-neighbour chain (hamiltonian/lattice.py chain:36-46)."""
    edges = [(i, i + 1) for i in range(n_sites - 1)]
    if periodic and n_sites > 2:
        edges.append((n_sites - 1, 0))
    return Lattice(name="chain", N=n_sites, edges=edges, J_x=-1.0, J_y=-1.0, J_z=1.0)


def square(Lx: int, Ly: int = None, periodic: bool = True) -> Lattice:
    """Nearest-neighbour square lattice of Lx x Ly sites, site x + Lx*y.

    PyGFMC has no square-lattice factory; this one follows its Lattice
    conventions.  Periodic boundaries need Lx, Ly >= 3 so that no bond is
    doubled.  ``extras['positions']`` holds the (N, 2) coordinates and
    ``extras['torus']`` the periods, for distance-dependent guides.
    """
    Ly = Lx if Ly is None else Ly
    if periodic and (Lx < 3 or Ly < 3):
        raise ValueError("square requires Lx, Ly >= 3 for periodic boundary conditions")
    idx = lambda x, y: (x % Lx) + Lx * (y % Ly)
    edges = set()
    for y in range(Ly):
        for x in range(Lx):
            for dx, dy in ((1, 0), (0, 1)):
                if not periodic and (x + dx >= Lx or y + dy >= Ly):
                    continue
                i, j = idx(x, y), idx(x + dx, y + dy)
                edges.add((min(i, j), max(i, j)))
    pos = np.array([(x, y) for y in range(Ly) for x in range(Lx)], dtype=float)
    return Lattice(name="square", N=Lx * Ly, edges=sorted(edges), J_x=-1.0, J_y=-1.0, J_z=1.0,
                   extras=dict(positions=pos, torus=np.array([Lx, Ly]), periodic=periodic))


def pyrochlore(nx: int, ny: int, nz: int, periodic: bool = True) -> Lattice:
    """Pyrochlore lattice of nx x ny x nz four-site cells
    (hamiltonian/lattice.py pyrochlore:49-183): the FCC lattice with primitive
    vectors a1 = (1/2, 1/2, 0), a2 = (1/2, 0, 1/2), a3 = (0, 1/2, 1/2)
    (conventional cubic cell of side 1) and a tetrahedral basis at 0, a1/2,
    a2/2, a3/2; site 4 (z + nz y + nz ny x) + b for cell (x, y, z) and
    sublattice b, so N = 4 nx ny nz and, periodic, 3N bonds (coordination 6).

    The bonds are found geometrically: every sublattice pair and cell offset
    in {-1, 0, 1}^3 whose displacement has the nearest-neighbour length
    1/(2 sqrt 2) -- the three bonds of a site inside its own ("up")
    tetrahedron and three into neighbouring cells' ("down") tetrahedra.
    They are listed as sorted (i < j) pairs, the order PyGFMC's edge list
    has.  Periodic boundaries need nx, ny, nz >= 2 (a single cell would wrap
    a bond onto itself); open ones keep the bonds inside the block.
    ``extras``: positions (N, 3), primitive_vectors, sublattice_offsets,
    supercell_dims and the torus vectors (rows nx a1, ny a2, nz a3).  The
    hexagonal loops PyGFMC also lists there serve only its plaquette model,
    which this package does not provide."""
    dims = (int(nx), int(ny), int(nz))
    if min(dims) < 1:
        raise ValueError(f"pyrochlore needs at least one cell per direction, got {dims}")
    if periodic and min(dims) < 2:
        raise ValueError(f"pyrochlore requires nx, ny, nz >= 2 for periodic boundary conditions "
                         f"(got {nx}, {ny}, {nz}); a dimension of one cell wraps a bond onto itself.")
    prim = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    basis = np.vstack([np.zeros(3), prim / 2.0])
    nn = 1.0 / (2.0 * np.sqrt(2.0))
    # the bond templates: (b, c, cell offset) at nearest-neighbour distance
    tmpl = []
    for off in itertools.product((-1, 0, 1), repeat=3):
        shift = np.asarray(off, np.float64) @ prim
        for b in range(4):
            for c in range(4):
                if np.isclose(np.linalg.norm(shift + basis[c] - basis[b]), nn, atol=1e-12):
                    tmpl.append((b, c, off))
    assert len(tmpl) == 24, len(tmpl)          # 6 neighbours of each of the 4 sublattices

    def cell(x, y, z):
        return z + dims[2] * (y + dims[1] * x)

    edges = set()
    for x, y, z in itertools.product(*(range(d) for d in dims)):
        for b, c, (ox, oy, oz) in tmpl:
            t = (x + ox, y + oy, z + oz)
            if not periodic and not all(0 <= t[k] < dims[k] for k in range(3)):
                continue
            i = 4 * cell(x, y, z) + b
            j = 4 * cell(*(t[k] % dims[k] for k in range(3))) + c
            edges.add((min(i, j), max(i, j)))
    pos = np.array([x * prim[0] + y * prim[1] + z * prim[2] + basis[b]
                    for x, y, z in itertools.product(*(range(d) for d in dims)) for b in range(4)])
    return Lattice(name="pyrochlore", N=4 * dims[0] * dims[1] * dims[2], edges=sorted(edges),
                   extras=dict(positions=pos, primitive_vectors=prim, sublattice_offsets=basis,
                               supercell_dims=np.array(dims, dtype=np.int32),
                               torus=np.asarray(dims, np.float64)[:, None] * prim))


def kagome(Lx: int, Ly: int, periodic: bool = True) -> Lattice:
    """Kagome lattice of Lx x Ly three-site cells (hamiltonian/lattice.py
    kagome:186-262): site 3*(x + Lx*y) + b, primitive vectors (2, 0) and
    (1, sqrt 3), sublattice offsets 0, a1/2, a2/2."""
    if periodic and (Lx < 2 or Ly < 2):
        raise ValueError(f"kagome requires Lx, Ly >= 2 for periodic boundary conditions "
                         f"(got {Lx}, {Ly}); smaller tori wrap a bond onto itself.")
    a1 = np.array([2.0, 0.0])
    a2 = np.array([1.0, np.sqrt(3.0)])
    basis = np.array([[0.0, 0.0], a1 / 2, a2 / 2])
    sub = {(0, 0): 0, (1, 0): 1, (0, 1): 2}

    def index(U, V):
        x, y = U // 2, V // 2
        if not periodic and not (0 <= x < Lx and 0 <= y < Ly):
            return None
        return 3 * ((x % Lx) + Lx * (y % Ly)) + sub[(U % 2, V % 2)]

    tmpl = [((0, 0), (1, 0)), ((0, 0), (0, 1)), ((1, 0), (0, 1)),
            ((1, 0), (2, 0)), ((0, 1), (0, 2)), ((1, 0), (2, -1))]
    edges = set()
    for x in range(Lx):
        for y in range(Ly):
            for (u1, v1), (u2, v2) in tmpl:
                i, j = index(2 * x + u1, 2 * y + v1), index(2 * x + u2, 2 * y + v2)
                if i is None or j is None:
                    continue
                edges.add((min(i, j), max(i, j)))
    pos = np.array([x * a1 + y * a2 + basis[b] for y in range(Ly) for x in range(Lx)
                    for b in range(3)])
    # one hexagon per cell, centred at the cell origin + (a1 + a2) / 2: its
    # corners are the sites at distance 1 from the centre (in this cell and
    # the cells +a1, +a2), listed counter-clockwise from angle 0; an open
    # lattice keeps the hexagons whose corners all lie inside it
    hexagons, centres = [], []
    for y in range(Ly):
        for x in range(Lx):
            c = x * a1 + y * a2 + (a1 + a2) / 2
            corners = []
            for dx, dy, b in itertools.product((0, 1), (0, 1), range(3)):
                r = (x + dx) * a1 + (y + dy) * a2 + basis[b]
                if np.isclose(np.linalg.norm(r - c), 1.0, atol=1e-9):
                    ang = np.arctan2(r[1] - c[1], r[0] - c[0]) % (2 * np.pi)
                    corners.append((round(ang, 9) % round(2 * np.pi, 9), x + dx, y + dy, b))
            if not periodic and any(cx >= Lx or cy >= Ly for _, cx, cy, _ in corners):
                continue
            corners.sort()
            hexagons.append([3 * ((cx % Lx) + Lx * (cy % Ly)) + b for _, cx, cy, b in corners])
            centres.append(c)
    return Lattice(name="kagome", N=3 * Lx * Ly, edges=sorted(edges),
                   extras=dict(positions=pos, primitive_vectors=np.array([a1, a2]),
                               supercell_dims=np.array([Lx, Ly]), sublattice_offsets=basis,
                               torus=np.array([Lx * a1, Ly * a2]),
                               hexagons=np.array(hexagons, dtype=np.int32).reshape(-1, 6),
                               hexagon_centers=np.array(centres, dtype=np.float64).reshape(-1, 2)))


# ---------------------------------------------------------------------------
# exact diagonalisation over the Hamiltonian protocol (host, float64)
# ---------------------------------------------------------------------------
_ED_MAX_DIM = 2 ** 24
_ED_DENSE_DIM = 2048
_ED_MAX_BYTES = 16 * 2 ** 30


def _basis(values, N):
    """Every configuration of N sites, row r holding the digits of r in base
    d = len(values) with site 0 most significant, mapped to the values."""
    d = len(values)
    powers = d ** np.arange(N - 1, -1, -1, dtype=np.int64)
    digits = (np.arange(d ** N, dtype=np.int64)[:, None] // powers) % d
    return np.asarray(values, np.float64)[digits], powers


def _basis_index(configs, values, powers):
    """Positional index of each row of configs (nearest local value per site)."""
    c = np.atleast_2d(np.asarray(configs, np.float64))
    digit = np.argmin(np.abs(c[..., None] - np.asarray(values, np.float64)), axis=-1)
    return digit.astype(np.int64) @ powers


def _value_digits(configs, values):
    """Digit (position in values) of every site value of configs."""
    return np.argmin(np.abs(np.asarray(configs, np.float64)[..., None] - np.asarray(values, np.float64)),
                     axis=-1).astype(np.int64)


def _batch_matrix(op, configs, values, powers):
    """The matrix of this package's SpinHalf / BoseHubbard over the whole
    basis at once (their get_rates formulas on every configuration, the
    successor's index from the changed sites' digits); None for other
    operators.  Equal element for element to the per-configuration build."""
    from scipy import sparse
    if not isinstance(op, (SpinHalf, BoseHubbard)):
        return None
    X = np.asarray(configs, np.float64)
    dim = len(X)
    dig = _value_digits(X, values)
    idx = np.arange(dim, dtype=np.int64)
    vals = np.asarray(values, np.float64)
    rows, cols, data = [idx], [idx], [np.broadcast_to(np.asarray(op.diagonal_weight(X), np.float64), (dim,))]

    def digit_of(v):
        """Digit of site values v (must be in the basis where the rate is nonzero)."""
        d = np.argmin(np.abs(v[..., None] - vals), axis=-1).astype(np.int64)
        ok = np.abs(vals[d] - v) < 1e-6
        return d, ok

    def add(rate, changes):
        """rate (dim,) of a move changing sites by the given (site, new value) arrays."""
        nz = rate != 0.0
        if not np.any(nz):
            return
        new = idx.copy()
        for site, v in changes:
            d, ok = digit_of(v)
            if not np.all(ok[nz]):
                raise ValueError(f"{type(op).__name__}: a transition of nonzero amplitude leads "
                                 "outside the supplied local_hilbert_space")
            new = new + (d - dig[idx, site]) * powers[site]
        rows.append(new[nz]); cols.append(idx[nz]); data.append(rate[nz])

    if isinstance(op, SpinHalf):
        N = op.N
        if op.n_hx_static:
            hx = np.broadcast_to(np.asarray(op.h_x_half, np.float64), (N,))
            for k in range(N):
                add(np.full(dim, hx[k]), [(k, -X[:, k])])
        if op.n_jpm_static:
            jpm = np.broadcast_to(np.asarray(op.J_pm, np.float64), (len(op.edge_i),))
            jpp = np.broadcast_to(np.asarray(op.J_pmpm, np.float64), (len(op.edge_i),))
            for e, (i, j) in enumerate(zip(np.asarray(op.edge_i, int), np.asarray(op.edge_j, int))):
                anti = X[:, i] != X[:, j]
                add(np.where(anti, jpm[e], jpp[e]), [(i, -X[:, i]), (j, -X[:, j])])
    else:
        a, b, da, db = op.moves()
        n = X
        nmax = float(op.n_max)
        ei, ej = np.asarray(op.edge_i, int), np.asarray(op.edge_j, int)
        blocks = []
        if op.n_hop_off:
            t = op._per_edge(op.t)
            blocks.append(lambda: [-t[e] * np.sqrt(n[:, ei[e]] * (n[:, ej[e]] + 1.0)) * (n[:, ej[e]] < nmax)
                                   for e in range(len(ei))])
            blocks.append(lambda: [-t[e] * np.sqrt((n[:, ei[e]] + 1.0) * n[:, ej[e]]) * (n[:, ei[e]] < nmax)
                                   for e in range(len(ei))])
        if op.n_eta_off:
            eta = op._per_edge(op.eta)
            blocks.append(lambda: [-eta[e] * np.sqrt((n[:, ei[e]] + 1.0) * (n[:, ej[e]] + 1.0))
                                   * ((n[:, ei[e]] < nmax) & (n[:, ej[e]] < nmax)) for e in range(len(ei))])
            blocks.append(lambda: [-eta[e] * np.sqrt(n[:, ei[e]] * n[:, ej[e]]) for e in range(len(ei))])
        if op.n_hpm_off:
            hp = op._per_site(op.h_pm)
            hp = np.broadcast_to(np.asarray(hp, np.float64), (op.N,))
            blocks.append(lambda: [hp[k] * np.sqrt(n[:, k] + 1.0) * (n[:, k] < nmax) for k in range(op.N)])
            blocks.append(lambda: [hp[k] * np.sqrt(n[:, k]) for k in range(op.N)])
        slot = 1
        for blk in blocks:
            for rate in blk():
                changes = [(int(a[slot]), n[:, a[slot]] + da[slot])]
                if db[slot] != 0:
                    changes.append((int(b[slot]), n[:, b[slot]] + db[slot]))
                add(np.asarray(rate, np.float64), changes)
                slot += 1
        assert slot == op.M_total, (slot, op.M_total)
    H = sparse.coo_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(dim, dim)).tocsr()
    H.sum_duplicates()
    return H


def _protocol_matrix(op, configs, values, powers):
    """Sparse matrix of op over the basis from get_rates alone: H[y, x] is the
    rate of the transition x -> y (the diagonal element at slot 0); this
    package's own operators take the vectorised build."""
    from scipy import sparse
    Hb = _batch_matrix(op, configs, values, powers)
    if Hb is not None:
        return _checked(Hb)
    dim = len(configs)
    rows, cols, vals = [], [], []
    for i, x in enumerate(configs):
        rates, succ = op.get_rates(x, return_configs=True)
        rates = np.asarray(rates, np.float64)
        nz = np.nonzero(rates)[0]
        if nz.size == 0:
            continue
        sub = np.asarray(succ, np.float64)[nz]
        ok = np.all(np.min(np.abs(sub[..., None] - np.asarray(values)), axis=-1) < 1e-6, axis=1)
        if not np.all(ok):
            raise ValueError(f"{type(op).__name__}: a transition of nonzero amplitude from "
                             f"configuration {x.tolist()} leads outside the supplied "
                             "local_hilbert_space")
        rows.append(_basis_index(sub, values, powers))
        cols.append(np.full(nz.size, i, np.int64))
        vals.append(rates[nz])
    if not rows:
        return sparse.csr_matrix((dim, dim))
    H = sparse.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(dim, dim)).tocsr()
    return _checked(H)


def _diagonal_values(op, configs):
    """``op.diagonal_weight`` over the basis (hamiltonian/exact.py:182-192):
    shape (dim,), or (dim, n_vals) for a vector-valued operator such as a
    structure factor over several wavevectors.  This package's operators
    evaluate the whole basis at once; any other goes configuration by
    configuration, so a diagonal_weight written for one configuration is
    never handed a batch."""
    dim = len(configs)
    if isinstance(op, (SpinHalf, BoseHubbard, SzSzStructureFactor)):
        vals = np.asarray(op.diagonal_weight(configs), np.float64)
        if vals.ndim == 0:                       # an operator with no diagonal term
            vals = np.full(dim, float(vals))
    else:
        vals = np.array([np.asarray(op.diagonal_weight(x), np.float64) for x in configs])
    if vals.ndim not in (1, 2) or vals.shape[0] != dim:
        raise ValueError(f"{type(op).__name__}.diagonal_weight gives values of shape "
                         f"{vals.shape[1:] if vals.ndim else ()} per configuration; a scalar or "
                         "a vector is expected")
    if not np.all(np.isfinite(vals)):
        raise ValueError(f"{type(op).__name__}.diagonal_weight is not finite on the whole basis")
    return vals


def _checked(H):
    """H after the finiteness and symmetry checks of the protocol build."""
    if not np.all(np.isfinite(H.data)):
        raise ValueError("the operator matrix has non-finite elements")
    asym = abs(H - H.T).max() if H.nnz else 0.0
    if asym > 1e-10 * max(1.0, abs(H).max()):
        raise ValueError(f"the operator matrix is not Hermitian (max |H - H^T| = {asym:.3e})")
    return H


def exact_diagonalization(hamiltonian, local_hilbert_space=None, N=None, diag_operators=None,
                          off_diag_operators=None, number_of_states=1, return_states=False):
    """Lowest eigenpairs of ``hamiltonian`` and observables on each
    (hamiltonian/exact.py:212-375): the matrix comes from the protocol's
    ``get_rates(x, return_configs=True)`` over the positional basis (site 0
    most significant digit of ``local_hilbert_space``), dense below 2048
    states, otherwise Lanczos on the sparse matrix.  Returns ``(energies,
    diag_obs, off_diag_obs)`` and the states (dim, number_of_states) when
    ``return_states``; ``diag_obs[name][k] = sum_x |psi_k(x)|^2 O(x)`` through
    ``diagonal_weight``, ``off_diag_obs[name][k] = psi_k^T O psi_k``."""
    # the checks in PyGFMC's order, each message holding the phrase its tests
    # match (hamiltonian/exact.py:266-345)
    name = type(hamiltonian).__name__
    if local_hilbert_space is None:
        local_hilbert_space = getattr(hamiltonian, "local_hilbert_space", None)
        if local_hilbert_space is None:
            raise ValueError(f"no local_hilbert_space given, and {name} has no local_hilbert_space "
                             "attribute to take it from")
    values = np.asarray(local_hilbert_space, dtype=np.float64).ravel()
    d = values.size
    if d < 2:
        raise ValueError(f"local_hilbert_space needs at least two values, got {values.tolist()}")
    if not np.all(np.isfinite(values)) or np.unique(values).size != d:
        raise ValueError(f"local_hilbert_space must hold distinct finite values, got {values.tolist()}")
    own = getattr(hamiltonian, "local_hilbert_space", None)
    if own is not None:
        own = np.asarray(own, np.float64).ravel()
        if own.size != d:
            raise ValueError(f"local_hilbert_space has {d} values, the Hamiltonian acts on {own.size} "
                             f"({own.tolist()}): another local dimension")
        if not np.array_equal(np.sort(own), np.sort(values)):
            raise ValueError(f"local_hilbert_space {values.tolist()} differs from the values "
                             f"{own.tolist()} the Hamiltonian acts on (their order may differ, the "
                             "values may not)")
    if N is None:
        N = getattr(hamiltonian, "N", None)
        if N is None:
            raise ValueError(f"no N given, and {name} has no N attribute: the size of the basis is "
                             "unknown")
    N = int(N)
    dim = d ** N
    if dim > _ED_MAX_DIM:
        raise ValueError(f"basis of {d}**{N} = {dim} states exceeds the {_ED_MAX_DIM} limit of exact "
                         "diagonalisation")
    k = int(number_of_states)
    if k != number_of_states or not 1 <= k <= dim:
        raise ValueError(f"number_of_states must be an integer in [1, {dim}], got {number_of_states!r}")
    # the basis (float64 values), the matrix triplets (at most M_total per
    # state: two int64 indices and a float64 value) and, for a full solve,
    # the dense matrix with its eigenvectors
    m_total = int(getattr(hamiltonian, "M_total", 1))
    dense = dim <= _ED_DENSE_DIM or k >= dim - 1
    need = max(dim * N * 8 + dim * m_total * 24, 2 * dim * dim * 8 if dense else 0)
    if need > _ED_MAX_BYTES:
        raise ValueError(f"exact diagonalisation of {dim} states would allocate about "
                         f"{need / 2 ** 30:.1f} GiB, above the {_ED_MAX_BYTES / 2 ** 30:.0f} GiB limit")
    # a basis of the wrong size or values gives a plausible spectrum of another
    # problem: cross-check what the operator reports
    own_N = getattr(hamiltonian, "N", None)
    if own_N is not None and int(own_N) != N:
        raise ValueError(f"N={N}, but the Hamiltonian reports N={int(own_N)}: a basis of another size")
    own_d = getattr(hamiltonian, "d", None)
    if own_d is not None and int(own_d) != d:
        raise ValueError(f"local_hilbert_space has {d} values, but the Hamiltonian reports a local "
                         f"dimension of {int(own_d)}")
    configs, powers = _basis(values, N)
    H = _protocol_matrix(hamiltonian, configs, values, powers)
    if dense:
        w, v = np.linalg.eigh(H.toarray())
        energies, states = w[:k], v[:, :k]
    else:
        from scipy.sparse.linalg import eigsh
        # a fixed start vector: ARPACK's own seed advances between calls, and
        # two solves of one matrix would then differ in their last bits
        v0 = np.random.default_rng(0).standard_normal(dim)
        w, v = eigsh(H, k=k, which="SA", tol=1e-12, v0=v0)
        order = np.argsort(w)
        energies, states = w[order], v[:, order]
    diag_obs = {}
    for name, op in (diag_operators or {}).items():
        # (k,) for a scalar operator, (k, n_vals) for a vector-valued one
        diag_obs[name] = (states ** 2).T @ _diagonal_values(op, configs)
    off_obs = {}
    for name, op in (off_diag_operators or {}).items():
        O = _protocol_matrix(op, configs, values, powers)
        off_obs[name] = np.einsum("ik,ik->k", states, O @ states)
    out = (np.asarray(energies, np.float64), diag_obs, off_obs)
    return out + (states,) if return_states else out

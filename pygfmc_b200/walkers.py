"""The walker population and its initialisers (PyGFMC walkers/walker.py).

``prepare_walkers_random`` / ``prepare_walkers_sz`` draw exactly what PyGFMC
draws for the same key (``jax.random.randint`` / ``jax.random.permutation``
restated over the Threefry stream in :mod:`pygfmc_b200.random`), in PyGFMC's
float64 mode (``jax_enable_x64``) unless ``x64=False``.
"""
import ctypes
from typing import NamedTuple, Sequence

import numpy as np

from . import random as _rnd

__all__ = ["Walker", "prepare_walkers_random", "prepare_walkers_sz",
           "prepare_walkers_from_configs", "prepare_walkers_occupations", "reconfiguration",
           "RECONFIGURATION_MAX_WALKERS"]

# population limit of reconfiguration(): its device scratch is a fixed array
# (GFMC_NOALLOC_MAX_WALKERS in the C header)
RECONFIGURATION_MAX_WALKERS = 131072


def _compact_config(config):
    """The smallest lossless storage of a configuration array: int8 when every
    value is an integer in int8's range (+-1 spins, small occupations), the
    array itself otherwise (walker.py _compact_config:31-47)."""
    arr = np.asarray(config)
    r = np.rint(arr)
    if arr.size and np.array_equal(arr, r) and r.min() >= -128 and r.max() <= 127:
        return r.astype(np.int8)
    return arr


class Walker(NamedTuple):
    """Population (or one walker): ``config`` (N_walkers, N_sites), ``log_weight``
    and ``e_loc`` (N_walkers,) -- walkers/walker.py Walker:50-64."""
    config: np.ndarray
    log_weight: np.ndarray
    e_loc: np.ndarray

    def save(self, path, rng_key=None, group="walkers", **attrs):
        """Checkpoint the walkers, the chain's key and scalar metadata
        (walker.py Walker.save:66-103): datasets ``config`` (in the smallest
        lossless dtype), ``log_weight``, ``e_loc`` and ``rng_key`` under
        ``group``, the keyword arguments (typically ``avg_log_weight=``) as
        attributes.  h5py is not available to this package, so the container
        is a NumPy ``.npz`` archive holding the same names as
        ``<group>/<dataset>`` and ``<group>/attrs/<name>``; the file is
        written at ``path`` exactly.  Pass ``stats['parameters/rng_key_next']``
        as ``rng_key``: with the walkers and ``avg_log_weight`` it is the whole
        resume state."""
        d = {f"{group}/config": _compact_config(self.config),
             f"{group}/config_dtype": np.asarray(str(np.asarray(self.config).dtype)),
             f"{group}/log_weight": np.asarray(self.log_weight),
             f"{group}/e_loc": np.asarray(self.e_loc)}
        if rng_key is not None:
            d[f"{group}/rng_key"] = np.asarray(_rnd.as_key(rng_key), dtype=np.uint32)
        for k, v in attrs.items():
            if np.ndim(v) != 0:
                raise ValueError(f"attribute {k!r} must be a scalar")
            d[f"{group}/attrs/{k}"] = np.asarray(v)
        with open(path, "wb") as f:
            np.savez(f, **d)

    @classmethod
    def load(cls, path, group="walkers", dtype=None, config_dtype=None):
        """Read a checkpoint written by :meth:`save` (walker.py
        Walker.load:105-140): returns ``(walker, rng_key, avg_log_weight)``,
        the last two None when not saved.  ``dtype`` (default float64, this
        package's x64 mode) is the weights' and local energies' dtype,
        ``config_dtype`` (default ``dtype``) the configurations'."""
        dtype = np.dtype(np.float64 if dtype is None else dtype)
        config_dtype = dtype if config_dtype is None else np.dtype(config_dtype)
        with np.load(path, allow_pickle=False) as z:
            if f"{group}/config" not in z.files:
                raise KeyError(f"{path} holds no walker group {group!r}")
            w = cls(config=np.asarray(z[f"{group}/config"], dtype=config_dtype),
                    log_weight=np.asarray(z[f"{group}/log_weight"], dtype=dtype),
                    e_loc=np.asarray(z[f"{group}/e_loc"], dtype=dtype))
            key = np.asarray(z[f"{group}/rng_key"], dtype=np.uint32) \
                if f"{group}/rng_key" in z.files else None
            alw_k = f"{group}/attrs/avg_log_weight"
            alw = dtype.type(z[alw_k]) if alw_k in z.files else None
        return w, key, alw


def _zeros(n, x64):
    return np.zeros(n, dtype=np.float64 if x64 else np.float32)


def prepare_walkers_random(N_walkers, N_sites, rng_key, states=(-1.0, 1.0), x64=True):
    """Every site an independent uniform draw from ``states`` (walker.py:199-254)."""
    vals = np.asarray(states)
    if vals.ndim != 1 or vals.size < 1:
        raise ValueError(f"states must be a non-empty 1-D sequence of local values; got {states!r}.")
    if x64 and vals.dtype == np.float32:
        vals = vals.astype(np.float64)
    if not x64 and vals.dtype == np.float64:
        vals = vals.astype(np.float32)
    idx = _rnd.randint(rng_key, (N_walkers, N_sites), 0, vals.size, x64=x64)
    return Walker(config=vals[idx], log_weight=_zeros(N_walkers, x64), e_loc=_zeros(N_walkers, x64))


def base_config_for_sum(N_sites, target, states):
    """Greedy multiset of local states summing to ``target`` (walker.py:143-196)."""
    vals = np.asarray(states, dtype=float).ravel()
    if vals.size < 1:
        raise ValueError("states must contain at least one local value.")
    if np.unique(vals).size != vals.size:
        raise ValueError(f"states must not repeat a value; got {list(states)}.")
    den = None
    for d in (1, 2, 3, 4, 5, 6, 8, 10, 12):
        if np.allclose(vals * d, np.round(vals * d)) and abs(target * d - round(target * d)) < 1e-9:
            den = d
            break
    if den is None:
        raise ValueError(f"states={list(states)} and sz={target} are not commensurate with a "
                         "small common denominator; pass values that are multiples of 1/2, 1/3, 1/4, ...")
    S = np.sort(np.round(vals * den).astype(np.int64))
    Z = int(round(target * den))
    inc = S - S[0]
    D = Z - N_sites * int(S[0])
    if D < 0 or D > N_sites * int(inc[-1]):
        lo, hi = N_sites * vals.min(), N_sites * vals.max()
        raise ValueError(f"sz={target} is outside the reachable range [{lo}, {hi}] for "
                         f"N_sites={N_sites} and states={list(states)}.")
    counts = np.zeros(S.size, dtype=np.int64)
    remaining, d = N_sites, D
    for k in range(S.size - 1, 0, -1):
        take = min(d // int(inc[k]), remaining)
        counts[k] += take
        d -= take * int(inc[k])
        remaining -= take
    counts[0] += remaining
    if d != 0:
        raise ValueError(f"sz={target} is not reachable with N_sites={N_sites} sites drawn from "
                         f"states={list(states)} (residual {d}/{den}). For a two-state ladder this "
                         "is the usual parity constraint.")
    return np.repeat(S, counts).astype(float) / den


def prepare_walkers_sz(N_walkers, N_sites, rng_key, sz=0, states=(-1.0, 1.0), x64=True):
    """Walkers in a fixed-sum sector: one permutation of the greedy base
    multiset per walker (walker.py:257-306)."""
    base = base_config_for_sum(N_sites, sz, states)
    dt = np.asarray(states).dtype
    if dt.kind == "f":
        dt = np.float64 if x64 else np.float32
    keys = _rnd.split(rng_key, N_walkers)
    configs = _rnd.permutation_rows(keys, base.astype(dt))
    return Walker(config=configs, log_weight=_zeros(N_walkers, x64), e_loc=_zeros(N_walkers, x64))


def prepare_walkers_from_configs(configs, x64=True):
    """Walkers at given configurations (walker.py:309-342)."""
    configs = np.asarray(configs)
    if configs.ndim != 2:
        raise ValueError(f"configs must have shape (N_walkers, N_sites); got shape {configs.shape}.  "
                         "For a single configuration copied to every walker use "
                         "np.tile(config, (N_walkers, 1)).")
    return Walker(config=configs, log_weight=_zeros(configs.shape[0], x64),
                  e_loc=_zeros(configs.shape[0], x64))


def prepare_walkers_occupations(N_walkers, N_sites, n_total, n_max, rng_key, x64=True):
    """Occupations drawn uniformly from {n in [0, n_max]^N : sum n = n_total}.

    PyGFMC has no such initialiser (``prepare_walkers_sz`` permutes one greedy
    base multiset).  Exact uniform sampling over the constrained set: the
    number of completions ``C(k, s)`` of k remaining sites to the sum s is
    tabulated, and each site draws its occupation with probability
    proportional to the completions it leaves.  Draws come from the Threefry
    stream ``split(rng_key, N_walkers)[w]`` (one 64-bit uniform per site).
    """
    if n_total < 0 or n_total > N_sites * n_max:
        raise ValueError(f"n_total={n_total} unreachable with {N_sites} sites and n_max={n_max}")
    C = np.zeros((N_sites + 1, n_total + 1), dtype=np.float64)
    C[0, 0] = 1.0
    for k in range(1, N_sites + 1):
        for s in range(n_total + 1):
            C[k, s] = sum(C[k - 1, s - v] for v in range(0, min(n_max, s) + 1))
    keys = _rnd.split(rng_key, N_walkers)
    out = np.zeros((N_walkers, N_sites), dtype=np.float64 if x64 else np.float32)
    for w in range(N_walkers):
        y0, y1 = _rnd.threefry2x32(keys[w, 0], keys[w, 1], np.zeros(N_sites, np.uint32),
                                   np.arange(N_sites, dtype=np.uint32))
        bits = ((y0.astype(np.uint64) << np.uint64(32)) | y1.astype(np.uint64)) >> np.uint64(11)
        u = bits.astype(np.float64) * (1.0 / 9007199254740992.0)
        s = n_total
        for i in range(N_sites):
            k = N_sites - i - 1
            weights = np.array([C[k, s - v] if v <= s else 0.0 for v in range(n_max + 1)])
            cdf = np.cumsum(weights) / weights.sum()
            v = int(np.searchsorted(cdf, u[i], side="right"))
            v = min(v, n_max)
            while weights[v] == 0:
                v -= 1
            out[w, i] = v
            s -= v
    return Walker(config=out, log_weight=_zeros(N_walkers, x64), e_loc=_zeros(N_walkers, x64))


def reconfiguration(walkers, rng_key):
    """Systematic resampling of a walker population on the GPU
    (walkers/reconfiguration.py:27-62): ``(new_walkers, log_G_n - log N,
    E_n, indices)`` with log G_n = logsumexp(log_weight), weights
    w = exp(log_weight - log G_n), E_n = sum w e_loc, the offset
    psi = uniform(rng_key) and indices[i] the first walker whose cumulative
    weight exceeds (i + psi) / N (capped at the last walker of positive
    weight, systematic_parents:9-24).  The new walkers are the parents'
    configurations and local energies with log weights reset to zero, in
    the dtype of the input's.

    The weights, the float64 cumulative sum, the search and E_n run on the
    device (``gfmc_reconfigure_noalloc``, the kernels of the engine's own
    resampling); the configurations stay where the caller keeps them (host
    arrays) and are gathered there through the returned parents.  At most
    ``RECONFIGURATION_MAX_WALKERS`` walkers per call (ValueError above).  A
    population whose weights sum to zero or overflow gives a non-finite
    log G and E_n, as the reference's does; its indices are then in range
    but carry no meaning.  Needs a CUDA device (no CPU fallback)."""
    from . import _lib
    from .engine import _torch
    config = np.asarray(walkers.config)
    log_w = np.asarray(walkers.log_weight)
    e_loc = np.asarray(walkers.e_loc)
    if log_w.ndim != 1 or e_loc.shape != log_w.shape or config.ndim < 1 or config.shape[0] != log_w.shape[0]:
        raise ValueError(f"walkers must hold log_weight and e_loc of shape (N_walkers,) and config of "
                         f"N_walkers rows; got {log_w.shape}, {e_loc.shape} and {config.shape}.")
    n = log_w.shape[0]
    if n < 1:
        raise ValueError("reconfiguration needs at least one walker.")
    if n > RECONFIGURATION_MAX_WALKERS:
        raise ValueError(f"reconfiguration takes at most {RECONFIGURATION_MAX_WALKERS} walkers per call; "
                         f"got {n}.  A larger population runs through run() / GFMCEngine, whose "
                         "resampling has no such limit.")
    key = np.ascontiguousarray(_rnd.as_key(rng_key), dtype=np.uint32)
    torch = _torch()
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    d_lw = torch.as_tensor(np.ascontiguousarray(log_w, dtype=np.float64)).to(dev, non_blocking=False)
    d_el = torch.as_tensor(np.ascontiguousarray(e_loc, dtype=np.float64)).to(dev, non_blocking=False)
    parents = torch.empty(n, dtype=torch.int32, device=dev)
    scalars = torch.empty(2, dtype=torch.float64, device=dev)      # log G_n - log N, E_n
    vp = lambda t: ctypes.c_void_p(t.data_ptr())                      # noqa: E731
    rc = lib.gfmc_reconfigure_noalloc(n, vp(d_lw), vp(d_el),
                                      key.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                      vp(parents), vp(scalars[0:1]), vp(scalars[1:2]),
                                      ctypes.c_void_p(stream.cuda_stream))
    _lib.check(rc, "reconfiguration")
    idx = parents.cpu().numpy()          # waits for the stream
    log_avg, E_n = scalars.cpu().numpy().tolist()
    new = Walker(config=config[idx], log_weight=np.zeros(n, dtype=log_w.dtype), e_loc=e_loc[idx])
    return new, log_avg, E_n, idx

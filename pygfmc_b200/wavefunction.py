"""Guiding wavefunctions with PyGFMC's constructors.

``JastrowSpinHalf(N, pairs, beta, h=None)`` follows
``wavefunction/jastrow_spin_half.py:42-157`` and
``JastrowBoseHubbard(N, pairs, beta, h=None, d=None, incremental=False)``
follows ``wavefunction/jastrow_bose_hubbard.py:65-125``: the same parameter
forms (tied scalars or per-pair/per-site arrays), the same conventions
(``log psi = -sum beta_ij x_i x_j + sum h_i x_i [- sum d_i x_i^2]``) and the
same validation errors.  ``log_psi`` and ``log_diff_from_operator`` are host
(numpy) versions for inspection and tests; the engine evaluates the ratios on
the device from the tables these objects lower to.
"""
import numpy as np

from .hamiltonian import BoseHubbard, edges_array

__all__ = ["JastrowSpinHalf", "JastrowBoseHubbard", "RBMSpinHalf", "MLPBoseHubbard", "ExactGroundState",
           "round_bf16"]

LAYOUT_ATTRS = ("n_hx_static", "n_jpm_static", "edge_i", "edge_j")


def require_spin_half_layout(op, guide_name):
    """wavefunction/_layout.py:14-19."""
    if not all(hasattr(op, name) for name in LAYOUT_ATTRS):
        raise TypeError(f"{guide_name} needs an operator with the SpinHalf transition layout "
                        f"({', '.join(LAYOUT_ATTRS)}); got {type(op).__name__}")


class JastrowSpinHalf:
    """psi_T(x) = exp(sum_{(i,j) in pairs} J_ij x_i x_j + sum_i h_i x_i), J = -beta.

    Stores what PyGFMC's ``JastrowSpinHalf`` stores
    (``wavefunction/jastrow_spin_half.py:79-157``): the parameters in the
    form they were given and rounded to ``dtype`` (``_J`` 0-d for a tied
    coupling or one per pair, ``_h`` None / 0-d / per site), the per-site
    partner tables ``site_other`` / ``site_valid_mask`` / ``_site_pair`` and
    the constructor order of the pairs (``_pair_site``, ``_pair_slot``).  The
    engine lowers a guide from exactly these attributes, so PyGFMC's own
    guide objects and this class are interchangeable.
    """

    def __init__(self, N, pairs, beta, h=None, dtype=np.float32):
        N = int(N)
        if pairs is None:
            raise ValueError("pairs must be provided (n_pairs, 2) int array)")
        pairs_np, _, n_min = edges_array(pairs)
        if n_min > N:
            raise ValueError(f"pair indices must lie in [0, {N}).")
        pairs_np = np.sort(pairs_np.astype(np.int32), axis=1)
        n_pairs = pairs_np.shape[0]
        dtype = np.dtype(dtype)
        # the broadcast rejects a beta of any other length than n_pairs
        J_np = -np.broadcast_to(np.asarray(beta, dtype=dtype), (n_pairs,))
        if h is not None:
            h_in = np.asarray(h, dtype=dtype)
            if h_in.ndim > 1 or (h_in.ndim == 1 and h_in.shape != (N,)):
                raise ValueError(f"h must be a scalar or have shape ({N},), got {h_in.shape}")
        partners = [[] for _ in range(N)]
        pair_site = np.zeros(n_pairs, dtype=np.int32)
        pair_slot = np.zeros(n_pairs, dtype=np.int32)
        for p, (a, b) in enumerate(pairs_np):
            pair_site[p] = a
            pair_slot[p] = len(partners[a])
            partners[a].append((int(b), p))
            partners[b].append((int(a), p))
        max_deg = max((len(s) for s in partners), default=0) or 1
        other = -np.ones((N, max_deg), dtype=np.int32)
        site_pair = np.zeros((N, max_deg), dtype=np.int32)
        for k in range(N):
            for slot, (o, p) in enumerate(partners[k]):
                other[k, slot] = o
                site_pair[k, slot] = p
        self.dtype = dtype
        self.N = N
        self.site_other = np.clip(other, 0, None)
        self.site_valid_mask = other >= 0
        self._pair_site = pair_site
        self._pair_slot = pair_slot
        self._site_pair = site_pair
        if np.ndim(beta) == 0:
            self._J = np.asarray(-float(np.asarray(beta)), dtype=dtype)
        else:
            self._J = np.array(J_np, dtype=dtype)
        if h is None:
            self._h = None
        elif np.ndim(h) == 0:
            self._h = np.asarray(float(np.asarray(h)), dtype=dtype)
        else:
            self._h = np.array(h_in, dtype=dtype)

    @property
    def tied_beta(self):
        return self._J.ndim == 0

    @property
    def site_J(self):
        """Couplings J = -beta per site and partner slot, (N, max_deg)."""
        J = self._J if self._J.ndim == 0 else self._J[self._site_pair]
        return np.where(self.site_valid_mask, J, 0).astype(self.dtype)

    @property
    def h(self):
        """One-body field per site, (N,) (zeros without a field)."""
        if self._h is None:
            return np.zeros(self.N, dtype=self.dtype)
        return np.broadcast_to(self._h, (self.N,))

    @property
    def beta(self):
        """Per-pair coupling beta = -J in constructor order."""
        return -np.broadcast_to(self._J, self._pair_site.shape)

    @property
    def pairs(self):
        """(n_pairs, 2) pairs (min, max) in constructor order."""
        return np.stack([self._pair_site, self.site_other[self._pair_site, self._pair_slot]], axis=1)

    def log_psi(self, config, cache=None):
        x = np.asarray(config, dtype=np.float64)
        pr = self.pairs
        J = -self.beta.astype(np.float64)
        pair = (J * x[..., pr[:, 0]] * x[..., pr[:, 1]]).sum(-1)
        return pair + (self.h.astype(np.float64) * x).sum(-1)

    def log_diff_from_configs(self, config, new_configs, cache=None):
        return self.log_psi(new_configs) - self.log_psi(config)

    def log_diff_from_operator(self, config, op, cache=None):
        """Host evaluation of the log-ratios in the SpinHalf layout."""
        require_spin_half_layout(op, type(self).__name__)
        M = 1 + op.n_hx_static + op.n_jpm_static
        x = np.asarray(config, dtype=np.float64)
        base = self.log_psi(x)
        out = np.zeros(M)
        for k in range(1, M):
            out[k] = self.log_psi(op.generate_state(x, k)) - base
        return out

    def build_cache(self, op):
        require_spin_half_layout(op, type(self).__name__)
        return None

    def save(self, path, group="jastrow_spin_half", **attrs):
        """Write the guide (jastrow_spin_half.py save:192-224): the pairs in
        constructor order, beta (0-d when tied, else per pair) and h (absent,
        0-d or per site) in the form they were given, N, and the keyword
        arguments as scalar attributes.  h5py is not available to this
        package, so the container is a NumPy ``.npz`` archive with the names
        ``<group>/<name>`` and ``<group>/attrs/<name>``, written at ``path``."""
        d = {f"{group}/pairs": self.pairs.astype(np.int32), f"{group}/beta": -np.asarray(self._J),
             f"{group}/attrs/N": np.asarray(self.N)}
        if self._h is not None:
            d[f"{group}/h"] = np.asarray(self._h)
        _put_attrs(d, group, attrs)
        with open(path, "wb") as f:
            np.savez(f, **d)

    @classmethod
    def load(cls, path, hamiltonian=None, group="jastrow_spin_half", dtype=np.float32):
        """A guide written by :meth:`save` (jastrow_spin_half.py load:226-266).
        With ``hamiltonian`` the site count is the largest of the saved N,
        the Hamiltonian's N and its highest edge index + 1, and a per-site h
        is padded with zeros to it."""
        with np.load(path, allow_pickle=False) as z:
            if f"{group}/pairs" not in z.files:
                raise KeyError(f"{path} holds no JastrowSpinHalf group {group!r}")
            pairs = np.asarray(z[f"{group}/pairs"], dtype=np.int64)
            beta = np.asarray(z[f"{group}/beta"])
            h = np.asarray(z[f"{group}/h"]) if f"{group}/h" in z.files else None
            N = int(z[f"{group}/attrs/N"])
        if hamiltonian is not None:
            edges = np.asarray(getattr(hamiltonian, "edges", np.zeros((0, 2))))
            N = max(N, int(edges.max(initial=-1)) + 1, int(hamiltonian.N))
            if h is not None and h.ndim == 1 and h.shape[0] < N:
                h = np.concatenate([h, np.zeros(N - h.shape[0], dtype=h.dtype)])
        return cls(N, pairs, float(beta) if beta.ndim == 0 else beta,
                   h=None if h is None else (float(h) if h.ndim == 0 else h), dtype=dtype)

    @classmethod
    def from_jax(cls, dtype, N, site_other, site_J, site_valid_mask, h, pair_site, pair_slot,
                 site_pair):
        """A guide from its stored arrays, bypassing the constructor
        (jastrow_spin_half.py from_jax:267-286): ``site_J`` is the coupling
        J = -beta as stored (0-d when tied, else per pair), ``h`` None / 0-d /
        per site, ``pair_site`` / ``pair_slot`` locate each pair in the
        per-site tables."""
        obj = object.__new__(cls)
        obj.dtype, obj.N = np.dtype(dtype), int(N)
        obj.site_other = np.asarray(site_other)
        obj._J = np.asarray(site_J)
        obj.site_valid_mask = np.asarray(site_valid_mask, dtype=bool)
        obj._h = None if h is None else np.asarray(h)
        obj._pair_site, obj._pair_slot = np.asarray(pair_site), np.asarray(pair_slot)
        obj._site_pair = np.asarray(site_pair)
        return obj


def _put_attrs(d, group, attrs):
    """Scalar attributes into a save dict under ``<group>/attrs/``."""
    for k, v in attrs.items():
        if np.ndim(v) != 0:
            raise ValueError(f"attribute {k!r} must be a scalar")
        d[f"{group}/attrs/{k}"] = np.asarray(v)


class JastrowBoseHubbard:
    """log psi_T(x) = -sum_pairs beta_ij x_i x_j + sum_i h_i x_i - sum_i d_i x_i^2.

    Stores what PyGFMC's ``JastrowBoseHubbard`` stores
    (``wavefunction/jastrow_bose_hubbard.py:97-125``): ``pair_i``, ``pair_j``
    and the parameters ``_beta``, ``_h``, ``_d`` in the form they were given
    (None, a 0-d tied value or one per pair / site), rounded to ``dtype``.
    The engine lowers a guide from exactly these attributes.

    ``incremental`` is kept as an attribute and does not change what runs:
    the device always carries each walker's weighted neighbour sums, updates
    them additively per move and rebuilds them every 100 steps (50 in the
    float32 build) -- the policy of PyGFMC's incremental mode
    (engine/evolution.py:167,181-189) -- so its
    ratios agree with both of PyGFMC's modes to rounding, not bit for bit
    with either.  The host methods of that mode (``init_state``,
    ``update_state``, the ``state=`` argument) exist for code that drives
    them itself.
    """

    def __init__(self, N, pairs, beta, h=None, d=None, dtype=np.float32, incremental=False):
        pairs, _, n_min = edges_array(pairs)
        if n_min > int(N):
            raise ValueError(f"pair indices must lie in [0, {N}).")
        if beta is None:
            raise ValueError("beta is required (a scalar or an (n_pairs,) array).")
        self.N = int(N)
        self.dtype = np.dtype(dtype)
        self.pair_i = pairs[:, 0].astype(np.int32)
        self.pair_j = pairs[:, 1].astype(np.int32)

        def param(v, n, name):
            # jastrow_bose_hubbard.py _param:36-45: the form given, rounded to dtype
            if v is None:
                return None
            a = np.asarray(v, dtype=np.float64)
            if a.ndim == 0:
                return np.asarray(float(a), dtype=self.dtype)
            if a.shape != (n,):
                raise ValueError(f"{name} must be a scalar or have shape ({n},), got {a.shape}")
            return np.asarray(a, dtype=self.dtype)
        self._beta = param(beta, len(pairs), "beta")
        self._h = param(h, self.N, "h")
        self._d = param(d, self.N, "d")
        self.incremental = bool(incremental)

    @property
    def beta(self):
        return np.broadcast_to(self._beta, self.pair_i.shape)

    @property
    def h(self):
        return np.zeros(self.N, self.dtype) if self._h is None else np.broadcast_to(self._h, (self.N,))

    @property
    def d(self):
        return np.zeros(self.N, self.dtype) if self._d is None else np.broadcast_to(self._d, (self.N,))

    def log_psi(self, config, cache=None):
        n = np.asarray(config, dtype=np.float64)
        d, beta, h = (np.asarray(v, np.float64) for v in (self.d, self.beta, self.h))
        out = -(d * n * n).sum(-1)
        out = out - (beta * n[..., self.pair_i] * n[..., self.pair_j]).sum(-1)
        return out + (h * n).sum(-1)

    def log_diff_from_operator(self, config, op, cache=None, state=None):
        """log psi(x') - log psi(x) for every transition of ``op`` (entry 0:
        0), from the successor configurations (jastrow_bose_hubbard.py
        log_diff_from_operator:253-286, whose non-BoseHubbard branch does the
        same).  ``state`` (the incremental neighbour sums) is accepted and
        not needed: the ratios come from log_psi directly."""
        n = np.asarray(config, dtype=np.float64)
        base = self.log_psi(n)
        if isinstance(op, BoseHubbard):
            out = np.zeros(op.M_total)
            for k in range(1, op.M_total):
                out[k] = self.log_psi(op.generate_state(n, k)) - base
            return out
        _, succ = op.get_rates(n, return_configs=True)
        return self.log_psi(np.asarray(succ, np.float64)) - base

    def build_cache(self, op):
        return None

    def _pair_weight(self):
        """Weight of each pair in the neighbour sums: -beta, or 1 for a tied
        beta (whose value then scales the sums)."""
        if np.ndim(self._beta) == 0:
            return np.ones(len(self.pair_i))
        return -np.asarray(self._beta, np.float64)

    def init_state(self, config, cache=None):
        """The incremental mode's per-walker state (jastrow_bose_hubbard.py
        init_state:230-235): the weighted neighbour sums
        S_a = sum over the pairs (a, b) of w_ab x_b, shape (N,)."""
        n = np.asarray(config, dtype=np.float64)
        w = self._pair_weight()
        s = np.zeros(self.N)
        np.add.at(s, self.pair_i, w * n[self.pair_j])
        np.add.at(s, self.pair_j, w * n[self.pair_i])
        return s

    def update_state(self, state, config, sites, deltas, cache=None):
        """``state`` after the move that adds ``deltas`` to ``sites`` (the
        form ``BoseHubbard.move`` returns; update_state:237-251): every
        partner q of a moved site s gains w_sq delta_s."""
        s = np.array(state, dtype=np.float64, copy=True)
        if len(self.pair_i) == 0:
            return s
        w = self._pair_weight()
        for k in range(2):
            site, dk = int(sites[k]), float(deltas[k])
            if dk == 0.0:
                continue
            on_i, on_j = self.pair_i == site, self.pair_j == site
            np.add.at(s, self.pair_j[on_i], w[on_i] * dk)
            np.add.at(s, self.pair_i[on_j], w[on_j] * dk)
        return s

    def save(self, path, group="jastrow_bose_hubbard", **attrs):
        """Write the guide (jastrow_bose_hubbard.py save:290-304): the pairs,
        beta, h and d in the form they were given (absent, 0-d or per pair /
        site), N, the incremental flag and the keyword arguments as scalar
        attributes, in a NumPy ``.npz`` archive written at ``path`` (names
        ``<group>/<name>``, ``<group>/attrs/<name>``)."""
        d = {f"{group}/pairs": np.stack([self.pair_i, self.pair_j], axis=1).astype(np.int32),
             f"{group}/attrs/N": np.asarray(self.N),
             f"{group}/attrs/incremental": np.asarray(int(self.incremental))}
        for name in ("beta", "h", "d"):
            v = getattr(self, "_" + name)
            if v is not None:
                d[f"{group}/{name}"] = np.asarray(v)
        _put_attrs(d, group, attrs)
        with open(path, "wb") as f:
            np.savez(f, **d)

    @classmethod
    def load(cls, path, group="jastrow_bose_hubbard", dtype=np.float32):
        """A guide written by :meth:`save` (jastrow_bose_hubbard.py
        load:306-316), every parameter back in its saved form."""
        with np.load(path, allow_pickle=False) as z:
            if f"{group}/pairs" not in z.files:
                raise KeyError(f"{path} holds no JastrowBoseHubbard group {group!r}")
            pairs = np.asarray(z[f"{group}/pairs"], dtype=np.int64)
            p = {}
            for name in ("beta", "h", "d"):
                v = np.asarray(z[f"{group}/{name}"]) if f"{group}/{name}" in z.files else None
                p[name] = None if v is None else (float(v) if v.ndim == 0 else v)
            N = int(z[f"{group}/attrs/N"])
            inc = bool(int(z[f"{group}/attrs/incremental"])) if f"{group}/attrs/incremental" in z.files \
                else False
        return cls(N, pairs, p["beta"], h=p["h"], d=p["d"], dtype=dtype, incremental=inc)


def round_bf16(x):
    """Round float values to the nearest bfloat16 (ties to even); returned as
    float32 arrays whose values are exactly representable in bf16."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


class RBMSpinHalf:
    """Restricted Boltzmann machine guide for spin-1/2 configurations:

        log psi(s) = sum_h log cosh(theta_h) + a . s,   theta = b + W s,

    s in {+-1}^N, W of shape (n_hidden, N) with bfloat16 values (stored as
    float32 arrays holding bf16-representable numbers), b (n_hidden,) and
    a (N,) float32.  A positive-amplitude guide; PyGFMC has no counterpart
    (its learned guides are the NetKet-trained cluster models).  The engine
    evaluates ratios on the device from theta, updated incrementally per move
    (theta' = theta - 2 s_i W[:, i] - 2 s_j W[:, j] for an edge flip)."""

    def __init__(self, N, n_hidden, W=None, b=None, a=None, seed=0, sigma=0.01, dtype=np.float32):
        N, H = int(N), int(n_hidden)
        if N <= 0 or H <= 0:
            raise ValueError("N and n_hidden must be positive")
        if H > 1024:
            raise ValueError(f"n_hidden={H} exceeds the engine's limit of 1024")
        rng = np.random.default_rng(seed)
        W = rng.normal(0.0, sigma, size=(H, N)) if W is None else np.asarray(W, dtype=np.float64)
        if W.shape != (H, N):
            raise ValueError(f"W must have shape ({H}, {N}), got {W.shape}")
        b = np.zeros(H) if b is None else np.broadcast_to(np.asarray(b, dtype=np.float64), (H,))
        a = np.zeros(N) if a is None else np.broadcast_to(np.asarray(a, dtype=np.float64), (N,))
        self.N, self.n_hidden = N, H
        self.dtype = np.dtype(dtype)
        self.W = round_bf16(W)
        self.b = np.asarray(b, dtype=np.float32).copy()
        self.a = np.asarray(a, dtype=np.float32).copy()

    def parameters(self):
        return {"W": self.W, "b": self.b, "a": self.a}

    def set_parameters(self, W=None, b=None, a=None):
        if W is not None:
            self.W = round_bf16(np.asarray(W).reshape(self.n_hidden, self.N))
        if b is not None:
            self.b = np.asarray(b, dtype=np.float32).reshape(self.n_hidden).copy()
        if a is not None:
            self.a = np.asarray(a, dtype=np.float32).reshape(self.N).copy()

    def theta(self, config):
        s = np.asarray(config, dtype=np.float64)
        return s @ self.W.astype(np.float64).T + self.b.astype(np.float64)

    def log_psi(self, config, cache=None):
        s = np.asarray(config, dtype=np.float64)
        t = self.theta(s)
        lc = np.abs(t) + np.log1p(np.exp(-2.0 * np.abs(t))) - np.log(2.0)
        return lc.sum(-1) + s @ self.a.astype(np.float64)

    def log_diff_from_configs(self, config, new_configs, cache=None):
        return self.log_psi(new_configs) - self.log_psi(config)

    def log_diff_from_operator(self, config, op, cache=None):
        """Host log-ratios in the SpinHalf rate layout (slot 0 = 0)."""
        require_spin_half_layout(op, type(self).__name__)
        x = np.asarray(config, dtype=np.float64)
        M = 1 + op.n_hx_static + op.n_jpm_static
        out = np.zeros(M)
        for k in range(op.n_hx_static):
            y = x.copy(); y[k] = -y[k]
            out[1 + k] = self.log_psi(y) - self.log_psi(x)
        for e in range(op.n_jpm_static):
            y = x.copy(); i, j = int(op.edge_i[e]), int(op.edge_j[e])
            y[i], y[j] = -y[i], -y[j]
            out[1 + op.n_hx_static + e] = self.log_psi(y) - self.log_psi(x)
        return out


def _bf16_round64(x):
    """float64 values rounded through float32 to the nearest bfloat16."""
    return round_bf16(np.asarray(x, dtype=np.float32)).astype(np.float64)


class MLPBoseHubbard:
    """Dense log-amplitude MLP guide for Bose-Hubbard occupations:

        x = one-hot occupations (site k, occupation n -> input k (n_max + 1) + n)
        h1 = tanh(W1 x + b1),  h2 = tanh(W2 bf16(h1) + b2),  log psi = w3 . h2 + b3

    W1 (H1, N (n_max + 1)), W2 (H2, H1) and w3 (H2,) hold bfloat16 values; the
    biases are float32.  The first layer's activations enter the second as
    bf16, as the tensor-core kernel consumes them.  No PyGFMC counterpart (its
    learned guides are NetKet-trained cluster models).  H1 in {64, 128, 192,
    256}, H2 a multiple of 16 up to 256."""

    def __init__(self, N, n_max, hidden=(256, 256), W1=None, b1=None, W2=None, b2=None, w3=None,
                 b3=0.0, seed=0, sigma=0.05, dtype=np.float32):
        N, n_max = int(N), int(n_max)
        H1, H2 = (int(hidden), int(hidden)) if np.ndim(hidden) == 0 else (int(hidden[0]), int(hidden[1]))
        if H1 not in (64, 128, 192, 256) or H2 < 16 or H2 > 256 or H2 % 16:
            raise ValueError(f"hidden sizes ({H1}, {H2}): H1 must be 64, 128, 192 or 256 and H2 a "
                             "multiple of 16 up to 256")
        if n_max < 1 or N < 1:
            raise ValueError("N and n_max must be positive")
        D = N * (n_max + 1)
        rng = np.random.default_rng(seed)
        W1 = rng.normal(0.0, sigma, (H1, D)) if W1 is None else np.asarray(W1, np.float64)
        W2 = rng.normal(0.0, sigma, (H2, H1)) if W2 is None else np.asarray(W2, np.float64)
        w3 = rng.normal(0.0, sigma, H2) if w3 is None else np.asarray(w3, np.float64)
        if W1.shape != (H1, D) or W2.shape != (H2, H1) or w3.shape != (H2,):
            raise ValueError("W1, W2, w3 shapes do not match (H1, N (n_max + 1)), (H2, H1), (H2,)")
        self.N, self.n_max, self.H1, self.H2 = N, n_max, H1, H2
        self.dtype = np.dtype(dtype)
        self.W1, self.W2, self.w3 = round_bf16(W1), round_bf16(W2), round_bf16(w3)
        self.b1 = np.broadcast_to(np.asarray(0.0 if b1 is None else b1, np.float32), (H1,)).copy()
        self.b2 = np.broadcast_to(np.asarray(0.0 if b2 is None else b2, np.float32), (H2,)).copy()
        self.b3 = float(np.float32(b3))

    def log_psi(self, config, cache=None):
        n = np.asarray(config, dtype=np.float64)
        idx = np.arange(self.N) * (self.n_max + 1) + n.astype(np.int64)
        z1 = self.W1.astype(np.float64)[:, idx].sum(-1).T if n.ndim > 1 else \
            self.W1.astype(np.float64)[:, idx].sum(-1)
        z1 = z1 + self.b1.astype(np.float64)
        h1 = _bf16_round64(np.tanh(z1))
        h2 = np.tanh(h1 @ self.W2.astype(np.float64).T + self.b2.astype(np.float64))
        return h2 @ self.w3.astype(np.float64) + self.b3

    def log_diff_from_configs(self, config, new_configs, cache=None):
        return self.log_psi(new_configs) - self.log_psi(config)


# floor on |psi_0| before the log: a node of the exact ground state gets a
# large negative log amplitude rather than -inf (exact_ground_state.py:36)
AMP_FLOOR = 1e-30


class ExactGroundState:
    """psi_T(x) = |psi_0[idx(x)]| with psi_0 the exact ground state
    (wavefunction/exact_ground_state.py:43-190): the zero-variance limit, in
    which every walker's local energy is E0.  ``idx`` is the positional basis
    index over ``local_hilbert_space`` (default the Hamiltonian's own), site 0
    the most significant digit.  ``log_amp`` (d^N values) is given, or taken
    from :func:`pygfmc_b200.hamiltonian.exact_diagonalization` (then ``E0`` is
    stored, else NaN), and kept rounded to ``dtype``.

    On the device (SpinHalf models, N <= 26) the ratio of a move is
    exp(log_amp[y] - log_amp[x]) in the run's precision, looked up at the
    walker's basis index; ``log_diff_from_configs`` is the host version."""

    def __init__(self, hamiltonian, *, log_amp=None, dtype=np.float32, local_hilbert_space=None,
                 N=None):
        name = type(hamiltonian).__name__
        values = local_hilbert_space
        if values is None:
            values = getattr(hamiltonian, "local_hilbert_space", None)
        if values is None:
            raise ValueError(f"{name} exposes no local_hilbert_space: pass local_hilbert_space=(...), "
                             "e.g. (1, -1) for spin-1/2")
        values = tuple(float(v) for v in np.asarray(values, dtype=float).ravel())
        if len(values) < 2:
            raise ValueError(f"local_hilbert_space needs at least two values, got {list(values)}")
        if N is None:
            N = getattr(hamiltonian, "N", None)
        if N is None:
            raise ValueError(f"{name} exposes no N: pass N=...")
        d, N = len(values), int(N)
        self.local_hilbert_space = values
        self.N = N
        self._powers = tuple(int(d ** k) for k in range(N - 1, -1, -1))
        if log_amp is None:
            from .hamiltonian import exact_diagonalization
            energies, _, _, states = exact_diagonalization(hamiltonian, values, N, number_of_states=1,
                                                           return_states=True)
            psi0 = np.asarray(states[:, 0])
            if psi0.min() < -1e-6 and psi0.max() > 1e-6:
                import warnings
                warnings.warn(f"ExactGroundState: psi_0 changes sign (min {psi0.min():.3e}, max "
                              f"{psi0.max():.3e}); the guide assumes a sign-problem-free Hamiltonian "
                              "and uses |psi_0|", UserWarning)
            self.E0 = float(energies[0])
            log_amp = np.log(np.maximum(np.abs(psi0), AMP_FLOOR))
        else:
            self.E0 = float("nan")
        log_amp = np.asarray(log_amp, dtype=dtype).ravel()
        if log_amp.shape[0] != d ** N:
            raise ValueError(f"log_amp has {log_amp.shape[0]} entries for a basis of {d}**{N} = "
                             f"{d ** N} states")
        self.log_amp = log_amp
        self.hamiltonian = hamiltonian
        self.dtype = np.dtype(dtype)
        self.M_total = int(hamiltonian.M_total)

    def basis_index(self, config):
        """Index of config (..., N) in log_amp (exact_ground_state.py:141-147)."""
        c = np.asarray(config, dtype=np.float64)
        digit = np.argmin(np.abs(c[..., None] - np.asarray(self.local_hilbert_space)), axis=-1)
        return digit.astype(np.int64) @ np.asarray(self._powers, dtype=np.int64)

    def log_psi(self, config, cache=None):
        return self.log_amp[self.basis_index(config)]

    def log_diff_from_configs(self, config, new_configs=None, cache=None):
        """log psi(y) - log psi(x) in ``dtype`` for the given successors, or
        for every transition of the bound Hamiltonian with element 0 pinned to
        0 (exact_ground_state.py:150-190); indices outside the basis (zero-rate
        transitions of a bounded local space) are clipped."""
        dim = self.log_amp.shape[0]
        old = self.log_amp[self.basis_index(config)]
        if new_configs is None:
            new_configs = np.stack([self.hamiltonian.generate_state(np.asarray(config), k)
                                    for k in range(self.M_total)])
            out = self.log_amp[np.clip(self.basis_index(new_configs), 0, dim - 1)] - old
            out[0] = 0
            return out.astype(self.dtype)
        new = np.clip(self.basis_index(new_configs), 0, dim - 1)
        return (self.log_amp[new] - old).astype(self.dtype)

    def save(self, path, group="exact_ground_state", **attrs):
        """``log_amp``, ``local_hilbert_space`` and the attributes N, family,
        E0 (plus keyword scalars) under ``group`` (exact_ground_state.py:
        193-210), in a NumPy ``.npz`` archive as ``Walker.save`` writes one."""
        d = {f"{group}/log_amp": np.asarray(self.log_amp),
             f"{group}/local_hilbert_space": np.asarray(self.local_hilbert_space, dtype=float),
             f"{group}/attrs/N": np.asarray(self.N),
             f"{group}/attrs/family": np.asarray(type(self.hamiltonian).__name__),
             f"{group}/attrs/E0": np.asarray(self.E0)}
        for k, v in attrs.items():
            if np.ndim(v) != 0:
                raise ValueError(f"attribute {k!r} must be a scalar")
            d[f"{group}/attrs/{k}"] = np.asarray(v)
        with open(path, "wb") as f:
            np.savez(f, **d)

    @classmethod
    def load(cls, path, hamiltonian, group="exact_ground_state", dtype=np.float32):
        """A guide written by :meth:`save`, bound to ``hamiltonian``
        (exact_ground_state.py:212-256); ValueError when the saved family or
        N differs from the Hamiltonian's."""
        with np.load(path, allow_pickle=False) as z:
            need = [f"{group}/{k}" for k in ("log_amp", "attrs/N", "attrs/family", "attrs/E0")]
            missing = [k for k in need if k not in z.files]
            if missing:
                raise ValueError(f"{path}:{group} is not an ExactGroundState file (missing {missing})")
            log_amp = np.asarray(z[f"{group}/log_amp"])
            family = str(z[f"{group}/attrs/family"])
            N = int(z[f"{group}/attrs/N"])
            E0 = float(z[f"{group}/attrs/E0"])
            lhs_k = f"{group}/local_hilbert_space"
            lhs = tuple(float(v) for v in z[lhs_k]) if lhs_k in z.files else None
        if family != type(hamiltonian).__name__:
            raise ValueError(f"saved guide family={family!r} but loading into "
                             f"{type(hamiltonian).__name__!r}")
        if getattr(hamiltonian, "N", None) is not None and N != int(hamiltonian.N):
            raise ValueError(f"saved guide N={N} but the Hamiltonian has N={int(hamiltonian.N)}")
        guide = cls(hamiltonian, log_amp=log_amp, dtype=dtype, local_hilbert_space=lhs, N=N)
        guide.E0 = E0
        return guide

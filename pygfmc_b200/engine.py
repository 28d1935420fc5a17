"""The GFMC driver: ``run`` / ``run_gfmc`` on one B200.

Mirrors PyGFMC's ``engine/multi_gpu.py run:822-868`` and
``engine/driver.py run_gfmc:1148-1547``: the same arguments, validation
order and errors, warm-up ramp (``_warmup_schedule:567``, side-streams
``_warmup_stage_key:48``), production key recurrence (``key, rng =
split(key); k1, k2 = fold_in(rng, 0/1)``, ``driver.py:218-221``), population
checks (``_check_population:913``) and return tuple ``(walkers, energy, obs,
stats, raw)``.  The per-step work runs in the CUDA engine through its C ABI
(``include/gfmc_b200.h``); this module only orchestrates chunks of steps,
pulls the per-step series and assembles the results.
"""
from __future__ import annotations

import ctypes
import math
import secrets
import time
from types import SimpleNamespace

import numpy as np

from . import _lib
from . import random as _rnd
from .hamiltonian import BoseHubbard, SpinHalf
from .walkers import Walker
from .wavefunction import JastrowBoseHubbard, JastrowSpinHalf, MLPBoseHubbard, RBMSpinHalf
from .estimators import (autocorrelation_stats, diagonal_estimates, off_diagonal_estimates,
                         validated_p_array, windowed_energy_host)

__all__ = ["run", "run_gfmc", "GFMCEngine", "DEFAULT_WARMUP_STEPS", "evolve_walkers",
           "estimate_average_log_branch_weight"]

DEFAULT_WARMUP_STEPS = 1000
_AUX_ROOT = 9_000
_WARMUP_CHUNK = 50


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.GFMCError("pygfmc_b200 needs a CUDA device (B200, sm_100a); none is visible -- "
                             "there is no CPU fallback")
    return torch


def _emit(msg, verbosity, level=1):
    if verbosity >= level:
        print(msg, flush=True)


def _validated_int(name, value, minimum):
    """_validation.py _validated_int:7-19."""
    if isinstance(value, (bool, np.bool_)):
        raise ValueError(f"{name} must be an integer >= {minimum}, got {value!r}.")
    try:
        result = int(value)
        ok = float(result) == float(value)
    except (TypeError, ValueError, OverflowError):
        ok, result = False, minimum - 1
    if not ok or result < minimum:
        raise ValueError(f"{name} must be an integer >= {minimum}, got {value!r}.")
    return result


def require_step_size(method, step_size):
    """engine/evolution.py require_step_size:744-758."""
    if not math.isfinite(float(step_size)):
        raise ValueError(f"step_size must be finite; got step_size={step_size!r}")
    if not (float(step_size) > 0):
        raise ValueError(f"step_size must be > 0; got step_size={step_size!r}")
    if method != "cont_time" and float(int(step_size)) != float(step_size):
        raise ValueError(f"method={method!r} requires an integer step_size; got step_size={step_size!r}")


def require_lam(method, lam):
    """engine/evolution.py require_lam:724-741."""
    if method == "cont_time":
        return None
    if method in ("single_step", "multi_step"):
        if lam is None:
            raise ValueError(
                f"method={method!r} needs the GFMC shift: pass lam=<float> with lam >= max_x H_xx "
                "over the reachable configurations (cont_time is the only method that does without it).")
        v = float(lam)
        if not math.isfinite(v):
            raise ValueError(f"lam must be finite; got lam={lam!r}")
        return v
    raise ValueError(f"Unknown method: {method!r}")


# ---- lowering of host objects to the C descriptors ---------------------------
class _Keep:
    """Keeps the numpy arrays a descriptor points into alive."""

    def __init__(self):
        self.arrays = []

    def f64(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        self.arrays.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def i32(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
        self.arrays.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))

    def f32(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
        self.arrays.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _is_spin_half(op):
    return all(hasattr(op, a) for a in ("n_hx_static", "n_jpm_static", "edge_i", "edge_j",
                                        "J_pm", "J_pmpm", "J_z"))


def _is_bose(op):
    return all(hasattr(op, a) for a in ("n_hop_off", "n_eta_off", "n_hpm_off", "n_max", "edge_i"))


def require_operator_protocol(op, role="hamiltonian"):
    """The engine runs the SpinHalf and BoseHubbard layouts; anything else is
    refused up front (engine/evolution.py require_operator_protocol:62-92)."""
    missing = [n for n in ("M_total", "get_rates") if not hasattr(op, n)]
    if missing:
        raise TypeError(f"{role} {type(op).__name__!r} is missing required attribute(s) "
                        f"{', '.join(missing)}; the operator protocol (pygfmc.Operator) requires "
                        "M_total, get_rates.")
    if not (_is_spin_half(op) or _is_bose(op)):
        raise TypeError(f"{role} {type(op).__name__!r} is not a SpinHalf or BoseHubbard operator; "
                        "the B200 engine has device kernels for those two transition layouts only.")


# The attributes a guide is lowered from: those PyGFMC's own guide classes
# store (wavefunction/jastrow_spin_half.py:79-157 and its beta / h
# properties:162-186; wavefunction/jastrow_bose_hubbard.py:97-125).  A guide
# carrying them -- PyGFMC's object or this package's -- lowers the same way.
SPIN_JASTROW_ATTRS = ("N", "site_other", "_pair_site", "_pair_slot", "beta", "h")
BOSE_JASTROW_ATTRS = ("N", "pair_i", "pair_j", "_beta", "_h", "_d")


def _is_spin_jastrow(guide):
    return all(hasattr(guide, a) for a in SPIN_JASTROW_ATTRS)


def _is_bose_jastrow(guide):
    return all(hasattr(guide, a) for a in BOSE_JASTROW_ATTRS) and not _is_spin_jastrow(guide)


EXACT_GUIDE_ATTRS = ("N", "log_amp", "local_hilbert_space", "basis_index")


def _is_exact_guide(guide):
    return all(hasattr(guide, a) for a in EXACT_GUIDE_ATTRS)


def exact_amplitude_table(guide):
    """log |psi_0| of an ExactGroundState-shaped guide in the device's basis
    order (bit N-1-i set for a down spin at site i: the digits of
    SpinHalf.local_hilbert_space (1, -1)), widened exactly to float64; a guide
    indexed over (-1, 1) has the complementary index, i.e. the reversed
    table."""
    values = tuple(float(v) for v in np.asarray(guide.local_hilbert_space, np.float64).ravel())
    if values not in ((1.0, -1.0), (-1.0, 1.0)):
        raise TypeError(f"the exact-amplitude guide runs on spin-1/2 configurations; its "
                        f"local_hilbert_space is {list(values)}")
    la = np.asarray(guide.log_amp, np.float64).ravel()
    if la.shape[0] != 2 ** int(guide.N):
        raise ValueError(f"log_amp has {la.shape[0]} entries for 2**{int(guide.N)} states")
    return np.ascontiguousarray(la if values == (1.0, -1.0) else la[::-1])


def require_guide_protocol(guide):
    if guide is None:
        return
    if not any(hasattr(guide, n) for n in ("log_diff_from_operator", "log_diff_from_configs", "log_psi")):
        raise TypeError(f"Guide {type(guide).__name__!r} must implement at least one of "
                        "log_diff_from_operator, log_diff_from_configs, or log_psi "
                        "(the guide protocol, pygfmc.Guide).")
    if not (_is_spin_jastrow(guide) or _is_bose_jastrow(guide) or _is_exact_guide(guide)
            or isinstance(guide, (RBMSpinHalf, MLPBoseHubbard)) or hasattr(guide, "_gfmc_guide_desc")):
        raise TypeError(f"Guide {type(guide).__name__!r} has no device implementation in the B200 "
                        "engine (supported: JastrowSpinHalf, JastrowBoseHubbard, ExactGroundState "
                        "on SpinHalf -- PyGFMC's or this package's -- RBMSpinHalf, MLPBoseHubbard).")


def spin_jastrow_tables(guide):
    """(pairs (n_pairs, 2) int32 in constructor order, J = -beta per pair,
    h per site) of a spin-1/2 Jastrow guide, read from the attributes PyGFMC's
    JastrowSpinHalf stores (its ``save``, jastrow_spin_half.py:205-210,
    recovers the pairs the same way).  The values are the guide's own,
    already rounded to its dtype; they are widened to float64 exactly."""
    a = np.asarray(guide._pair_site, dtype=np.int64)
    slot = np.asarray(guide._pair_slot, dtype=np.int64)
    b = np.asarray(guide.site_other)[a, slot]
    pairs = np.stack([a, b], axis=1).astype(np.int32)
    J = -np.asarray(guide.beta, dtype=np.float64).reshape(-1)
    N = int(guide.N)
    h = np.broadcast_to(np.asarray(guide.h, dtype=np.float64), (N,))
    if J.shape != (len(pairs),):
        raise ValueError(f"JastrowSpinHalf guide has {J.shape[0]} couplings for {len(pairs)} pairs")
    return pairs, J, h


def model_desc(op, keep):
    d = _lib.ModelDesc()
    E = int(len(op.edge_i))
    N = int(op.N)
    d.n_sites, d.n_edges = N, E
    d.edge_i, d.edge_j = keep.i32(op.edge_i), keep.i32(op.edge_j)
    if _is_spin_half(op):
        d.kind = _lib.MODEL_SPIN_HALF
        d.n_hx, d.n_jpm = int(op.n_hx_static), int(op.n_jpm_static)
        d.has_jz, d.uniform_jz, d.has_hz = int(op.has_jz), int(op.uniform_jz), int(op.has_hz)
        jz = np.asarray(op.J_z, np.float64)
        d.jz = keep.f64(jz[:1] if op.uniform_jz else np.broadcast_to(jz, (E,)))
        d.jpm = keep.f64(np.broadcast_to(np.asarray(op.J_pm, np.float64), (E,)) if E else np.zeros(1))
        d.jpmpm = keep.f64(np.broadcast_to(np.asarray(op.J_pmpm, np.float64), (E,)) if E else np.zeros(1))
        if op.h_z is not None:
            d.hz = keep.f64(np.broadcast_to(np.asarray(op.h_z, np.float64), (N,)))
        if op.h_x_half is not None:
            d.hx_half = keep.f64(np.broadcast_to(np.asarray(op.h_x_half, np.float64), (N,)))
    else:
        d.kind = _lib.MODEL_BOSE_HUBBARD
        d.n_max = int(op.n_max)
        d.n_hop, d.n_eta, d.n_hpm = int(op.n_hop_off), int(op.n_eta_off), int(op.n_hpm_off)
        d.has_U, d.has_mu = int(op.has_U), int(op.has_mu)
        if E:
            d.t = keep.f64(np.broadcast_to(np.asarray(op.t, np.float64), (E,)))
            d.eta = keep.f64(np.broadcast_to(np.asarray(op.eta, np.float64), (E,)))
        d.U = keep.f64(np.broadcast_to(np.asarray(op.U, np.float64), (N,)))
        d.mu = keep.f64(np.broadcast_to(np.asarray(op.mu, np.float64), (N,)))
        if op.h_pm is not None:
            d.hpm = keep.f64(np.broadcast_to(np.asarray(op.h_pm, np.float64), (N,)))
    return d


def diag_desc(op, n_sites, keep):
    """A diagonal operator (diag_operators) lowered to gfmc_diag_desc:
    SpinHalf / BoseHubbard diagonal_weight or SzSzStructureFactor."""
    from .hamiltonian import SzSzStructureFactor
    d = _lib.DiagDesc()
    d.n_sites = int(n_sites)
    if isinstance(op, SzSzStructureFactor) or all(hasattr(op, a) for a in ("cos", "sin", "offset")):
        cos = np.asarray(op.cos, np.float64)
        if cos.shape[1] != n_sites:
            raise ValueError(f"SzSzStructureFactor has {cos.shape[1]} positions for {n_sites} sites")
        d.kind = _lib.DIAG_SZSZ
        d.n_k = cos.shape[0]
        d.cos_kr, d.sin_kr = keep.f64(cos), keep.f64(np.asarray(op.sin, np.float64))
        d.offset = float(op.offset)
        return d, int(cos.shape[0])
    if _is_spin_half(op):
        d.kind = _lib.DIAG_SPIN_HALF
        E = int(len(op.edge_i))
        d.n_edges = E
        d.edge_i, d.edge_j = keep.i32(op.edge_i), keep.i32(op.edge_j)
        d.has_jz, d.uniform_jz, d.has_hz = int(op.has_jz), int(op.uniform_jz), int(op.has_hz)
        jz = np.asarray(op.J_z, np.float64)
        d.jz = keep.f64(jz[:1] if op.uniform_jz else np.broadcast_to(jz, (E,)))
        if op.h_z is not None:
            d.hz = keep.f64(np.broadcast_to(np.asarray(op.h_z, np.float64), (n_sites,)))
        return d, 1
    if _is_bose(op):
        d.kind = _lib.DIAG_BOSE_HUBBARD
        d.has_U, d.has_mu = int(op.has_U), int(op.has_mu)
        d.U = keep.f64(np.broadcast_to(np.asarray(op.U, np.float64), (n_sites,)))
        d.mu = keep.f64(np.broadcast_to(np.asarray(op.mu, np.float64), (n_sites,)))
        return d, 1
    raise TypeError(f"diagonal operator {type(op).__name__!r} has no device implementation "
                    "(supported: SpinHalf, BoseHubbard, SzSzStructureFactor)")


def guide_desc(guide, op, keep):
    g = _lib.GuideDesc()
    if guide is None:
        g.kind = _lib.GUIDE_NONE
        return g
    if hasattr(guide, "_gfmc_guide_desc"):
        return guide._gfmc_guide_desc(op, keep)
    if _is_exact_guide(guide):
        if not _is_spin_half(op):
            raise TypeError(f"the exact-amplitude guide runs on SpinHalf models only; got "
                            f"{type(op).__name__}")
        N = int(guide.N)
        if N != int(op.N) or N > 26:
            raise ValueError(f"ExactGroundState over {N} sites for an operator of {int(op.N)} sites "
                             "(the device table holds at most 2**26 amplitudes)")
        g.kind = _lib.GUIDE_EXACT_SPIN_HALF
        g.exact_n_sites = N
        g.exact_log_amp = keep.f64(exact_amplitude_table(guide))
        return g
    if _is_spin_jastrow(guide):
        if not _is_spin_half(op):
            raise TypeError(f"JastrowSpinHalf needs an operator with the SpinHalf transition layout "
                            f"(n_hx_static, n_jpm_static, edge_i, edge_j); got {type(op).__name__}")
        if int(guide.N) != int(op.N):
            raise ValueError(f"JastrowSpinHalf guide has N={int(guide.N)} for {int(op.N)} sites")
        pairs, J, h = spin_jastrow_tables(guide)
        g.kind = _lib.GUIDE_JASTROW_SPIN_HALF
        g.n_pairs = len(pairs)
        g.pair_i, g.pair_j = keep.i32(pairs[:, 0]), keep.i32(pairs[:, 1])
        g.pair_w = keep.f64(J)
        g.h = keep.f64(h)
        return g
    if _is_bose_jastrow(guide):
        if not _is_bose(op):
            raise TypeError(f"JastrowBoseHubbard needs a BoseHubbard operator; got {type(op).__name__}")
        g.kind = _lib.GUIDE_JASTROW_BOSE_HUBBARD
        P = len(guide.pair_i)
        g.n_pairs = P
        g.pair_i, g.pair_j = keep.i32(guide.pair_i), keep.i32(guide.pair_j)
        tied = np.ndim(guide._beta) == 0
        g.beta_tied = int(tied)
        g.beta0 = float(np.asarray(guide._beta)) if tied else 0.0
        g.pair_w = keep.f64(np.ones(P) if tied else -np.asarray(guide._beta, np.float64))
        for name in ("h", "d"):
            v = getattr(guide, "_" + name)
            mode = 0 if v is None else (1 if np.ndim(v) == 0 else 2)
            setattr(g, name + "_mode", mode)
            if mode == 1:
                setattr(g, name + "0", float(np.asarray(v)))
            elif mode == 2:
                setattr(g, name, keep.f64(np.asarray(v, np.float64)))
        return g
    if isinstance(guide, RBMSpinHalf):
        if not _is_spin_half(op):
            raise TypeError(f"RBMSpinHalf needs a SpinHalf operator; got {type(op).__name__}")
        if guide.N != int(op.N):
            raise ValueError(f"RBMSpinHalf has {guide.N} visible units for {int(op.N)} sites")
        g.kind = _lib.GUIDE_RBM_SPIN_HALF
        g.n_hidden = guide.n_hidden
        g.rbm_W, g.rbm_b, g.rbm_a = keep.f32(guide.W), keep.f32(guide.b), keep.f32(guide.a)
        return g
    if isinstance(guide, MLPBoseHubbard):
        if not _is_bose(op):
            raise TypeError(f"MLPBoseHubbard needs a BoseHubbard operator; got {type(op).__name__}")
        if guide.N != int(op.N) or guide.n_max != int(op.n_max):
            raise ValueError(f"MLPBoseHubbard is built for {guide.N} sites with n_max {guide.n_max}; "
                             f"the operator has {int(op.N)} sites with n_max {int(op.n_max)}")
        g.kind = _lib.GUIDE_MLP_BOSE_HUBBARD
        g.mlp_H1, g.mlp_H2 = guide.H1, guide.H2
        g.mlp_W1, g.mlp_b1 = keep.f32(guide.W1), keep.f32(guide.b1)
        g.mlp_W2, g.mlp_b2 = keep.f32(guide.W2), keep.f32(guide.b2)
        g.mlp_w3, g.mlp_b3 = keep.f32(guide.w3), float(guide.b3)
        return g
    raise TypeError(f"Guide {type(guide).__name__!r} has no device implementation")


class GFMCEngine:
    """Device state of one walker population on one model/guide pair.

    Holds the packed configurations (``cfg``, ``cfg_tmp``), the parent map
    of the last reconfiguration, and the per-walker float64 weights and
    local energies, all as torch CUDA tensors; every step runs in the CUDA
    engine (``gfmc_run_steps``) on the current torch stream.
    """

    def __init__(self, hamiltonian, guide, n_walkers, precision="fp64"):
        torch = _torch()
        self.torch = torch
        L = _lib.load()
        self.L = L
        self.hamiltonian, self.guide = hamiltonian, guide
        self.n = int(n_walkers)
        self.N = int(hamiltonian.N)
        self.family = _lib.MODEL_SPIN_HALF if _is_spin_half(hamiltonian) else _lib.MODEL_BOSE_HUBBARD
        self.precision = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
        keep = _Keep()
        md = model_desc(hamiltonian, keep)
        gd = guide_desc(guide, hamiltonian, keep)
        h = ctypes.c_void_p()
        _lib.check(L.gfmc_create(ctypes.byref(md), ctypes.byref(gd), self.precision, ctypes.byref(h)),
                   "gfmc_create")
        self.h = h
        self.cfg_bytes = L.gfmc_config_bytes(h)
        self.M = L.gfmc_n_transitions(h)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.cfg = torch.zeros(self.n * self.cfg_bytes, dtype=torch.uint8, device=dev)
        self.cfg_tmp = torch.zeros_like(self.cfg)
        self.parents = torch.arange(self.n, dtype=torch.int32, device=dev)
        self.parents_valid = 0
        self.log_w = torch.zeros(self.n, dtype=torch.float64, device=dev)
        self.e_loc = torch.zeros(self.n, dtype=torch.float64, device=dev)

    def __del__(self):
        try:
            if getattr(self, "h", None) is not None and self.h.value:
                self.L.gfmc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr())

    def load(self, config, e_loc=None):
        """Packs a host or device (n, N) configuration array into ``cfg``."""
        torch = self.torch
        c = torch.as_tensor(np.asarray(config) if not torch.is_tensor(config) else config)
        c = c.to(device=self.device, dtype=torch.float64).contiguous()
        if tuple(c.shape) != (self.n, self.N):
            raise ValueError(f"walker configurations must have shape ({self.n}, {self.N}); got {tuple(c.shape)}")
        _lib.check(self.L.gfmc_pack(self.h, self.n, self._ptr(c), self._ptr(self.cfg), self._stream()),
                   "gfmc_pack")
        st = self.status()
        if st & _lib.STATUS_BAD_CONFIG:
            raise ValueError("walker configurations hold values outside the model's local basis "
                             "(+-1 for spin-1/2, integers in [0, n_max] for bosons)")
        self.parents_valid = 0
        if e_loc is not None:
            self.e_loc.copy_(torch.as_tensor(np.asarray(e_loc), dtype=torch.float64))

    def set_max_iters(self, max_iters):
        _lib.check(self.L.gfmc_set_max_iters(self.h, int(max_iters)), "gfmc_set_max_iters")

    def carry_mode(self, mode=-1):
        """Sets the carried-guide-state mode of a sparse Jastrow guide (1: carry
        while it fits, 0: rebuild per walker every step; -1: unchanged) and
        returns whether the handle carries guide state (gfmc_carry_mode)."""
        v = ctypes.c_int(0)
        _lib.check(self.L.gfmc_carry_mode(self.h, int(mode), ctypes.byref(v)), "gfmc_carry_mode")
        return bool(v.value)

    def status(self):
        v = ctypes.c_int(0)
        _lib.check(self.L.gfmc_read_status(self.h, ctypes.byref(v), self._stream()), "gfmc_read_status")
        return v.value

    def local_energy(self):
        """e_L of the current population (float64 device tensor)."""
        out = self.torch.empty(self.n, dtype=self.torch.float64, device=self.device)
        par = self._ptr(self.parents) if self.parents_valid else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_local_energy(self.h, self.n, self._ptr(self.cfg), par, self._ptr(out),
                                            self._stream()), "gfmc_local_energy")
        return out

    def local_energy_parts(self):
        """(e_L, H_xx) of the current population (float64 device tensors)."""
        e = self.torch.empty(self.n, dtype=self.torch.float64, device=self.device)
        d = self.torch.empty_like(e)
        par = self._ptr(self.parents) if self.parents_valid else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_local_energy_parts(self.h, self.n, self._ptr(self.cfg), par,
                                                  self._ptr(e), self._ptr(d), self._stream()),
                   "gfmc_local_energy_parts")
        return e, d

    def packed_population(self):
        """The current population's packed configurations (host uint8 (n, bytes))."""
        cfg = self.cfg
        if self.parents_valid:
            cfg = self.torch.empty_like(self.cfg)
            _lib.check(self.L.gfmc_gather(self.h, self.n, self._ptr(self.parents), self._ptr(self.cfg),
                                          self._ptr(cfg), ctypes.c_void_p(0), ctypes.c_void_p(0),
                                          ctypes.c_void_p(0), self._stream()), "gfmc_gather")
        return cfg.view(self.n, self.cfg_bytes).cpu().numpy()

    def steps(self, method, step, lam, alw, keys, logG, E, hops=None):
        """len(keys) branching steps; keys is a (n_steps, 4) uint32 host array."""
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        ns = keys.shape[0]
        _lib.check(self.L.gfmc_run_steps(
            self.h, _lib.METHODS[method], float(step), float(lam if lam is not None else 0.0),
            float(alw), ns, keys.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), self.n,
            self._ptr(self.cfg), self._ptr(self.cfg_tmp), self._ptr(self.parents),
            int(self.parents_valid), self._ptr(self.log_w), self._ptr(self.e_loc),
            self._ptr(logG), self._ptr(E), self._ptr(hops) if hops is not None else ctypes.c_void_p(0),
            self._stream()), "gfmc_run_steps")
        self.parents_valid = 1

    def population(self):
        """The current walkers (config float64 (n, N), e_loc) as device tensors."""
        torch = self.torch
        cfg = self.cfg
        e = self.e_loc
        if self.parents_valid:
            cfg = torch.empty_like(self.cfg)
            e = torch.empty_like(self.e_loc)
            _lib.check(self.L.gfmc_gather(self.h, self.n, self._ptr(self.parents), self._ptr(self.cfg),
                                          self._ptr(cfg), self._ptr(self.e_loc), self._ptr(e),
                                          ctypes.c_void_p(0), self._stream()), "gfmc_gather")
        out = torch.empty((self.n, self.N), dtype=torch.float64, device=self.device)
        _lib.check(self.L.gfmc_unpack(self.h, self.n, self._ptr(cfg), self._ptr(out), self._stream()),
                   "gfmc_unpack")
        return out, e

    def set_diag_operators(self, ops, m_array):
        """Diagonal operators (name -> op) measured by forward walking at the
        windows m_array; returns the per-operator column widths."""
        keep = _Keep()
        descs, widths = [], []
        for name, op in ops.items():
            d, w = diag_desc(op, self.N, keep)
            if (d.kind == _lib.DIAG_BOSE_HUBBARD) != (self.family == _lib.MODEL_BOSE_HUBBARD) and \
                    d.kind != _lib.DIAG_SZSZ:
                raise TypeError(f"diagonal operator {name!r} does not act on this model's configurations")
            descs.append(d)
            widths.append(w)
        arr = (_lib.DiagDesc * max(1, len(descs)))(*descs)
        m = np.ascontiguousarray(m_array, dtype=np.int32)
        _lib.check(self.L.gfmc_set_diag_operators(self.h, len(descs), arr, len(m),
                                                  m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                   "gfmc_set_diag_operators")
        self.diag_widths = widths
        self.diag_width = self.L.gfmc_diag_width(self.h)
        return widths

    def reset_diag(self):
        _lib.check(self.L.gfmc_reset_diag(self.h, self.n, self._stream()), "gfmc_reset_diag")

    def set_diag_output(self, out):
        _lib.check(self.L.gfmc_set_diag_output(self.h, self._ptr(out) if out is not None
                                               else ctypes.c_void_p(0)), "gfmc_set_diag_output")

    def rbm_theta(self):
        """theta = b + W s of the current population on the tensor cores
        (float32 device tensor (n, Hp), Hp = n_hidden padded to 256)."""
        Hp = self.L.gfmc_rbm_hidden_padded(self.h)
        _lib.check(Hp if Hp < 0 else 0, "gfmc_rbm_hidden_padded")
        out = self.torch.empty((self.n, Hp), dtype=self.torch.float32, device=self.device)
        _lib.check(self.L.gfmc_rbm_theta(self.h, self.n, self._ptr(self.cfg), self._ptr(self.parents),
                                         int(self.parents_valid), self._ptr(out), self._stream()),
                   "gfmc_rbm_theta")
        return out

    def rbm_gradient(self, omega=None):
        """Variance-loss gradient of the RBM guide over the current population:
        (dW (H, N), db (H,), da (N,)) float32 device tensors and (E, var)."""
        torch = self.torch
        g = self.guide
        gW = torch.empty((g.n_hidden, self.N), dtype=torch.float32, device=self.device)
        gb = torch.empty(g.n_hidden, dtype=torch.float32, device=self.device)
        ga = torch.empty(self.N, dtype=torch.float32, device=self.device)
        st = np.zeros(2, dtype=np.float64)
        om = self._ptr(omega) if omega is not None else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_rbm_gradient(
            self.h, self.n, self._ptr(self.cfg), self._ptr(self.parents), int(self.parents_valid), om,
            self._ptr(gW), self._ptr(gb), self._ptr(ga),
            st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()), "gfmc_rbm_gradient")
        return gW, gb, ga, (float(st[0]), float(st[1]))

    def rbm_train_step(self, lr, omega=None):
        """One Adam step of the RBM guide on the current population; returns
        (E, var) of the population before the step."""
        st = np.zeros(2, dtype=np.float64)
        om = self._ptr(omega) if omega is not None else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_rbm_train_step(
            self.h, self.n, self._ptr(self.cfg), self._ptr(self.parents), int(self.parents_valid), om,
            float(lr), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
            "gfmc_rbm_train_step")
        return float(st[0]), float(st[1])

    def rbm_parameters(self):
        """The guide's current (W, b, a) as host float32 arrays."""
        g = self.guide
        W = np.zeros((g.n_hidden, self.N), dtype=np.float32)
        b = np.zeros(g.n_hidden, dtype=np.float32)
        a = np.zeros(self.N, dtype=np.float32)
        P = ctypes.POINTER(ctypes.c_float)
        _lib.check(self.L.gfmc_rbm_get_params(self.h, W.ctypes.data_as(P), b.ctypes.data_as(P),
                                              a.ctypes.data_as(P)), "gfmc_rbm_get_params")
        return W, b, a

    def _mlp_split(self, flat):
        """The MLP parameter order W1 (H1, D), b1, W2 (H2, H1), b2, w3 as views."""
        g = self.guide
        H1, H2, D = g.H1, g.H2, g.N * (g.n_max + 1)
        sizes = [("W1", (H1, D)), ("b1", (H1,)), ("W2", (H2, H1)), ("b2", (H2,)), ("w3", (H2,))]
        out, o = {}, 0
        for name, shp in sizes:
            k = int(np.prod(shp))
            out[name] = flat[o:o + k].reshape(shp)
            o += k
        return out

    def mlp_gradient(self, omega=None):
        """Variance-loss gradient of the MLP guide over the current population:
        a dict of float32 device tensors (W1, b1, W2, b2, w3) and (E, var)."""
        torch = self.torch
        np_ = int(self.L.gfmc_mlp_param_count(self.h))
        _lib.check(np_ if np_ < 0 else 0, "gfmc_mlp_param_count")
        grad = torch.empty(np_, dtype=torch.float32, device=self.device)
        st = np.zeros(2, dtype=np.float64)
        om = self._ptr(omega) if omega is not None else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_mlp_gradient(
            self.h, self.n, self._ptr(self.cfg), self._ptr(self.parents), int(self.parents_valid), om,
            self._ptr(grad), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
            "gfmc_mlp_gradient")
        return self._mlp_split(grad), (float(st[0]), float(st[1]))

    def mlp_train_step(self, lr, omega=None):
        """One Adam step of the MLP guide on the current population; returns
        (E, var) of the population before the step."""
        st = np.zeros(2, dtype=np.float64)
        om = self._ptr(omega) if omega is not None else ctypes.c_void_p(0)
        _lib.check(self.L.gfmc_mlp_train_step(
            self.h, self.n, self._ptr(self.cfg), self._ptr(self.parents), int(self.parents_valid), om,
            float(lr), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
            "gfmc_mlp_train_step")
        return float(st[0]), float(st[1])

    def mlp_parameters(self):
        """The guide's current parameters as used (bf16 weight values): a dict
        of host float32 arrays W1, b1, W2, b2, w3."""
        np_ = int(self.L.gfmc_mlp_param_count(self.h))
        _lib.check(np_ if np_ < 0 else 0, "gfmc_mlp_param_count")
        flat = np.zeros(np_, dtype=np.float32)
        _lib.check(self.L.gfmc_mlp_get_params(self.h, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                   "gfmc_mlp_get_params")
        return {k: v.copy() for k, v in self._mlp_split(flat).items()}

    def copy_population_from(self, other):
        """This engine's population := other's current population (gathered
        through its parent map); weights and local energies restart."""
        par = other.parents if other.parents_valid else self.torch.arange(
            self.n, dtype=self.torch.int32, device=self.device)
        _lib.check(self.L.gfmc_gather(self.h, self.n, self._ptr(par), self._ptr(other.cfg),
                                      self._ptr(self.cfg), self._ptr(other.e_loc), self._ptr(self.e_loc),
                                      self._ptr(self.log_w), self._stream()), "gfmc_gather")
        self.parents_valid = 0

    def forward_walk(self, op, main, method, step, lam, alw, apply_key, shadow_keys, m_array,
                     val_out, norm_out):
        """One forward walk of operator handle ``op`` from ``main``'s current
        population with this engine as the shadow chain (gfmc_forward_walk);
        writes mean values and log norms at the depths m_array into the
        float64 device views val_out, norm_out (n_p each)."""
        torch = self.torch
        if getattr(self, "_fw_vals", None) is None:
            self._fw_vals = torch.empty(self.n, dtype=torch.float64, device=self.device)
            self._fw_vals_tmp = torch.empty_like(self._fw_vals)
        apply_key = np.ascontiguousarray(apply_key, dtype=np.uint32)
        sk = np.ascontiguousarray(shadow_keys, dtype=np.uint32)
        m = np.ascontiguousarray(m_array, dtype=np.int32)
        P = ctypes.POINTER(ctypes.c_uint32)
        _lib.check(self.L.gfmc_forward_walk(
            self.h, op.h, _lib.METHODS[method], float(step), float(lam if lam is not None else 0.0),
            float(alw), apply_key.ctypes.data_as(P), sk.ctypes.data_as(P) if sk.size else None,
            self.n, self._ptr(main.cfg), self._ptr(main.parents), int(main.parents_valid),
            self._ptr(self.cfg), self._ptr(self.cfg_tmp), self._ptr(self.parents),
            self._ptr(self.log_w), self._ptr(self.e_loc), self._ptr(self._fw_vals),
            self._ptr(self._fw_vals_tmp), len(m), m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            self._ptr(val_out), self._ptr(norm_out), self._stream()), "gfmc_forward_walk")
        self.parents_valid = 1

    def windowed_energy(self, logG, E, p_array):
        p = np.ascontiguousarray(p_array, dtype=np.int32)
        out = np.zeros(len(p), dtype=np.float64)
        _lib.check(self.L.gfmc_windowed_energy(
            int(logG.numel()), self._ptr(logG), self._ptr(E), len(p),
            p.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self._stream()),
            "gfmc_windowed_energy")
        return dict(zip([int(v) for v in p], out.tolist()))


class OperatorHandle:
    """Device tables of a measurement operator under the run's guide -- the
    analogue of ``guide.build_cache(op)`` (engine/driver.py:1476-1477) --
    for gfmc_apply_operator / gfmc_forward_walk / gfmc_operator_min_rate."""

    def __init__(self, op, guide, precision):
        L = _lib.load()
        self.L = L
        keep = _Keep()
        md = model_desc(op, keep)
        gd = guide_desc(guide, op, keep)
        h = ctypes.c_void_p()
        _lib.check(L.gfmc_create(ctypes.byref(md), ctypes.byref(gd),
                                 {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision],
                                 ctypes.byref(h)), "gfmc_create (operator)")
        self.h = h
        self.M = L.gfmc_n_transitions(h)

    def __del__(self):
        try:
            if getattr(self, "h", None) is not None and self.h.value:
                self.L.gfmc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def min_rates(self, eng, count):
        """Smallest rate per walker of the first ``count`` walkers of
        ``eng``'s population (host float64; NaN where a rate is not finite)."""
        torch = eng.torch
        out = torch.empty(eng.n, dtype=torch.float64, device=eng.device)
        _lib.check(self.L.gfmc_operator_min_rate(self.h, eng.n, eng._ptr(eng.cfg), eng._ptr(eng.parents),
                                                 int(eng.parents_valid), eng._ptr(out), eng._stream()),
                   "gfmc_operator_min_rate")
        return out[:count].cpu().numpy()

    def apply(self, eng, key):
        """apply_operator_one over ``eng``'s population: (packed successor
        configurations, values) as device tensors."""
        torch = eng.torch
        cfg_out = torch.empty_like(eng.cfg)
        vals = torch.empty(eng.n, dtype=torch.float64, device=eng.device)
        key = np.ascontiguousarray(key, dtype=np.uint32)
        _lib.check(self.L.gfmc_apply_operator(self.h, key.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                              eng.n, eng._ptr(eng.cfg), eng._ptr(eng.parents),
                                              int(eng.parents_valid), eng._ptr(cfg_out), eng._ptr(vals),
                                              eng._stream()), "gfmc_apply_operator")
        return cfg_out, vals


def _is_vector_op(op):
    """Whether diagonal_weight returns a vector (keeps its value axis)."""
    return all(hasattr(op, a) for a in ("cos", "sin", "offset"))


def key_schedule(key, n_steps):
    """(n_steps, 4) production keys (k1, k2 per step) and the next key."""
    L = _lib.load()
    key = np.ascontiguousarray(_rnd.as_key(key))
    out = np.zeros((n_steps, 4), dtype=np.uint32)
    nxt = np.zeros(2, dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    _lib.check(L.gfmc_key_schedule(key.ctypes.data_as(P), int(n_steps), out.ctypes.data_as(P),
                                   nxt.ctypes.data_as(P)), "gfmc_key_schedule")
    return out, nxt


_AUX_POSITIVITY = 10_001
_AUX_STATISTICS = 10_002
_POSITIVITY_PROBE_STEPS = 100
_N_POSITIVITY_CHECK = 100


def measurement_plan(n_steps, p_array, n_off_ops, off_diag_stride, return_raw):
    """Window grid and off-diagonal measurement grid of one call
    (engine/driver.py _measurement_plan:478-551).  Off-diagonal rows are
    measured at the steps t with (t + 1) % stride == 0; without raw series
    (return_raw False) only in the band every window can use, so every p
    rests on the same measurements."""
    p = list(p_array)
    m = [v // 2 for v in p]
    equal = not bool(return_raw)
    p_max = p[-1] if p else 0
    m_od = p_max // 2
    if p_max >= n_steps:
        raise ValueError(f"every p value must be smaller than n_steps: got n_steps={n_steps} and "
                         f"max(p)={p_max}")
    if n_off_ops > 0 and n_steps <= p_max + m_od:
        raise ValueError(f"off-diagonal operators need n_steps > 1.5*max(p) (max(p) + max(p)//2 = "
                         f"{p_max + m_od}: every window p needs p past and p//2 future steps in this "
                         f"call), got n_steps={n_steps}")
    gate = n_off_ops > 0 and (off_diag_stride > 1 or equal)
    if equal and n_off_ops > 0:
        offset = next((k for k in range(p_max, p_max + off_diag_stride)
                       if (k + 1) % off_diag_stride == 0), p_max)
        if not any((k + 1) % off_diag_stride == 0 for k in range(p_max, n_steps - m_od)):
            raise ValueError(
                f"equal off-diagonal windows (return_raw=False) measure only the steps "
                f"{p_max}..{n_steps - m_od - 1} (n_steps={n_steps} minus the lead-in max(p)={p_max} "
                f"and the tail max(p)//2={m_od}), and none of them is a multiple of "
                f"off_diag_stride={off_diag_stride} (counted from 1); raise n_steps or lower the stride")
    else:
        offset = off_diag_stride - 1
    return SimpleNamespace(p_array=p, m_array=m, p_max=p_max, m_max=max(m) if m else 0,
                           n_off_ops=n_off_ops, off_diag_stride=off_diag_stride,
                           equal_windows=equal, gate_off_diag=gate, off_diag_offset=offset)


def measured_steps(n_steps, plan):
    """The 0-based production steps that measure the off-diagonal operators
    (engine/driver.py _measured_steps:554-564)."""
    t = np.arange(n_steps)
    meas = (t + 1) % plan.off_diag_stride == 0
    if plan.equal_windows and plan.n_off_ops > 0:
        meas &= (t >= plan.p_max) & (t <= n_steps - plan.p_max // 2 - 1)
    return t[meas]


def key_schedule_ex(key, n_steps, n_sub):
    """(n_steps, n_sub, 2) sub-keys fold_in(rng_s, j) of the production key
    recurrence and the key after n_steps (gfmc_key_schedule_ex)."""
    L = _lib.load()
    key = np.ascontiguousarray(_rnd.as_key(key))
    out = np.zeros((n_steps, n_sub, 2), dtype=np.uint32)
    nxt = np.zeros(2, dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    _lib.check(L.gfmc_key_schedule_ex(key.ctypes.data_as(P), int(n_steps), int(n_sub),
                                      out.ctypes.data_as(P), nxt.ctypes.data_as(P)),
               "gfmc_key_schedule_ex")
    return out, nxt


def _warmup_keys(rngs):
    """k1, k2 = split(rng) for every step of a warm-up chunk (driver.py:183-185)."""
    out = np.zeros((len(rngs), 4), dtype=np.uint32)
    for i, r in enumerate(rngs):
        ks = _rnd.split(r, 2)
        out[i, :2], out[i, 2:] = ks[0], ks[1]
    return out


def warmup_schedule(method, step_f, warmup_steps):
    """engine/driver.py _warmup_schedule:567-584."""
    if warmup_steps <= 0:
        return []
    base, extra = divmod(warmup_steps, 4)
    counts = [base + (i < extra) for i in range(4)]
    if method == "cont_time":
        sizes = [step_f / 8.0, step_f / 4.0, step_f / 2.0, step_f]
    else:
        nb = int(step_f)
        sizes = [float(max(1, nb // 8)), float(max(1, nb // 4)), float(max(1, nb // 2)), float(nb)]
    return [(s, c) for s, c in zip(sizes, counts) if c > 0]


def _logsumexp(a):
    a = np.asarray(a, dtype=np.float64)
    m = np.max(a)
    if not np.isfinite(m):
        return float(m)
    return float(np.log(np.sum(np.exp(a - m))) + m)


def _check_population(log_G_chunk, step0, E_chunk=None):
    """engine/driver.py _check_population:913-937."""
    bad = np.flatnonzero(~np.isfinite(log_G_chunk))
    if bad.size:
        raise ValueError(
            f"[gfmc] population extinct at step {step0 + int(bad[0])}: the mean branch weight of "
            "the step is not finite, i.e. every walker's weight is zero (or one overflowed).  The "
            "ensemble cannot be renormalised; check lam against the diagonal elements (discrete "
            "methods), the step size and the guide.")
    if E_chunk is not None:
        bad = np.flatnonzero(~np.isfinite(E_chunk))
        if bad.size:
            raise ValueError(
                f"[gfmc] non-finite energy at step {step0 + int(bad[0])}: the weighted mean of the "
                "local energies is not finite while the branch weights are, i.e. a walker's local "
                "energy overflowed (a guide ratio or a rate of its configuration is inf or NaN); "
                "check the guide and the Hamiltonian on the configurations the walk reaches.")


def _device_status_check(eng):
    st = eng.status()
    if st & _lib.STATUS_HOP_CAP:
        raise _lib.GFMCError("a walker exceeded the per-step iteration cap (max_hops_per_step, "
                             "default 2**22 holds): the escape rate times the step size is far "
                             "too large for this model")
    if st & _lib.STATUS_TIMEOUT:
        raise _lib.GFMCError("a bounded wait on the tensor-core pipeline ran out (theta GEMM); "
                             "the results of this call are not valid")


def _weight_dtype(lw):
    dt = getattr(lw, "dtype", None)
    if dt is None:
        return np.dtype(np.float64)
    name = str(dt).replace("torch.", "")
    return np.dtype(np.float32) if name in ("float32", "bfloat16", "float16") else np.dtype(np.float64)


def _population_engine(walkers, hamiltonian, guide, precision):
    """A GFMCEngine holding the host population ``walkers`` (validated)."""
    config = np.asarray(walkers.config)
    n = config.shape[0] if config.ndim == 2 else -1
    if n < 1 or np.shape(walkers.log_weight) != (n,) or np.shape(walkers.e_loc) != (n,):
        raise ValueError(f"walkers must hold config (N_walkers, N_sites) with N_walkers >= 1 and "
                         f"log_weight, e_loc of shape (N_walkers,); got {config.shape}, "
                         f"{np.shape(walkers.log_weight)} and {np.shape(walkers.e_loc)}.")
    require_operator_protocol(hamiltonian)
    if guide is not None:
        require_guide_protocol(guide)
    if precision not in (None, "fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64', 'mixed' or None, got {precision!r}")
    if precision is None:
        precision = "fp64" if _weight_dtype(walkers.log_weight) == np.float64 \
            and not isinstance(guide, MLPBoseHubbard) else "mixed"
    eng = GFMCEngine(hamiltonian, guide, n, precision=precision)
    eng.load(config)
    return eng


def evolve_walkers(walkers, hamiltonian, step_size, guide, method, rng_key, avg_log_weight,
                   lam=None, cache=None, rates=None, state=None, return_rates=False, precision=None):
    """One evolution of the whole population without resampling, on the GPU
    (engine/evolution.py evolve_walkers:761-843): walker i draws from
    split(rng_key, N_walkers)[i]; its log weight accumulates onto
    ``walkers.log_weight`` (the step's terms added to the incoming value in
    PyGFMC's order, then avg_log_weight x beta or x n_bra subtracted); its
    ``e_loc`` is the local energy of its final configuration.  ``step_size``
    is beta for cont_time and the number of sub-steps for the discrete
    methods, which need ``lam``.

    ``cache``, ``rates`` and ``state`` are accepted for PyGFMC's signature
    and not needed: the device builds the tables and the guide state from the
    configurations, which gives the same walk (in PyGFMC they only spare a
    recomputation).  ``return_rates=True`` is refused: the device keeps each
    walker's evaluation itself, and chained steps belong to ``run`` /
    ``GFMCEngine``.  Float64 weights select the fp64 build, float32 the mixed
    build (log weights accumulate in float64 there and are returned in the
    input's dtype), or pass ``precision``.  Returns a Walker of host arrays
    in the input's dtypes."""
    require_step_size(method, step_size)
    lam = require_lam(method, lam)
    if return_rates:
        raise ValueError("return_rates=True is not available: the device engine carries each walker's "
                         "rate evaluation from step to step itself; use run() or GFMCEngine for "
                         "chained steps.")
    eng = _population_engine(walkers, hamiltonian, guide, precision)
    torch = eng.torch
    lw = torch.as_tensor(np.ascontiguousarray(walkers.log_weight, dtype=np.float64)).to(eng.device)
    cfg_out = torch.empty_like(eng.cfg)
    key = np.ascontiguousarray(_rnd.as_key(rng_key), dtype=np.uint32)
    _lib.check(eng.L.gfmc_evolve_walkers(
        eng.h, _lib.METHODS[method], float(step_size), float(lam if lam is not None else 0.0),
        float(avg_log_weight), key.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), eng.n,
        eng._ptr(eng.cfg), eng._ptr(cfg_out), eng._ptr(lw), eng._ptr(eng.e_loc), ctypes.c_void_p(0),
        eng._stream()), "evolve_walkers")
    _device_status_check(eng)
    out = torch.empty((eng.n, eng.N), dtype=torch.float64, device=eng.device)
    _lib.check(eng.L.gfmc_unpack(eng.h, eng.n, eng._ptr(cfg_out), eng._ptr(out), eng._stream()),
               "gfmc_unpack")
    cfg_dt = np.asarray(walkers.config).dtype
    return Walker(config=out.cpu().numpy().astype(cfg_dt, copy=False),
                  log_weight=lw.cpu().numpy().astype(np.asarray(walkers.log_weight).dtype, copy=False),
                  e_loc=eng.e_loc.cpu().numpy().astype(np.asarray(walkers.e_loc).dtype, copy=False))


def estimate_average_log_branch_weight(walkers, hamiltonian, guide, method="cont_time", lam=None,
                                       cache=None, precision=None):
    """The starting avg_log_weight of a run (engine/estimators.py:722-751):
    mean(-e_L) for cont_time (per unit imaginary time), mean(log(lam - e_L))
    for the discrete methods (per sub-step), e_L = the sum of the
    guide-transformed rates of each walker's configuration, evaluated on the
    GPU.  ``cache`` is accepted for PyGFMC's signature and not needed."""
    lam = require_lam(method, lam)
    eng = _population_engine(walkers, hamiltonian, guide, precision)
    e = eng.local_energy().cpu().numpy()
    _device_status_check(eng)
    return float(np.mean(-e)) if method == "cont_time" else float(np.mean(np.log(lam - e)))


def run_gfmc(walkers, n_steps, hamiltonian, step_size, guide, p_array, *, method="cont_time",
             rng_key=None, lam=None, diag_operators=None, off_diag_operators=None,
             return_raw=True, avg_log_weight=None, warmup_steps=None, verbosity=7,
             number_of_outputs=100, off_diag_stride=1, off_diag_batch_size=None,
             precision=None, max_hops_per_step=None, _step_offset=0, _shards=None):
    """GFMC on one B200 with PyGFMC's run_gfmc signature and return tuple.

    ``precision``: ``"fp64"`` (every step quantity in float64, the build that
    reproduces PyGFMC's float64 runs) or ``"mixed"`` (rates, ratios, local
    energies in float32; weights, resampling sums and energies in float64).
    Default: ``"fp64"`` for float64 walker weights, ``"mixed"`` for float32.
    """
    wall_start = time.time()
    if rng_key is None:
        seed = secrets.randbits(32)
        _emit(f"[gfmc] - [run_gfmc] - rng_key not given; using jax.random.PRNGKey({seed})", verbosity, 1)
        rng_key = _rnd.PRNGKey(seed)
    rng_key = _rnd.as_key(rng_key)
    rng_key_in = rng_key.copy()
    aux_root = _rnd.fold_in(rng_key, _AUX_ROOT)
    config = walkers.config
    N_walker = int(np.shape(config)[0])
    if N_walker == 0:
        raise ValueError("At least one walker is required.")
    weight_dtype = _weight_dtype(walkers.log_weight)
    n_steps = _validated_int("n_steps", n_steps, 1)
    require_step_size(method, step_size)
    if warmup_steps is None:
        warmup_steps = DEFAULT_WARMUP_STEPS if avg_log_weight is None else 0
    warmup_steps = _validated_int("warmup_steps", warmup_steps, 0)
    number_of_outputs = _validated_int("number_of_outputs", number_of_outputs, 1)
    off_diag_stride = _validated_int("off_diag_stride", off_diag_stride, 1)
    if off_diag_batch_size is not None:
        off_diag_batch_size = _validated_int("off_diag_batch_size", off_diag_batch_size, 1)
        if N_walker % off_diag_batch_size:
            raise ValueError(f"off_diag_batch_size={off_diag_batch_size} must divide "
                             f"N_walkers={N_walker} (a remainder would compile a second shape "
                             "for the tail; keep one shape so throughput and memory stay predictable)")
    lam_given = lam
    lam = require_lam(method, lam)
    require_operator_protocol(hamiltonian, role="hamiltonian")
    for name, op in (off_diag_operators or {}).items():
        require_operator_protocol(op, role=f"off-diagonal operator {name!r}")
    require_guide_protocol(guide)
    p_in = len(p_array) if p_array is not None else 0
    p_array = validated_p_array(p_array)
    if len(p_array) != p_in:
        _emit(f"[gfmc.run_gfmc] dedup'd p_array: {p_in - len(p_array)} duplicate value(s) "
              f"dropped, using {p_array}", verbosity)
    off_names = list(off_diag_operators.keys()) if off_diag_operators else []
    diag_names = list(diag_operators.keys()) if diag_operators else []
    collisions = set(diag_names) & set(off_names)
    if collisions:
        raise ValueError(
            f"diag_operators and off_diag_operators share name(s) {sorted(collisions)}; the returned "
            "obs dict is keyed by name, so colliding entries would silently overwrite each other.")
    if off_diag_operators is not None:
        # the shadow chain is m = p // 2 steps deep (driver.py:1453-1463)
        if any(int(op.M_total) > 1 for op in off_diag_operators.values()):
            bad = [p for p in p_array if p % 2 != 0]
            if bad:
                raise ValueError("All p values must be divisible by 2 when off_diag_operators have "
                                 f"off-diagonal elements (M_total > 1); got {bad}")
    plan = measurement_plan(n_steps, p_array, len(off_names), off_diag_stride, return_raw)
    m_array = plan.m_array
    if avg_log_weight is None and warmup_steps == 0:
        raise ValueError(
            "warmup_steps=0 needs an avg_log_weight: without a warm-up nothing measures it. Pass "
            "avg_log_weight=stats['avg_log_weight'] of the run being continued (run_from_HDF5 does "
            f"this), or leave warmup_steps unset for the default warm-up of {DEFAULT_WARMUP_STEPS} steps.")
    if precision is None:
        # the MLP guide's kernel exists in the float32 build only
        precision = "fp64" if weight_dtype == np.float64 and not isinstance(guide, MLPBoseHubbard) \
            else "mixed"
    step_f = float(step_size)

    torch = _torch()
    n_dev = 1
    if _shards is not None:
        # a population sharded over GPUs (no measurement operators here)
        from .distributed import ShardedPopulation
        n_dev, shard_devices = _shards
        if shard_devices is None:
            import torch.distributed as dist
            grouped = dist.is_available() and dist.is_initialized() and dist.get_world_size() == n_dev
            if not grouped:
                if torch.cuda.device_count() < n_dev:
                    raise ValueError(f"n_devices={n_dev} but {torch.cuda.device_count()} GPU(s) are "
                                     "visible and no torch.distributed group of that size is set up")
                shard_devices = [f"cuda:{d}" for d in range(n_dev)]
        if N_walker % n_dev:
            raise ValueError(f"N_walkers={N_walker} must be divisible by n_devices={n_dev}")
        eng = ShardedPopulation(hamiltonian, guide, N_walker, precision=precision,
                                devices=shard_devices)
    else:
        eng = GFMCEngine(hamiltonian, guide, N_walker, precision=precision)
    if max_hops_per_step is not None:
        eng.set_max_iters(_validated_int("max_hops_per_step", max_hops_per_step, 1))
    eng.load(np.asarray(config) if not torch.is_tensor(config) else config)

    # ---- warm-up (driver.py _warmup:747-788)
    alw_pinned = avg_log_weight is not None
    if not alw_pinned:
        e = eng.local_energy().cpu().numpy()
        alw = float(np.mean(-e)) if method == "cont_time" else float(np.mean(np.log(lam - e)))
    else:
        alw = float(avg_log_weight)
    dev = eng.device
    stages = warmup_schedule(method, step_f, warmup_steps)
    for i, (step_, n_w) in enumerate(stages):
        t0 = time.time()
        sub = _rnd.fold_in(_rnd.fold_in(aux_root, int(n_w)), int(step_ * 1000))
        remaining = n_w
        lg_all = []
        while remaining > 0:
            mm = min(_WARMUP_CHUNK, remaining)
            sub, k = _rnd.split(sub, 2)
            keys = _warmup_keys(_rnd.split(k, mm))
            lg = torch.empty(mm, dtype=torch.float64, device=dev)
            Ee = torch.empty(mm, dtype=torch.float64, device=dev)
            eng.steps(method, step_, lam, alw, keys, lg, Ee)
            lg_all.append(lg.cpu().numpy())
            remaining -= mm
        _device_status_check(eng)
        measured = alw + (_logsumexp(np.concatenate(lg_all)) - math.log(n_w)) / step_
        label = f"{i + 1}/{len(stages)}"
        el = max(time.time() - t0, 1e-9)
        if method == "cont_time":
            _emit(f"[gfmc] - [run_warmup {label}] - step={step_}, {n_w} steps @ {n_w / el:.1f} it/s, "
                  f"avg_log_weight = {measured:.6f}", verbosity, 8)
        else:
            _emit(f"[gfmc] - [run_warmup {label}] - step={step_}, {n_w} steps @ {n_w / el:.1f} it/s, "
                  f"average_b_x = {math.exp(measured):.6f}", verbosity, 8)
        if alw_pinned:
            _emit(f"[gfmc] - [run_warmup {label}] - alw pinned at {alw:.6f}; this stage would have "
                  f"measured {measured:.6f}", verbosity, 8)
        else:
            alw = measured
    if not stages:
        _emit(f"[gfmc] - [run_gfmc] - no warmup (warmup_steps=0), avg_log_weight={alw:.6f}", verbosity, 8)

    # ---- off-diagonal operators: device tables, shadow chain, positivity
    #      probe on a side-stream (driver.py _positivity_probe:791-807)
    op_handles, shadow = [], None
    if off_names:
        op_handles = [OperatorHandle(off_diag_operators[nm], guide, precision) for nm in off_names]
        shadow = GFMCEngine(hamiltonian, guide, N_walker, precision=precision)
        if max_hops_per_step is not None:
            shadow.set_max_iters(int(max_hops_per_step))
        shadow.copy_population_from(eng)
        rngs = _rnd.split(_rnd.fold_in(aux_root, _AUX_POSITIVITY), _POSITIVITY_PROBE_STEPS)
        lgp = torch.empty(_POSITIVITY_PROBE_STEPS, dtype=torch.float64, device=dev)
        Ep = torch.empty_like(lgp)
        shadow.steps(method, step_f, lam, alw, _warmup_keys(rngs), lgp, Ep)
        n_check = min(_N_POSITIVITY_CHECK, N_walker)
        for nm, oh in zip(off_names, op_handles):
            if oh.M == 1:
                continue
            mins = oh.min_rates(shadow, n_check)
            if not np.all(np.isfinite(mins) & (mins >= 0)):
                raise ValueError(f"Operator '{nm}': negative rate detected (min = {float(np.min(mins)):.6f}). "
                                 "All rates must be >= 0.")
        _emit("[estimators] - [check_off_diag_operator_positivity] - all operators passed positivity "
              f"check ({n_check} configs, {len(off_names)} operators)", verbosity, 1)

    # ---- diagonal forward walking: ring buffers start after the warm-up
    #      (driver.py _diag_ring_buffers:810-838, called after _warmup)
    n_p = len(p_array)
    diag_d = None
    if diag_names:
        widths = eng.set_diag_operators(diag_operators, m_array)
        eng.reset_diag()
        diag_d = torch.zeros((n_steps, eng.diag_width, n_p), dtype=torch.float64, device=dev)

    # ---- production (driver.py _production:940-1143), chunked and pipelined
    print_every = max(1, n_steps // max(1, number_of_outputs))
    chunk = print_every if verbosity >= 1 else n_steps
    logG_d = torch.empty(n_steps, dtype=torch.float64, device=dev)
    E_d = torch.empty(n_steps, dtype=torch.float64, device=dev)
    hops_d = torch.zeros(n_steps, dtype=torch.int64, device=dev)
    logG_h = torch.empty(n_steps, dtype=torch.float64, pin_memory=True)
    E_h = torch.empty(n_steps, dtype=torch.float64, pin_memory=True)
    key = rng_key.copy()
    prod_start = time.time()
    pending = []
    step0 = 0
    last_print_t, last_print_step = prod_start, 0
    meas = measured_steps(n_steps, plan) if off_names else np.zeros(0, dtype=np.int64)
    n_meas = len(meas)
    od_d = on_d = None
    if off_names:
        od_d = torch.full((n_meas, len(off_names), n_p), float("nan"), dtype=torch.float64, device=dev)
        on_d = torch.full_like(od_d, float("nan"))
    m_max_od = plan.m_max if off_names else 0
    row = 0

    def run_range(a, b, keys, step0):
        """Main-chain steps step0+a .. step0+b-1 of the chunk."""
        sl = slice(step0 + a, step0 + b)
        if diag_d is not None:
            eng.set_diag_output(diag_d[sl])
        eng.steps(method, step_f, lam, alw, keys[a:b], logG_d[sl], E_d[sl], hops_d[sl])

    while step0 < n_steps:
        cs = min(chunk, n_steps - step0)
        keys, key_after = key_schedule(key, cs)
        sl = slice(step0, step0 + cs)
        if not off_names:
            run_range(0, cs, keys, step0)
        else:
            # forward walks right after each measured step's reconfiguration;
            # the shadow replays the main chain's next m_max steps' keys
            # (driver.py:291-316): the chunk's schedule runs m_max further
            kx, _ = key_schedule_ex(key, cs + m_max_od, 3)
            a = 0
            for t in meas[(meas >= step0) & (meas < step0 + cs)] - step0:
                t = int(t)
                run_range(a, t + 1, keys, step0)
                a = t + 1
                k3 = kx[t, 2]
                ak0, ak1 = _rnd.threefry2x32(k3[0], k3[1], np.zeros(len(off_names), np.uint32),
                                              np.arange(len(off_names), dtype=np.uint32))
                sk = np.ascontiguousarray(kx[t + 1:t + 1 + m_max_od, :2].reshape(m_max_od, 4))
                for i, oh in enumerate(op_handles):
                    shadow.forward_walk(oh, eng, method, step_f, lam, alw,
                                        np.array([ak0[i], ak1[i]], dtype=np.uint32), sk, m_array,
                                        od_d[row, i], on_d[row, i])
                row += 1
            if a < cs:
                run_range(a, cs, keys, step0)
        key = key_after
        logG_h[sl].copy_(logG_d[sl], non_blocking=True)
        E_h[sl].copy_(E_d[sl], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        pending.append((step0, cs, ev))
        step0 += cs
        # process every chunk but the one just dispatched (pipelining)
        while len(pending) > 1 or (pending and step0 >= n_steps):
            s0, c0, e0 = pending.pop(0)
            e0.synchronize()
            lgc = logG_h[s0:s0 + c0].numpy()
            Ec = E_h[s0:s0 + c0].numpy()
            _check_population(lgc, s0, Ec)
            done = s0 + c0
            if verbosity >= 1 and done - 1 > p_array[-1]:
                now = time.time()
                rate = (done - last_print_step) / max(now - last_print_t, 1e-9)
                line = f"[gfmc] - [run_gfmc] - step: {done}/{n_steps}, {rate:.1f} it/s"
                if verbosity >= 3:
                    est = windowed_energy_host(p_array, logG_h[:done].numpy(), E_h[:done].numpy())
                    line += f" Energy[p]: {est}"
                _emit(line, verbosity)
                last_print_t, last_print_step = now, done
    torch.cuda.current_stream().synchronize()
    runtime = time.time() - prod_start
    _device_status_check(eng)
    weights_np = logG_h.numpy().copy()
    E_np = E_h.numpy().copy()
    energy = eng.windowed_energy(logG_d, E_d, p_array)

    cfg_d, e_d = eng.population()
    diag_np = additional_diag_np = None
    if diag_d is not None:
        def split_cols(arr):
            out, c = {}, 0
            for name, w in zip(diag_names, widths):
                a = arr[:, c:c + w, :]
                out[name] = a[:, 0, :].copy() if w == 1 and not _is_vector_op(diag_operators[name]) \
                    else a.copy()
                c += w
            return out
        diag_np = split_cols(diag_d.cpu().numpy())
        m_max = max(m_array)
        if m_max > 0:
            # the lead-in a continuation substitutes for its first rows: m_max
            # further steps walked with this run's ancestry (driver.py:1101-1127);
            # the returned walkers stay the production-final ones
            keys_x, _ = key_schedule(key, m_max)
            extra = torch.zeros((m_max, eng.diag_width, n_p), dtype=torch.float64, device=dev)
            eng.set_diag_output(extra)
            lgx = torch.empty(m_max, dtype=torch.float64, device=dev)
            Ex = torch.empty(m_max, dtype=torch.float64, device=dev)
            eng.steps(method, step_f, lam, alw, keys_x, lgx, Ex)
            additional_diag_np = split_cols(extra.cpu().numpy())
        eng.set_diag_output(None)
    cfg_np = cfg_d.cpu().numpy()
    in_dtype = np.asarray(config).dtype if not torch.is_tensor(config) else np.float64
    if in_dtype.kind == "f":
        cfg_np = cfg_np.astype(in_dtype)
    out_w = Walker(config=cfg_np, log_weight=np.zeros(N_walker, dtype=weight_dtype),
                   e_loc=e_d.cpu().numpy().astype(weight_dtype))
    hops_np = hops_d.cpu().numpy()
    # whether the steps carried guide state through the parent maps (a sparse
    # guide's optional state is rebuilt per step when it does not fit; the
    # float64 results then differ from a carried run in the last bits only)
    carried = eng.carry_mode()

    # the end-of-run statistics pass from the production-final walkers, on
    # its own side-stream (driver.py _run_stats:627-660)
    from .diagnostics import statistics as _statistics
    _, end_stats = _statistics(out_w, hamiltonian, step_f, guide, method,
                               _rnd.fold_in(aux_root, _AUX_STATISTICS), alw, lam=lam,
                               quiet=verbosity < 1, m_array=m_array, precision=precision)
    stats = dict(end_stats)
    stats.update({
        "avg_log_weight": float(alw),
        "it_per_sec": n_steps / runtime,
        "runtime": runtime,
        "total_wall_time": time.time() - wall_start,
        "number_of_devices": n_dev,
        "guide_state_carried": int(carried),
        "moves_per_walker_step": hops_np / float(N_walker),
        "parameters/n_steps": int(n_steps),
        "parameters/n_walkers": N_walker,
        "parameters/n_sites": int(np.shape(config)[1]),
        "parameters/step_size": step_f,
        "parameters/lam": float(lam_given) if lam_given is not None else float("nan"),
        "parameters/p_array": np.asarray(p_array, dtype=np.int64),
        "parameters/m_array": np.asarray(m_array, dtype=np.int64),
        "parameters/warmup_steps": int(warmup_steps),
        "parameters/verbosity": int(verbosity),
        "parameters/number_of_outputs": int(number_of_outputs),
        "parameters/off_diag_stride": int(off_diag_stride),
        "parameters/off_diag_offset": int(plan.off_diag_offset),
        "parameters/off_diag_equal_windows": int(bool(plan.equal_windows)),
        "parameters/n_off_diag_operators": len(off_names),
        "parameters/off_diag_operators": np.asarray(off_names, dtype="S64"),
        "parameters/method": np.asarray(str(method), dtype="S32"),
        "parameters/guide": np.asarray(type(guide).__name__ if guide is not None else "none", dtype="S32"),
        "parameters/hamiltonian": np.asarray(type(hamiltonian).__name__, dtype="S32"),
        "parameters/has_guide": int(guide is not None),
        "parameters/precision": np.asarray(precision, dtype="S32"),
        "parameters/rng_key": rng_key_in,
        "parameters/rng_key_next": key,
    })
    off_np = off_norm_np = off_steps_np = None
    if off_names:
        od = od_d.cpu().numpy()
        on = on_d.cpu().numpy()
        off_np = {nm: od[:, i].copy() for i, nm in enumerate(off_names)}
        off_norm_np = {nm: on[:, i].copy() for i, nm in enumerate(off_names)}
        off_steps_np = meas.astype(np.int64)
    stats.update(autocorrelation_stats(E_np, weights_np, diag_np=diag_np, off_diag_np=off_np,
                                       off_diag_stride=off_diag_stride))
    stats["parameters/diag_operators"] = np.asarray(diag_names, dtype="S64")
    stats["parameters/n_diag_operators"] = len(diag_names)
    # with both kinds measured, every window starts at i >= max(m)
    # (engine/estimators.py:596-619)
    m_common = max(m_array) if (diag_np and off_names) else 0
    obs = diagonal_estimates(p_array, weights_np, diag_np, m_common) if diag_np else {}
    if off_names:
        obs.update(off_diagonal_estimates(p_array, m_array, weights_np, off_np, off_norm_np,
                                          off_steps_np, m_common))
    if return_raw:
        raw = dict(log_weights=weights_np, energy=E_np, diag=diag_np, off_diag=off_np,
                   off_diag_norm=off_norm_np, off_diag_steps=off_steps_np,
                   additional_diag=additional_diag_np,
                   p_array=list(p_array), m_array=list(m_array),
                   diag_operators=list(diag_names) or None,
                   off_diag_operators=list(off_names) or None)
        return out_w, energy, obs, stats, raw
    return out_w, energy, obs, stats


def _default_n_devices():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_world_size()
    except Exception:
        pass
    return 1


def run(walkers, n_steps, hamiltonian, step_size, guide, p_array, *, method="cont_time",
        rng_key=None, lam=None, **kwargs):
    """Drop-in for ``pygfmc.run`` (engine/multi_gpu.py:822-868): the run on
    one GPU, or with ``n_devices > 1`` a population sharded over GPUs.

    ``n_devices`` (default: the world size of an initialised torch.distributed
    group, else 1; PyGFMC's default is every visible device): with a process
    group of that size, one shard per process (torchrun, one process per
    GPU); otherwise the shards live in this process on ``cuda:0 ..
    cuda:n_devices-1`` (``shard_devices=[...]`` names other devices, and may
    repeat one to emulate the ranks on a single GPU).  The walker count must
    be divisible by ``n_devices``.  Each process passes the whole population
    and gets the whole final population back.  Unlike PyGFMC's sharded run,
    the trajectory does not depend on the device count: every walker keeps
    its global random stream and the resampling is global, so the sharded run
    follows the one-GPU run (identical configurations, weights to rounding).
    As in PyGFMC, runs with ``diag_operators`` stay on one device; so do runs
    with ``off_diag_operators`` here (PyGFMC shards those)."""
    n_devices = kwargs.pop("n_devices", None)
    shard_devices = kwargs.pop("shard_devices", None)
    n_devices = _default_n_devices() if n_devices is None else _validated_int("n_devices", n_devices, 1)
    if shard_devices is not None and len(shard_devices) != n_devices:
        raise ValueError(f"shard_devices names {len(shard_devices)} devices for n_devices={n_devices}")
    if n_devices > 1 and (kwargs.get("diag_operators") or kwargs.get("off_diag_operators")):
        _emit(f"[gfmc] - [run] - n_devices={n_devices} with measurement operators: running on one "
              "device", kwargs.get("verbosity", 7), 1)
        n_devices = 1
    if n_devices > 1:
        return run_gfmc(walkers, n_steps, hamiltonian, step_size, guide, p_array, method=method,
                        rng_key=rng_key, lam=lam, _shards=(n_devices, shard_devices), **kwargs)
    return run_gfmc(walkers, n_steps, hamiltonian, step_size, guide, p_array, method=method,
                    rng_key=rng_key, lam=lam, **kwargs)

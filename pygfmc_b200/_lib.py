"""ctypes binding of the engine's C ABI (include/gfmc_b200.h).

The shared library is built in-tree (``pygfmc_b200/_lib/libgfmc_b200.so``)
by ``pygfmc_b200/csrc/Makefile``.  There is no fallback: a missing library
or a missing GPU raises.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libgfmc_b200.so")

GFMC_OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_UNSUPPORTED = -3
ERR_DEVICE = -4

MODEL_SPIN_HALF = 0
MODEL_BOSE_HUBBARD = 1
GUIDE_NONE = 0
GUIDE_JASTROW_SPIN_HALF = 1
GUIDE_JASTROW_BOSE_HUBBARD = 2
GUIDE_RBM_SPIN_HALF = 3
GUIDE_MLP_BOSE_HUBBARD = 4
GUIDE_EXACT_SPIN_HALF = 5
METHODS = {"cont_time": 0, "single_step": 1, "multi_step": 2}
PRECISION_FP64 = 0
PRECISION_MIXED = 1
STATUS_HOP_CAP = 1
STATUS_BAD_CONFIG = 2
STATUS_NONFINITE = 4
STATUS_TIMEOUT = 8

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_vp = ctypes.c_void_p
_fp = ctypes.POINTER(ctypes.c_float)


class ModelDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n_sites", ctypes.c_int), ("n_edges", ctypes.c_int),
                ("edge_i", _i32p), ("edge_j", _i32p),
                ("n_hx", ctypes.c_int), ("n_jpm", ctypes.c_int), ("has_jz", ctypes.c_int),
                ("uniform_jz", ctypes.c_int), ("has_hz", ctypes.c_int),
                ("jz", _dp), ("jpm", _dp), ("jpmpm", _dp), ("hz", _dp), ("hx_half", _dp),
                ("n_max", ctypes.c_int), ("n_hop", ctypes.c_int), ("n_eta", ctypes.c_int),
                ("n_hpm", ctypes.c_int), ("has_U", ctypes.c_int), ("has_mu", ctypes.c_int),
                ("t", _dp), ("eta", _dp), ("U", _dp), ("mu", _dp), ("hpm", _dp)]


class GuideDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n_pairs", ctypes.c_int),
                ("pair_i", _i32p), ("pair_j", _i32p), ("pair_w", _dp), ("h", _dp),
                ("beta_tied", ctypes.c_int), ("beta0", ctypes.c_double),
                ("h_mode", ctypes.c_int), ("h0", ctypes.c_double),
                ("d_mode", ctypes.c_int), ("d0", ctypes.c_double), ("d", _dp),
                ("n_hidden", ctypes.c_int), ("rbm_W", _fp), ("rbm_b", _fp), ("rbm_a", _fp),
                ("mlp_H1", ctypes.c_int), ("mlp_H2", ctypes.c_int), ("mlp_W1", _fp),
                ("mlp_b1", _fp), ("mlp_W2", _fp), ("mlp_b2", _fp), ("mlp_w3", _fp),
                ("mlp_b3", ctypes.c_double),
                ("exact_n_sites", ctypes.c_int), ("exact_log_amp", _dp)]


class DiagDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n_sites", ctypes.c_int), ("n_edges", ctypes.c_int),
                ("edge_i", _i32p), ("edge_j", _i32p),
                ("has_jz", ctypes.c_int), ("uniform_jz", ctypes.c_int), ("has_hz", ctypes.c_int),
                ("jz", _dp), ("hz", _dp), ("has_U", ctypes.c_int), ("has_mu", ctypes.c_int),
                ("U", _dp), ("mu", _dp), ("n_k", ctypes.c_int), ("cos_kr", _dp), ("sin_kr", _dp),
                ("offset", ctypes.c_double)]


DIAG_SPIN_HALF = 0
DIAG_BOSE_HUBBARD = 1
DIAG_SZSZ = 2

# name -> (restype, argtypes); every symbol include/gfmc_b200.h declares
SIGNATURES = {
    "gfmc_create": (ctypes.c_int, [ctypes.POINTER(ModelDesc), ctypes.POINTER(GuideDesc),
                                   ctypes.c_int, ctypes.POINTER(_vp)]),
    "gfmc_destroy": (ctypes.c_int, [_vp]),
    "gfmc_config_bytes": (ctypes.c_int, [_vp]),
    "gfmc_n_transitions": (ctypes.c_int, [_vp]),
    "gfmc_pack": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "gfmc_unpack": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "gfmc_run_steps": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, _u32p, ctypes.c_int,
                                      _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gfmc_local_energy": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "gfmc_local_energy_parts": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "gfmc_gather": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "gfmc_windowed_energy": (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, _i32p, _dp, _vp]),
    "gfmc_set_max_iters": (ctypes.c_int, [_vp, ctypes.c_int]),
    "gfmc_carry_mode": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "gfmc_set_diag_operators": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(DiagDesc),
                                               ctypes.c_int, _i32p]),
    "gfmc_diag_width": (ctypes.c_int, [_vp]),
    "gfmc_reset_diag": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "gfmc_set_diag_output": (ctypes.c_int, [_vp, _vp]),
    "gfmc_apply_operator": (ctypes.c_int, [_vp, _u32p, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                           _vp, _vp]),
    "gfmc_forward_walk": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, _u32p, _u32p, ctypes.c_int, _vp, _vp,
                                         ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                         ctypes.c_int, _i32p, _vp, _vp, _vp]),
    "gfmc_operator_min_rate": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp]),
    "gfmc_rbm_theta": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp]),
    "gfmc_rbm_hidden_padded": (ctypes.c_int, [_vp]),
    "gfmc_rbm_gradient": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                         _vp, _dp, _vp]),
    "gfmc_rbm_train_step": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                           ctypes.c_double, _dp, _vp]),
    "gfmc_rbm_get_params": (ctypes.c_int, [_vp, _fp, _fp, _fp]),
    "gfmc_mlp_param_count": (ctypes.c_longlong, [_vp]),
    "gfmc_mlp_gradient": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _dp,
                                         _vp]),
    "gfmc_mlp_train_step": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                           ctypes.c_double, _dp, _vp]),
    "gfmc_mlp_get_params": (ctypes.c_int, [_vp, _fp]),
    "gfmc_evolve": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, _u32p, ctypes.c_longlong, ctypes.c_int, _vp,
                                   _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "gfmc_evolve_walkers": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, _u32p, ctypes.c_int, _vp, _vp, _vp, _vp,
                                           _vp, _vp]),
    "gfmc_dist_local_max": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _dp, _vp]),
    "gfmc_dist_local_sums": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_double, _dp,
                                            _vp]),
    "gfmc_dist_local_max_dev": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp]),
    "gfmc_dist_local_sums_dev": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "gfmc_dist_parents": (ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_longlong,
                                         ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "gfmc_reconfigure_noalloc": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _u32p, _vp, _vp, _vp, _vp]),
    "gfmc_read_status": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), _vp]),
    "gfmc_key_schedule": (ctypes.c_int, [_u32p, ctypes.c_int, _u32p, _u32p]),
    "gfmc_key_schedule_ex": (ctypes.c_int, [_u32p, ctypes.c_int, ctypes.c_int, _u32p, _u32p]),
    "gfmc_threefry2x32": (ctypes.c_int, [ctypes.c_uint32] * 4 + [_u32p]),
    "gfmc_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "gfmc_version": (ctypes.c_char_p, []),
}

_lib = None


class GFMCError(RuntimeError):
    """An engine call failed (CUDA error or invalid use of the C ABI)."""


def build(force=False):
    """Compile the CUDA engine for sm_100a (``make -C pygfmc_b200/csrc``)."""
    args = ["make", "-s", "-C", os.path.join(_HERE, "csrc")]
    if force:
        subprocess.run(args + ["clean"], check=True)
    subprocess.run(args, check=True)


def load():
    """The loaded engine library; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise GFMCError(
            f"the CUDA engine is not built ({LIB_PATH} missing); run "
            "`make -C pygfmc_b200/csrc` or __graft_entry__.build() -- there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().gfmc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc, what=""):
    if rc != GFMC_OK:
        msg = last_error()
        if rc == ERR_INVALID:
            raise ValueError(f"{what}: {msg}")
        raise GFMCError(f"{what} failed ({rc}): {msg}")
    return rc

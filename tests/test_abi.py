"""The C ABI library loads (no GPU needed) and exports every symbol that
include/gfmc_b200.h declares; host-only entry points work on the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gfmc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gfmc_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from pygfmc_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    from pygfmc_b200 import _lib
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_key_schedule_matches_the_reference_recurrence(lib, oracle):
    from pygfmc_b200.engine import key_schedule
    key = oracle.case_key("spinhalf_jastrow_cont_time")
    keys, nxt = key_schedule(key, 300)
    k = key.copy()
    for s in range(300):
        k, r = oracle.split(k, 2)
        assert np.array_equal(keys[s, :2], oracle.fold_in(r, 0))
        assert np.array_equal(keys[s, 2:], oracle.fold_in(r, 1))
    assert np.array_equal(nxt, [4201513499, 1131088919])


def test_key_schedule_ex_sub_keys(lib, oracle):
    """fold_in(rng, j) for j < n_sub per step; the (k1, k2) columns equal
    gfmc_key_schedule's, and the measurement key is fold_in(rng, 2)."""
    from pygfmc_b200.engine import key_schedule, key_schedule_ex
    key = oracle.case_key("bose_none_cont_time")
    kx, nxt = key_schedule_ex(key, 40, 3)
    k4, nxt4 = key_schedule(key, 40)
    assert np.array_equal(kx[:, :2].reshape(40, 4), k4) and np.array_equal(nxt, nxt4)
    k = key.copy()
    for s in range(40):
        k, r = oracle.split(k, 2)
        assert np.array_equal(kx[s, 2], oracle.fold_in(r, 2))


def test_last_error_and_invalid_arguments(lib):
    from pygfmc_b200 import _lib
    rc = lib.gfmc_key_schedule(None, 3, None, None)
    assert rc == _lib.ERR_INVALID
    assert "gfmc_key_schedule" in _lib.last_error()
    with pytest.raises(ValueError):
        _lib.check(rc, "gfmc_key_schedule")
    assert lib.gfmc_carry_mode(None, 1, None) == _lib.ERR_INVALID
    assert "gfmc_carry_mode" in _lib.last_error()


def test_create_rejects_edges_without_arrays(lib):
    """gfmc_create checks the edge list before touching the device: a
    positive n_edges without edge_i / edge_j, or a negative n_edges, is an
    invalid argument (no GPU needed)."""
    from pygfmc_b200 import _lib
    for n_edges in (4, -1):
        md = _lib.ModelDesc()
        md.kind = _lib.MODEL_SPIN_HALF
        md.n_sites = 4
        md.n_edges = n_edges
        h = ctypes.c_void_p()
        rc = lib.gfmc_create(ctypes.byref(md), None, _lib.PRECISION_FP64, ctypes.byref(h))
        assert rc == _lib.ERR_INVALID
        assert "edge_i" in _lib.last_error()
        assert not h.value

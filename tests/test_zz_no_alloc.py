"""gfmc_reconfigure_noalloc, the resampling entry point that allocates no
device memory (for callers that must not allocate inside a call, e.g. a host
framework owning the device through its own pool allocator), against the
resampling inside gfmc_run_steps on the same pre-resampling weights and key:
identical parent maps and log G / E to 1e-12, on two calls in a row.  Kept in
its own file, collected last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_reconfigure_matches_run_steps():
    import torch
    import pygfmc_b200 as P
    L = P._lib.load()
    e = P.chain(32).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)
    G = P.JastrowSpinHalf(32, e, beta=0.3)
    n = 3000                                  # three reconfiguration tiles, a ragged last one
    eng = P.GFMCEngine(H, G, n, precision="fp64")
    eng.load(P.prepare_walkers_sz(n, 32, P.PRNGKey(3), sz=0).config)
    dev = eng.device
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    key = P.PRNGKey(11)
    for call in range(2):
        keys, key = P.engine.key_schedule(key, 1)
        lg = torch.empty(1, dtype=torch.float64, device=dev)
        En = torch.empty(1, dtype=torch.float64, device=dev)
        eng.steps("cont_time", 0.1, None, -1.2, keys, lg, En)   # existing entry point
        par = torch.full((n,), -7, dtype=torch.int32, device=dev)
        lg2 = torch.empty(1, dtype=torch.float64, device=dev)
        En2 = torch.empty(1, dtype=torch.float64, device=dev)
        k2 = np.ascontiguousarray(keys[0, 2:], dtype=np.uint32)
        rc = L.gfmc_reconfigure_noalloc(n, _ptr(eng.log_w), _ptr(eng.e_loc),
                                        k2.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                        _ptr(par), _ptr(lg2), _ptr(En2), stream)
        assert rc == 0, P._lib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(par, eng.parents), f"call {call}: parent maps differ"
        np.testing.assert_allclose(lg2.item(), lg.item(), rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(En2.item(), En.item(), rtol=1e-12, atol=1e-14)


def test_noalloc_rejects_populations_above_its_limit():
    import pygfmc_b200 as P
    L = P._lib.load()
    k = np.zeros(2, dtype=np.uint32)
    big = 131072 + 1
    rc = L.gfmc_reconfigure_noalloc(big, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                    k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                    ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8),
                                    ctypes.c_void_p(0))
    assert rc == P._lib.ERR_INVALID
    assert "GFMC_NOALLOC_MAX_WALKERS" in P._lib.last_error()

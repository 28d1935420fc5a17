"""Sharded resampling: the host logic over two gloo ranks on CPU, and the
device pieces with emulated ranks on one GPU.  Both must give the systematic
resampling of the concatenated population (walkers/reconfiguration.py:9-62,
as restated by the oracle)."""
import math
import os
import tempfile

import numpy as np
import pytest

from pygfmc_b200.distributed import exchange_plan, slot_ranges


def test_slot_ranges_partition_and_plan():
    S = [0.0, 2.0, 1.0, 0.5]
    r = slot_ranges(S, 0.37, 16)
    assert r[0] == (0, 0) and r[-1][1] == 16
    assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
    # the slots of a rank are those whose point falls in its weight interval
    tot, off = sum(S), np.concatenate([[0.0], np.cumsum(S)])
    for k, (lo, hi) in enumerate(r):
        for i in range(lo, hi):
            U = (i + 0.37) / 16 * tot
            assert off[k] <= U < off[k + 1] + 1e-12
    plan = exchange_plan(r, 4)
    moved = sorted((a, b) for a, b in plan.values())
    assert sum(b - a for a, b in moved) == 16
    assert all(b <= (a // 4 + 1) * 4 for a, b in moved)
    with pytest.raises(ValueError):
        slot_ranges([0.0, 0.0], 0.5, 4)


def _local_parents(lw, shift, offset, S_tot, psi, N, lo, cnt):
    """The per-rank parent rule (gfmc_dist_parents) restated in numpy."""
    w = np.exp(lw - shift)
    cdf = offset + np.cumsum(w)
    last = int(np.flatnonzero(w > 0)[-1]) if np.any(w > 0) else 0
    out = []
    for i in range(lo, lo + cnt):
        U = (i + psi) / N * S_tot
        k = min(int(np.searchsorted(cdf, U, side="right")), last)
        while k > 0 and not w[k] > 0:
            k -= 1
        out.append(k)
    return np.asarray(out, dtype=np.int64)


def _rank_main(rank, world, port, n, seed, path):
    import torch
    import torch.distributed as dist
    from pygfmc_b200 import random as rnd
    from pygfmc_b200.distributed import exchange
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    rng = np.random.default_rng(seed)
    lw_all = rng.normal(0, 1.5, n * world)
    lw_all[rng.integers(0, n * world, 5)] = -np.inf
    lw = lw_all[rank * n:(rank + 1) * n]
    mt = torch.tensor([np.max(lw)])
    dist.all_reduce(mt, op=dist.ReduceOp.MAX)
    shift = float(mt.item())
    S_r = torch.tensor([float(np.sum(np.exp(lw - shift)))], dtype=torch.float64)
    allS = [torch.zeros_like(S_r) for _ in range(world)]
    dist.all_gather(allS, S_r)
    S = [float(a.item()) for a in allS]
    key2 = rnd.PRNGKey(seed + 7)
    psi = rnd.uniform(key2)
    ranges = slot_ranges(S, psi, n * world)
    lo, hi = ranges[rank]
    par = _local_parents(lw, shift, math.fsum(S[:rank]), math.fsum(S), psi, n * world, lo, hi - lo)
    # payload: the global walker id of each selected walker
    sel = torch.as_tensor((rank * n + par).reshape(-1, 1), dtype=torch.int64)
    new = torch.full((n, 1), -1, dtype=torch.int64)
    exchange(sel, new, exchange_plan(ranges, n), lo, n, rank)
    got = [torch.zeros_like(new) for _ in range(world)]
    dist.all_gather(got, new)
    if rank == 0:
        np.save(path, np.concatenate([g.numpy().ravel() for g in got]))
        np.save(path + ".lw.npy", lw_all)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,n,seed", [(2, 37, 1), (3, 64, 2)])
def test_gloo_sharded_resampling_equals_the_concatenated_one(oracle, world, n, seed):
    import torch.multiprocessing as mp
    port = 29600 + seed
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "parents.npy")
        mp.start_processes(_rank_main, args=(world, port, n, seed, path), nprocs=world,
                           start_method="spawn")
        got = np.load(path)
        lw = np.load(path + ".lw.npy")
    from pygfmc_b200 import random as rnd
    cfg = np.arange(n * world, dtype=np.float64)[:, None]
    par, _, _ = oracle.reconfigure(rnd.PRNGKey(seed + 7), cfg.copy(), lw.copy(),
                                   np.zeros(n * world))
    assert np.array_equal(got, par)


@pytest.mark.gpu
@pytest.mark.parametrize("R,guide", [(1, "nn"), (3, "nn"), (3, "dense")])
def test_sharded_steps_follow_the_unsharded_run(R, guide):
    """R emulated ranks on one GPU (evolve with global walker offsets, the
    device resampling pieces, the exchange plan applied by copies) against
    one engine over the whole population: identical configurations after
    every step, log G and E_n to 1e-12."""
    import ctypes
    import torch
    import pygfmc_b200 as P
    from pygfmc_b200 import _lib
    from pygfmc_b200 import random as rnd
    from pygfmc_b200.distributed import evolve_shard
    e = P.chain(24).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)
    if guide == "dense":
        # all pairs: the shards' guide state is built as one product per call
        pairs = np.array([(i, j) for i in range(24) for j in range(i + 1, 24)])
        r = np.minimum(pairs[:, 1] - pairs[:, 0], 24 - (pairs[:, 1] - pairs[:, 0]))
        G = P.JastrowSpinHalf(24, pairs, beta=0.3 / r)
    else:
        G = P.JastrowSpinHalf(24, e, beta=0.3)
    n = 200
    N = n * R
    cfg = P.prepare_walkers_random(N, 24, P.PRNGKey(3)).config
    ref = P.GFMCEngine(H, G, N)
    ref.load(cfg)
    shards = [P.GFMCEngine(H, G, n) for _ in range(R)]
    for r, eng in enumerate(shards):
        eng.load(cfg[r * n:(r + 1) * n])
    tmp = [torch.empty_like(eng.cfg) for eng in shards]
    keys, _ = P.engine.key_schedule(P.PRNGKey(9), 6)
    alw = 1.0
    lg = torch.empty(1, dtype=torch.float64, device=ref.device)
    En = torch.empty_like(lg)
    B = ref.cfg_bytes
    for s in range(6):
        ref.steps("cont_time", 0.15, None, alw, keys[s:s + 1], lg, En)
        k1, k2 = keys[s, :2], keys[s, 2:]
        for r, eng in enumerate(shards):
            evolve_shard(eng, "cont_time", 0.15, None, alw, k1, r * n, tmp[r])
        mx = []
        for eng in shards:
            m = ctypes.c_double()
            _lib.check(eng.L.gfmc_dist_local_max(eng.h, n, eng._ptr(eng.log_w), ctypes.byref(m),
                                                 eng._stream()), "max")
            mx.append(m.value)
        shift = max(mx)
        outs = []
        for eng in shards:
            o = np.zeros(3)
            _lib.check(eng.L.gfmc_dist_local_sums(eng.h, n, eng._ptr(eng.log_w), eng._ptr(eng.e_loc),
                                                  shift, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  eng._stream()), "sums")
            outs.append(o)
        S = [o[0] for o in outs]
        psi = rnd.uniform(k2)
        ranges = slot_ranges(S, psi, N)
        sels = []
        for r, eng in enumerate(shards):
            lo, hi = ranges[r]
            sel = torch.empty((max(hi - lo, 1), B), dtype=torch.uint8, device=eng.device)
            if hi > lo:
                par = torch.empty(hi - lo, dtype=torch.int32, device=eng.device)
                _lib.check(eng.L.gfmc_dist_parents(eng.h, n, eng._ptr(eng.log_w), shift, sum(S[:r]),
                                                   sum(S), psi, N, lo, hi - lo, int(outs[r][2]),
                                                   eng._ptr(par), eng._stream()), "parents")
                _lib.check(eng.L.gfmc_gather(eng.h, hi - lo, eng._ptr(par), eng._ptr(tmp[r]),
                                             eng._ptr(sel), ctypes.c_void_p(0), ctypes.c_void_p(0),
                                             ctypes.c_void_p(0), eng._stream()), "gather")
            sels.append(sel)
        for (src, dst), (a, b) in exchange_plan(ranges, n).items():
            lo = ranges[src][0]
            shards[dst].cfg.view(n, B)[a - dst * n:b - dst * n].copy_(sels[src][a - lo:b - lo])
        for eng in shards:
            eng.parents_valid = 0
        logG = math.log(math.fsum(S)) + shift - math.log(N)
        E_n = math.fsum(o[1] for o in outs) / math.fsum(S)
        np.testing.assert_allclose(logG, lg.item(), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(E_n, En.item(), rtol=1e-12, atol=1e-12)
        whole = ref.packed_population()
        mine = np.concatenate([eng.cfg.view(n, B).cpu().numpy() for eng in shards])
        assert np.array_equal(whole, mine), f"step {s}"

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


def _chain_system(P, guide):
    e = P.chain(24).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.2, dtype=np.float64)
    if guide == "dense":
        # all pairs: the shards' guide state is built as one product per call
        pairs = np.array([(i, j) for i in range(24) for j in range(i + 1, 24)])
        r = np.minimum(pairs[:, 1] - pairs[:, 0], 24 - (pairs[:, 1] - pairs[:, 0]))
        G = P.JastrowSpinHalf(24, pairs, beta=0.3 / r)
    else:
        G = P.JastrowSpinHalf(24, e, beta=0.3)
    return H, G


@pytest.mark.gpu
@pytest.mark.parametrize("R,guide", [(1, "nn"), (3, "nn"), (3, "dense"), (4, "nn")])
def test_sharded_population_follows_the_unsharded_engine(R, guide):
    """ShardedPopulation with R shards emulated on one GPU (evolve with the
    global walker offsets, the device-side max and sums, the parents and the
    exchange of configuration + local-energy rows) against one engine over
    the whole population, step by step: identical configurations, local
    energies to 1e-12 with zero log weights, log G and E_n to 1e-12."""
    import torch
    import pygfmc_b200 as P
    from pygfmc_b200.distributed import ShardedPopulation
    H, G = _chain_system(P, guide)
    n = 200
    N = n * R
    cfg = P.prepare_walkers_random(N, 24, P.PRNGKey(3)).config
    ref = P.GFMCEngine(H, G, N)
    ref.load(cfg)
    sp = ShardedPopulation(H, G, N, devices=["cuda:0"] * R)
    sp.load(cfg)
    keys, _ = P.engine.key_schedule(P.PRNGKey(9), 6)
    alw = 1.0
    lg = torch.empty(1, dtype=torch.float64, device=ref.device)
    En = torch.empty_like(lg)
    lg2, En2 = torch.empty_like(lg), torch.empty_like(lg)
    h1 = torch.zeros(1, dtype=torch.int64, device=ref.device)
    h2 = torch.zeros_like(h1)
    for s in range(6):
        ref.steps("cont_time", 0.15, None, alw, keys[s:s + 1], lg, En, h1)
        sp.steps("cont_time", 0.15, None, alw, keys[s:s + 1], lg2, En2, h2)
        np.testing.assert_allclose(lg2.item(), lg.item(), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(En2.item(), En.item(), rtol=1e-12, atol=1e-12)
        assert h1.item() == h2.item()
        c_ref, e_ref = ref.population()
        c_sp, e_sp = sp.population()
        assert torch.equal(c_ref, c_sp), f"step {s}"
        np.testing.assert_allclose(e_sp.cpu().numpy(), e_ref.cpu().numpy(), rtol=1e-12, atol=1e-12)
        for sh in sp.shards:
            assert not torch.any(sh.log_w != 0)
    assert sp.status() == 0


@pytest.mark.gpu
def test_device_and_host_shard_sums_agree():
    """gfmc_dist_local_sums_dev (shift read from device memory) gives the host
    entry point's (S_r, sum w e, last positive) bit for bit."""
    import ctypes
    import torch
    import pygfmc_b200 as P
    H, G = _chain_system(P, "nn")
    eng = P.GFMCEngine(H, G, 3000)
    eng.load(P.prepare_walkers_random(3000, 24, P.PRNGKey(4)).config)
    eng.log_w.copy_(torch.as_tensor(np.random.default_rng(1).normal(0, 2, 3000)))
    eng.e_loc.copy_(torch.as_tensor(np.random.default_rng(2).normal(-5, 1, 3000)))
    L = eng.L
    m = ctypes.c_double()
    P._lib.check(L.gfmc_dist_local_max(eng.h, 3000, eng._ptr(eng.log_w), ctypes.byref(m),
                                       eng._stream()), "max")
    md = torch.empty(1, dtype=torch.float64, device=eng.device)
    P._lib.check(L.gfmc_dist_local_max_dev(eng.h, 3000, eng._ptr(eng.log_w), eng._ptr(md),
                                           eng._stream()), "max dev")
    assert md.item() == m.value == float(eng.log_w.max().item())
    host = np.zeros(3)
    P._lib.check(L.gfmc_dist_local_sums(eng.h, 3000, eng._ptr(eng.log_w), eng._ptr(eng.e_loc), m.value,
                                        host.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        eng._stream()), "sums")
    out = torch.empty(4, dtype=torch.float64, device=eng.device)
    P._lib.check(L.gfmc_dist_local_sums_dev(eng.h, 3000, eng._ptr(eng.log_w), eng._ptr(eng.e_loc),
                                            eng._ptr(md), eng._ptr(out), eng._stream()), "sums dev")
    o = out.cpu().numpy()
    assert o[0] == m.value and np.array_equal(o[1:], host)


def _run_system(P):
    H, G = _chain_system(P, "nn")
    w = P.prepare_walkers_sz(240, 24, P.PRNGKey(5), sz=0)
    return H, G, w


@pytest.mark.gpu
def test_run_with_n_devices_follows_the_one_device_run():
    """run(..., n_devices=3) with the shards emulated on one GPU reproduces
    run(...) on one device: identical final walkers, series to 1e-10."""
    import pygfmc_b200 as P
    H, G, w = _run_system(P)
    kw = dict(rng_key=P.PRNGKey(6), warmup_steps=30, verbosity=0)
    w1, E1, _, st1, raw1 = P.run(w, 40, H, 0.1, G, [4, 8], **kw)
    w3, E3, _, st3, raw3 = P.run(w, 40, H, 0.1, G, [4, 8], n_devices=3,
                                 shard_devices=["cuda:0"] * 3, **kw)
    assert st3["number_of_devices"] == 3 and st1["number_of_devices"] == 1
    assert np.array_equal(w1.config, w3.config)
    np.testing.assert_allclose(w3.e_loc, w1.e_loc, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw3["log_weights"], raw1["log_weights"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(raw3["energy"], raw1["energy"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(st3["avg_log_weight"], st1["avg_log_weight"], rtol=1e-10)
    for p in (4, 8):
        np.testing.assert_allclose(E3[p], E1[p], rtol=1e-10)
    assert np.array_equal(st3["parameters/rng_key_next"], st1["parameters/rng_key_next"])
    with pytest.raises(ValueError, match="divisible"):
        P.run(P.prepare_walkers_sz(100, 24, P.PRNGKey(5), sz=0), 4, H, 0.1, G, [2], n_devices=3,
              shard_devices=["cuda:0"] * 3, **kw)


def _group_rank_main(rank, world, port, path):
    """One rank of a gloo process group on the one GPU: run(..., n_devices=2)
    with one shard per process (global_reconfigure, exchange through host
    memory)."""
    import torch
    import torch.distributed as dist
    import pygfmc_b200 as P
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
    try:
        H, G, w = _run_system(P)
        wf, E, _, st, raw = P.run(w, 40, H, 0.1, G, [4, 8], rng_key=P.PRNGKey(6), warmup_steps=30,
                                  verbosity=0)
        assert st["number_of_devices"] == world
        np.savez(path + f".{rank}.npz", config=wf.config, e_loc=wf.e_loc, lw=raw["log_weights"],
                 E=raw["energy"], alw=st["avg_log_weight"])
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_gloo_process_group_run_follows_the_one_device_run():
    """Two processes of a gloo group sharing the one GPU (no kernel of one
    waits for the other: the ranks meet only in host collectives), each with
    one shard: run() shards over the group (global_reconfigure, point-to-point
    exchange through host memory) and every rank returns the one-device run's
    walkers and series."""
    import torch.multiprocessing as mp
    import pygfmc_b200 as P
    H, G, w = _run_system(P)
    w1, _, _, st1, raw1 = P.run(w, 40, H, 0.1, G, [4, 8], rng_key=P.PRNGKey(6), warmup_steps=30,
                                verbosity=0)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "run")
        mp.start_processes(_group_rank_main, args=(2, 29655, path), nprocs=2, start_method="spawn")
        for r in range(2):
            got = np.load(path + f".{r}.npz")
            assert np.array_equal(got["config"], w1.config), f"rank {r}"
            np.testing.assert_allclose(got["e_loc"], w1.e_loc, rtol=1e-10, atol=1e-12)
            np.testing.assert_allclose(got["lw"], raw1["log_weights"], rtol=1e-10, atol=1e-12)
            np.testing.assert_allclose(got["E"], raw1["energy"], rtol=1e-10, atol=1e-12)
            np.testing.assert_allclose(got["alw"], st1["avg_log_weight"], rtol=1e-10)

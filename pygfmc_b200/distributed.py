"""Walkers sharded over GPUs: one process per GPU, contiguous walker blocks,
global systematic resampling with the data moved once.

The reference's multi-device path (engine/multi_gpu.py:91-155) all-gathers
every configuration to every device and resamples there.  Here each rank
resamples only its own output slots: the ranks exchange their weight sums
(one float64 per rank), each rank finds the parents of the global slots
whose resampling points fall in its own weight interval (``slot_ranges``),
and sends those walkers to the ranks that own the slots -- contiguous blocks,
so a rank talks to at most a few neighbours.  The result is the systematic
resampling of the concatenated population, and with ``evolve_shard`` (the
per-walker random streams numbered by the global walker index) a sharded run
follows the same trajectory as the unsharded one.

``slot_ranges`` and ``exchange_plan`` are host logic; ``global_reconfigure``
runs the device pieces (``gfmc_dist_*``) and the exchange (torch.distributed
point-to-point: NCCL over NVLink between GPUs, gloo in the CPU tests).
"""
import ctypes
import math

import numpy as np

from . import _lib
from . import random as _rnd

__all__ = ["slot_ranges", "exchange_plan", "exchange", "global_reconfigure", "evolve_shard",
           "sharded_step"]


def slot_ranges(S, psi, N_total):
    """Global output slots owned by each rank: rank r takes the slots i whose
    point U_i = (i + psi) / N * S_total lies in [O_r, O_r + S_r),
    O_r = sum_{k<r} S_k.  Returns [(lo, hi)] (hi exclusive), a partition of
    [0, N_total) that every rank computes identically from the same sums."""
    S = [float(x) for x in S]
    tot = math.fsum(S)
    if not (tot > 0.0) or not math.isfinite(tot):
        raise ValueError("the population is extinct (zero or non-finite total weight)")
    out, off, lo = [], 0.0, 0
    for r, s in enumerate(S):
        if r == len(S) - 1:
            hi = N_total
        else:
            off = off + s
            hi = int(math.ceil(off / tot * N_total - psi))
            hi = min(max(hi, lo), N_total)
        out.append((lo, hi))
        lo = hi
    return out


def exchange_plan(ranges, n_per_rank):
    """Which slots move where: {(src, dst): (a, b)} for every pair where src
    resampled the global slots [a, b) that dst owns ([dst n, (dst + 1) n))."""
    plan = {}
    for src, (lo, hi) in enumerate(ranges):
        if hi <= lo:
            continue
        for dst in range(lo // n_per_rank, (hi - 1) // n_per_rank + 1):
            a, b = max(lo, dst * n_per_rank), min(hi, (dst + 1) * n_per_rank)
            if b > a:
                plan[(src, dst)] = (a, b)
    return plan


def exchange(sel, new, plan, lo, n, rank, group=None):
    """Moves the rows of the plan: ``sel`` holds this rank's resampled walkers
    for its slots [lo, lo + len(sel)), one row per slot; ``new`` (n rows)
    receives the walkers of the slots this rank owns.  Same-rank blocks are
    copied, the others go point to point."""
    import torch
    import torch.distributed as dist
    ops, recvs = [], []
    for (src, dst), (a, b) in sorted(plan.items()):
        if src == rank and dst == rank:
            new[a - dst * n:b - dst * n].copy_(sel[a - lo:b - lo])
        elif src == rank:
            ops.append(dist.P2POp(dist.isend, sel[a - lo:b - lo].contiguous(), dst, group))
        elif dst == rank:
            buf = torch.empty((b - a,) + tuple(new.shape[1:]), dtype=new.dtype, device=new.device)
            ops.append(dist.P2POp(dist.irecv, buf, src, group))
            recvs.append((a - dst * n, b - dst * n, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for a, b, buf in recvs:
        new[a:b].copy_(buf)


def global_reconfigure(eng, cfg_out, key2, group=None):
    """Systematic resampling over all ranks of the walkers this rank just
    evolved (``cfg_out`` with ``eng.log_w``, ``eng.e_loc``; n walkers per
    rank); leaves the resampled population in ``eng.cfg`` (identity parents)
    and returns (log G_n, E_n), identical on every rank."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    n = eng.n
    N = n * world
    L, s = eng.L, eng._stream()
    dev = eng.device
    m = ctypes.c_double()
    _lib.check(L.gfmc_dist_local_max(eng.h, n, eng._ptr(eng.log_w), ctypes.byref(m), s),
               "gfmc_dist_local_max")
    mt = torch.tensor([m.value], dtype=torch.float64, device=dev)
    dist.all_reduce(mt, op=dist.ReduceOp.MAX, group=group)
    shift = float(mt.item())
    if not math.isfinite(shift):
        shift = 0.0
    out = np.zeros(3, dtype=np.float64)
    _lib.check(L.gfmc_dist_local_sums(eng.h, n, eng._ptr(eng.log_w), eng._ptr(eng.e_loc), shift,
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), s),
               "gfmc_dist_local_sums")
    mine = torch.tensor(out, dtype=torch.float64, device=dev)
    allv = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(allv, mine, group=group)
    allv = [a.cpu().numpy() for a in allv]
    S = [a[0] for a in allv]
    S_tot = math.fsum(S)
    ranges = slot_ranges(S, _rnd.uniform(key2), N)
    logG = math.log(S_tot) + shift - math.log(N)
    E_n = math.fsum(a[1] for a in allv) / S_tot
    lo, hi = ranges[rank]
    cnt = hi - lo
    B = eng.cfg_bytes
    sel = torch.empty((max(cnt, 1), B), dtype=torch.uint8, device=dev)
    if cnt > 0:
        par = torch.empty(cnt, dtype=torch.int32, device=dev)
        last = int(out[2]) if out[2] >= 0 else 0
        _lib.check(L.gfmc_dist_parents(eng.h, n, eng._ptr(eng.log_w), shift, math.fsum(S[:rank]),
                                       S_tot, _rnd.uniform(key2), N, lo, cnt, last, eng._ptr(par), s),
                   "gfmc_dist_parents")
        _lib.check(L.gfmc_gather(eng.h, cnt, eng._ptr(par), eng._ptr(cfg_out), eng._ptr(sel),
                                 ctypes.c_void_p(0), ctypes.c_void_p(0), ctypes.c_void_p(0), s),
                   "gfmc_gather")
    torch.cuda.current_stream().synchronize()
    exchange(sel, eng.cfg.view(n, B), exchange_plan(ranges, n), lo, n, rank, group)
    eng.parents_valid = 0
    return logG, E_n


def evolve_shard(eng, method, step, lam, alw, k1, walker_offset, cfg_out):
    """The evolve half of a step for this rank's walkers, the global walkers
    [walker_offset, walker_offset + n) (gfmc_evolve): the same per-walker
    streams as in the unsharded population."""
    key = np.ascontiguousarray(_rnd.as_key(k1), dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    _lib.check(eng.L.gfmc_evolve(eng.h, _lib.METHODS[method], float(step),
                                 float(lam if lam is not None else 0.0), float(alw),
                                 key.ctypes.data_as(P), int(walker_offset), eng.n,
                                 eng._ptr(eng.cfg), eng._ptr(eng.parents), int(eng.parents_valid),
                                 eng._ptr(cfg_out), eng._ptr(eng.log_w), eng._ptr(eng.e_loc),
                                 ctypes.c_void_p(0), eng._stream()), "gfmc_evolve")


def sharded_step(eng, method, step, lam, alw, k1, k2, cfg_tmp, group=None):
    """One branching step of a population sharded over the ranks (rank r holds
    the global walkers [r n, (r + 1) n)).  Returns (log G_n, E_n), identical on
    every rank."""
    import torch.distributed as dist
    evolve_shard(eng, method, step, lam, alw, k1, dist.get_rank(group) * eng.n, cfg_tmp)
    return global_reconfigure(eng, cfg_tmp, k2, group)

"""Walkers sharded over GPUs: contiguous walker blocks, global systematic
resampling with the data moved once.

The reference's multi-device path (engine/multi_gpu.py:91-155) all-gathers
every configuration to every device and resamples there.  Here each shard
resamples only its own output slots: the shards exchange their weight sums
(four float64 values each), each finds the parents of the global slots whose
resampling points fall in its own weight interval (``slot_ranges``), and
sends those walkers -- configuration and local energy, one row each -- to the
shards that own the slots: contiguous blocks, so a shard talks to at most a
few neighbours.  The result is the systematic resampling of the concatenated
population (walkers/reconfiguration.py:9-62: the new walkers carry their
parents' local energies and zero log weights), and with ``gfmc_evolve`` (the
per-walker random streams numbered by the global walker index) a sharded run
follows the same trajectory as the unsharded one.

Two ways to hold the shards, with the same step:

* ``ShardedPopulation(..., devices=[...])``: every shard in this process,
  one per listed device (several shards on one device emulate the ranks).
  The exchange is a device-to-device copy per block.
* ``ShardedPopulation(..., group=g)`` (or a process group already set up
  with ``torch.distributed``): one shard per process, as launched by
  torchrun.  The max and the sums are reduced on device buffers (NCCL), the
  blocks go point to point; a gloo group stages them through host memory.

Per step: one evolve launch per shard, the max of the log weights reduced
over shards on the device, one 4-double gather whose host copy is the step's
only wait (the block sizes of the exchange are decided on the host), the
parents and the gather of the selected rows, one exchange.
"""
import ctypes
import math

import numpy as np

from . import _lib
from . import random as _rnd

__all__ = ["slot_ranges", "exchange_plan", "exchange", "global_reconfigure", "evolve_shard",
           "sharded_step", "ShardedPopulation"]


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


def exchange(sel, new, plan, lo, n, rank, group=None, host_staging=False):
    """Moves the rows of the plan between processes: ``sel`` holds this
    rank's resampled rows for its slots [lo, lo + len(sel)), one row per slot;
    ``new`` (n rows) receives the rows of the slots this rank owns.
    Same-rank blocks are copied, the others go point to point (through host
    memory when ``host_staging``: a gloo group)."""
    import torch
    import torch.distributed as dist
    ops, recvs = [], []
    for (src, dst), (a, b) in sorted(plan.items()):
        if src == rank and dst == rank:
            new[a - dst * n:b - dst * n].copy_(sel[a - lo:b - lo])
        elif src == rank:
            t = sel[a - lo:b - lo].contiguous()
            ops.append(dist.P2POp(dist.isend, t.cpu() if host_staging else t, dst, group))
        elif dst == rank:
            dev = "cpu" if host_staging else new.device
            buf = torch.empty((b - a,) + tuple(new.shape[1:]), dtype=new.dtype, device=dev)
            ops.append(dist.P2POp(dist.irecv, buf, src, group))
            recvs.append((a - dst * n, b - dst * n, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for a, b, buf in recvs:
        new[a:b].copy_(buf)


# ---------------------------------------------------------------------------
# communication between shards
# ---------------------------------------------------------------------------
class _LocalShards:
    """Every shard in this process (one per device, or several per device)."""

    def __init__(self, devices):
        self.devices = list(devices)
        self.world = len(self.devices)
        self.rank0 = 0

    def max_(self, torch, vals):
        """vals: one (1,) float64 device tensor per local shard -> the max over
        all shards, as one (1,) tensor on each shard's device."""
        d0 = vals[0].device
        m = torch.stack([v.to(d0) for v in vals]).max().reshape(1)
        return [m.to(v.device) for v in vals]

    def gather(self, torch, rows):
        d0 = rows[0].device
        return torch.stack([r.to(d0) for r in rows]).cpu().numpy()

    def sum_(self, torch, vals):
        d0 = vals[0].device
        s = torch.stack([v.to(d0) for v in vals]).sum(0)
        return [s.to(v.device) for v in vals]

    def all_rows(self, torch, parts):
        d0 = parts[0].device
        return torch.cat([p.to(d0) for p in parts])

    def exchange(self, torch, plan, payloads, news, n):
        """payloads[r] = (lo_r, rows of the slots [lo_r, hi_r)); news[r] the
        (n, width) receive buffer of shard r."""
        for (src, dst), (a, b) in sorted(plan.items()):
            lo = payloads[src][0]
            news[dst][a - dst * n:b - dst * n].copy_(payloads[src][1][a - lo:b - lo])


class _ProcessGroup:
    """One shard per process over a torch.distributed group: NCCL reduces and
    gathers device buffers; a gloo group stages them through host memory."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.world = dist.get_world_size(group)
        self.rank0 = dist.get_rank(group)
        self.host = dist.get_backend(group) != "nccl"

    def _op(self, torch, t, fn):
        x = t.cpu() if self.host else t
        fn(x)
        if x is not t:
            t.copy_(x)
        return t

    def max_(self, torch, vals):
        d = self.dist
        return [self._op(torch, vals[0], lambda x: d.all_reduce(x, op=d.ReduceOp.MAX,
                                                               group=self.group))]

    def sum_(self, torch, vals):
        d = self.dist
        return [self._op(torch, vals[0], lambda x: d.all_reduce(x, op=d.ReduceOp.SUM,
                                                               group=self.group))]

    def gather(self, torch, rows):
        x = rows[0].cpu() if self.host else rows[0]
        parts = [torch.empty_like(x) for _ in range(self.world)]
        self.dist.all_gather(parts, x, group=self.group)
        return torch.stack(parts).cpu().numpy()

    def all_rows(self, torch, parts):
        x = parts[0].cpu() if self.host else parts[0]
        out = [torch.empty_like(x) for _ in range(self.world)]
        self.dist.all_gather(out, x, group=self.group)
        return torch.cat(out).to(parts[0].device)

    def exchange(self, torch, plan, payloads, news, n):
        lo, sel = payloads[0]
        exchange(sel, news[0], plan, lo, n, self.rank0, self.group, host_staging=self.host)


# ---------------------------------------------------------------------------
# the sharded step
# ---------------------------------------------------------------------------
def evolve_shard(eng, method, step, lam, alw, k1, walker_offset, cfg_out, hops=None):
    """The evolve half of a step for one shard, the global walkers
    [walker_offset, walker_offset + n) (gfmc_evolve): the same per-walker
    streams as in the unsharded population."""
    key = np.ascontiguousarray(_rnd.as_key(k1), dtype=np.uint32)
    P = ctypes.POINTER(ctypes.c_uint32)
    _lib.check(eng.L.gfmc_evolve(eng.h, _lib.METHODS[method], float(step),
                                 float(lam if lam is not None else 0.0), float(alw),
                                 key.ctypes.data_as(P), int(walker_offset), eng.n,
                                 eng._ptr(eng.cfg), eng._ptr(eng.parents), int(eng.parents_valid),
                                 eng._ptr(cfg_out), eng._ptr(eng.log_w), eng._ptr(eng.e_loc),
                                 eng._ptr(hops) if hops is not None else ctypes.c_void_p(0),
                                 eng._stream()), "gfmc_evolve")


def _resample(torch, shards, cfg_outs, key2, comm):
    """Systematic resampling over all shards of the walkers just evolved into
    ``cfg_outs`` (with each shard's ``log_w``, ``e_loc``).  Leaves the new
    population in each shard's ``cfg`` / ``e_loc`` with zero ``log_w``;
    returns (log G_n, E_n), identical on every shard."""
    n = shards[0].n
    N = n * comm.world
    B = shards[0].cfg_bytes
    psi = _rnd.uniform(key2)
    mx = []
    for sh in shards:
        with torch.cuda.device(sh.device):
            t = torch.empty(1, dtype=torch.float64, device=sh.device)
            _lib.check(sh.L.gfmc_dist_local_max_dev(sh.h, n, sh._ptr(sh.log_w), sh._ptr(t),
                                                    sh._stream()), "gfmc_dist_local_max_dev")
            mx.append(t)
    shift_d = comm.max_(torch, mx)
    rows = []
    for sh, sd in zip(shards, shift_d):
        with torch.cuda.device(sh.device):
            r = torch.empty(4, dtype=torch.float64, device=sh.device)
            _lib.check(sh.L.gfmc_dist_local_sums_dev(sh.h, n, sh._ptr(sh.log_w), sh._ptr(sh.e_loc),
                                                     sh._ptr(sd), sh._ptr(r), sh._stream()),
                       "gfmc_dist_local_sums_dev")
            rows.append(r)
    g = comm.gather(torch, rows)            # (world, 4) on the host: the step's one wait
    shift = float(g[0, 0])
    S = [float(x) for x in g[:, 1]]
    S_tot = math.fsum(S)
    ranges = slot_ranges(S, psi, N)
    logG = math.log(S_tot) + shift - math.log(N)
    E_n = math.fsum(float(x) for x in g[:, 2]) / S_tot
    payloads, news = [], []
    for j, (sh, cfg_out) in enumerate(zip(shards, cfg_outs)):
        r = comm.rank0 + j
        lo, hi = ranges[r]
        cnt = hi - lo
        with torch.cuda.device(sh.device):
            rows_ = torch.empty((max(cnt, 1), B + 8), dtype=torch.uint8, device=sh.device)
            if cnt > 0:
                par = torch.empty(cnt, dtype=torch.int32, device=sh.device)
                last = int(g[r, 3]) if g[r, 3] >= 0 else 0
                _lib.check(sh.L.gfmc_dist_parents(sh.h, n, sh._ptr(sh.log_w), shift, math.fsum(S[:r]),
                                                  S_tot, psi, N, lo, cnt, last, sh._ptr(par),
                                                  sh._stream()), "gfmc_dist_parents")
                c_sel = torch.empty(cnt * B, dtype=torch.uint8, device=sh.device)
                e_sel = torch.empty(cnt, dtype=torch.float64, device=sh.device)
                _lib.check(sh.L.gfmc_gather(sh.h, cnt, sh._ptr(par), sh._ptr(cfg_out), sh._ptr(c_sel),
                                            sh._ptr(sh.e_loc), sh._ptr(e_sel), ctypes.c_void_p(0),
                                            sh._stream()), "gfmc_gather")
                rows_[:cnt, :B].copy_(c_sel.view(cnt, B))
                rows_[:cnt, B:].copy_(e_sel.view(torch.uint8).view(cnt, 8))
            payloads.append((lo, rows_[:cnt]))
            news.append(torch.empty((n, B + 8), dtype=torch.uint8, device=sh.device))
    comm.exchange(torch, exchange_plan(ranges, n), payloads, news, n)
    for sh, new in zip(shards, news):
        with torch.cuda.device(sh.device):
            sh.cfg.view(n, B).copy_(new[:, :B])
            sh.e_loc.copy_(new[:, B:].contiguous().view(torch.float64).view(n))
            sh.log_w.zero_()
            sh.parents_valid = 0
    return logG, E_n


def global_reconfigure(eng, cfg_out, key2, group=None):
    """Systematic resampling over all processes of a torch.distributed group
    of the walkers this rank just evolved (``cfg_out`` with ``eng.log_w``,
    ``eng.e_loc``; n walkers per rank).  Leaves the resampled population in
    ``eng.cfg`` (identity parents) with the parents' local energies in
    ``eng.e_loc`` and zero ``eng.log_w``; returns (log G_n, E_n), identical on
    every rank."""
    import torch
    return _resample(torch, [eng], [cfg_out], key2, _ProcessGroup(group))


def sharded_step(eng, method, step, lam, alw, k1, k2, cfg_tmp, group=None):
    """One branching step of a population sharded over the processes of a
    group (rank r holds the global walkers [r n, (r + 1) n)).  Returns
    (log G_n, E_n), identical on every rank."""
    import torch.distributed as dist
    evolve_shard(eng, method, step, lam, alw, k1, dist.get_rank(group) * eng.n, cfg_tmp)
    return global_reconfigure(eng, cfg_tmp, k2, group)


class ShardedPopulation:
    """A walker population split into equal contiguous shards, one engine
    handle per shard; the step's evolve runs per shard with the global
    walker streams and the resampling is global, so the trajectory is the
    unsharded one (configurations identical, weights to rounding: the
    sharded evolve rebuilds the guide state each step instead of carrying
    it).

    ``devices``: the devices of the shards held by this process (several
    entries may name one device, which emulates the ranks); ``group``: one
    shard per process of this torch.distributed group (default: the
    initialised default group, when ``devices`` is not given).  The public
    methods mirror ``GFMCEngine``'s (``load``, ``local_energy``, ``steps``,
    ``population``, ``status``), each over the whole population.
    """

    def __init__(self, hamiltonian, guide, n_walkers, precision="fp64", devices=None, group=None):
        import torch
        from .engine import GFMCEngine
        self.torch = torch
        if devices is None:
            import torch.distributed as dist
            if not (dist.is_available() and dist.is_initialized()):
                raise ValueError("ShardedPopulation needs a list of devices or an initialised "
                                 "torch.distributed process group")
            self.comm = _ProcessGroup(group)
            devices = [torch.device("cuda", torch.cuda.current_device())]
        else:
            devices = [torch.device(d) for d in devices]
            self.comm = _LocalShards(devices)
        world = self.comm.world
        n_walkers = int(n_walkers)
        if n_walkers % world:
            raise ValueError(f"n_walkers={n_walkers} must be divisible by the number of shards "
                             f"({world})")
        self.n = n_walkers
        self.n_local = n_walkers // world
        self.N = int(hamiltonian.N)
        self.world = world
        self.shards, self.tmp = [], []
        for d in devices:
            with torch.cuda.device(d):
                sh = GFMCEngine(hamiltonian, guide, self.n_local, precision=precision)
                self.shards.append(sh)
                self.tmp.append(torch.empty_like(sh.cfg))
        self.device = self.shards[0].device
        self.cfg_bytes = self.shards[0].cfg_bytes

    def _offset(self, j):
        return (self.comm.rank0 + j) * self.n_local

    def set_max_iters(self, max_iters):
        for sh in self.shards:
            sh.set_max_iters(max_iters)

    def carry_mode(self, mode=-1):
        """The sharded evolve rebuilds the guide state every step."""
        return False

    def load(self, config):
        """Loads the whole population (n_walkers, N); each shard takes its block."""
        torch = self.torch
        c = config if torch.is_tensor(config) else torch.as_tensor(np.asarray(config))
        if tuple(c.shape) != (self.n, self.N):
            raise ValueError(f"walker configurations must have shape ({self.n}, {self.N}); "
                             f"got {tuple(c.shape)}")
        for j, sh in enumerate(self.shards):
            a = self._offset(j)
            with torch.cuda.device(sh.device):
                sh.load(c[a:a + self.n_local])

    def local_energy(self):
        """e_L of the whole population (float64, host tensor)."""
        torch = self.torch
        parts = []
        for sh in self.shards:
            with torch.cuda.device(sh.device):
                parts.append(sh.local_energy())
        return self.comm.all_rows(torch, parts).cpu()

    def status(self):
        torch = self.torch
        st = 0
        for sh in self.shards:
            with torch.cuda.device(sh.device):
                st |= sh.status()
        if isinstance(self.comm, _ProcessGroup):
            g = self.comm.gather(torch, [torch.tensor([st], dtype=torch.int64, device=self.device)])
            st = int(np.bitwise_or.reduce(g.ravel()))
        return st

    def steps(self, method, step, lam, alw, keys, logG, E, hops=None):
        """len(keys) branching steps of the whole population (keys: (n, 4)
        uint32 = k1, k2 per step); log G_n, E_n into the device tensors logG, E
        and, when given, the hops of each step summed over all walkers."""
        torch = self.torch
        keys = np.ascontiguousarray(keys, dtype=np.uint32)
        ns = keys.shape[0]
        lgs, Es = np.zeros(ns), np.zeros(ns)
        hb = None
        if hops is not None:
            hb = []
            for sh in self.shards:
                hb.append(torch.zeros(ns, dtype=torch.int64, device=sh.device))
        for s in range(ns):
            for j, sh in enumerate(self.shards):
                with torch.cuda.device(sh.device):
                    evolve_shard(sh, method, step, lam, alw, keys[s, :2], self._offset(j),
                                 self.tmp[j], hb[j][s:s + 1] if hb is not None else None)
            lgs[s], Es[s] = _resample(torch, self.shards, self.tmp, keys[s, 2:], self.comm)
        logG[:ns].copy_(torch.as_tensor(lgs, dtype=torch.float64))
        E[:ns].copy_(torch.as_tensor(Es, dtype=torch.float64))
        if hb is not None:
            hops[:ns].copy_(self.comm.sum_(torch, hb)[0].to(hops.device))

    def population(self):
        """(configurations float64 (n_walkers, N), e_loc (n_walkers,)) of the
        whole population, on this process's first shard device."""
        torch = self.torch
        cs, es = [], []
        for sh in self.shards:
            with torch.cuda.device(sh.device):
                c, e = sh.population()
                cs.append(c)
                es.append(e)
        return (self.comm.all_rows(torch, cs).to(self.device),
                self.comm.all_rows(torch, es).to(self.device))

    def windowed_energy(self, logG, E, p_array):
        sh = self.shards[0]
        with self.torch.cuda.device(sh.device):
            return sh.windowed_energy(logG.to(sh.device), E.to(sh.device), p_array)

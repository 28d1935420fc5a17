"""Benchmark of the GFMC branching step on B200 (walker-steps/s).

Workload (the headline configuration): periodic 16x16 square-lattice
Heisenberg model in the Marshall-rotated frame (J_x = J_y = -1, J_z = +1,
512 bonds, M_total = 513), long-range Jastrow guide on all 32640 pairs with
beta_ij = v(r_ij) = 0.3 / r (periodic minimum-image distance), 32768 walkers
initialised as random Sz = 0 bitstrings, cont_time with tau = 0.05.  Inputs
are synthetic (the configuration itself; no dataset is involved).

A step is one production branching step (evolve + systematic resampling)
over the whole population.  ``value`` times steps with the population
resident in HBM; L2 is flushed (a 256 MB write) before every timed step, and
each step is timed with CUDA events on the launching stream.  ``e2e`` times
the same step through the C ABI with the walkers in pinned host memory
(packed configurations copied in, and configurations, parent map and the
step's log G / E copied out, every step).

Multi-GPU (torchrun): every rank runs its own population (replicas, weak
scaling, no data-path collective); time is the max over ranks.

``--impl reference``: the reference's algorithm on the host cores -- PyGFMC
itself is JAX-based and cannot run here, so its CPU restatement (``oracle/``,
C + OpenMP on every host thread) runs a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_WALKERS = 32768
L = 16
TAU = 0.05
# untimed oracle steps that bring the reference arm's fresh sample to the
# equilibrated population before its timed steps
REF_EQUILIBRATION_STEPS = 100


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one
# evolve_kernel launch of this workload, from a one-pass ncu capture of
# `bench.py --steps 20 --warmup 3 --no-cpu-baseline` (32768 walkers, float64;
# mean of 3 carried-state launches): 77.8 MB read + 34.4 MB written; part of
# the carried fields and evaluation records stays in L2 across the step, so
# DRAM sees less than the algorithmic bytes.
EVOLVE_TRAFFIC_BYTES = {("fp64", 32768): 112.1e6}

# DRAM traffic of one rbm_theta_persist launch (16x16, H = 512, 65536
# walkers), from the `--set full` capture of
# `bench.py --guide rbm --steps 3 --warmup 3` (-k regex:rbm_theta_persist
# -s 2 -c 1): 3.0 MB read + 74.6 MB written (the rest of the 134 MB output
# is still in L2 when the kernel ends).
THETA_TRAFFIC_BYTES = {(256, 512, 65536): 77.6e6}


def build_system(P, precision):
    lat = P.square(L)
    H = P.SpinHalf.create(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    pos = lat.extras["positions"]
    n = lat.N
    iu = np.triu_indices(n, 1)
    pairs = np.stack(iu, axis=1)
    d = np.abs(pos[pairs[:, 0]] - pos[pairs[:, 1]])
    d = np.minimum(d, L - d)
    r = np.sqrt((d ** 2).sum(1))
    G = P.JastrowSpinHalf(n, pairs, beta=0.3 / r)
    # the couplings as the guide stores them (rounded to its float32 dtype)
    return lat, H, G, pairs, np.asarray(G.beta, np.float64)


CLOCK_FIELDS = ("uuid,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    """nvidia-smi sampling this process's GPU every 50 ms while it runs (one
    nvidia-smi process, stopped through its own handle).  start() returns once
    the first sample has arrived, so the samples cover what runs after it."""

    def __init__(self, uuid):
        self.uuid = (uuid or "").lower()
        self.lines, self.proc, self.th = [], None, None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self

        def read():
            for ln in self.proc.stdout:
                ln = ln.strip()
                if ln and (not self.uuid or self.uuid in ln.split(",")[0].strip().lower()):
                    self.lines.append(ln)

        self.th = threading.Thread(target=read, daemon=True)
        self.th.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10 and self.proc.poll() is None:
            time.sleep(0.01)
        self.n0 = len(self.lines)
        return self

    def stop(self):
        """The samples taken between start() and now."""
        if self.proc is None:
            return []
        n1 = len(self.lines)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.th.join(timeout=2)
        return self.lines[max(self.n0 - 1, 0):n1]


def gpu_uuid(torch, dev):
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return ""


def summarize_clocks(lines):
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in lines:
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 10:
            continue
        try:
            sm.append(float(f[2]))
            mx = float(f[3])
        except ValueError:
            continue
        for nm, v in zip(names, f[6:10]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_reference(P, cfg_sample, alw, steps, warmup, seed_key, min_seconds=0.0, max_steps=1000):
    """The oracle (C, OpenMP) on a sample of walkers: walker-steps/s, the
    threads used, the timed seconds and the timed steps (at least `steps`,
    more until `min_seconds` of timed work or `max_steps`)."""
    from oracle import oracle as O
    O.build()
    lat, H, G, pairs, beta = build_system(P, "fp64")
    m = O.spin_half(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
    g = O.jastrow_spin_half(lat.N, pairs, beta, None, m)
    cfg = np.array(cfg_sample, dtype=np.float64, copy=True)
    lw = np.zeros(len(cfg)); el = np.zeros(len(cfg))
    key = np.asarray(seed_key, np.uint32)
    threads = O.lib().om_threads()
    times = []
    s = 0
    while s < warmup + steps or (sum(times) < min_seconds and len(times) < max_steps):
        key, r = O.split(key, 2)
        k1, k2 = O.fold_in(r, 0), O.fold_in(r, 1)
        t0 = time.perf_counter()
        O.evolve(m, g, "cont_time", TAU, None, alw, k1, cfg, lw, el)
        O.reconfigure(k2, cfg, lw, el)
        if s >= warmup:
            times.append(time.perf_counter() - t0)
        s += 1
    return len(cfg) * len(times) / sum(times), threads, sum(times), len(times)


def study_system(P, args):
    """The learned-vs-plain workloads of the sigma study: the RBM on the 16x16
    Heisenberg or the kagome lattice (see rbm_system), or the dense MLP
    (320 -> 256 -> 256 -> 1) on the 64-site Bose-Hubbard ring against the
    Gutzwiller + density-Jastrow guide (32768 walkers, tau = 0.02,
    p = [16, 64])."""
    if args.lattice == "bose64":
        e, H, GJ = bose_chain(P)
        G0 = P.MLPBoseHubbard(64, 4, hidden=(256, 256), seed=0, sigma=0.01)

        def walk(n, key):
            return P.prepare_walkers_occupations(n, 64, 64, 4, key)

        def train(w, G):
            return P.learn.train_mlp_guide(w, H, G, n_iterations=args.train_iters,
                                           steps_per_iteration=3, step_size=0.02, lr=args.train_lr,
                                           rng_key=P.PRNGKey(14), warmup_steps=100, verbosity=0)
        return {"name": "bose_hubbard_ring64", "H": H, "plain": GJ, "G0": G0, "N": 64,
                "learned": "mlp_256x256_mixed", "n_learned": N_WALKERS, "n_plain": N_WALKERS,
                "tau": 0.02,
                "p": [16, 64], "walk": walk, "train": train,
                "plain_name": "gutzwiller_density_jastrow"}
    lat, H, G, hid, tau, n_rbm, name = rbm_system(P, args.lattice)
    N = lat.N

    def walk(n, key):
        return P.prepare_walkers_sz(n, N, key, sz=0)

    def train(w, G0):
        return P.learn.train_rbm_guide(w, H, G0, n_iterations=args.train_iters,
                                       steps_per_iteration=3, step_size=tau, lr=args.train_lr,
                                       rng_key=P.PRNGKey(14), warmup_steps=100, verbosity=0)
    return {"name": name, "H": H, "plain": G, "G0": P.RBMSpinHalf(N, hid, seed=0, sigma=0.01),
            "N": N, "learned": f"rbm_h{hid}_mixed", "n_learned": n_rbm,
            "n_plain": N_WALKERS if args.lattice == "square16" else n_rbm, "tau": tau,
            "p": [8, 32, 128] if args.lattice == "square16" else [16, 64, 256], "walk": walk,
            "train": train,
            "plain_name": "longrange_jastrow" if args.lattice == "square16" else "nn_jastrow"}


def sigma_study(P, args):
    """GPU seconds to sigma(E/N) = 1e-5: the plain Jastrow engine (float64 and
    float32) against a learned guide trained on the run's own walkers by
    variance minimisation, on the workload of study_system.  Each method runs
    warm-up + production through run(); the blocked jackknife error at the
    largest window gives sigma(E/N); the time to the target is the production
    GPU time x (sigma / 1e-5)^2 (errors fall as 1/sqrt(steps)).  The learned
    guide's training time is reported beside it."""
    import torch
    S = study_system(P, args)
    H, N, tau, p_arr = S["H"], S["N"], S["tau"], S["p"]
    pm = p_arr[-1]
    out = {}

    def measure(key, guide, n, steps, warm, precision):
        w = S["walk"](n, P.PRNGKey(11))
        torch.cuda.synchronize()
        wf, E, _, st, raw = P.run(w, steps, H, tau, guide, p_arr, rng_key=P.PRNGKey(12),
                                  warmup_steps=warm, verbosity=0, precision=precision)
        Ej, err = P.estimators.jackknife_energy([pm], raw["log_weights"], raw["energy"], 20)
        sig = err[pm] / N
        t = st["runtime"]
        out[key] = {"E_per_site": Ej[pm] / N, "sigma_per_site": sig, "n_walkers": n,
                    "steps": steps, "warmup": warm, "precision": precision,
                    "production_gpu_s": t, "gpu_s_to_1e-5": t * (sig / 1e-5) ** 2,
                    "walker_steps_per_s": n * steps / t,
                    "local_energy_var_per_site": float(np.var(wf.e_loc) / N)}

    measure("jastrow_fp64", S["plain"], S["n_plain"], args.study_steps, 2000, "fp64")
    measure("jastrow_mixed", S["plain"], S["n_plain"], args.study_steps, 2000, "mixed")
    trained, hist = S["train"](S["walk"](S["n_learned"], P.PRNGKey(13)), S["G0"])
    rk = S["learned"]
    measure(rk, trained, S["n_learned"], args.rbm_steps, 500, "mixed")
    r = out[rk]
    r["training_gpu_s"] = hist["seconds"]
    r["train_var_per_site_first_last"] = [float(hist["variance"][0] / N),
                                          float(hist["variance"][-1] / N)]
    r["train_iterations"] = len(hist["variance"])
    r["train_lr"] = args.train_lr
    r["train_collapsed"] = bool(hist["collapsed"])
    r["gpu_s_to_1e-5_with_training"] = r["gpu_s_to_1e-5"] + hist["seconds"]
    j = out["jastrow_fp64"]
    diff = abs(j["E_per_site"] - r["E_per_site"]) / np.hypot(j["sigma_per_site"], r["sigma_per_site"])
    line = {"metric": "GPU-s to sigma(E/N)=1e-5", "value": r["gpu_s_to_1e-5"], "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
            "config": {"workload": f"{S['name']}_{rk}_vs_{S['plain_name']}", "tau": tau, "p": pm,
                       "jackknife_blocks": 20},
            "methods": out,
            "learned_over_jastrow_fp64_time_ratio": r["gpu_s_to_1e-5"] / j["gpu_s_to_1e-5"],
            "energy_difference_in_sigma": diff}
    print(json.dumps(line))


def rbm_system(P, lattice):
    """The RBM workloads: the periodic 16x16 Heisenberg lattice (H = 512,
    tau = 0.05, 65536 walkers) or the 12x12 kagome XXZ lattice (432 sites,
    864 bonds, J_x = J_y = -1, J_z = 1; H = 432, tau = 0.02, 131072 walkers),
    each with the plain guide it is compared with (long-range Jastrow v(r) =
    0.3 / r on the square lattice, nearest-neighbour Jastrow beta = 0.3 on
    kagome)."""
    if lattice == "kagome12":
        lat = P.kagome(12, 12)
        H = P.SpinHalf.create(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
        GJ = P.JastrowSpinHalf(lat.N, lat.edges, beta=0.3)
        return lat, H, GJ, 432, 0.02, 131072, "kagome_12x12_xxz"
    lat, H, GJ, pairs, beta = build_system(P, "fp64")
    return lat, H, GJ, 512, TAU, 65536, "heisenberg_16x16"


def measure_rbm(P, lattice, hid, n, steps, warmup):
    """The RBM-guided branching step (float32 build, L2 flushed before each
    timed step), one training step (gfmc_rbm_train_step) and the tensor-core
    theta GEMM of one population: a dict of times and rates."""
    import torch
    lat, H, GJ, _, tau, _, name = rbm_system(P, lattice)
    N = lat.N
    G = P.RBMSpinHalf(N, hid, seed=0, sigma=0.01)
    w = P.prepare_walkers_sz(n, N, P.PRNGKey(0), sz=0)
    eng = P.GFMCEngine(H, G, n, precision="mixed")
    eng.load(w.config)
    stream = torch.cuda.current_stream()
    alw = float((-eng.local_energy()).mean().item())
    step_ms, hpw = timed_steps(P, eng, alw, tau, steps, warmup, P.PRNGKey(1000))
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    eng.rbm_theta()
    torch.cuda.synchronize()
    # ten launches back to back: the host's per-call overhead overlaps the
    # kernels instead of sitting inside one call's bracket
    a.record(stream)
    for _ in range(10):
        eng.rbm_theta()
    b.record(stream)
    b.synchronize()
    gemm_ms = a.elapsed_time(b) / 10
    eng.rbm_train_step(1e-4)
    torch.cuda.synchronize()
    a.record(stream)
    eng.rbm_train_step(1e-4)
    b.record(stream)
    b.synchronize()
    train_ms = a.elapsed_time(b)
    del eng
    pk, pk_kind = peaks()
    Hp = ((hid + 255) // 256) * 256
    Np = ((N + 63) // 64) * 64
    gemm_tflops = 2.0 * n * Hp * Np / (gemm_ms / 1e3) / 1e12
    # the float32 output is the GEMM's one unavoidable HBM traffic
    out_bytes = 4.0 * n * Hp
    return {"workload": f"{name}_rbm_h{hid}_cont_time", "n_walkers": n, "n_sites": N, "tau": tau,
            "value": n / (step_ms / 1e3), "unit": "walker-steps/s", "ms_per_step": step_ms,
            "steps": steps, "hops_per_walker_step": hpw, "train_step_ms": train_ms,
            "theta_gemm": {"kernel": "rbm_theta_persist", "ms": gemm_ms, "tflops": gemm_tflops,
                           "peak_tflops": pk["bf16_tflops"], "peak_source": pk_kind,
                           "frac": gemm_tflops / pk["bf16_tflops"], "out_bytes": out_bytes,
                           "hbm_floor_ms": out_bytes / (pk["hbm_gbs"] * 1e9) * 1e3,
                           "hbm_frac": out_bytes / (gemm_ms / 1e3) / (pk["hbm_gbs"] * 1e9)},
            "_jastrow": GJ, "_H": H, "_w": w, "_tau": tau, "_name": name}


def rbm_bench(P, args):
    """Learned-guide workload: an RBM guide (bf16 weights N(0, 0.01^2)),
    float32 build, cont_time.  Times the branching step (L2 flushed before
    each), one training step (gfmc_rbm_train_step), the tensor-core theta
    GEMM and, beside them, the plain Jastrow-guided step on the same lattice
    (float64 and float32)."""
    lat, H, GJ, hid, tau, n_def, name = rbm_system(P, args.lattice)
    if args.hidden_set:
        hid = args.hidden
    n = args.walkers if args.walkers_set else n_def
    wk = max(args.warmup, 3)
    r = measure_rbm(P, args.lattice, hid, n, args.steps, wk)
    plain = {}
    for prec in ("fp64", "mixed"):
        ej = P.GFMCEngine(H, GJ, n, precision=prec)
        ej.load(r["_w"].config)
        alw_j = float((-ej.local_energy()).mean().item())
        ms_j, _ = timed_steps(P, ej, alw_j, tau, args.steps, wk, P.PRNGKey(1000))
        plain[prec] = {"value": n / (ms_j / 1e3), "ms_per_step": ms_j}
        del ej
    g = r["theta_gemm"]
    line = {"metric": "walker-steps/s", "value": r["value"], "unit": "walker-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": wk, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
            "data": "synthetic",
            "config": {"workload": r["workload"], "n_walkers": n, "n_sites": lat.N,
                       "tau": tau, "l2": "flushed (256 MB write) before every timed step",
                       "hops_per_walker_step": r["hops_per_walker_step"]},
            "train_step_ms": r["train_step_ms"],
            "jastrow_fp64": plain["fp64"], "jastrow_mixed": plain["mixed"],
            "roofline": {"bound": "tensor", "kernel": "rbm_theta_persist", "achieved": g["tflops"],
                         "peak": g["peak_tflops"], "unit": "TFLOP/s", "frac": g["frac"],
                         "traffic": THETA_TRAFFIC_BYTES.get((lat.N, hid, n)),
                         "peak_source": g["peak_source"],
                         "hbm_floor_ms": g["hbm_floor_ms"], "hbm_frac": g["hbm_frac"],
                         "note": "the GEMM's floor is its float32 output through HBM (hbm_floor_ms); "
                                 "the branching step itself is bound by the per-slot product "
                                 "chains and block barriers of its float32 kernel (see profiles/)"}}
    print(json.dumps(line))


def bose_chain(P):
    """Bose-Hubbard ring of 64 sites, 64 bosons, n_max = 4, t = 1, U = 3
    (M = 129), with the Gutzwiller + density-Jastrow guide."""
    e = P.chain(64).edges
    H = P.BoseHubbard.create(e, t=1.0, U=3.0, n_max=4, dtype=np.float64)
    GJ = P.JastrowBoseHubbard(64, e, beta=0.05, d=0.3)
    return e, H, GJ


def timed_steps(P, eng, alw, tau, steps, warmup, key):
    """Mean CUDA-event time of one cont_time branching step (L2 flushed by a
    256 MB write before each) and the hops per walker-step."""
    import torch
    dev = eng.device
    keys, key = P.engine.key_schedule(key, warmup)
    lg = torch.empty(warmup, dtype=torch.float64, device=dev)
    eng.steps("cont_time", tau, None, alw, keys, lg, torch.empty_like(lg))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    keys, key = P.engine.key_schedule(key, steps)
    logG = torch.empty(1, dtype=torch.float64, device=dev)
    Es = torch.empty_like(logG)
    hops = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream()
    ms, tot_hops = [], 0
    for st in range(steps):
        flush.fill_(float(st))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.steps("cont_time", tau, None, alw, keys[st:st + 1], logG, Es, hops)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        tot_hops += int(hops.item())
    return float(np.mean(ms)), tot_hops / (eng.n * steps)


# The reference's published throughput (paper/images/Fig3/data.csv, 1 H200,
# iterations/s x walkers): walker-steps/s by population.
FIG3_H200 = {1024: 1.16e6, 32768: 2.68e7, 65536: 3.63e7, 131072: 4.68e7, 1 << 20: 5.67e7,
             1 << 24: 5.69e7}


def fig3_bench(P, args):
    """The reference's own throughput workload (its paper's Fig. 3): periodic
    Heisenberg chain L = 100 (J_xy = -1, J_z = 1), no guide, single_step with
    n_bra = 6 and lam = n_edges J_z / 4 = 25, every walker starting from the
    Neel state, a branching step = 6 sub-steps + resampling.  Same timing
    rules as the headline line (W warm-up steps, CUDA events per step on the
    launching stream, L2 flushed before each, clocks sampled); the line adds
    the published H200 number at the same population where there is one, and
    the oracle on the host cores (C + OpenMP, ~10 s) beside it."""
    import torch
    L_ = 100
    e = P.chain(L_).edges
    H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    n = args.walkers
    neel = np.where(np.arange(L_) % 2 == 0, 1.0, -1.0)
    eng = P.GFMCEngine(H, None, n, precision=args.precision)
    dev = eng.device
    # one Neel row expanded on the device (no n x L host array)
    eng.load(torch.as_tensor(neel, dtype=torch.float64, device=dev).expand(n, L_))
    n_bra, lam = 6, 25.0
    e0 = eng.local_energy()
    alw = float(torch.log(lam - e0).mean().item())
    wk = max(args.warmup, 3)
    keys, key = P.engine.key_schedule(P.PRNGKey(1), wk)
    lgw = torch.empty(wk, dtype=torch.float64, device=dev)
    eng.steps("single_step", n_bra, lam, alw, keys, lgw, torch.empty_like(lgw))
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    logG = torch.empty(1, dtype=torch.float64, device=dev)
    Es = torch.empty_like(logG)
    keys, key = P.engine.key_schedule(key, args.steps)
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(gpu_uuid(torch, dev)).start()
    torch.cuda.synchronize()
    ms = []
    for st in range(args.steps):
        flush.fill_(float(st))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.steps("single_step", n_bra, lam, alw, keys[st:st + 1], logG, Es)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    torch.cuda.synchronize()
    clocks = summarize_clocks(sampler.stop())
    t = float(np.sum(ms)) / 1e3
    value = n * args.steps / t
    ref = FIG3_H200.get(n)
    # per step: evolve + the one-launch resampling when every 1024-walker tile
    # fits on the GPU at once (2 per SM), else evolve + three resampling
    # launches + the series reduction
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    per_step = 2 if (n + 1023) // 1024 <= 2 * sms else 5
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1,
            "gpu_launches": per_step * args.steps,
            "steps": args.steps, "warmup": wk, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (value / ref) if ref else None,   # the published 1-H200 number
            "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
            "config": {"workload": "heisenberg_chain100_noguide_single_step_nbra6_lam25",
                       "n_walkers": n, "precision": args.precision, "init": "neel",
                       "l2": "flushed (256 MB write) before every timed step"},
            "published_h200_walker_steps_per_s": ref,
            "vs_published_h200": (value / ref) if ref else None,
            "clocks": clocks}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0)
        g = O.no_guide()
        c = np.tile(neel, (args.cpu_sample, 1))
        lw = np.zeros(len(c)); el = np.zeros(len(c))
        k = np.asarray(P.PRNGKey(7), np.uint32)
        times = []
        while sum(times) < 10.0 and len(times) < 1000:
            k, r = O.split(k, 2)
            k1, k2 = O.fold_in(r, 0), O.fold_in(r, 1)
            t0 = time.perf_counter()
            O.evolve(m, g, "single_step", n_bra, lam, alw, k1, c, lw, el)
            O.reconfigure(k2, c, lw, el)
            times.append(time.perf_counter() - t0)
        line["cpu_baseline"] = {"value": len(c) * len(times) / sum(times), "unit": "walker-steps/s",
                                "cores": O.lib().om_threads(), "kind": "port",
                                "sample": f"{args.cpu_sample} walkers x {len(times)} steps "
                                          f"({sum(times):.1f} s), C+OpenMP restatement of the "
                                          "reference"}
    print(json.dumps(line))


def measure_mlp(P, hid, n, steps, warmup):
    """The MLP-guided branching step on the 64-site Bose-Hubbard ring (float32
    build, L2 flushed before each timed step) and one training step
    (gfmc_mlp_train_step): a dict of times and rates, with the second-layer
    MMA work over the whole step against the bf16 peak."""
    import torch
    e, H, GJ = bose_chain(P)
    G = P.MLPBoseHubbard(64, 4, hidden=(hid, hid), seed=0, sigma=0.01)
    w = P.prepare_walkers_occupations(n, 64, 64, 4, P.PRNGKey(0))
    tau = 0.02
    eng = P.GFMCEngine(H, G, n, precision="mixed")
    eng.load(w.config)
    alw = float((-eng.local_energy()).mean().item())
    ms, hpw = timed_steps(P, eng, alw, tau, steps, warmup, P.PRNGKey(1000))
    train_ms = None
    if hid % 64 == 0:
        stream = torch.cuda.current_stream()
        eng.mlp_train_step(1e-4)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.mlp_train_step(1e-4)
        b.record(stream)
        b.synchronize()
        train_ms = a.elapsed_time(b)
    del eng
    torch.cuda.synchronize()
    # tiles of 128 moves per walker-step: one rate evaluation per hop and one
    # for the final hold (M - 1 = 128 moves); the walker's own amplitude is
    # carried (its tile on the steps that rebuild the carried state, every
    # 50th, is not counted)
    tflops = 2.0 * 128 * hid * hid * n * (1.0 + hpw) / (ms / 1e3) / 1e12
    pk, pk_kind = peaks()
    return {"workload": f"bose_hubbard_ring64_mlp_{hid}x{hid}_cont_time", "n_walkers": n,
            "tau": tau, "value": n / (ms / 1e3), "unit": "walker-steps/s", "ms_per_step": ms,
            "steps": steps, "hops_per_walker_step": hpw, "train_step_ms": train_ms,
            "mma": {"kernel": "mlp_evolve_kernel", "tflops": tflops, "peak_tflops": pk["bf16_tflops"],
                    "peak_source": pk_kind, "frac": tflops / pk["bf16_tflops"]},
            "_jastrow": GJ, "_H": H, "_w": w}


def mlp_bench(P, args):
    """Learned-guide workload for bosons: the 64-site Bose-Hubbard ring with
    64 bosons (n_max = 4, t = 1, U = 3; M = 129), dense MLP guide
    320 -> 256 -> 256 -> 1 (tanh, bf16 weights N(0, 0.01^2)), float32 build,
    32768 walkers drawn uniformly with sum n = 64, cont_time tau = 0.02.
    Times the MLP-guided branching step, one training step
    (gfmc_mlp_train_step) and, beside them, the same branching step under the
    Gutzwiller + density-Jastrow guide (float64 and float32 builds)."""
    hid = min(args.hidden, 256)
    n = args.walkers
    wk = max(args.warmup, 3)
    r = measure_mlp(P, hid, n, args.steps, wk)
    plain = {}
    for prec in ("fp64", "mixed"):
        eng = P.GFMCEngine(r["_H"], r["_jastrow"], n, precision=prec)
        eng.load(r["_w"].config)
        alw = float((-eng.local_energy()).mean().item())
        ms, _ = timed_steps(P, eng, alw, 0.02, args.steps, wk, P.PRNGKey(1000))
        plain[prec] = {"value": n / (ms / 1e3), "ms_per_step": ms}
        del eng
    m = r["mma"]
    line = {"metric": "walker-steps/s", "value": r["value"], "unit": "walker-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": wk, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
            "data": "synthetic",
            "config": {"workload": r["workload"], "n_walkers": n,
                       "tau": 0.02, "l2": "flushed (256 MB write) before every timed step",
                       "hops_per_walker_step": r["hops_per_walker_step"]},
            "train_step_ms": r["train_step_ms"],
            "jastrow_fp64": plain["fp64"], "jastrow_mixed": plain["mixed"],
            "roofline": {"bound": "tensor", "kernel": "mlp_evolve_kernel", "achieved": m["tflops"],
                         "peak": m["peak_tflops"], "unit": "TFLOP/s", "frac": m["frac"],
                         "traffic": None, "peak_source": m["peak_source"],
                         "note": "second-layer MMA flops (128 x H x H per tile) over the whole step; "
                                 "the step is bound by the first-layer rows and tanh on the CUDA "
                                 "cores (see profiles/)"}}
    print(json.dumps(line))


def measure_plain(P, H, G, w, tau, precision, steps, warmup, workload):
    """A plain (Jastrow-guided) branching step of population w."""
    eng = P.GFMCEngine(H, G, len(w.config), precision=precision)
    eng.load(w.config)
    alw = float((-eng.local_energy()).mean().item())
    ms, hpw = timed_steps(P, eng, alw, tau, steps, warmup, P.PRNGKey(1000))
    n = eng.n
    del eng
    return {"workload": workload, "precision": precision, "n_walkers": n, "tau": tau,
            "value": n / (ms / 1e3), "unit": "walker-steps/s", "ms_per_step": ms, "steps": steps,
            "hops_per_walker_step": hpw}


def secondary_measurements(P, steps_scale=1.0):
    """The other workloads' steps, each timed like the headline (W >= 3
    warm-up steps, CUDA events per step on the launching stream, L2 flushed
    by a 256 MB write before every timed step, clocks sampled throughout):
    the 16x16 long-range Jastrow step in the mixed build, the RBM step on
    16x16 (H = 512, 65536 walkers) with its training step and theta GEMM,
    the MLP step on the 64-site Bose ring (320-256-256-1, 32768 walkers) with
    its training step, the Gutzwiller + density-Jastrow step on that ring,
    the kagome nearest-neighbour step (432 sites, 131072 walkers) and the
    100-site chain (1024 walkers); then the short sigma study
    (sigma_short)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    sampler = ClockSampler(gpu_uuid(torch, dev)).start()
    k = lambda x: max(3, int(x * steps_scale))   # noqa: E731
    out = {}
    lat, H, G, _, _ = build_system(P, "mixed")
    w = P.prepare_walkers_sz(N_WALKERS, L * L, P.PRNGKey(0), sz=0)
    out["c1_square16_longrange_mixed"] = measure_plain(
        P, H, G, w, TAU, "mixed", k(200), 5, "heisenberg_16x16_longrange_jastrow_cont_time")
    r = measure_rbm(P, "square16", 512, 65536, k(12), 3)
    out["c2_square16_rbm_h512_mixed"] = {a: b for a, b in r.items() if not a.startswith("_")}
    r = measure_mlp(P, 256, N_WALKERS, k(30), 3)
    out["c3_bose_ring64_mlp_256_mixed"] = {a: b for a, b in r.items() if not a.startswith("_")}
    out["c3_bose_ring64_jastrow_fp64"] = measure_plain(
        P, r["_H"], r["_jastrow"], r["_w"], 0.02, "fp64", k(100), 5,
        "bose_hubbard_ring64_gutzwiller_density_jastrow_cont_time")
    kg = P.kagome(12, 12)
    Hk = P.SpinHalf.create(kg.edges, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    Gk = P.JastrowSpinHalf(kg.N, kg.edges, beta=0.3)
    out["c4_kagome12_nn_jastrow_fp64"] = measure_plain(
        P, Hk, Gk, P.prepare_walkers_sz(131072, kg.N, P.PRNGKey(0), sz=0), 0.02, "fp64", k(40), 4,
        "kagome_12x12_xxz_nn_jastrow_cont_time")
    ec = P.chain(100).edges
    Hc = P.SpinHalf.create(ec, J_x=-1.0, J_y=-1.0, J_z=1.0, dtype=np.float64)
    Gc = P.JastrowSpinHalf(100, ec, beta=0.3)
    out["c0_chain100_nn_jastrow_fp64"] = measure_plain(
        P, Hc, Gc, P.prepare_walkers_sz(1024, 100, P.PRNGKey(0), sz=0), 0.2, "fp64", k(200), 5,
        "heisenberg_chain100_nn_jastrow_cont_time")
    torch.cuda.synchronize()
    out["clocks"] = summarize_clocks(sampler.stop())
    out["sigma_short"] = sigma_short(P, steps_scale)
    return out


def sigma_short(P, steps_scale=1.0):
    """A short version of the sigma study (--study sigma) on the 16x16
    Heisenberg lattice: an RBM (H = 512) trained by variance minimisation for
    150 iterations on 32768 walkers, then fixed-length productions of the
    trained RBM (float32 build, 1000 steps) and of the long-range Jastrow
    guide (float64 build, 5000 steps), 32768 walkers each, tau = 0.05,
    blocked jackknife (10 blocks, each at least three times the p = 32
    window) at p = 32; GPU seconds to sigma(E/N) = 1e-5
    = production time x (sigma / 1e-5)^2.  Short runs: the ratio is an
    estimate (the full study trains for 600 iterations and runs longer)."""
    import torch
    lat, H, GJ, _, _ = build_system(P, "fp64")
    n = N_WALKERS
    trained, hist = P.learn.train_rbm_guide(
        P.prepare_walkers_sz(n, 256, P.PRNGKey(13), sz=0), H, P.RBMSpinHalf(256, 512, seed=0, sigma=0.01),
        n_iterations=max(10, int(150 * steps_scale)), steps_per_iteration=3, step_size=TAU, lr=3e-4,
        rng_key=P.PRNGKey(14), warmup_steps=100, verbosity=0)
    res = {}
    for key, G, steps, prec in (("rbm_h512_mixed", trained, max(40, int(1000 * steps_scale)), "mixed"),
                                ("jastrow_fp64", GJ, max(200, int(5000 * steps_scale)), "fp64")):
        w = P.prepare_walkers_sz(n, 256, P.PRNGKey(11), sz=0)
        torch.cuda.synchronize()
        wf, _, _, st, raw = P.run(w, steps, H, TAU, G, [8, 32], rng_key=P.PRNGKey(12),
                                  warmup_steps=200, verbosity=0, precision=prec)
        Ej, err = P.estimators.jackknife_energy([32], raw["log_weights"], raw["energy"], 10)
        sig = err[32] / 256
        res[key] = {"E_per_site": Ej[32] / 256, "sigma_per_site": sig, "steps": steps,
                    "production_gpu_s": st["runtime"],
                    "gpu_s_to_1e-5": st["runtime"] * (sig / 1e-5) ** 2,
                    "local_energy_var_per_site": float(np.var(wf.e_loc) / 256)}
    r, j = res["rbm_h512_mixed"], res["jastrow_fp64"]
    return {"workload": "heisenberg_16x16_rbm_h512_vs_longrange_jastrow", "n_walkers": n, "tau": TAU,
            "p": 32, "jackknife_blocks": 10, "train_iterations": len(hist["variance"]),
            "train_gpu_s": hist["seconds"], "methods": res,
            "learned_over_jastrow_fp64_time_ratio": r["gpu_s_to_1e-5"] / j["gpu_s_to_1e-5"],
            "energy_difference_in_sigma": abs(r["E_per_site"] - j["E_per_site"])
            / float(np.hypot(r["sigma_per_site"], j["sigma_per_site"]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--walkers", type=int, default=N_WALKERS)
    ap.add_argument("--cpu-sample", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the other workloads' steps (the line's 'secondary' object; N=1 only)")
    ap.add_argument("--study", default=None, choices=["sigma"],
                    help="sigma: GPU seconds to sigma(E/N)=1e-5, RBM vs Jastrow (minutes)")
    ap.add_argument("--study-steps", type=int, default=4000)
    ap.add_argument("--rbm-steps", type=int, default=1000,
                    help="--study sigma: production steps of the learned guide")
    ap.add_argument("--train-iters", type=int, default=600)
    ap.add_argument("--train-lr", type=float, default=3e-4)
    ap.add_argument("--guide", default="jastrow", choices=["jastrow", "rbm", "mlp"],
                    help="rbm: the learned-guide workload (RBM, float32); mlp: the Bose-Hubbard "
                         "ring with the dense MLP guide")
    ap.add_argument("--hidden", type=int, default=None,
                    help="hidden units of the learned guide (default: the workload's)")
    ap.add_argument("--workload", default="headline", choices=["headline", "fig3"],
                    help="fig3: the reference's published throughput workload (Heisenberg chain "
                         "L = 100, no guide, single_step n_bra = 6, lam = 25; --walkers, "
                         "--precision)")
    ap.add_argument("--lattice", default="square16", choices=["square16", "kagome12", "bose64"],
                    help="--guide rbm / --study sigma: the 16x16 Heisenberg, the 432-site kagome "
                         "XXZ workload, or (--study sigma) the 64-site Bose-Hubbard ring with the "
                         "MLP guide")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    import pygfmc_b200 as P

    if args.study == "sigma":
        if rank == 0:
            sigma_study(P, args)
        return
    if args.workload == "fig3":
        if rank == 0:
            fig3_bench(P, args)
        return
    args.hidden_set = args.hidden is not None
    args.walkers_set = args.walkers != N_WALKERS
    if args.hidden is None:
        args.hidden = 256 if args.guide == "mlp" else 512
    if args.guide == "rbm" and args.lattice == "bose64":
        ap.error("--guide rbm runs on --lattice square16 or kagome12")
    if args.guide == "rbm":
        if rank == 0:
            rbm_bench(P, args)
        return
    if args.guide == "mlp":
        if rank == 0:
            mlp_bench(P, args)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        w = P.prepare_walkers_sz(args.cpu_sample, L * L, P.PRNGKey(0), sz=0)
        # alw: minus the mean local energy of the sample (what the warm-up starts from)
        lat, H, G, pairs, beta = build_system(P, "fp64")
        from oracle import oracle as O
        O.build()
        m = O.spin_half(lat.edges, J_x=-1.0, J_y=-1.0, J_z=1.0)
        g = O.jastrow_spin_half(lat.N, pairs, beta, None, m)
        alw = O.initial_alw(m, g, "cont_time", None, w.config)
        steps = max(1, args.steps)
        # the fresh sample first relaxes to the equilibrated population the
        # GPU arm times (8.3 hops per walker-step fresh, 6.8-6.9 after ~100
        # steps on this workload), untimed, then the run's W warm-up steps
        val, threads, secs, _ = cpu_reference(P, w.config, alw, steps,
                                              REF_EQUILIBRATION_STEPS + args.warmup, P.PRNGKey(7))
        line = {"metric": "walker-steps/s", "value": val, "unit": "walker-steps/s", "n_gpus": 0,
                "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": "heisenberg_16x16_longrange_jastrow_cont_time",
                           "n_walkers_sample": args.cpu_sample, "tau": TAU},
                "cpu_baseline": {"value": val, "unit": "walker-steps/s", "cores": threads,
                                 "kind": "port",
                                 "sample": f"{args.cpu_sample} walkers x {steps} steps of the "
                                           f"headline workload after {REF_EQUILIBRATION_STEPS} "
                                           "untimed equilibration steps (PyGFMC is JAX-based "
                                           "and not runnable here; C restatement of its "
                                           "algorithm)"},
                "e2e": {"value": val, "unit": "walker-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    lat, H, G, pairs, beta = build_system(P, args.precision)
    n = args.walkers
    w = P.prepare_walkers_sz(n, L * L, P.PRNGKey(rank), sz=0)
    eng = P.GFMCEngine(H, G, n, precision=args.precision)
    eng.load(w.config)
    e0 = eng.local_energy()
    alw = float((-e0).mean().item())
    stream = torch.cuda.current_stream()
    # log G and E_n of a step side by side: the e2e leg reads both in one copy
    lgE = torch.empty(2, dtype=torch.float64, device=dev)
    logG, Es = lgE[0:1], lgE[1:2]
    key = P.PRNGKey(1000 + rank)
    # warm-up: equilibrate (also refines alw)
    wk = max(args.warmup, 3)
    keys, key = P.engine.key_schedule(key, wk)
    lgw = torch.empty(wk, dtype=torch.float64, device=dev)
    Ew = torch.empty(wk, dtype=torch.float64, device=dev)
    eng.steps("cont_time", TAU, None, alw, keys, lgw, Ew)
    torch.cuda.synchronize()
    alw = alw + float(torch.logsumexp(lgw, 0).item() - np.log(wk)) / TAU
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    hops = torch.zeros(1, dtype=torch.int64, device=dev)
    keys, key = P.engine.key_schedule(key, args.steps)

    sampler = ClockSampler(gpu_uuid(torch, dev)).start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms = []
    evolve_ms = []
    total_hops = 0
    for s in range(args.steps):
        flush.fill_(float(s))
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.steps("cont_time", TAU, None, alw, keys[s:s + 1], logG, Es, hops)
        b.record(stream)
        b.synchronize()
        step_ms.append(a.elapsed_time(b))
        total_hops += int(hops.item())
    torch.cuda.synchronize()
    clock_lines = sampler.stop()
    if world > 1:
        torch.distributed.barrier()
    t_step = float(np.sum(step_ms)) / 1e3
    if world > 1:
        t = torch.tensor([t_step], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_step = float(t.item())
    value = n * args.steps * world / t_step
    ms_per_step = 1e3 * t_step / args.steps

    # ---- e2e: host-resident walkers through the C ABI, every step
    import ctypes
    packed_h = torch.empty(n * eng.cfg_bytes, dtype=torch.uint8, pin_memory=True)
    packed_h.copy_(eng.cfg)
    out_h = torch.empty(2, dtype=torch.float64, pin_memory=True)
    e2e_steps = max(1, min(args.steps, 50))
    e2e_warm = 3
    keys2, key = P.engine.key_schedule(key, e2e_steps + e2e_warm)
    null = ctypes.c_void_p(0)
    torch.cuda.synchronize()
    for s in range(e2e_steps + e2e_warm):
        if s == e2e_warm:
            t0 = time.perf_counter()
        # the host population in, one step (evolve + resampling), the resampled
        # population (configurations gathered through the parents) and
        # log G, E out
        eng.cfg.copy_(packed_h, non_blocking=True)
        eng.parents_valid = 0
        eng.steps("cont_time", TAU, None, alw, keys2[s:s + 1], logG, Es)
        P._lib.check(eng.L.gfmc_gather(eng.h, n, eng._ptr(eng.parents), eng._ptr(eng.cfg),
                                       eng._ptr(eng.cfg_tmp), null, null, null, eng._stream()),
                     "gfmc_gather")
        packed_h.copy_(eng.cfg_tmp, non_blocking=True)
        out_h.copy_(lgE, non_blocking=True)
        stream.synchronize()
    t_e2e = time.perf_counter() - t0
    if world > 1:
        te = torch.tensor([t_e2e], device=dev)
        torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
        t_e2e = float(te.item())
    e2e_val = n * e2e_steps / t_e2e * world

    pk, pk_kind = peaks()
    clocks = summarize_clocks(clock_lines)
    C = eng.cfg_bytes
    # evolve (gather fused) + reconfiguration, the carried guide fields (N
    # values per walker, read through the parent map and written back) and
    # the carried evaluation record (68 values per walker, the same way)
    tsz = 8 if args.precision == "fp64" else 4
    fbytes = 2 * (L * L) * tsz + 2 * 68 * tsz
    alg_bytes = 4 + 2 * C + 16 + (2 * C + 36) + fbytes
    achieved_gbs = alg_bytes * n / (ms_per_step / 1e3) / 1e9
    line = {
        "metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": wk, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": "heisenberg_16x16_longrange_jastrow_cont_time", "n_walkers": n,
                   "n_sites": 256, "n_bonds": 512, "jastrow_pairs": int(len(pairs)), "tau": TAU,
                   "precision": args.precision, "l2": "flushed (256 MB write) before every timed step",
                   "hops_per_walker_step": total_hops / (n * args.steps),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_val, "unit": "walker-steps/s", "h2d_bytes_per_step": n * C,
                "d2h_bytes_per_step": n * C + 16},
        # per step: evolve and the one-launch resampling (which also sums the
        # step's E_n); plus the population guide-state product on each
        # refresh of the carried state (every 100 steps in float64, 50 in
        # float32)
        "gpu_launches": 2 * args.steps + args.steps // (100 if args.precision == "fp64" else 50),
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved_gbs / pk["hbm_gbs"],
                     "traffic": EVOLVE_TRAFFIC_BYTES.get((args.precision, n)),
                     "algorithmic_bytes_per_launch": alg_bytes * n,
                     "peak_source": pk_kind,
                     "note": f"algorithmic bytes per walker-step {alg_bytes} (packed configs "
                             "in/out, parent index, weights, resampling, carried guide fields "
                             "and evaluation record in/out); the step is compute-bound "
                             "(guide-ratio arithmetic over 512 bonds per rate evaluation), "
                             "see profiles/"},
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        cfg_d, _ = eng.population()
        sample = cfg_d[: args.cpu_sample].cpu().numpy()
        val, threads, secs, nst = cpu_reference(P, sample, alw, 2, 0, P.PRNGKey(7), min_seconds=10.0)
        line["cpu_baseline"] = {"value": val, "unit": "walker-steps/s", "cores": threads,
                                "kind": "port",
                                "sample": f"{args.cpu_sample} equilibrated walkers x {nst} steps "
                                          f"({secs:.1f} s), C+OpenMP restatement of the reference"}
    if world == 1 and not args.no_secondary:
        del eng
        torch.cuda.synchronize()
        line["secondary"] = secondary_measurements(P)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()

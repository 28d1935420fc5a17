"""Extract the golden fixtures this repository's tests pin against.

Source: PyGFMC's own golden-output file
``tests/core/reference_data/golden_cpu.npz`` (jax 0.9.2, CPU, float64), which
its ``tests/core/test_golden_outputs.py`` writes and checks.  Only the cases
of the hot path are kept (SpinHalf and BoseHubbard, without a guide and with
their Jastrow guides, for the three propagators), plus the Threefry key chain
of every case.  Run from the repository root with the path of PyGFMC's file:

    python tests/golden/make_golden.py <PyGFMC>/tests/core/reference_data/golden_cpu.npz

Writes ``tests/golden/golden_subset.npz``.
"""
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_subset.npz")

CASES = [f"{sys_}_{g}_{m}" for sys_ in ("spinhalf", "bose") for g in ("none", "jastrow")
         for m in ("cont_time", "single_step", "multi_step")]
KEEP = ("config", "log_weight", "e_loc", "energy/", "obs/", "raw/log_weights", "raw/energy",
        "raw/diag/", "raw/off_diag/", "raw/off_diag_norm/", "raw/additional_diag/",
        "stats/avg_log_weight", "stats/parameters/rng_key", "stats/parameters/rng_key_next",
        "stats/parameters/n_steps", "stats/parameters/warmup_steps",
        "stats/parameters/step_size", "stats/parameters/lam",
        "stats/hops_per_step_mean", "stats/offspring_k0")


def main(src):
    g = np.load(src, allow_pickle=False)
    out = {"__jax_version__": g["__jax_version__"]}
    for k in g.files:
        case, _, rest = k.partition("/")
        if case in CASES and any(rest == p or (p.endswith("/") and rest.startswith(p))
                                 for p in KEEP):
            a = g[k]
            if rest == "config":
                a = a.astype(np.int8)          # +-1 spins / small occupations, lossless
            out[k] = a
        elif rest in ("stats/parameters/rng_key", "stats/parameters/rng_key_next",
                      "stats/parameters/n_steps"):
            out[k] = g[k]                       # key-chain KATs of every case
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <PyGFMC>/tests/core/reference_data/golden_cpu.npz")
    main(sys.argv[1])

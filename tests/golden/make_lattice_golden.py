"""Write the lattice fixtures this repository's tests pin against.

Source: PyGFMC's ``codes/pygfmc/hamiltonian/lattice.py``, which needs only
numpy and is loaded on its own from the given path (without importing the
pygfmc package, which needs jax).  For each case the fixture holds the edge
list (sorted (i < j) pairs, the order that fixes the transition slots of a
Hamiltonian built on it), the site positions and, for kagome, the hexagonal
loops with their centres.  Run from the repository
root with the path of PyGFMC's file:

    python tests/golden/make_lattice_golden.py <PyGFMC>/codes/pygfmc/hamiltonian/lattice.py

Writes ``tests/golden/lattices.npz``.
"""
import importlib.util
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lattices.npz")

# (name, builder, arguments, periodic)
CASES = [("pyrochlore_2x2x2", "pyrochlore", (2, 2, 2), True),
         ("pyrochlore_3x2x4", "pyrochlore", (3, 2, 4), True),
         ("pyrochlore_4x4x4", "pyrochlore", (4, 4, 4), True),
         ("pyrochlore_2x3x2_open", "pyrochlore", (2, 3, 2), False),
         ("pyrochlore_1x1x1_open", "pyrochlore", (1, 1, 1), False),
         ("kagome_12x12", "kagome", (12, 12), True),
         ("kagome_3x2_open", "kagome", (3, 2), False),
         ("chain_100", "chain", (100,), True),
         ("chain_7_open", "chain", (7,), False)]


def main(src):
    spec = importlib.util.spec_from_file_location("pygfmc_lattice", src)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod           # dataclasses look their module up here
    spec.loader.exec_module(mod)
    out = {}
    for name, fn, args, periodic in CASES:
        lat = getattr(mod, fn)(*args, periodic=periodic)
        out[f"{name}/N"] = np.asarray(lat.N, dtype=np.int64)
        out[f"{name}/edges"] = np.asarray(lat.edges, dtype=np.int32).reshape(-1, 2)
        pos = lat.extras.get("positions") if lat.extras else None
        if pos is not None:
            out[f"{name}/positions"] = np.asarray(pos, dtype=np.float64)
        if fn == "kagome":                  # the hexagonal loops, one per cell
            out[f"{name}/hexagons"] = np.asarray(lat.extras["hexagons"], dtype=np.int32).reshape(-1, 6)
            out[f"{name}/hexagon_centers"] = np.asarray(lat.extras["hexagon_centers"],
                                                        dtype=np.float64).reshape(-1, 2)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(CASES)} lattices")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])

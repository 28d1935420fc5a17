"""Oracle guides built from an engine guide's stored parameters.

A Jastrow guide keeps its couplings rounded to its dtype (float32 unless
given otherwise), as PyGFMC's does; the oracle is handed those stored values,
widened exactly to float64, so that both sides run the same guide."""
import numpy as np


def oracle_guide(O, G, m):
    """The oracle restatement of guide G (JastrowSpinHalf or
    JastrowBoseHubbard, PyGFMC's attribute set) for oracle model m."""
    if hasattr(G, "site_other"):
        a = np.asarray(G._pair_site, np.int64)
        b = np.asarray(G.site_other)[a, np.asarray(G._pair_slot, np.int64)]
        h = None if G._h is None else np.asarray(G.h, np.float64)
        return O.jastrow_spin_half(int(G.N), np.stack([a, b], axis=1),
                                   np.asarray(G.beta, np.float64), h, m)
    pairs = np.stack([np.asarray(G.pair_i), np.asarray(G.pair_j)], axis=1)

    def form(v):
        if v is None:
            return None
        return float(np.asarray(v)) if np.ndim(v) == 0 else np.asarray(v, np.float64)
    return O.jastrow_bose_hubbard(int(G.N), pairs, form(G._beta), m, h=form(G._h), d=form(G._d))

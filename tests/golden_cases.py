"""The golden-file systems of PyGFMC's tests/core/test_golden_outputs.py
(_spinhalf:196-216, _bose:233-245), built for the oracle and for the engine."""
import numpy as np

CASES = [f"{s}_{g}_{m}" for s in ("spinhalf", "bose") for g in ("none", "jastrow")
         for m in ("cont_time", "single_step", "multi_step")]


def oracle_system(O, name):
    if name.startswith("spinhalf"):
        e = O.chain_edges(8)
        m = O.spin_half(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5)
        cfg = O.prepare_walkers_random(64, 8, O.case_key("spinhalf walkers"))
        g = O.jastrow_spin_half(8, e, 0.3, 0.05, m) if "_jastrow_" in name else O.no_guide()
        return m, cfg, g, 0.2, 4.0
    e = O.chain_edges(6)
    m = O.bose_hubbard(e, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2)
    cfg = O.prepare_walkers_sz(64, 6, O.case_key("bose walkers"), sz=6, states=(0.0, 1.0, 2.0))
    g = O.jastrow_bose_hubbard(6, e, 0.05, m, h=0.1, d=0.3) if "_jastrow_" in name else O.no_guide()
    return m, cfg, g, 0.1, 20.0


def engine_system(P, name):
    if name.startswith("spinhalf"):
        e = P.chain(8).edges
        H = P.SpinHalf.create(e, J_x=-1.0, J_y=-1.0, J_z=1.0, h_x=0.5, dtype=np.float64)
        w = P.prepare_walkers_random(64, 8, P.random.PRNGKey(_crc("spinhalf walkers")))
        g = P.JastrowSpinHalf(8, e, beta=0.3, h=0.05, dtype=np.float64) if "_jastrow_" in name else None
        return H, w, g, 0.2, 4.0
    e = P.chain(6).edges
    H = P.BoseHubbard.create(e, t=1.0, eta=0.3, U=2.0, mu=0.5, h_pm=0.2, n_max=2, dtype=np.float64)
    w = P.prepare_walkers_sz(64, 6, P.random.PRNGKey(_crc("bose walkers")), sz=6,
                             states=(0.0, 1.0, 2.0))
    g = (P.JastrowBoseHubbard(6, e, beta=0.05, h=0.1, d=0.3, dtype=np.float64)
         if "_jastrow_" in name else None)
    return H, w, g, 0.1, 20.0


def engine_diag_ops(P, name):
    """The diagonal operators of the golden systems (test_golden_outputs.py
    _spinhalf:196-216, _bose:233-245)."""
    if name.startswith("spinhalf"):
        e = P.chain(8).edges
        pos = np.arange(8, dtype=float)[:, None]
        ks = (2 * np.pi * np.arange(3) / 8)[:, None]
        return {"zz": P.SpinHalf.create(e, J_z=1.0, dtype=np.float64),
                "sf": P.hamiltonian.SzSzStructureFactor(pos, ks, dtype=np.float64)}
    return {"nn": P.BoseHubbard.create(P.chain(6).edges, U=2.0, n_max=2, dtype=np.float64)}


def oracle_off_ops(O, name):
    """The off-diagonal operators of the golden systems as oracle models, each
    with the case's guide built against the operator (guide.build_cache(op)):
    [(name, op_model, op_guide)] (test_golden_outputs.py:180-193, 206-209,
    236-237)."""
    jas = "_jastrow_" in name
    if name.startswith("spinhalf"):
        e = O.chain_edges(8)
        W = 1.0 + np.cos(np.ones(len(e)) * np.pi / 2)
        ops = [("spsm", O.spin_half(e, J_x=2.0, J_y=2.0, J_z=0.0)),
               ("sx", O.spin_half(e, h_x=-1.0)),
               ("sfx", O.spin_half(e, J_x=4.0 * W, J_y=0.0 * W, J_z=0.0, N=8))]
        return [(nm, m, O.jastrow_spin_half(8, e, 0.3, 0.05, m) if jas else O.no_guide())
                for nm, m in ops]
    e = O.chain_edges(6)
    ops = [("hop", O.bose_hubbard(e, t=-1.0, n_max=2)),
           ("pair", O.bose_hubbard(e, eta=-0.3, n_max=2))]
    return [(nm, m, O.jastrow_bose_hubbard(6, e, 0.05, m, h=0.1, d=0.3) if jas else O.no_guide())
            for nm, m in ops]


def engine_off_ops(P, name):
    """The off-diagonal operators of the golden systems for the engine
    (test_golden_outputs.py:180-193, 206-209, 236-237)."""
    if name.startswith("spinhalf"):
        e = P.chain(8).edges
        W = 1.0 + np.cos(np.ones(len(e)) * np.pi / 2)
        return {"spsm": P.SpinHalf.create(e, J_x=2.0, J_y=2.0, J_z=0.0, sign_check=False,
                                          dtype=np.float64),
                "sx": P.SpinHalf.create(e, h_x=-1.0, sign_check=False, dtype=np.float64),
                "sfx": P.SpinHalf.create(np.asarray(e, dtype=np.int32), J_x=4.0 * W, J_y=0.0 * W,
                                         J_z=0.0, N=8, dtype=np.float64, sign_check=False)}
    e = P.chain(6).edges
    return {"hop": P.BoseHubbard.create(e, t=-1.0, n_max=2, sign_check=False, dtype=np.float64),
            "pair": P.BoseHubbard.create(e, eta=-0.3, n_max=2, sign_check=False, dtype=np.float64)}


def _crc(s):
    import zlib
    return zlib.crc32(s.encode())


def method_of(name):
    for m in ("cont_time", "single_step", "multi_step"):
        if name.endswith(m):
            return m

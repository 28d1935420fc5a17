"""Training the learned guides on the walkers of a GFMC run (no PyGFMC
counterpart; PyGFMC trains its learned guides by NetKet VMC).

``train_rbm_guide`` and ``train_mlp_guide`` alternate GFMC steps under the
current guide with Adam steps on the local-energy variance of the current
population, so the guide is fitted on the mixed distribution the GFMC run
itself samples.  Every step runs on the device: the branching steps in the
guide's step kernel, the loss gradient on the tensor cores
(``gfmc_rbm_train_step``: theta GEMM + fused tanh / tcgen05 contraction;
``gfmc_mlp_train_step``: the second layer forward, its backward and dW2 as
tcgen05 GEMMs, the one-hot first layer by accumulation)."""
import math
import time

import numpy as np

from . import random as _rnd
from .engine import GFMCEngine, _device_status_check, _emit, key_schedule
from .wavefunction import MLPBoseHubbard, RBMSpinHalf

__all__ = ["train_rbm_guide", "train_mlp_guide"]


def train_rbm_guide(walkers, hamiltonian, guide, *, n_iterations=200, steps_per_iteration=5,
                    step_size=0.05, method="cont_time", lam=None, rng_key=None, lr=3e-4,
                    warmup_steps=100, verbosity=1, collapse_tol=0.05, snapshot_every=10):
    """Variance-minimisation training of an ``RBMSpinHalf`` guide.

    Returns ``(trained_guide, history)``: a new ``RBMSpinHalf`` with the
    trained (bf16-valued) parameters, and a dict of per-iteration arrays
    ``energy`` (population mean local energy), ``variance`` (the loss), the
    total ``seconds`` and ``collapsed`` (see below).  The walkers are evolved
    in the float32 build; ``walkers.config`` is the starting population.

    Collapse guard: the population's mean local energy estimates the ground
    energy whatever the guide, so a jump of more than ``collapse_tol`` (relative)
    away from its running mean over the last 20 iterations means the guide has
    switched the moves off (the zero-variance degenerate solution of variance
    minimisation on walkers the guide itself steers).  Training then stops and
    the parameters of the last snapshot (every ``snapshot_every`` iterations)
    are returned."""
    if not isinstance(guide, RBMSpinHalf):
        raise TypeError("train_rbm_guide needs an RBMSpinHalf guide")
    return _train(walkers, hamiltonian, guide, "rbm", n_iterations, steps_per_iteration, step_size,
                  method, lam, rng_key, lr, warmup_steps, verbosity, collapse_tol, snapshot_every)


def train_mlp_guide(walkers, hamiltonian, guide, *, n_iterations=200, steps_per_iteration=5,
                    step_size=0.02, rng_key=None, lr=3e-4, warmup_steps=100, verbosity=1,
                    collapse_tol=0.05, snapshot_every=10):
    """Variance-minimisation training of an ``MLPBoseHubbard`` guide (cont_time,
    float32 build); same protocol, return value and collapse guard as
    ``train_rbm_guide``.  ``mlp_H2`` must be a multiple of 64."""
    if not isinstance(guide, MLPBoseHubbard):
        raise TypeError("train_mlp_guide needs an MLPBoseHubbard guide")
    if guide.H2 % 64:
        raise ValueError(f"train_mlp_guide needs H2 a multiple of 64, got {guide.H2}")
    return _train(walkers, hamiltonian, guide, "mlp", n_iterations, steps_per_iteration, step_size,
                  "cont_time", None, rng_key, lr, warmup_steps, verbosity, collapse_tol,
                  snapshot_every)


def _train(walkers, hamiltonian, guide, kind, n_iterations, steps_per_iteration, step_size, method,
           lam, rng_key, lr, warmup_steps, verbosity, collapse_tol, snapshot_every):
    name = f"train_{kind}_guide"
    n_iterations = int(n_iterations)
    steps_per_iteration = int(steps_per_iteration)
    if n_iterations < 1 or steps_per_iteration < 1:
        raise ValueError("n_iterations and steps_per_iteration must be positive")
    if not lr > 0:
        raise ValueError("lr must be positive")
    if method != "cont_time" and lam is None:
        raise ValueError(f"method={method!r} needs the GFMC shift lam")
    config = np.asarray(walkers.config)
    n = config.shape[0]
    key = _rnd.as_key(rng_key if rng_key is not None else _rnd.PRNGKey(0))
    t0 = time.time()
    eng = GFMCEngine(hamiltonian, guide, n, precision="mixed")
    eng.load(config)
    torch = eng.torch
    e = eng.local_energy().cpu().numpy()
    alw = float(np.mean(-e)) if method == "cont_time" else float(np.mean(np.log(lam - e)))
    lg = torch.empty(max(warmup_steps, steps_per_iteration, 1), dtype=torch.float64,
                     device=eng.device)
    E = torch.empty_like(lg)
    if warmup_steps > 0:
        keys, key = key_schedule(key, warmup_steps)
        eng.steps(method, step_size, lam, alw, keys, lg[:warmup_steps], E[:warmup_steps])
    hist_e, hist_v = [], []
    params = eng.rbm_parameters if kind == "rbm" else eng.mlp_parameters
    train_step = eng.rbm_train_step if kind == "rbm" else eng.mlp_train_step
    snapshot = params()
    collapsed = False
    for it in range(n_iterations):
        keys, key = key_schedule(key, steps_per_iteration)
        eng.steps(method, step_size, lam, alw, keys, lg[:steps_per_iteration],
                  E[:steps_per_iteration])
        em, var = train_step(lr)
        hist_e.append(em)
        hist_v.append(var)
        recent = hist_e[-21:-1]
        if (not (math.isfinite(em) and math.isfinite(var))) or (
                len(recent) >= 20 and abs(em - np.mean(recent)) > collapse_tol * abs(np.mean(recent))):
            collapsed = True
            _emit(f"[learn] - [{name}] - collapse at iteration {it + 1} (E = {em:.6g}); "
                  "returning the last snapshot", verbosity)
            break
        if (it + 1) % snapshot_every == 0:
            snapshot = params()
        if verbosity >= 2 or (verbosity >= 1 and (it % max(1, n_iterations // 10) == 0
                                                  or it == n_iterations - 1)):
            _emit(f"[learn] - [{name}] - iteration {it + 1}/{n_iterations}: "
                  f"E/N = {em / hamiltonian.N:.6f}, var(e_L)/N = {var / hamiltonian.N:.6f}",
                  verbosity)
    _device_status_check(eng)
    final = snapshot if collapsed else params()
    if kind == "rbm":
        W, b, a = final
        trained = RBMSpinHalf(guide.N, guide.n_hidden, W=W, b=b, a=a, dtype=guide.dtype)
    else:
        trained = MLPBoseHubbard(guide.N, guide.n_max, hidden=(guide.H1, guide.H2), W1=final["W1"],
                                 b1=final["b1"], W2=final["W2"], b2=final["b2"], w3=final["w3"],
                                 b3=guide.b3, dtype=guide.dtype)
    torch.cuda.current_stream().synchronize()
    return trained, {"energy": np.asarray(hist_e), "variance": np.asarray(hist_v),
                     "seconds": time.time() - t0, "collapsed": collapsed}

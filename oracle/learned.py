"""CPU oracle of the learned guides -- TEST INFRASTRUCTURE ONLY.

The RBM and MLP guides and their variance-minimisation trainer have no counterpart in
the reference (PyGFMC trains its guides by NetKet VMC), so the checker is a
direct float64 statement of the definitions with torch's CPU autograd for
the derivatives:

  log psi(s) = sum_h log cosh(b_h + sum_i W_hi s_i) + a . s
  e_L(x)     = H_xx + sum_s c_s(x) psi(x'_s) / psi(x)
  L          = sum_w omega_w (e_L(x_w) - E)^2 / sum_w omega_w

over every walker's connected configurations x'_s (the SpinHalf slots: site
flips, then edges; the BoseHubbard moves: hops, pair terms, b+ / b-; with
their couplings c_s(x) before the guide).  The MLP guide,

  log psi(x) = w3 . tanh(W2 bf16(tanh(W1 onehot(x) + b1)) + b2) + b3,

passes its bf16 rounding straight through the derivative.  Only tests use
it.
"""
import numpy as np
import torch


def _slots(model, x):
    """Couplings (n, n_off) and flipped configurations (n, n_off, N) of the
    SpinHalf slots of the configurations x (n, N) (hamiltonian/SpinHalf.py
    get_rates:316-369 without the guide), and the diagonal (n,)."""
    x = np.asarray(x, dtype=np.float64)
    n, N = x.shape
    ei = np.asarray(model.edge_i, dtype=np.int64)
    ej = np.asarray(model.edge_j, dtype=np.int64)
    E = len(ei)
    coup, succ = [], []
    if model.n_hx_static:
        hx = np.broadcast_to(np.asarray(model.h_x_half, np.float64), (N,))
        for k in range(N):
            y = x.copy(); y[:, k] = -y[:, k]
            coup.append(np.full(n, hx[k])); succ.append(y)
    if model.n_jpm_static:
        jpm = np.broadcast_to(np.asarray(model.J_pm, np.float64), (E,))
        jpp = np.broadcast_to(np.asarray(model.J_pmpm, np.float64), (E,))
        for e in range(E):
            anti = x[:, ei[e]] != x[:, ej[e]]
            y = x.copy(); y[:, ei[e]] = -y[:, ei[e]]; y[:, ej[e]] = -y[:, ej[e]]
            coup.append(np.where(anti, jpm[e], jpp[e])); succ.append(y)
    diag = np.asarray(model.diagonal_weight(x), dtype=np.float64)
    return np.stack(coup, 1), np.stack(succ, 1), diag


def variance_loss_and_grads(model, W, b, a, x, omega=None):
    """(E, L, dL/dW, dL/db, dL/da) in float64 for RBM parameters (W, b, a) on
    the configurations x (n, N)."""
    c, xs, diag = _slots(model, x)
    Wt = torch.tensor(np.asarray(W, np.float64), requires_grad=True)
    bt = torch.tensor(np.asarray(b, np.float64), requires_grad=True)
    at = torch.tensor(np.asarray(a, np.float64), requires_grad=True)

    def logpsi(s):
        th = s @ Wt.T + bt
        return (torch.abs(th) + torch.log1p(torch.exp(-2.0 * torch.abs(th))) - np.log(2.0)).sum(-1) \
            + s @ at

    X = torch.tensor(np.asarray(x, np.float64))
    XS = torch.tensor(xs)
    C = torch.tensor(c)
    lp = logpsi(X)
    lps = logpsi(XS)
    e = torch.tensor(diag) + (C * torch.exp(lps - lp[:, None])).sum(1)
    om = torch.ones_like(e) if omega is None else torch.tensor(np.asarray(omega, np.float64))
    Em = (om * e).sum() / om.sum()
    L = (om * (e - Em) ** 2).sum() / om.sum()
    L.backward()
    Em, L = Em.detach(), L.detach()
    return (Em.item(), L.item(), Wt.grad.numpy().copy(), bt.grad.numpy().copy(),
            at.grad.numpy().copy())


def _bose_moves(model, x):
    """Couplings (n, n_off), successor occupations (n, n_off, N) (clipped to
    [0, n_max] where a move has no element) and the diagonal (n,) of the
    BoseHubbard moves (hamiltonian/bose_hubbard.py get_rates:285-393)."""
    x = np.asarray(x, dtype=np.float64)
    a, b, da, db = model.moves()
    coup = np.stack([model.get_rates(xi)[0] for xi in x])
    succ = np.repeat(x[:, None, :], len(a), axis=1)
    k = np.arange(len(a))
    succ[:, k, a] += da
    succ[:, k, b] += db
    succ = np.clip(succ, 0, model.n_max)
    return coup[:, 1:], succ[:, 1:], coup[:, 0]


def mlp_variance_loss_and_grads(model, W1, b1, W2, b2, w3, b3, x, omega=None, round_h1=True):
    """(E, L, grads) in float64 for MLP parameters on the occupations x (n, N);
    grads is a dict W1, b1, W2, b2, w3.  round_h1=False drops the bf16
    rounding of the first layer (the loss is then smooth, for finite
    differences)."""
    c, xs, diag = _bose_moves(model, x)
    N, nm = int(model.N), int(model.n_max)
    T = {k: torch.tensor(np.asarray(v, np.float64), requires_grad=True)
         for k, v in (("W1", W1), ("b1", b1), ("W2", W2), ("b2", b2), ("w3", w3))}

    def logpsi(nconf):
        nconf = np.asarray(nconf, np.int64)
        onehot = np.zeros(nconf.shape[:-1] + (N * (nm + 1),))
        np.put_along_axis(onehot, np.arange(N) * (nm + 1) + nconf, 1.0, axis=-1)
        z1 = torch.tensor(onehot) @ T["W1"].T + T["b1"]
        h1 = torch.tanh(z1)
        if not round_h1:
            h1b = h1
        else:
            h1r = h1.detach().float().bfloat16().double()
            h1b = h1 + (h1r - h1).detach()
        h2 = torch.tanh(h1b @ T["W2"].T + T["b2"])
        return h2 @ T["w3"] + float(b3)

    lp = logpsi(x)
    lps = logpsi(xs)
    C = torch.tensor(c)
    e = torch.tensor(diag) + (C * torch.exp(lps - lp[:, None])).sum(1)
    om = torch.ones_like(e) if omega is None else torch.tensor(np.asarray(omega, np.float64))
    Em = (om * e).sum() / om.sum()
    L = (om * (e - Em) ** 2).sum() / om.sum()
    L.backward()
    return (Em.item(), L.item(), {k: v.grad.numpy().copy() for k, v in T.items()})

"""CPU oracle of the learned guide -- TEST INFRASTRUCTURE ONLY.

The RBM guide and its variance-minimisation trainer have no counterpart in
the reference (PyGFMC trains its guides by NetKet VMC), so the checker is a
direct float64 statement of the definitions with torch's CPU autograd for
the derivatives:

  log psi(s) = sum_h log cosh(b_h + sum_i W_hi s_i) + a . s
  e_L(x)     = H_xx + sum_s c_s(x) psi(x'_s) / psi(x)
  L          = sum_w omega_w (e_L(x_w) - E)^2 / sum_w omega_w

over every walker's connected configurations x'_s (the SpinHalf slots: site
flips, then edges, with their couplings c_s(x) before the guide).  Only
tests use it.
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

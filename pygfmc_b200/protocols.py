"""The interfaces of a Hamiltonian, a measurement operator and a guiding
wavefunction (PyGFMC protocols.py:1-143), as :class:`typing.Protocol`
classes: a class satisfies one by having the members, not by inheriting, so
PyGFMC's objects, this package's and user classes all qualify as they are.
The classes name the interfaces for type hints; the engine checks them at the
start of a run (``engine.require_operator_protocol``,
``engine.require_guide_protocol``).

``config`` is one basis configuration, an array of shape (N_sites,).  The
methods are the host-side definition of the model: this package's host tools
(``exact_diagonalization``, the tests) call them, while the propagation runs
on the device from tables the engine lowers from the objects' attributes.
What the device lowering reads, beyond the protocol:

* Operators -- the SpinHalf transition layout (``n_hx_static``,
  ``n_jpm_static``, ``edge_i``, ``edge_j``, ``J_pm``, ``J_pmpm``, ``J_z``, and
  the fields) or the BoseHubbard one (``n_hop_off``, ``n_eta_off``,
  ``n_hpm_off``, ``n_max``, ``edge_i``, ``edge_j`` and the couplings); an
  operator with neither is refused with TypeError, as PyGFMC refuses an
  object without the protocol.
* Diagonal operators -- SpinHalf, BoseHubbard and SzSzStructureFactor
  layouts.
* Guides -- the attribute sets of the Jastrow guides
  (``engine.SPIN_JASTROW_ATTRS``, ``engine.BOSE_JASTROW_ATTRS``), of the
  exact-amplitude guide (``engine.EXACT_GUIDE_ATTRS``), and this package's
  learned guides (RBMSpinHalf, MLPBoseHubbard); a guide with the protocol but
  none of these layouts is refused with TypeError.
"""
from typing import Any, Optional, Protocol

import numpy as np

__all__ = ["Operator", "DiagonalOperator", "Guide"]


class Operator(Protocol):
    """The rate protocol of a Hamiltonian or an off-diagonal observable:
    H = sum of ``M_total`` terms, each taking a basis state to at most one
    other; term 0 is the diagonal."""

    M_total: int
    """Number of terms (1 + the off-diagonal transition slots)."""

    def get_rates(self, config: np.ndarray, return_configs: bool = False):
        """The ``M_total`` matrix elements H[x', x] of ``config`` = x, slot 0
        the diagonal one; with ``return_configs`` also the successor
        configurations x' (M_total, N_sites), slot 0 being x itself.  A slot
        whose move is impossible has rate 0."""
        ...

    def generate_state(self, config: np.ndarray, idx: int) -> np.ndarray:
        """The successor of ``config`` through slot ``idx`` (needed when
        M_total > 1)."""
        ...

    def move(self, config: np.ndarray, idx: int):
        """Optional: slot ``idx`` as ``(sites, deltas)``, the sites it
        changes and the amounts added to them (the incremental guides' form
        of a move)."""
        ...


class DiagonalOperator(Protocol):
    """A diagonal observable, measured by forward walking."""

    def diagonal_weight(self, config: np.ndarray) -> np.ndarray:
        """O(x): a scalar, or a vector (one value per component, e.g. per
        wavevector) of fixed length."""
        ...


class Guide(Protocol):
    """A guiding wavefunction psi_T.  The propagation needs only the ratios
    psi_T(x') / psi_T(x) to the successors of x, so a guide has at least one
    of the three ratio methods; ``build_cache`` and the incremental members
    are optional."""

    def log_diff_from_operator(self, config: np.ndarray, op: Operator, cache: Any = None,
                               state: Any = None) -> np.ndarray:
        """log psi_T(x') - log psi_T(x) for every slot of ``op`` (slot 0: 0)."""
        ...

    def log_diff_from_configs(self, config: np.ndarray, new_configs: np.ndarray,
                              cache: Any = None) -> np.ndarray:
        """log psi_T(x') - log psi_T(x) for each row x' of ``new_configs``."""
        ...

    def log_psi(self, config: np.ndarray, cache: Any = None) -> np.ndarray:
        """log |psi_T(x)|."""
        ...

    def build_cache(self, op: Operator) -> Any:
        """Optional: tables for ``op`` computed once per run."""
        ...

    incremental: bool
    """Optional: True when the guide keeps a per-walker state updated move by
    move (``init_state`` / ``update_state``)."""

    def init_state(self, config: np.ndarray, cache: Any = None) -> Any:
        """Optional (incremental mode): the per-walker state of ``config``."""
        ...

    def update_state(self, state: Any, config: np.ndarray, sites: np.ndarray,
                     deltas: np.ndarray, cache: Optional[Any] = None) -> Any:
        """Optional (incremental mode): ``state`` after adding ``deltas`` to
        ``sites`` of ``config``."""
        ...

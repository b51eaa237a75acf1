"""Order continuation on the device: solve at P0 first, then raise the order
one step at a time up to the target, prolonging the state between phases.

Restates core/utils/order_continuation.py (paths relative to the reference's
src/autoflowcfd):

* ``linear_interp_matrix_3d``: _build_linear_interp_matrix_3d (:14-60), the
  operator of scipy's ``RegularGridInterpolator(method="linear",
  fill_value=None)`` between two Gauss-Legendre tensor grids.  It is the
  tensor product of 1-D linear interpolation with linear extrapolation past
  the end nodes (a one-node grid gives a constant); each column is the
  product of three 1-D weights, as the reference's unit-basis probe yields.
* ``interpolate_to_new_order``: interpolate_to_new_order_checked (:62-205):
  the state (and the SST fields) prolonged by that matrix on the device
  (``afr_prolong``), the dual-time history dropped.
* ``run_order_continuation``: run_order_continuation (:207-425): restart from
  the uniform free stream at P0, phases P0..P with ``max_iter // n_phases``
  steps each, phase tolerance ``tol * 10**(P - p)``, and an early move to the
  next order once the residual has dropped 100x after at least 20 steps.

The solver is a ``B200FRSolver`` built with ``case_for_order``: one device
handle per phase, built from that order's tables of the same mesh; the handle
of a finished phase is released (the reference likewise keeps only the
current order's geometry).
"""

from typing import Callable, Optional

import numpy as np

from .solver import SolverResult


def gauss_legendre_nodes(n: int) -> np.ndarray:
    """1-D Gauss-Legendre points on (-1, 1) (fr/quadrature_points.py:16-28)."""
    return np.polynomial.legendre.leggauss(n)[0]


def _linear_weights_1d(old: np.ndarray, new: np.ndarray) -> np.ndarray:
    """(len(new), len(old)) weights of 1-D linear interpolation on the nodes
    ``old`` (ascending), extrapolating linearly past either end; a single
    node gives weight 1 everywhere."""
    n_old = len(old)
    W = np.zeros((len(new), n_old))
    if n_old == 1:
        W[:, 0] = 1.0
        return W
    for a, x in enumerate(new):
        # interval i with old[i] <= x < old[i+1], clamped to the first / last
        i = int(np.searchsorted(old, x)) - 1
        i = min(max(i, 0), n_old - 2)
        t = (x - old[i]) / (old[i + 1] - old[i])
        W[a, i] += 1.0 - t
        W[a, i + 1] += t
    return W


def linear_interp_matrix_3d(old_sps_1d: np.ndarray, new_sps_1d: np.ndarray) -> np.ndarray:
    """(n_new^3, n_old^3) trilinear interpolation matrix between tensor grids,
    points ordered with the first coordinate slowest (meshgrid "ij" ravel)."""
    w = _linear_weights_1d(np.asarray(old_sps_1d, float), np.asarray(new_sps_1d, float))
    n_new, n_old = w.shape
    W = np.zeros((n_new**3, n_old**3))
    for a0 in range(n_new):
        for a1 in range(n_new):
            for a2 in range(n_new):
                row = (a0 * n_new + a1) * n_new + a2
                for b0 in range(n_old):
                    for b1 in range(n_old):
                        for b2 in range(n_old):
                            W[row, (b0 * n_old + b1) * n_old + b2] = w[a0, b0] * w[a1, b1] * w[a2, b2]
    return W


def prolongation_matrix(old_order: int, new_order: int) -> np.ndarray:
    """The matrix interpolate_to_new_order applies between two orders."""
    return linear_interp_matrix_3d(gauss_legendre_nodes(old_order + 1), gauss_legendre_nodes(new_order + 1))


def interpolate_to_new_order(solver, new_order: int) -> None:
    """Prolong the solver's state to ``new_order`` on the device and continue
    on a handle of that order (interpolate_to_new_order_checked)."""
    solver._change_order(new_order, prolongation_matrix(solver.current_order, new_order))


def run_order_continuation(solver, max_iter: int, dt: float, tol: float,
                           checkpoint_callback: Optional[Callable] = None,
                           log: Optional[Callable[[str], None]] = None) -> SolverResult:
    """P0 -> P1 -> ... -> ``solver.order`` with the reference's phase rules.

    ``checkpoint_callback(solver, total_iteration)`` runs after every step.
    Returns the reference's SolverResult(converged, iterations, final_residual)."""
    say = log or (lambda msg: None)
    original_order = solver.order
    if solver.n_sps != 1:
        # restart from the uniform free stream at P0 (:236-288)
        solver._restart_at_p0()
        say(f"[INFO] Reinitialized to P0 (1 SP/cell)")
    orders = list(range(0, original_order + 1))
    total_iter = 0
    final_residual = 1e10
    for target_p in orders:
        if target_p > 0:
            interpolate_to_new_order(solver, target_p)
        if solver.n_sps != (target_p + 1) ** 3:
            raise RuntimeError(f"Order Continuation dimension mismatch after interpolation to P{target_p}: "
                               f"state has {solver.n_sps} SPs, expected {(target_p + 1) ** 3}")
        phase_max_iter = max_iter // len(orders)
        phase_tol = tol * (10 ** (original_order - target_p))
        initial = None
        drop_threshold = 1e2
        min_iter_before_transition = 20
        converged = False
        for i in range(phase_max_iter):
            res = solver.step(dt)
            final_residual = res
            total_iter += 1
            if initial is None:
                initial = res
            say(f"P{target_p} Iter {i + 1}: Residual = {res:.6e} | Drop: {initial / max(res, 1e-30):.1f}x")
            if checkpoint_callback is not None:
                checkpoint_callback(solver, total_iter)
            if res < phase_tol:
                converged = True
                break
            if (target_p < original_order and i >= min_iter_before_transition and initial > 0
                    and initial / max(res, 1e-30) >= drop_threshold):
                break
        if target_p == original_order and converged:
            return SolverResult(converged=True, iterations=total_iter, final_residual=final_residual)
    return SolverResult(converged=False, iterations=total_iter, final_residual=final_residual)

"""Order continuation (P0 -> ... -> P) without a GPU: the prolongation matrix,
the oracle against the reference's continuation runs, and the phase rules of
the product's driver on a scripted solver.

The fixtures cont_*.npz hold the reference's own FRSolver.solve runs
(core/utils/order_continuation.py:207-425) with every phase's tables."""
import os

import numpy as np
import pytest

from autoflowcfd_b200 import continuation as C
from conftest import golden_path
from oracle import fr_oracle as O

CONT_CASES = ["cont_prism_p2_ns", "cont_tet_p2_uniform", "cont_prism_p2_sst"]
# Absolute tolerance of the step residuals.  cont_tet_p2_uniform starts from
# the uniform free stream on a periodic box: its residuals (4e-8 .. 1.5) are
# the rounding noise of free-stream preservation on fluxes of ~2e5, so any
# change of summation order moves them by up to ~1e-4; the states agree to
# 1e-13 all the same.  cont_prism_p2_ns has residuals ~1e5-1e6 of real flow.
# cont_prism_p2_sst starts its P0 phase from the free stream too: residuals
# 0.03 .. 0.5 against fluxes of ~1e5, moved by ~1e-8 absolute by the device's
# summation orders (measured 9e-9).
RES_ATOL = {"cont_prism_p2_ns": 0.0, "cont_tet_p2_uniform": 1e-3, "cont_prism_p2_sst": 1e-6}
# Relative tolerance of the step residuals.  In cont_prism_p2_sst the P1 / P2
# states change by ~1e-5 relative per step, so the RMS of dU/dt carries the
# rounding of a different summation order at up to ~1e-10 relative (oracle:
# 9e-10 at most) while every state, k, omega and nu_t agree to ~1e-15.
RES_RTOL = {"cont_prism_p2_ns": 1e-12, "cont_tet_p2_uniform": 1e-12, "cont_prism_p2_sst": 2e-9}
REF_SRC = os.path.join(os.environ.get("AFR_REFERENCE", "/root/reference"), "src")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("old,new", [(0, 1), (1, 2), (2, 3), (0, 2), (1, 3)])
def test_prolongation_matrix_matches_the_interpolator_probe(old, new):
    """The product's closed-form trilinear matrix equals the reference's
    construction (scipy's linear RegularGridInterpolator probed with unit
    vectors) to rounding: rows still sum to one."""
    gl = lambda n: np.polynomial.legendre.leggauss(n)[0]
    W = C.prolongation_matrix(old, new)
    Wr = O.interp_matrix_3d(gl(old + 1), gl(new + 1))
    assert W.shape == ((new + 1) ** 3, (old + 1) ** 3)
    assert np.max(np.abs(W - Wr)) <= 4e-16
    assert np.allclose(W.sum(axis=1), 1.0, atol=1e-14)


@pytest.mark.parametrize("name", CONT_CASES)
def test_oracle_continuation_matches_reference(golden, name):
    g = golden(name)
    order = int(g["order"])
    so, sr, states, result = O.order_continuation(
        lambda p: O.case_from_prefix(g, f"p{p}/"), order, float(g["mu"]), bool(g["inviscid_only"]),
        g["freestream"], int(g["max_iter"]), float(g["dt"]), float(g["tol"]), turb=str(g["turb"]),
        wall_distance=g["wall_distance"] if "wall_distance" in g else None)
    assert list(so) == list(g["step_order"])
    assert np.allclose(sr, g["step_residual"], rtol=RES_RTOL[name], atol=RES_ATOL[name])
    for k, v in states.items():
        assert rel(v, g[k]) < 1e-12, k
    assert rel(states[f"U_end_p{order}"], g["U_final"]) < 1e-12
    assert result[0] == bool(g["result"][0]) and result[1] == int(g["result"][1])
    assert abs(result[2] - g["result"][2]) <= RES_RTOL[name] * abs(g["result"][2]) + RES_ATOL[name]


class Scripted:
    """A solver whose residuals follow a script per phase; records the
    order changes the continuation asks for."""

    def __init__(self, order, script, start_sps=None):
        self.order = order
        self.current_order = order
        self.n_sps = (order + 1) ** 3 if start_sps is None else start_sps
        self.script = script
        self.calls = []
        self.i = 0

    def _restart_at_p0(self):
        self.calls.append("restart")
        self.current_order, self.n_sps, self.i = 0, 1, 0

    def _change_order(self, p, W):
        assert W.shape == ((p + 1) ** 3, self.n_sps)
        self.calls.append(p)
        self.current_order, self.n_sps, self.i = p, (p + 1) ** 3, 0

    def step(self, dt):
        r = self.script(self.current_order, self.i)
        self.i += 1
        return r


def _run(order, script, max_iter, tol):
    s = Scripted(order, script)
    seen = []
    r = C.run_order_continuation(s, max_iter, 1e-3, tol, checkpoint_callback=lambda sol, it: seen.append(
        (sol.current_order, it)))
    return s, seen, r


def test_phase_budget_without_convergence():
    s, seen, r = _run(2, lambda p, i: 1.0, max_iter=30, tol=1e-6)
    assert s.calls == ["restart", 1, 2]
    assert [p for p, _ in seen] == [0] * 10 + [1] * 10 + [2] * 10
    assert [it for _, it in seen] == list(range(1, 31))
    assert (r.converged, r.iterations, r.final_residual) == (False, 30, 1.0)


def test_early_move_after_a_hundredfold_drop():
    # P0 drops 100x at its 23rd step (i = 22): moves on then; P1 never drops
    def script(p, i):
        return 1.0 if p > 0 else (1.0 if i < 22 else 0.009)

    s, seen, r = _run(2, script, max_iter=90, tol=1e-12)
    phases = [p for p, _ in seen]
    assert phases.count(0) == 23 and phases.count(1) == 30 and phases.count(2) == 30
    assert not r.converged and r.iterations == 83


def test_drop_needs_twenty_steps_first():
    # a 1000x drop at the second step does not move on before i >= 20
    s, seen, r = _run(1, lambda p, i: 1.0 if i == 0 else 1e-3, max_iter=60, tol=1e-12)
    phases = [p for p, _ in seen]
    assert phases.count(0) == 21 and phases.count(1) == 30


def test_phase_tolerance_and_converged_return():
    # phase tolerance tol * 10**(P - p): 1e-4 at P0, 1e-5 at P1, 1e-6 at P2
    levels = {0: 5e-5, 1: 5e-6, 2: 5e-7}
    s, seen, r = _run(2, lambda p, i: levels[p] * (10.0 if i < 2 else 1.0), max_iter=30, tol=1e-6)
    assert [p for p, _ in seen] == [0, 0, 0, 1, 1, 1, 2, 2, 2]
    assert (r.converged, r.iterations, r.final_residual) == (True, 9, 5e-7)


def test_a_lower_phase_converging_does_not_end_the_run():
    levels = {0: 1e-9, 1: 1.0}
    s, seen, r = _run(1, lambda p, i: levels[p], max_iter=8, tol=1e-6)
    assert [p for p, _ in seen] == [0, 1, 1, 1, 1]
    assert not r.converged and r.iterations == 5


def _reference_available():
    try:
        import importlib.util

        return os.path.isdir(os.path.join(REF_SRC, "autoflowcfd")) and importlib.util.find_spec("numba") is not None
    except Exception:
        return False


@pytest.mark.skipif(not _reference_available(), reason="the reference checkout is not installed here")
@pytest.mark.parametrize("case", ["budget", "drop", "tol"])
def test_phase_rules_match_the_reference_driver(case, monkeypatch):
    """The reference's run_order_continuation and the product's driver take
    the same steps on the same scripted residuals."""
    import sys
    from types import SimpleNamespace

    if REF_SRC not in sys.path:
        monkeypatch.syspath_prepend(REF_SRC)
    from autoflowcfd.core.utils import order_continuation as ref

    scripts = {"budget": (lambda p, i: 1.0, 30, 1e-6),
               "drop": (lambda p, i: 1.0 if p > 0 or i < 22 else 0.009, 90, 1e-12),
               "tol": (lambda p, i: {0: 5e-5, 1: 5e-6, 2: 5e-7}[p] * (10.0 if i < 2 else 1.0), 30, 1e-6)}
    script, max_iter, tol = scripts[case]
    ref_log = []

    class RefFake:
        def __init__(self):
            self.order = 2
            self.current_order = 0
            self.state = SimpleNamespace(U=np.zeros((3, 1, 5)), n_cells=3, n_vars=5)
            self.mesh = SimpleNamespace(set_order=lambda p: None, _order_geometry_cache={})
            self.ops = None
            self.turb_model = None
            self.wall_distance = None
            self.freestream = {"rho_inf": 1.0, "vel_inf": 1.0, "p_inf": 1.0}
            self.i = 0

        def _interpolate_to_new_order(self, p):
            self.state.U = np.zeros((3, (p + 1) ** 3, 5))
            self.current_order, self.i = p, 0

        def step(self, dt):
            r = script(self.current_order, self.i)
            self.i += 1
            ref_log.append(self.current_order)
            return r

    r_ref = ref.run_order_continuation(RefFake(), max_iter, 1e-3, tol)
    s, seen, r = _run(2, script, max_iter, tol)
    assert [p for p, _ in seen] == ref_log
    assert (r.converged, r.iterations, r.final_residual) == (r_ref.converged, r_ref.iterations, r_ref.final_residual)

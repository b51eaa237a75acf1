"""Known-answer physics checks of the CUDA path in both forms, after the
reference's own unit tests: free-stream preservation
(tests/unit/test_fr_residual_inviscid.py:129-141 of the reference) and a zero
viscous residual for a uniform flow (tests/unit/test_fr_viscous_flux.py:56-77).
They run on the triply periodic tet mesh of the isentropic-vortex case, where
a uniform state is an exact steady solution, so every residual must vanish to
rounding.  The scale is the residual of the vortex state on the same mesh."""
import numpy as np
import pytest

from autoflowcfd_b200.solver import B200FRSolver

pytestmark = pytest.mark.gpu


def make(case, precision):
    free = case["freestream"]
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=float(case["mu"]), rho_inf=free[0],
                     vel_inf=free[1], p_inf=free[2], precision=precision)
    s.set_state_from_cpu(case["U0"])
    return s


# Bars relative to the vortex residual: FP64 rounding through the collapsed
# P1 tet operators (row l1 norms up to 2e4); the mixed form adds FP32 fluxes.
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_uniform_flow_is_preserved(golden, precision, tol):
    case = golden("tet_p1_vortex")
    s = make(case, precision)
    scale = float(s.compute_inviscid_residual()[..., :5].abs().max())
    assert scale > 0.0
    U0 = case["U0"]
    uniform = np.broadcast_to(U0.reshape(-1, U0.shape[-1]).mean(0), U0.shape).copy()
    s.set_state_from_cpu(uniform)
    ri = float(s.compute_inviscid_residual()[..., :5].abs().max())
    rv = float(s.compute_viscous_residual()[..., :5].abs().max())
    assert ri <= tol * scale, (ri, scale)
    assert rv <= tol * scale, (rv, scale)
    s.cleanup()

"""Order continuation and the order-0 path on the device, against the
reference's own FRSolver.solve runs (core/utils/order_continuation.py:207-425):
every step's residual, the state at the end of every phase and the result.

Tolerances as in test_continuation.py: 1e-12 relative on states; residuals
1e-12 relative, plus an absolute 1e-3 for the uniform-stream case whose
residuals are the rounding noise of free-stream preservation."""
import numpy as np
import pytest

from test_continuation import CONT_CASES, RES_ATOL, RES_RTOL

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def phase_cases(g):
    def case_at(p):
        pre = f"p{p}/"
        return {k[len(pre):]: g[k] for k in g if k.startswith(pre)}

    return case_at


@pytest.mark.parametrize("name", CONT_CASES)
def test_device_continuation_matches_reference(golden, name):
    from autoflowcfd_b200.solver import B200FRSolver

    g = golden(name)
    order = int(g["order"])
    case_at = phase_cases(g)
    free = g["freestream"]
    sst = str(g["turb"]) == "SST"
    target = dict(case_at(order))
    if sst:
        target["wall_distance"] = g["wall_distance"]  # the target order's field
    s = B200FRSolver(target, turb_model_name=str(g["turb"]), mu_molecular=float(g["mu"]), rho_inf=free[0],
                     vel_inf=free[1], p_inf=free[2], inviscid_only=bool(g["inviscid_only"]), case_for_order=case_at)
    ends, turb_ends, orders = {}, {}, []

    def cb(sol, it):
        orders.append(sol.current_order)
        ends[sol.current_order] = sol.U.detach().cpu().numpy()
        if sst:
            turb_ends[sol.current_order] = [x.detach().cpu().numpy() for x in (sol.k, sol.omega, sol.nu_t)]

    r = s.solve(max_iter=int(g["max_iter"]), dt=float(g["dt"]), tol=float(g["tol"]), checkpoint_callback=cb)
    assert orders == list(g["step_order"])
    assert np.allclose(r["residual_history"], g["step_residual"], rtol=RES_RTOL[name], atol=RES_ATOL[name])
    for p, U in ends.items():
        assert rel(U, g[f"U_end_p{p}"]) < 1e-12, p
    for p, (k, w, nut) in turb_ends.items():
        assert rel(k, g[f"k_end_p{p}"]) < 1e-12 and rel(w, g[f"w_end_p{p}"]) < 1e-12, p
        assert rel(nut, g[f"nut_end_p{p}"]) < 1e-12, p
    assert rel(s.U, g["U_final"]) < 1e-12
    assert r["converged"] == bool(g["result"][0]) and r["iterations"] == int(g["result"][1])
    assert s.current_order == order and s.n_sps == (order + 1) ** 3
    s.cleanup()


def test_prolongation_on_the_device_matches_einsum(golden):
    """afr_prolong against np.einsum("ab,cbv->cav") on a random field."""
    import torch

    from autoflowcfd_b200 import continuation as C
    from autoflowcfd_b200.solver import B200FRSolver

    g = golden("cont_prism_p2_ns")
    case_at = phase_cases(g)
    s = B200FRSolver(case_at(1), mu_molecular=float(g["mu"]), case_for_order=case_at)
    rng = np.random.default_rng(3)
    U1 = rng.standard_normal((s.n_cells, 8, 5)) * 1e3
    s.set_state_from_cpu(U1)
    W = C.prolongation_matrix(1, 2)
    s._change_order(2, W)
    want = np.einsum("ab,cbv->cav", W, U1)
    assert s.current_order == 2 and tuple(s.U.shape) == (s.n_cells, 27, 5)
    assert rel(s.U, want) < 1e-14
    s.cleanup()

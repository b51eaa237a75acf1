"""The dual-time (BDF1 on the first physical step, BDF2 after) and IMEX
Euler schemes through the C-ABI against the reference's own steps
(core/time_integration/dual.py, imex.py; fixtures made by
tests/golden/make_golden.py with the reference's FRSolver).

Plain form: every conserved variable, the turbulence fields and the norms at
1e-12.  Mixed form: field L2 <= 1e-6 per field (its accuracy target); its
pseudo-time control flow reads the same norms to ~1e-8, so it takes the same
inner iterations."""
import numpy as np
import pytest

from autoflowcfd_b200.solver import B200FRSolver
from conftest import SCHEME_CASES
from fields import per_field, scalar, worst

pytestmark = pytest.mark.gpu


def make(case, precision):
    free = case["freestream"]
    s = B200FRSolver(case, turb_model_name=str(case["turb"]), mu_molecular=float(case["mu"]), rho_inf=free[0],
                     vel_inf=free[1], p_inf=free[2], inviscid_only=bool(case["inviscid_only"]),
                     precision=precision, time_scheme=str(case["time_scheme"]),
                     dual_time_inner_iter=int(case["dual_time_inner_iter"]))
    s.set_state_from_cpu(case["U0"])
    if str(case["turb"]) == "SST":
        s.set_turbulence(case["k0"], case["omega0"], case["nu_t0"])
    return s


@pytest.mark.parametrize("name", SCHEME_CASES)
def test_plain_form_scheme_steps_match_reference(golden, name):
    case = golden(name)
    s = make(case, "fp64")
    dt = float(case["dt_step"])
    for i in range(len(case["norms"])):
        n = s.step(dt)
        assert worst(per_field(s.U, case[f"U_step{i + 1}"])) < 1e-12, i
        assert abs(n - case["norms"][i]) <= 1e-12 * case["norms"][i], i
        if s.k is not None:
            for a, key in ((s.k, "k"), (s.omega, "w"), (s.nu_t, "nut")):
                assert scalar(a, case[f"{key}_step{i + 1}"])[1] < 1e-12, key
    if "cd_cl" in case:
        c = s.compute_aerodynamic_coefficients(1.0)
        assert np.allclose([c["Cd"], c["Cl"], c["Cs"]], case["cd_cl"], rtol=1e-10, atol=0)
    s.cleanup()


@pytest.mark.parametrize("name", SCHEME_CASES)
def test_mixed_form_scheme_steps_against_reference(golden, name):
    case = golden(name)
    s = make(case, "mixed")
    dt = float(case["dt_step"])
    for i in range(len(case["norms"])):
        s.step(dt)
        errs = per_field(s.U, case[f"U_step{i + 1}"])
        if s.k is not None:
            errs["k"] = scalar(s.k, case[f"k_step{i + 1}"])
            errs["omega"] = scalar(s.omega, case[f"w_step{i + 1}"])
        print(f"{name} mixed step {i + 1}: " + " ".join(f"{k} {v[0]:.1e}/{v[1]:.1e}" for k, v in errs.items()))
        assert worst(errs, 0) < 1e-6, i
    s.cleanup()

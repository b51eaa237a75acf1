"""Resume from a checkpoint on the GPU: a run interrupted after two steps,
written to a checkpoint, and resumed in a fresh handle continues bitwise as
the uninterrupted run (SST with SSP-RK3, and the dual-time scheme whose
BDF2 steps need the saved previous level)."""
import numpy as np
import pytest

from autoflowcfd_b200.solver import B200FRSolver

pytestmark = pytest.mark.gpu


def make(case, scheme):
    free = case["freestream"]
    s = B200FRSolver(case, turb_model_name=str(case["turb"]), mu_molecular=float(case["mu"]), rho_inf=free[0],
                     vel_inf=free[1], p_inf=free[2], time_scheme=scheme)
    s.set_state_from_cpu(case["U0"])
    if str(case["turb"]) == "SST":
        s.set_turbulence(case["k0"], case["omega0"], case["nu_t0"])
    return s


@pytest.mark.parametrize("name,scheme,dt", [("prism_p2_sst", "ssp_rk3", 1e-3),
                                            ("prism_p1_ns_dual_time", "dual_time", 2e-5)])
def test_resume_continues_bitwise(golden, tmp_path, name, scheme, dt):
    case = golden(name)
    ref = make(case, scheme)
    for _ in range(4):
        ref.step(dt)
    a = make(case, scheme)
    for _ in range(2):
        a.step(dt)
    path = a.save_checkpoint(str(tmp_path / "ck"), iteration=2)
    a.cleanup()
    b = make(case, scheme)
    assert b.resume_from_checkpoint(path) == 2
    for _ in range(2):
        b.step(dt)
    assert np.array_equal(b.U.cpu().numpy(), ref.U.cpu().numpy())
    if b.k is not None:
        assert np.array_equal(b.k.cpu().numpy(), ref.k.cpu().numpy())
        assert np.array_equal(b.nu_t.cpu().numpy(), ref.nu_t.cpu().numpy())
    assert b.residual_history == ref.residual_history
    ref.cleanup()
    b.cleanup()

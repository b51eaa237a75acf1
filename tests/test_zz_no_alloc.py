"""The allocation-free entry point, afr_rms_norm_noalloc.

Callers that may not allocate at call time (CUDA graph capture, real-time step
loops, applications owning the device memory pool) get the step's residual
norm from a fixed static scratch array.  Its result must equal the norm
afr_step reports for the same stage-0 residual, on two calls in a row.  Kept
in a file of its own that pytest collects last."""
import ctypes

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def test_noalloc_norm_matches_step_norm_on_two_calls():
    import torch

    from autoflowcfd_b200._lib import AFR_EINVAL, AFR_OK, LIB
    from autoflowcfd_b200.solver import B200FRSolver

    z = np.load(golden_path("prism_p1_ns"))
    case = {k: z[k] for k in z.files}
    free = case["freestream"]
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=float(case["mu"]), rho_inf=free[0],
                     vel_inf=free[1], p_inf=free[2])
    s.set_state_from_cpu(case["U0"])
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        R = (s.compute_inviscid_residual() + s.compute_viscous_residual()).contiguous()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = LIB.afr_rms_norm_noalloc(ctypes.c_void_p(R.data_ptr()), R.numel(), ctypes.c_void_p(out.data_ptr()),
                                      stream)
        torch.cuda.synchronize()
        assert rc == AFR_OK
        if call == 1:  # after the first call loaded the module: no device memory taken
            assert torch.cuda.mem_get_info()[0] == free_before
        got = float(out.item())
        ref = s.step()  # RMS of dU/dt at stage 0 of this state (step() advances the state)
        assert abs(got - ref) / ref < 1e-12, (call, got, ref)
    # sizes beyond the fixed scratch are refused before any launch
    rc = LIB.afr_rms_norm_noalloc(ctypes.c_void_p(R.data_ptr()), 4096 * 65536 + 1, ctypes.c_void_p(out.data_ptr()),
                                  stream)
    assert rc == AFR_EINVAL
    s.cleanup()

"""Mixed form against the plain FP64 form on a generated C2-style box large
enough that every persistent CTA of the mixed pre-pass and volume kernels runs
several tiles (24x20x18 hex -> 17,280 P2 prisms: 2,160 pre-pass tiles on at
most 296 CTAs, 1,080 volume tiles on 148), RANS-SST with a no-slip wall and
farfield planes, local dt.  The golden fixtures are too small for that: there
each CTA runs at most one tile, so the copies a CTA issues for its next tile
while the current one runs are never exercised.

Bars: the inviscid and viscous residuals of the start state within 1e-3 and
2e-2 relative max-norm of the FP64 form's (measured on B200: 2.6e-5 and 3.7e-3;
the viscous residual depends on the gradients the pre-pass forms from each
tile's inverse-Jacobian rows, and a build whose tiles could read the next
tile's rows measured 37.5), per-field relative L2 after each of two steps
<= 1e-6 (measured: 2e-9 .. 3e-8), Cd within 1e-4 relative.
"""
import os
import sys

import numpy as np
import pytest
import torch

from autoflowcfd_b200.solver import B200FRSolver

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402  (the bench's seeded generator and flow conditions)


@pytest.fixture(scope="module")
def box():
    spec = dict(bench.SMALL)
    case = bench.make_case(spec)
    U, k, om, nut, mu = bench.initial_state(case, spec)
    return case, U, k, om, nut, mu


def make(box, precision):
    case, U, k, om, nut, mu = box
    rho, u, p, *_ = bench.flow_conditions()
    s = B200FRSolver(dict(case), turb_model_name="SST", mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p,
                     precision=precision)
    s.set_state_from_cpu(U)
    s.set_turbulence(k, om, nut)
    return s


def rel_max(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_mixed_residuals_on_a_multi_tile_box(box):
    s64, smx = make(box, "fp64"), make(box, "mixed")
    ri = rel_max(smx.compute_inviscid_residual(), s64.compute_inviscid_residual())
    rv = rel_max(smx.compute_viscous_residual(), s64.compute_viscous_residual())
    print(f"residual rel max: inviscid {ri:.2e}, viscous {rv:.2e}")
    s64.cleanup()
    smx.cleanup()
    assert ri < 1e-3 and rv < 2e-2, (ri, rv)


def run(box, precision, steps):
    s = make(box, precision)
    out = []
    for _ in range(steps):
        s.step(want_norm=True)
        torch.cuda.synchronize()
        out.append((s.U.clone(), s.k.clone(), s.omega.clone()))
    cd = s.compute_aerodynamic_coefficients()["Cd"] if hasattr(s, "compute_aerodynamic_coefficients") else None
    s.cleanup()
    return out, cd


def test_mixed_form_tracks_fp64_on_a_multi_tile_box(box):
    mixed, cd_m = run(box, "mixed", 2)
    plain, cd_p = run(box, "fp64", 2)
    for step, ((Um, km, wm), (Up, kp, wp)) in enumerate(zip(mixed, plain), start=1):
        err = bench.per_field_errors(Um, km, wm, Up, kp, wp)
        worst = {f: e["l2_rel"] for f, e in err.items()}
        print(f"step {step}: " + ", ".join(f"{f} {v:.2e}" for f, v in worst.items()))
        for f, v in worst.items():
            assert np.isfinite(v) and v <= 1e-6, (step, f, v)
    if cd_m is not None and cd_p is not None:
        assert abs(cd_m - cd_p) <= 1e-4 * abs(cd_p)

"""Multi-step runs of the CUDA path against trajectories of the reference's own
FRSolver.step (tests/golden/traj_*.npz, made by tests/golden/make_golden.py),
through the C-ABI, on meshes the box-mesh generator rebuilds bit for bit.

- Small configuration at full size (24,576 periodic tets, P1 isentropic
  vortex, Euler, global dt 3 min(dt_local)), 100 steps: the plain form against
  the reference's state after steps 1 and 100 and its per-step residual norm
  and field sums; the mixed form against the reference's step-100 state per
  field.
- The C2 generator's 576-prism sample (P2, SST, the benchmark's start state),
  20 steps: the plain form follows the reference step by step through the SST
  growth (k max and nu_t max every step, fields at steps 1, 6 and 12); the
  mixed form's per-field errors against the reference over steps 1-6, before
  the growth.
- P3 precision stress at 3,072 tets: finite after one step at the P3 bar,
  non-finite after the second, as in the reference.

Per-field errors are relative L2 / relative max (tests/fields.py).  Prism
tables from the generator differ from a fresh reference build by up to 3e-10
(Newton location noise in the reference's matrices), which sets the prism bars.
"""
import numpy as np
import pytest

import bench
import flows
from autoflowcfd_b200 import boxgeom, boxmesh
from autoflowcfd_b200._lib import AfrError
from autoflowcfd_b200.solver import B200FRSolver
from conftest import golden_path
from fields import per_field, scalar, worst

pytestmark = pytest.mark.gpu


def load(name):
    z = np.load(golden_path(name), allow_pickle=False)
    return {k: z[k] for k in z.files}


def report(tag, errs):
    print(f"{tag}: " + " ".join(f"{k} {v[0]:.2e}/{v[1]:.2e}" for k, v in errs.items()))


@pytest.fixture(scope="module")
def c1():
    box = boxmesh.tet_box(16, 16, 16, (1.0, 1.0, 1.0), jitter=0.0, periodic=True)
    case = boxgeom.build_case(box, 1, None, wall_distance=False, want_sps_coords=True)
    U, u0 = flows.c1_vortex(case.pop("sps_coords"))
    return case, U, u0, load("traj_c1_vortex")


def c1_solver(case, U, u0, precision):
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=1.8e-5, rho_inf=flows.RHO, vel_inf=u0,
                     p_inf=flows.P, inviscid_only=True, global_dt_factor=3.0, precision=precision)
    s.set_state_from_cpu(U)
    return s


def test_c1_plain_form_follows_reference_100_steps(c1):
    case, U, u0, g = c1
    st = int(g["stride"])
    assert np.array_equal(U[::st], g["U0_sample"])
    s = c1_solver(case, U, u0, "fp64")
    for it in range(1, 101):
        n = s.step()
        assert abs(n - g["step_norm"][it - 1]) <= 1e-10 * g["step_norm"][it - 1], it
        l2 = s.U.norm(dim=(0, 1)).cpu().numpy()
        assert np.all(np.abs(l2 - g["step_l2"][it - 1]) <= 1e-10 * g["step_l2"][it - 1]), it
        if it in (1, 100):
            errs = per_field(s.U.cpu().numpy()[::st], g[f"U_s{it}"])
            report(f"c1 fp64 step {it}", errs)
            assert worst(errs) < (1e-12 if it == 1 else 1e-10)
    s.cleanup()


def test_c1_mixed_form_against_reference_after_100_steps(c1):
    case, U, u0, g = c1
    st = int(g["stride"])
    s = c1_solver(case, U, u0, "mixed")
    for _ in range(100):
        s.step(want_norm=False)
    a = s.U.cpu().numpy()[::st]
    assert np.all(np.isfinite(a))
    errs = per_field(a, g["U_s100"])
    report("c1 mixed step 100 vs reference", errs)
    assert worst(errs, 0) < 1e-6  # the field relative L2 target of the mixed form
    assert worst(errs, 1) < 1e-5
    s.cleanup()


@pytest.fixture(scope="module")
def c2s():
    spec = bench.SAMPLE
    case = bench.make_case(spec)
    U, k, om, nut, mu = bench.initial_state(case, spec)
    return case, (U, k, om, nut, mu), load("traj_c2_sample")


def c2_solver(case, st, precision):
    U, k, om, nut, mu = st
    rho, u, p, *_ = bench.flow_conditions()
    s = B200FRSolver(case, turb_model_name="SST", mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p,
                     precision=precision)
    s.set_state_from_cpu(U)
    s.set_turbulence(k, om, nut)
    return s


def test_c2_sample_plain_form_follows_reference_through_sst_growth(c2s):
    case, st, g = c2s
    assert np.array_equal(st[0], g["U0_sample"])
    s = c2_solver(case, st, "fp64")
    for it in range(1, int(g["n_steps_run"]) + 1):
        n = s.step()
        assert abs(n - g["step_norm"][it - 1]) <= (1e-10 if it <= 16 else 1e-7) * g["step_norm"][it - 1], it
        assert abs(float(s.k.max()) - g["step_k_max"][it - 1]) <= 1e-9 * g["step_k_max"][it - 1], it
        assert abs(float(s.nu_t.max()) - g["step_nut_max"][it - 1]) <= 1e-9 * g["step_nut_max"][it - 1], it
        if f"U_s{it}" in g:
            assert worst(per_field(s.U, g[f"U_s{it}"])) < 1e-9, it
            for a, key in ((s.k, "k"), (s.omega, "w"), (s.nu_t, "nut")):
                assert scalar(a, g[f"{key}_s{it}"])[1] < 1e-8, (it, key)
    s.cleanup()


def test_c2_sample_mixed_form_per_field_errors_before_sst_growth(c2s):
    """Mixed form against the reference at steps 1 and 6 (before the growth
    that the reference's SST closure starts at step 7): per-field relative L2
    and max for rho, rho u, rho v, rho w, E, k and omega."""
    case, st, g = c2s
    s = c2_solver(case, st, "mixed")
    worst_l2 = 0.0
    for it in range(1, 7):
        s.step(want_norm=False)
        if f"U_s{it}" in g:
            errs = per_field(s.U, g[f"U_s{it}"])
            errs["k"] = scalar(s.k, g[f"k_s{it}"])
            errs["omega"] = scalar(s.omega, g[f"w_s{it}"])
            report(f"c2 sample mixed step {it} vs reference", errs)
            worst_l2 = max(worst_l2, worst(errs, 0))
    assert worst_l2 < 1e-6
    s.cleanup()


def test_p3_plain_form_blows_up_like_the_reference():
    g = load("traj_p3_tgv")
    st = int(g["stride"])
    box = boxmesh.tet_box(8, 8, 8, (1.0, 1.0, 1.0), jitter=0.05, seed=7, periodic=True)
    case = boxgeom.build_case(box, 3, None, wall_distance=False, want_sps_coords=True)
    U, u0 = flows.c3_tgv(case.pop("sps_coords"))
    s = B200FRSolver(case, turb_model_name="NONE", mu_molecular=1.8e-5, rho_inf=flows.RHO, vel_inf=u0,
                     p_inf=flows.P, inviscid_only=True, global_dt_factor=3.0)
    s.set_state_from_cpu(U)
    s.step()
    assert worst(per_field(s.U.cpu().numpy()[::st], g["U_s1"])) < 1e-3
    nonfinite = False
    try:
        n = s.step()
        nonfinite = not np.isfinite(n) or not bool(np.all(np.isfinite(s.U.cpu().numpy())))
    except AfrError as e:
        nonfinite = "non-finite" in str(e)
    assert nonfinite
    s.cleanup()

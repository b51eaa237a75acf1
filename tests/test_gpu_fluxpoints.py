"""Flux-point construction on the device (afr_flux_point_jobs) against the
reference's own construction (tests/golden/fp_*.npz): located coordinates,
location residuals and every cross-interpolation matrix; then the residual
of a case built from the constructed tables against the reference's.

Tolerances: the located coordinates and the matrices follow the reference's
arithmetic operation for operation (no multiply-add contraction, the same
integer-power rounding, the same inverse Vandermonde bit for bit), so most
entries agree exactly; the remaining differences are the last-bit effects of
sqrt / division sequences through the Newton iteration, amplified in the
matrices by the condition number of the modal Vandermonde matrix (~1e9 for
P3 tets)."""
import numpy as np
import pytest

from autoflowcfd_b200 import facegeom as FG
from test_fluxpoints import FP_CASES, face_conn, load

pytestmark = pytest.mark.gpu

# relative max-norm bars of the matrices by case
MAT_TOL = {"fp_prism_p1": 1e-12, "fp_prism_p2": 1e-11, "fp_prism_p3_bump": 1e-10, "fp_tet_p2": 1e-9,
           "fp_tet_p3": 1e-6}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", FP_CASES)
def test_construction_matches_reference(name):
    g = load(name)
    t = FG.flux_point_tables(face_conn(g), g["prism_conn"], g["tet_conn"], g["nodes"], int(g["order"]))
    for k in ("owner_cell", "neighbor_cell", "is_boundary", "owner_axis", "neighbor_axis", "owner_is_primary",
              "neighbor_is_primary", "nb_src0_cell", "nb_src1_idx", "nb_src1_cell", "ow_src0_cell", "ow_src1_idx",
              "ow_src1_cell", "colors"):
        assert np.array_equal(np.asarray(t[k]).astype(np.int64), np.asarray(g[k]).astype(np.int64)), k
    for k in ("owner_side", "neighbor_side", "true_normal"):
        assert np.array_equal(t[k], g[k]), k
    assert np.allclose(t["true_area_weight"], g["true_area_weight"], rtol=1e-15, atol=0)
    # located free coordinates of every record side and the residuals
    # (the reference's own residuals include the full periodic offset of the
    # tet faces it locates by projection: 2.0 on the unit box)
    for side in ("nb", "ow"):
        assert np.max(np.abs(t[side + "_fc"] - g[side + "_fc"])) < 1e-12, side
        assert np.allclose(t[side + "_resid"], g[side + "_resid"], rtol=1e-6, atol=1e-12), side
    for k in ("nb_src0_mat", "ow_src0_mat", "nb_src1_mat", "ow_src1_mat"):
        if g[k].size:
            assert rel(t[k], g[k]) < MAT_TOL[name], (k, rel(t[k], g[k]))
            # zero exactly where the reference's is zero (rows outside a half)
            assert np.array_equal(t[k] == 0, g[k] == 0) or rel(t[k], g[k]) < 1e-14, k


def test_case_from_constructed_tables_reproduces_reference_residuals(golden):
    """prism_p2_sst's mesh is fp_prism_p2's box: replace its face tables by
    the constructed ones and evaluate through the C-ABI."""
    from autoflowcfd_b200.solver import B200FRSolver

    g = load("fp_prism_p2")
    case = dict(golden("prism_p2_sst"))
    t = FG.flux_point_tables(face_conn(g), g["prism_conn"], g["tet_conn"], g["nodes"], 2)
    for k in ("owner_is_primary", "neighbor_is_primary", "true_normal", "nb_src0_cell", "nb_src0_mat", "nb_src1_idx",
              "nb_src1_cell", "nb_src1_mat", "ow_src0_cell", "ow_src0_mat", "ow_src1_idx", "ow_src1_cell",
              "ow_src1_mat", "colors", "true_area_weight"):
        case[k] = t[k]
    free = case["freestream"]
    s = B200FRSolver(case, turb_model_name="SST", mu_molecular=float(case["mu"]), rho_inf=free[0], vel_inf=free[1],
                     p_inf=free[2])
    s.set_state_from_cpu(case["U0"])
    s.set_turbulence(case["k0"], case["omega0"], case["nu_t0"])
    assert rel(s.compute_inviscid_residual().cpu().numpy(), case["R_inv"]) < 1e-9
    assert rel(s.compute_viscous_residual().cpu().numpy(), case["R_visc"]) < 1e-9
    s.cleanup()


def test_exporter_builds_the_face_tables_on_the_device(golden):
    """export_case(..., flux_points="device") on stand-ins of the reference's
    objects for prism_p2_sst (whose box is fp_prism_p2's): the constructed face
    tables and, through the C-ABI, the reference's residuals."""
    import refstandins
    from autoflowcfd_b200.reference_io import export_case
    from autoflowcfd_b200.solver import B200FRSolver

    case = dict(golden("prism_p2_sst"))
    fp = load("fp_prism_p2")
    mesh, ops, _ = refstandins.mesh_ops_flat(case)
    mesh.face_connectivity = type("FC", (), face_conn(fp))()
    mesh._fixed_prism_conn, mesh._fixed_tet_conn, mesh._node_coords = fp["prism_conn"], None, fp["nodes"]
    ext = case["boundary_extrap"]
    ops.boundary_extrap_prism = {(a, s): ext[0, a, i] for a in range(3) for i, s in enumerate((-1.0, 1.0))}
    ops.boundary_extrap_tet = {(a, s): ext[1, a, i] for a in range(3) for i, s in enumerate((-1.0, 1.0))}
    ops.g_left, ops.g_right = case["g_left"], case["g_right"]
    out = export_case(mesh, ops, refstandins.provider(case), wall_distance=case["wall_distance"],
                      flux_points="device")
    for k in ("owner_is_primary", "neighbor_is_primary", "nb_src1_idx", "ow_src1_idx", "colors", "dist_fp_of_sp",
              "dist_axis_coord_of_sp", "bc_group"):
        assert np.array_equal(np.asarray(out[k]).astype(np.int64), np.asarray(case[k]).astype(np.int64)), k
    assert rel(out["nb_src0_mat"], case["nb_src0_mat"]) < 1e-11
    assert np.array_equal(out["boundary_extrap"], case["boundary_extrap"])
    for k in ("freestream", "U0", "k0", "omega0", "nu_t0", "mu", "turb", "R_inv", "R_visc"):
        out[k] = case[k]
    free = case["freestream"]
    s = B200FRSolver(out, turb_model_name="SST", mu_molecular=float(case["mu"]), rho_inf=free[0], vel_inf=free[1],
                     p_inf=free[2])
    s.set_state_from_cpu(case["U0"])
    s.set_turbulence(case["k0"], case["omega0"], case["nu_t0"])
    assert rel(s.compute_inviscid_residual().cpu().numpy(), case["R_inv"]) < 1e-9
    assert rel(s.compute_viscous_residual().cpu().numpy(), case["R_visc"]) < 1e-9
    s.cleanup()

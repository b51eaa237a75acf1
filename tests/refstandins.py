"""Objects shaped like the reference's HighOrderMesh, FROperators,
FlatFaceGeometry and BoundaryGhostStateProvider, rebuilt from a golden
fixture's arrays.  They let the drop-in constructor run where the reference
is not installed (the GPU machine); the fixtures hold the reference's own
arrays, so the stand-ins carry the same numbers as the real objects."""

from types import SimpleNamespace

import numpy as np

BC_NAMES = {0: "WALL", 1: "FARFIELD", 2: "INLET", 3: "OUTLET", 4: "SYMMETRY"}


def mesh_ops_flat(g):
    N, S, Fn = int(g["n_cells"]), int(g["n_sps"]), int(g["n_fine"])
    mesh = SimpleNamespace(
        order=int(g["order"]), n_cells=N, n_sps_per_cell=S, n_sps_per_cell_fine=Fn,
        n_prism_cells=int(g["n_prism"]),
        jacobians={"det_jacs": g["det_jacs"].reshape(-1), "inv_jacs": g["inv_jacs"].reshape(-1, 3, 3)},
        jacobians_fine={"det_jacs": g["det_jacs_fine"].reshape(-1), "inv_jacs": g["inv_jacs_fine"].reshape(-1, 3, 3)},
        get_all_cell_volumes=lambda: g["cell_volumes"],
        face_flux_points=SimpleNamespace(true_area_weight=g["true_area_weight"]))
    ops = SimpleNamespace(
        D_3d_prism=g["D_3d_prism"], D_3d_tet=g["D_3d_tet"], overint_interp_c2f_prism=g["c2f_prism"],
        overint_interp_c2f_tet=g["c2f_tet"], overint_D_fine_prism=g["Dfine_prism"], overint_D_fine_tet=g["Dfine_tet"],
        overint_restrict_f2c_prism=g["f2c_prism"], overint_restrict_f2c_tet=g["f2c_tet"],
        filter_prism=g["filter_prism"], filter_tet=g["filter_tet"])
    col = g["colors"]
    P = g["true_normal"].shape[1]
    flat = SimpleNamespace(
        n_faces=len(col), n_fp=P, n_sps=S, n_prism=int(g["n_prism"]),
        owner_cell=g["owner_cell"], neighbor_cell=g["neighbor_cell"], is_boundary=g["is_boundary"].astype(bool),
        owner_axis=g["owner_axis"], owner_side=g["owner_side"], neighbor_axis=g["neighbor_axis"],
        neighbor_side=g["neighbor_side"], owner_is_primary=g["owner_is_primary"].astype(bool),
        neighbor_is_primary=g["neighbor_is_primary"].astype(bool), true_normal=g["true_normal"],
        neighbor_src0_cell=g["nb_src0_cell"], neighbor_src0_mat=g["nb_src0_mat"],
        neighbor_src1_idx=g["nb_src1_idx"], neighbor_src1_cell=g["nb_src1_cell"],
        neighbor_src1_mat=g["nb_src1_mat"], owner_src0_cell=g["ow_src0_cell"], owner_src0_mat=g["ow_src0_mat"],
        owner_src1_idx=g["ow_src1_idx"], owner_src1_cell=g["ow_src1_cell"], owner_src1_mat=g["ow_src1_mat"],
        boundary_extrap=g["boundary_extrap"], g_left=g["g_left"], g_right=g["g_right"],
        dist_fp_of_sp=g["dist_fp_of_sp"], dist_axis_coord_of_sp=g["dist_axis_coord_of_sp"],
        color_face_indices=[np.flatnonzero(col == c) for c in range(int(col.max()) + 1)])
    return mesh, ops, flat


def provider(g):
    """A table-form provider with the fixture's boundary tables: one group
    code per table row, the last row the default configuration."""
    rows = len(g["bc_type"])
    default = rows - 1

    def cfg(i):
        t = BC_NAMES[int(g["bc_type"][i])]
        c = {"type": t, "is_no_slip": bool(g["bc_noslip"][i]), "wall_velocity": list(g["bc_wall_vel"][i])}
        if t == "FARFIELD":
            c["Q_free"] = list(g["bc_Q"][i])
        if t == "INLET":
            c["Q_inlet"] = list(g["bc_Q"][i])
        if t == "OUTLET":
            c["p_outlet"] = float(g["bc_p_out"][i])
        return c

    gc = np.where(g["bc_group"] == default, -1, g["bc_group"]).astype(np.int64)
    return SimpleNamespace(group_code=gc, code_to_config={i: cfg(i) for i in range(default)},
                           default_config=cfg(default))

"""The box-mesh generator reproduces the reference's flattened tables.

The golden meshes were built by the reference's own loader from the same
BoxMesh; the generator must give bit-identical geometry and, through the
oracle, the reference's residuals: 1e-12 on tets, 1e-9 on prisms.  On prisms
the reference's own cross-interpolation matrices differ by up to 3e-10
(relative) between topologically identical faces (Newton location noise), so
the replayed template matrices can only agree to that level."""
import numpy as np
import pytest

from autoflowcfd_b200 import boxgeom, boxmesh
from conftest import golden_path
from oracle import fr_oracle as O

BOXES = {
    "prism_p2_sst": lambda: boxmesh.prism_box(4, 3, 3, (4.0, 2.0, 1.5), jitter=0.1, seed=7),
    "prism_p1_ns": lambda: boxmesh.prism_box(4, 3, 2, (2.0, 1.0, 1.0), jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3)),
    "tet_p1_vortex": lambda: boxmesh.tet_box(3, 3, 3, (1.0, 1.0, 1.0), jitter=0.0, periodic=True),
    # order 0 (finite volume): the same boxes as prism_p1_ns and tet_p1_vortex
    "prism_p0_ns": lambda: boxmesh.prism_box(4, 3, 2, (2.0, 1.0, 1.0), jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3)),
    "tet_p0_vortex": lambda: boxmesh.tet_box(3, 3, 3, (1.0, 1.0, 1.0), jitter=0.0, periodic=True),
}


def plane_cfg_from(g):
    inv = {v: k for k, v in boxgeom.BC_CODES.items()}
    cfg = {}
    for i, pn in enumerate(boxmesh.PLANE_NAMES):
        t = inv[int(g["bc_type"][i])]
        d = {"type": t, "is_no_slip": bool(g["bc_noslip"][i])}
        if t == "FARFIELD":
            d["Q_free"] = list(g["bc_Q"][i])
        if t == "INLET":
            d["Q_inlet"] = list(g["bc_Q"][i])
        if t == "OUTLET":
            d["p_outlet"] = float(g["bc_p_out"][i])
        cfg[pn] = d
    return cfg


def expand(case):
    c = dict(case)
    tab = c.pop("src_mat_table")
    for k in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        c[k] = tab[c.pop(k + "_index")]
    return c


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", sorted(BOXES))
def test_generator_matches_reference_build(golden, name):
    g = golden(name)
    box = BOXES[name]()
    cfg = None if box.periodic else plane_cfg_from(g)
    sst = str(g["turb"]) == "SST"
    c = boxgeom.build_case(box, int(g["order"]), cfg, wall_distance=sst, want_sps_coords=True)
    for k in ("det_jacs", "inv_jacs", "det_jacs_fine", "inv_jacs_fine", "cell_volumes", "sps_coords"):
        assert np.array_equal(c[k], g[k]), k
    if sst:
        assert np.array_equal(c["wall_distance"], g["wall_distance"])
    assert len(c["owner_cell"]) == len(g["owner_cell"])
    assert int(np.sum(c["is_boundary"])) == int(np.sum(g["is_boundary"]))
    if "cd_wall_face" in g:
        assert int(c["cd_wall_face"].sum()) == int(g["cd_wall_face"].sum())
    ce = expand(c)
    for k in ("mu", "turb", "freestream", "U0", "k0", "omega0", "nu_t0"):
        if k in g:
            ce[k] = g[k]
    m = O.Mesh.from_case(ce)
    U = g["U0"]
    Q = O.state_primitives(U)
    mu = float(g["mu"])
    mu_t = Q[:, :, 0] * g["nu_t0"] if sst else None
    tol = 1e-12 if box.kind == "tet" else 1e-9
    assert rel(O.inviscid_residual(m, U), g["R_inv"][..., :5]) < tol
    assert rel(O.viscous_residual(m, U, mu, mu_t), g["R_visc"][..., :5]) < tol
    assert rel(O.local_dt(m, Q, mu, mu_t), g["dt_local"]) < 1e-15


def test_coloring_is_valid_and_greedy():
    from autoflowcfd_b200._lib import greedy_face_coloring

    box = boxmesh.prism_box(5, 4, 3, jitter=0.1, seed=1)
    c = boxgeom.build_case(box, 1, None)
    col = greedy_face_coloring(c["owner_cell"], c["neighbor_cell"], c["is_boundary"], c["n_cells"])
    # no cell receives two faces of one color
    cells = np.concatenate([c["owner_cell"], np.where(c["is_boundary"].astype(bool), -1, c["neighbor_cell"])])
    cols = np.concatenate([col, col])
    ok = cells >= 0
    pairs = cells[ok] * 1000 + cols[ok]
    assert len(np.unique(pairs)) == len(pairs)
    assert col.min() == 0

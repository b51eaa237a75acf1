"""Box meshes of any size, flattened into the reference's face-table format.

``build_case(box, order, ...)`` returns the same mapping of arrays the
reference's ``HighOrderMesh`` + ``FlatFaceGeometry`` produce for a mesh
(keys as in ``tests/golden/make_golden.py``), without the reference and fast
enough for millions of cells:

* geometry is recomputed from the node coordinates with the reference's
  closed forms: Duffy-collapsed prism / tet maps and their exact Jacobians
  (grid/curved_mapping/curved_mapping_exact_jacobian.py:39-119), closed-form
  3x3 determinant and inverse (grid/curved_mapping/curved_mapping.py:39-91),
  Gauss-Legendre cell volumes (grid/high_order/high_order_mesh.py:335-354),
  vertex-average-oriented face normals and areas
  (grid/mesh_gen/background/face_geometry_finalize.py:95-176), KD-tree wall
  distance (core/fr_solver/turbulence.py:112-125);
* face records (which records exist, owner / neighbour roles, primary flags,
  interpolation sources and their matrices) are replayed from a 3x3x3-hex
  template the reference itself flattened (``data/tmpl_<kind>_p<order>.npz``,
  made by ``tests/golden/make_tables.py``): every cell copies the records of the
  template cell in the same topological position (low boundary / interior /
  high boundary per axis);
* face colors come from the reference's greedy rule (C++ in libafr_b200.so).

The interpolation matrices are returned in indexed form (a small table plus
per-record indices) that ``afr_create`` expands on the device into the
reference's dense per-record layout.
"""

import os
from typing import Dict, Optional

import numpy as np

from . import boxmesh
from .boxmesh import BoxMesh, PLANE_NAMES

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
BC_CODES = {"WALL": 0, "FARFIELD": 1, "INLET": 2, "OUTLET": 3, "SYMMETRY": 4}
_TEMPLATES: Dict[tuple, dict] = {}


def load_template(kind: str, order: int) -> dict:
    key = (kind, order)
    if key not in _TEMPLATES:
        z = np.load(os.path.join(DATA, f"tmpl_{kind}_p{order}.npz"), allow_pickle=False)
        _TEMPLATES[key] = {k: z[k] for k in z.files}
    return _TEMPLATES[key]


def ref_grid(pts_1d):
    a, b, c = np.meshgrid(pts_1d, pts_1d, pts_1d, indexing="ij")
    return np.column_stack([a.ravel(), b.ravel(), c.ravel()])


# ---------------------------------------------------------------------------
# element maps and exact Jacobians
# ---------------------------------------------------------------------------
def prism_map(ref, X):
    """map_prism_to_physical: ref (n,3), X (N,6,3) -> (N,n,3)."""
    a, b, c = ref[:, 0], ref[:, 1], ref[:, 2]
    r = (1.0 + a) * (1.0 - b) / 2.0 - 1.0
    s = b
    l1, l2, l3 = -(r + s) / 2.0, (1.0 + r) / 2.0, (1.0 + s) / 2.0
    bot = l1[None, :, None] * X[:, None, 0] + l2[None, :, None] * X[:, None, 1] + l3[None, :, None] * X[:, None, 2]
    top = l1[None, :, None] * X[:, None, 3] + l2[None, :, None] * X[:, None, 4] + l3[None, :, None] * X[:, None, 5]
    return 0.5 * (1.0 - c)[None, :, None] * bot + 0.5 * (1.0 + c)[None, :, None] * top


def tet_map(ref, X):
    """map_tet_to_physical: ref (n,3), X (N,4,3) -> (N,n,3)."""
    a, b, c = ref[:, 0], ref[:, 1], ref[:, 2]
    t = c
    s = (1.0 + b) * (1.0 - c) / 2.0 - 1.0
    r = -(1.0 + a) * (s + t) / 2.0 - 1.0
    L = [-(1.0 + r + s + t) / 2.0, (1.0 + r) / 2.0, (1.0 + s) / 2.0, (1.0 + t) / 2.0]
    out = L[0][None, :, None] * X[:, None, 0]
    for k in range(1, 4):
        out = out + L[k][None, :, None] * X[:, None, k]
    return out


def prism_jacobian(ref, X):
    """prism_exact_jacobian (curved_mapping_exact_jacobian.py:76-119), vectorised: -> (N,n,3,3)."""
    a, b, c = ref[:, 0], ref[:, 1], ref[:, 2]
    p = [X[:, None, i, :] for i in range(6)]  # (N,1,3)
    e = lambda v: v[None, :, None]  # noqa: E731
    d_bot_da = e((1.0 - b) / 4.0) * (p[1] - p[0])
    d_top_da = e((1.0 - b) / 4.0) * (p[4] - p[3])
    d_bot_db = e(-(1.0 - a) / 4.0) * p[0] + e(-(1.0 + a) / 4.0) * p[1] + 0.5 * p[2]
    d_top_db = e(-(1.0 - a) / 4.0) * p[3] + e(-(1.0 + a) / 4.0) * p[4] + 0.5 * p[5]
    r = (1.0 + a) * (1.0 - b) / 2.0 - 1.0
    s = b
    l1, l2, l3 = -(r + s) / 2.0, (1.0 + r) / 2.0, (1.0 + s) / 2.0
    bot = e(l1) * p[0] + e(l2) * p[1] + e(l3) * p[2]
    top = e(l1) * p[3] + e(l2) * p[4] + e(l3) * p[5]
    J = np.empty(X.shape[:1] + ref.shape[:1] + (3, 3))
    J[..., 0] = 0.5 * e(1.0 - c) * d_bot_da + 0.5 * e(1.0 + c) * d_top_da
    J[..., 1] = 0.5 * e(1.0 - c) * d_bot_db + 0.5 * e(1.0 + c) * d_top_db
    J[..., 2] = 0.5 * (top - bot)
    return J


def tet_jacobian(ref, X):
    """tet_exact_jacobian (curved_mapping_exact_jacobian.py:39-73), vectorised: -> (N,n,3,3)."""
    a, b, c = ref[:, 0], ref[:, 1], ref[:, 2]
    p0, p1, p2, p3 = (X[:, None, i, :] for i in range(4))
    e1 = (p1 - p0) / 2.0
    e2 = (p2 - p0) / 2.0
    e3 = (p3 - p0) / 2.0
    s = (1.0 + b) * (1.0 - c) / 2.0 - 1.0
    t = c
    e = lambda v: v[None, :, None]  # noqa: E731
    J = np.empty(X.shape[:1] + ref.shape[:1] + (3, 3))
    J[..., 0] = e(-(s + t) / 2.0) * e1
    J[..., 1] = e(-(1.0 + a) * (1.0 - c) / 4.0) * e1 + e((1.0 - c) / 2.0) * e2
    J[..., 2] = e(-(1.0 + a) * (1.0 - b) / 4.0) * e1 + e(-(1.0 + b) / 2.0) * e2 + e3
    return J


def det_inv(J):
    """batched_det_inv_3x3 (grid/curved_mapping/curved_mapping.py:39-91): cofactor closed form."""
    m = [[J[..., i, j] for j in range(3)] for i in range(3)]
    c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1]
    c01 = -(m[1][0] * m[2][2] - m[1][2] * m[2][0])
    c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0]
    c10 = -(m[0][1] * m[2][2] - m[0][2] * m[2][1])
    c11 = m[0][0] * m[2][2] - m[0][2] * m[2][0]
    c12 = -(m[0][0] * m[2][1] - m[0][1] * m[2][0])
    c20 = m[0][1] * m[1][2] - m[0][2] * m[1][1]
    c21 = -(m[0][0] * m[1][2] - m[0][2] * m[1][0])
    c22 = m[0][0] * m[1][1] - m[0][1] * m[1][0]
    d = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02
    inv_d = 1.0 / d
    inv = np.empty(J.shape)
    inv[..., 0, 0], inv[..., 0, 1], inv[..., 0, 2] = c00 * inv_d, c10 * inv_d, c20 * inv_d
    inv[..., 1, 0], inv[..., 1, 1], inv[..., 1, 2] = c01 * inv_d, c11 * inv_d, c21 * inv_d
    inv[..., 2, 0], inv[..., 2, 1], inv[..., 2, 2] = c02 * inv_d, c12 * inv_d, c22 * inv_d
    return d, inv


def _geometry(X, kind, ref, chunk=16384):
    """det / inverse Jacobian at ``ref`` points of every cell, in cell chunks
    spread over host threads (numpy releases the GIL in these kernels)."""
    from concurrent.futures import ThreadPoolExecutor

    jac = prism_jacobian if kind == "prism" else tet_jacobian
    N, n = X.shape[0], ref.shape[0]
    det = np.empty((N, n))
    inv = np.empty((N, n, 3, 3))

    def work(s):
        d, iv = det_inv(jac(ref, X[s:s + chunk]))
        det[s:s + chunk] = d
        inv[s:s + chunk] = iv

    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        list(ex.map(work, range(0, N, chunk)))
    if np.any(det <= 0):
        raise ValueError("non-positive Jacobian determinant: the mesh is tangled")
    return det, inv


# ---------------------------------------------------------------------------
# template replay
# ---------------------------------------------------------------------------
def _cell_index(box: BoxMesh, H, kind):
    nx, ny, nz = box.shape
    i, j, k = H[..., 0], H[..., 1], H[..., 2]
    if box.kind == "prism":
        return ((i * ny + j) * 2 + kind) * nz + k
    return ((i * ny + j) * nz + k) * 6 + kind


def _template_pos(H, n):
    """Topological position along an axis: 0 low boundary, 1 interior, 2 high boundary."""
    return np.where(H == 0, 0, np.where(H == n - 1, 2, 1))


def _rel_cells(box, H, rel):
    """Cells at hex H + rel[:, :3] of kind rel[:, 3] (-1 where kind < 0)."""
    out = np.full(H.shape[0], -1, np.int64)
    ok = rel[:, 3] >= 0
    Hn = H[ok] + rel[ok, :3]
    n = np.array(box.shape)
    if box.periodic:
        Hn = Hn % n
    elif np.any((Hn < 0) | (Hn >= n)):
        raise ValueError("template replay left the box")
    out[ok] = _cell_index(box, Hn, rel[ok, 3])
    return out


def build_case(box: BoxMesh, order: int, plane_cfg: Optional[dict] = None, wall_distance: bool = False,
               want_sps_coords: bool = False, colorer=None) -> Dict[str, np.ndarray]:
    """Flattened FR case for ``box`` at polynomial order ``order``.

    Args:
        colorer: ``f(owner, neighbor, is_boundary, n_cells) -> colors``; the
            default is the library's C++ greedy coloring.  A caller that must
            not load the library passes another implementation of the same
            rule.
        plane_cfg: boundary configuration per plane name (PLANE_NAMES), dicts
            as the reference's BoundaryGhostStateProvider takes
            ({"type": "WALL", "is_no_slip": True}, {"type": "FARFIELD",
            "Q_free": [...]}, ...); ignored for periodic boxes.
        wall_distance: compute the SP wall distance to the WALL planes.
    """
    T = load_template(box.kind, order)
    n1d = order + 1
    S, P = n1d**3, n1d**2
    if box.periodic and min(box.shape) < 3:
        raise ValueError("periodic boxes need at least 3 hexes per axis")
    conn = boxmesh.orient_cells(box)
    X = box.nodes[conn]
    N = box.n_cells
    is_prism = box.kind == "prism"
    case: Dict[str, np.ndarray] = dict(
        order=np.int32(order), n_cells=np.int32(N), n_prism=np.int32(N if is_prism else 0), n_sps=np.int32(S),
        box_kind=np.array(box.kind), box_shape=np.array(box.shape), box_lengths=np.array(box.lengths),
        periodic=np.int32(box.periodic))
    # ---- geometry ----
    ref = ref_grid(T["sps_1d"])
    reff = ref_grid(T["fine_1d"])
    case["n_fine"] = np.int32(reff.shape[0])
    case["det_jacs"], case["inv_jacs"] = _geometry(X, box.kind, ref)
    case["det_jacs_fine"], case["inv_jacs_fine"] = _geometry(X, box.kind, reff)
    w = T["w_1d"]
    wx, wy, wz = np.meshgrid(w, w, w, indexing="ij")
    w3 = (wx * wy * wz).ravel()
    case["cell_volumes"] = np.sum(case["det_jacs"] * w3[None, :], axis=1)
    # ---- operators ----
    for k in ("D_3d_prism", "D_3d_tet", "c2f_prism", "c2f_tet", "Dfine_prism", "Dfine_tet", "f2c_prism",
              "f2c_tet", "filter_prism", "filter_tet", "boundary_extrap", "g_left", "g_right", "dist_fp_of_sp",
              "dist_axis_coord_of_sp"):
        if k in T:  # order 0 has no over-integration operators
            case[k] = T[k]
    # ---- face records replayed from the template ----
    n = np.array(box.shape)
    H = box.hex_index
    tpos = _template_pos(H, n[None, :])
    tmpl_box_shape = (int(T["template"]),) * 3
    tc = _cell_index(BoxMesh(box.kind, None, None, None, None, tmpl_box_shape, (1.0, 1.0, 1.0)), tpos,
                     box.local_kind)
    ptr = T["cell_ptr"]
    cnt = ptr[tc + 1] - ptr[tc]
    owner = np.repeat(np.arange(N, dtype=np.int64), cnt)
    start = np.repeat(ptr[tc], cnt)
    within = np.arange(owner.shape[0]) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    r = start + within  # template record per full record
    Ho = H[owner]
    F = owner.shape[0]
    case["owner_cell"] = owner
    case["neighbor_cell"] = _rel_cells(box, Ho, T["rec_nb"][r])
    for k_out, k_in in (("owner_axis", "rec_o_axis"), ("owner_side", "rec_o_side"), ("neighbor_axis", "rec_n_axis"),
                        ("neighbor_side", "rec_n_side"), ("is_boundary", "rec_is_boundary"),
                        ("owner_is_primary", "rec_o_primary"), ("neighbor_is_primary", "rec_n_primary")):
        case[k_out] = T[k_in][r]
    mat = T["rec_mat"][r]  # (F,4): nb0, ow0, nb1, ow1 indices into T["mats"]
    case["src_mat_table"] = T["mats"]
    for which, c0k, c1k, col0, col1 in (("nb", "rec_nb_src0", "rec_nb_src1", 0, 2),
                                          ("ow", "rec_ow_src0", "rec_ow_src1", 1, 3)):
        c0 = _rel_cells(box, Ho, T[c0k][r])
        c1 = _rel_cells(box, Ho, T[c1k][r])
        case[which + "_src0_cell"] = c0
        case[which + "_src0_mat_index"] = mat[:, col0].astype(np.int32)
        has1 = c1 >= 0
        idx1 = np.full(F, -1, np.int64)
        idx1[has1] = np.arange(int(has1.sum()))
        case[which + "_src1_idx"] = idx1
        case[which + "_src1_cell"] = c1[has1]
        case[which + "_src1_mat_index"] = mat[has1, col1].astype(np.int32)
    # ---- face normals and areas from the owner's triangle ----
    lat = Ho[:, None, :] + T["rec_tri"][r]  # (F,3,3) node lattice coordinates
    nx, ny, _ = box.shape
    nid = lat[..., 0] + (nx + 1) * lat[..., 1] + (nx + 1) * (ny + 1) * lat[..., 2]
    nid = np.sort(nid, axis=1)
    p0, p1, p2 = (box.nodes[nid[:, i]] for i in range(3))
    avec = 0.5 * np.cross(p1 - p0, p2 - p0)
    fcen = (p0 + p1 + p2) / 3.0
    ocen = np.mean(box.nodes[conn], axis=1)[owner]
    flip = np.sum(avec * (fcen - ocen), axis=1) < 0
    avec[flip] *= -1
    area = np.linalg.norm(avec, axis=1)
    nrm = avec / area[:, None]
    case["true_normal"] = np.ascontiguousarray(np.broadcast_to(nrm[:, None, :], (F, P, 3)))
    wx2, wy2 = np.meshgrid(w, w, indexing="ij")
    rel_w = (wx2 * wy2).ravel()
    rel_w = rel_w / np.sum(rel_w)
    case["true_area_weight"] = np.outer(area, rel_w)
    case["face_node_ids"] = nid
    # ---- colors ----
    if colorer is None:
        from ._lib import greedy_face_coloring as colorer
    case["colors"] = colorer(owner, case["neighbor_cell"], case["is_boundary"], N)
    # ---- boundary conditions ----
    isb = case["is_boundary"].astype(bool)
    plane = np.full(F, -1, np.int64)
    if np.any(isb):
        plane[isb] = box.plane_of_faces(nid[isb])
        if np.any(plane[isb] < 0):
            raise ValueError("boundary face off the box planes")
    _bc_tables(case, plane, plane_cfg, box, conn)
    if wall_distance or want_sps_coords:
        xyz = (prism_map if is_prism else tet_map)(ref, X)
        if want_sps_coords:
            case["sps_coords"] = xyz
        if wall_distance:
            case["wall_distance"] = _wall_distance(box, plane_cfg, xyz)
    return case


def _bc_tables(case, plane, plane_cfg, box, conn):
    """Boundary table rows = planes (+ a FARFIELD default row), as the
    reference's face-exact ghost provider (tests/validation/_channel_mesh.py:19-66)."""
    n = len(PLANE_NAMES) + 1
    t = np.full(n, BC_CODES["FARFIELD"], np.int32)
    ns = np.ones(n, np.int32)
    wv = np.zeros((n, 3))
    Q = np.zeros((n, 5))
    po = np.zeros(n)
    cfg = plane_cfg or {}
    for i, name in enumerate(PLANE_NAMES):
        c = cfg.get(name)
        if c is None:
            continue
        t[i] = BC_CODES[c["type"]]
        ns[i] = 1 if c.get("is_no_slip", True) else 0
        if c.get("wall_velocity") is not None:
            wv[i] = c["wall_velocity"]
        if "Q_free" in c:
            Q[i] = c["Q_free"]
        if "Q_inlet" in c:
            Q[i] = c["Q_inlet"]
        po[i] = float(c.get("p_outlet", 0.0))
    default = cfg.get("_default_Q", [1.225, 0.0, 0.0, 0.0, 101325.0])
    Q[n - 1] = default
    g = np.where(plane >= 0, plane, n - 1).astype(np.int32)
    case.update(bc_group=g, bc_type=t, bc_noslip=ns, bc_wall_vel=wv, bc_Q=Q, bc_p_out=po, bc_default=np.int32(n - 1))
    # force-integration faces: the reference tags a boundary face with the
    # last plane group (x_min..z_max order) containing its owner cell
    # (grid/connectivity/face_connectivity.py:234-272), WALL no-slip planes count
    if plane_cfg is not None:
        ijk = box.node_ijk(conn)
        owner = case["owner_cell"]
        code = np.full(owner.shape[0], -1, np.int64)
        isb = case["is_boundary"].astype(bool)
        for gi, (ax, val) in enumerate(((0, 0), (0, box.shape[0]), (1, 0), (1, box.shape[1]), (2, 0),
                                        (2, box.shape[2]))):
            member = (ijk[:, :, ax] == val).sum(axis=1) >= 3
            code[isb & member[owner]] = gi
        wall_planes = [i for i, nme in enumerate(PLANE_NAMES)
                       if cfg.get(nme, {}).get("type") == "WALL" and cfg.get(nme, {}).get("is_no_slip", True)]
        case["cd_wall_face"] = np.isin(code, wall_planes).astype(np.uint8)


def _wall_distance(box, plane_cfg, xyz):
    """Distance from every SP to the nearest node of a no-slip WALL plane
    (compute_wall_distance_field, core/fr_solver/turbulence.py:112-125)."""
    from scipy.spatial import cKDTree

    cfg = plane_cfg or {}
    lat = box.node_ijk(np.arange(box.nodes.shape[0]))
    mask = np.zeros(box.nodes.shape[0], bool)
    for i, (ax, val) in enumerate(((0, 0), (0, box.shape[0]), (1, 0), (1, box.shape[1]), (2, 0), (2, box.shape[2]))):
        c = cfg.get(PLANE_NAMES[i], {})
        if c.get("type") == "WALL":
            mask |= lat[:, ax] == val
    if not np.any(mask):
        raise ValueError("wall distance requested but no WALL plane configured")
    tree = cKDTree(box.nodes[mask])
    d, _ = tree.query(xyz.reshape(-1, 3), k=1, workers=-1)
    return d.reshape(xyz.shape[:2])

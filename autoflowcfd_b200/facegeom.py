"""Flux-point construction: the flattened face tables of a prism / tet mesh
(owner and neighbour sides, primary flags, normals, area weights, the
cross-interpolation matrices and the face colors) from its face connectivity,
with the per-face Newton location and interpolation rows on the device
(``afr_flux_point_jobs``).

Restates (paths relative to the reference's src/autoflowcfd):

* build_face_flux_points, fr/face_flux_points_merge.py:51-434: one record per
  (cell, cube face) group is primary (prism quad faces are split into two
  records; the lower face index of a group is primary), the neighbour side of
  an owner-primary record and the owner side of a neighbour-primary record
  are located on the other cell, a prism quad face's primary record carries
  the rows of its half of the quad (the diagonal classification) and a
  second-source matrix with the other half, located on the other record's
  cell;
* _prism_quad_diagonal_local / _quad_half_sets / _classify_half,
  fr/face_flux_points_data.py:123-187;
* _get_v_sps_lu, fr/face_flux_points.py:59-74: the inverse of the modal
  Vandermonde matrix at the solution points by an LU solve;
* tet_modal_basis_and_grad / prism_modal_basis_and_grad (values),
  fr/collapsed_basis.py:51-231;
* build_flat_face_geometry, core/fr_operators/face_kernels.py:228-341: the
  flattened arrays and the greedy face colors.

The per-record work (Newton or closed-form location of every flux point, the
modal basis at the located points and the rows V * V_inv) runs in
``csrc/afr_facegeom.cu``, one warp per record side.  The host does the O(F)
grouping and the small dense LU.
"""

import ctypes
from typing import Dict

import numpy as np

from . import _lib
from ._lib import LIB

FACE_AXIS = np.array([0, 0, 1, 1, 2, 2], dtype=np.int64)
FACE_SIDE = np.array([-1.0, 1.0, -1.0, 1.0, -1.0, 1.0])
QUAD_CODES = (0, 1, 2)  # a=-1, a=+1, b=-1: the prism's quad faces
# local corner indices of the prism's faces by cube-face code (grid/curved_mapping/curved_mapping.py:236-242)
QUAD_LOCAL = np.array([[0, 2, 5, 3], [1, 2, 5, 4], [0, 1, 4, 3]], dtype=np.int64)


def gauss_legendre(n: int):
    """1-D Gauss-Legendre points and weights (fr/quadrature_points.py:16-28)."""
    return np.polynomial.legendre.leggauss(n)


def jacobi(x: np.ndarray, alpha: float, beta: float, n: int) -> np.ndarray:
    """Unnormalised Jacobi polynomial P_n^(alpha,beta)(x), three-term recurrence."""
    P0 = np.ones_like(x)
    if n == 0:
        return P0
    P1 = 0.5 * ((alpha - beta) + (alpha + beta + 2.0) * x)
    if n == 1:
        return P1
    Pm, P = P0, P1
    for k in range(1, n):
        a1 = 2.0 * (k + 1) * (k + alpha + beta + 1) * (2 * k + alpha + beta)
        a2 = (2 * k + alpha + beta + 1) * (alpha**2 - beta**2)
        a3 = (2 * k + alpha + beta) * (2 * k + alpha + beta + 1) * (2 * k + alpha + beta + 2)
        a4 = 2.0 * (k + alpha) * (k + beta) * (2 * k + alpha + beta + 2)
        Pm, P = P, ((a2 + a3 * x) * P - a4 * Pm) / a1
    return P


def int_power(x: np.ndarray, n: int) -> np.ndarray:
    """x**n for an integer n >= 1 by square-and-multiply from 1 (the
    rounding of the reference's compiled ``x**i`` with an integer exponent)."""
    r = np.ones_like(x)
    a = np.array(x, dtype=np.float64, copy=True)
    e = n
    while True:
        if e & 1:
            r = r * a
        e >>= 1
        if not e:
            break
        a = a * a
    return r


def modal_vandermonde(kind: str, order: int, a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """(n_pts, (order+1)^3) values of the collapsed modal basis, modes flat =
    i*(order+1)^2 + j*(order+1) + k:
    prism phi = g_ij(a,b) P_k(c); tet psi = g_ij(a,b) ((1-c)/2)^(i+j) P_k^(2i+2j+2,0)(c),
    g_ij = P_i(a) ((1-b)/2)^i P_j^(2i+1,0)(b)."""
    n1d = order + 1
    V = np.zeros((len(a), n1d**3))
    h1b, h1c = (1.0 - b) / 2.0, (1.0 - c) / 2.0
    for i in range(n1d):
        fi = jacobi(a, 0.0, 0.0, i)
        wi = np.ones_like(h1b) if i == 0 else int_power(h1b, i)
        for j in range(n1d):
            g = fi * (wi * jacobi(b, float(2 * i + 1), 0.0, j))
            p = i + j
            w = np.ones_like(h1c) if p == 0 else int_power(h1c, p)
            for k in range(n1d):
                flat = i * n1d * n1d + j * n1d + k
                if kind == "prism":
                    V[:, flat] = g * jacobi(c, 0.0, 0.0, k)
                else:
                    V[:, flat] = g * (w * jacobi(c, float(2 * i + 2 * j + 2), 0.0, k))
    return V


def vandermonde_inverse(kind: str, order: int) -> np.ndarray:
    """V_sps^-1 from an LU solve of V_sps^T (the solution points are the
    Gauss-Legendre tensor grid)."""
    from scipy.linalg import lu_factor, lu_solve

    sps = gauss_legendre(order + 1)[0]
    ga, gb, gc = np.meshgrid(sps, sps, sps, indexing="ij")
    V = modal_vandermonde(kind, order, ga.ravel(), gb.ravel(), gc.ravel())
    return np.ascontiguousarray(lu_solve(lu_factor(V.T), np.eye(V.shape[0])).T)


def _groups(member: np.ndarray, key: np.ndarray):
    """Faces of ``member`` grouped by ``key``: (non-first members, the second
    member of each group indexed by its first member (the first itself for a
    group of one))."""
    F = member.shape[0]
    idx = np.flatnonzero(member)
    k = key[idx]
    order = np.lexsort((idx, k))
    sidx, sk = idx[order], k[order]
    start = np.ones(len(sidx), bool)
    start[1:] = sk[1:] != sk[:-1]
    gstart = np.flatnonzero(start)
    glen = np.diff(np.append(gstart, len(sidx)))
    second = np.full(F, -1, np.int64)
    if len(gstart):
        second[sidx[gstart]] = np.where(glen >= 2, sidx[np.minimum(gstart + 1, len(sidx) - 1)], sidx[gstart])
    return sidx[~start], second


def _same_pair(a, b, c, d):
    return ((a == c) & (b == d)) | ((a == d) & (b == c))


def half_masks(cells6: np.ndarray, codes: np.ndarray, face_nodes: np.ndarray, order: int) -> np.ndarray:
    """Bit p set where flux point p of the prism quad face ``codes`` of the
    cells ``cells6`` (global node ids) lies in the half covered by the record
    with corner ids ``face_nodes`` (_classify_half with the diagonal rule of
    the mesh's quad triangulation: bottom corners sorted by global id
    v0' < v1' < v2', diagonals v0'-w1', v1'-w2', v0'-w2')."""
    n = cells6.shape[0]
    if n == 0:
        return np.zeros(0, np.uint32)
    quad = QUAD_LOCAL[codes]
    srt = np.argsort(cells6[:, :3], axis=1, kind="stable")
    v, w = srt, srt + 3
    e0, e1 = quad[:, 0], quad[:, 1]
    m01 = _same_pair(e0, e1, v[:, 0], v[:, 1])
    m12 = _same_pair(e0, e1, v[:, 1], v[:, 2])
    m02 = _same_pair(e0, e1, v[:, 0], v[:, 2])
    if not np.all(m01 | m12 | m02):
        raise RuntimeError("prism quad face whose bottom edge is not an edge of the base triangle")
    d_bot = np.where(m01, v[:, 0], np.where(m12, v[:, 1], v[:, 0]))
    d_top = np.where(m01, w[:, 1], np.where(m12, w[:, 2], w[:, 2]))
    i0, i1, i2, i3 = quad.T
    std = _same_pair(d_bot, d_top, i0, i2)
    flip = _same_pair(d_bot, d_top, i1, i3)
    if not np.all(std | flip):
        raise RuntimeError("quad diagonal is not a diagonal of its corners")
    lower = np.where(std[:, None], np.stack([i0, i1, i2], 1), np.stack([i0, i1, i3], 1))
    upper = np.where(std[:, None], np.stack([i0, i2, i3], 1), np.stack([i1, i2, i3], 1))
    lower_g = np.sort(np.take_along_axis(cells6, lower, 1), 1)
    upper_g = np.sort(np.take_along_axis(cells6, upper, 1), 1)
    fs = np.sort(face_nodes, 1)
    is_low = np.all(fs == lower_g, 1)
    is_up = np.all(fs == upper_g, 1)
    if not np.all(is_low | is_up):
        raise RuntimeError("face corners match neither half of the prism quad face")
    sps = gauss_legendre(order + 1)[0]
    g1, g2 = np.meshgrid(sps, sps, indexing="ij")
    low_std, low_flip = (g1.ravel() >= g2.ravel()), (g1.ravel() + g2.ravel()) <= 0.0
    is_lower = np.where(std[:, None], low_std[None, :], low_flip[None, :])
    m = np.where(is_low[:, None], is_lower, ~is_lower)
    return (m.astype(np.uint64) << np.arange(m.shape[1], dtype=np.uint64)).sum(1).astype(np.uint32)


def distribution_maps(n1d: int):
    """(fp_of_sp, axis_coord_of_sp), each (3, n1d^3): the lifting of a face's
    flux-point row onto the solution points along `axis` (the index form of
    _distribute_from_face, core/fr_operators/face_kernels.py:68-115): point
    (i0, i1, i2) takes g'[i_axis] times flux point (i_o0 * n1d + i_o1), o0 < o1
    the other two axes."""
    S = n1d**3
    idx = np.array(np.unravel_index(np.arange(S), (n1d, n1d, n1d)))  # (3, S): i0, i1, i2
    fp = np.empty((3, S), np.int64)
    co = np.empty((3, S), np.int64)
    for ax in range(3):
        o0, o1 = [a for a in range(3) if a != ax]
        fp[ax] = idx[o0] * n1d + idx[o1]
        co[ax] = idx[ax]
    return fp, co


def operator_face_tables(ops, order: int) -> Dict[str, np.ndarray]:
    """The per-order face tables that come from the operators, not the mesh:
    the boundary extrapolation matrices by (cell type, axis, side), g' at the
    two ends and the distribution maps (core/fr_operators/face_kernels.py:297-305)."""
    n1d = order + 1
    P, S = n1d * n1d, n1d**3
    ext = np.zeros((2, 3, 2, P, S))
    for axis in range(3):
        for si, side in enumerate((-1.0, 1.0)):
            ext[0, axis, si] = ops.boundary_extrap_prism[(axis, side)]
            ext[1, axis, si] = ops.boundary_extrap_tet[(axis, side)]
    fp, co = distribution_maps(n1d)
    return dict(boundary_extrap=ext, g_left=np.asarray(ops.g_left, np.float64),
                g_right=np.asarray(ops.g_right, np.float64), dist_fp_of_sp=fp, dist_axis_coord_of_sp=co)


def _get(fc, name):
    return np.asarray(fc[name] if isinstance(fc, dict) else getattr(fc, name))


def plan_jobs(face_conn, prism_conn, tet_conn, order: int) -> Dict:
    """Host half of the construction: primary flags, the split-quad halves
    and the locate jobs (one per face side that reads the other cell): the
    owner-primary records' neighbour sides, the neighbour-primary records'
    owner sides, then the second halves of split prism quad faces."""
    prism_conn = np.asarray(prism_conn, np.int64).reshape(-1, 6)
    tet_conn = np.asarray(tet_conn, np.int64).reshape(-1, 4)
    n_prism = prism_conn.shape[0]
    oc = _get(face_conn, "owner_cell").astype(np.int64)
    nc = _get(face_conn, "neighbor_cell").astype(np.int64)
    occ = _get(face_conn, "owner_cube_face").astype(np.int64)
    ncc = _get(face_conn, "neighbor_cube_face").astype(np.int64)
    fnodes = np.asarray(_get(face_conn, "face_node_ids"), np.int64)
    isb = _get(face_conn, "is_boundary").astype(bool)
    F = oc.shape[0]
    inner = ~isb
    o_pq = (oc < n_prism) & np.isin(occ, QUAD_CODES)
    n_pq = inner & (nc >= 0) & (nc < n_prism) & np.isin(ncc, QUAD_CODES)

    # primary records: the first (lowest face index) of each (cell, cube face) group
    own_key, nb_key = oc * 6 + occ, np.where(nc >= 0, nc, 0) * 6 + np.where(ncc >= 0, ncc, 0)
    own_drop, own_second = _groups(inner & o_pq, own_key)
    nb_drop, nb_second = _groups(n_pq, nb_key)
    bnd_drop, _ = _groups(isb & o_pq, own_key)
    opr = np.ones(F, bool)
    npr = np.ones(F, bool)
    opr[own_drop] = False
    opr[bnd_drop] = False
    npr[nb_drop] = False

    ms_nb = np.flatnonzero(inner & opr & o_pq)
    ms_ow = np.flatnonzero(inner & npr & n_pq)
    nb_mask = np.zeros(F, np.uint32)
    ow_mask = np.zeros(F, np.uint32)
    nb_mask[ms_nb] = half_masks(prism_conn[oc[ms_nb]], occ[ms_nb], fnodes[ms_nb], order)
    ow_mask[ms_ow] = half_masks(prism_conn[nc[ms_ow]], ncc[ms_ow], fnodes[ms_ow], order)

    main_nb = np.flatnonzero(inner & opr)
    main_ow = np.flatnonzero(inner & npr)
    sec_nb_other, sec_ow_other = own_second[ms_nb], nb_second[ms_ow]
    jobs = {
        "face": np.concatenate([main_nb, main_ow, ms_nb, ms_ow]),
        "src_cell": np.concatenate([oc[main_nb], nc[main_ow], oc[ms_nb], nc[ms_ow]]),
        "src_code": np.concatenate([occ[main_nb], ncc[main_ow], occ[ms_nb], ncc[ms_ow]]),
        "tgt_cell": np.concatenate([nc[main_nb], oc[main_ow], nc[sec_nb_other], oc[sec_ow_other]]),
        "tgt_code": np.concatenate([ncc[main_nb], occ[main_ow], ncc[sec_nb_other], occ[sec_ow_other]]),
        "sign": np.concatenate([np.full(len(main_nb), -1), np.full(len(main_ow), 1), np.full(len(ms_nb), -1),
                                np.full(len(ms_ow), 1)]),
        "mode": np.concatenate([o_pq[main_nb].astype(np.int64), n_pq[main_ow].astype(np.int64),
                                np.full(len(ms_nb), 2), np.full(len(ms_ow), 2)]),
        "mask": np.concatenate([nb_mask[main_nb], ow_mask[main_ow], nb_mask[ms_nb], ow_mask[ms_ow]]),
    }
    return dict(F=F, oc=oc, nc=nc, occ=occ, ncc=ncc, isb=isb, opr=opr, npr=npr, ms_nb=ms_nb, ms_ow=ms_ow,
                main_nb=main_nb, main_ow=main_ow, nb_mask=nb_mask, ow_mask=ow_mask, jobs=jobs,
                prism_conn=prism_conn, tet_conn=tet_conn)


def flux_point_tables(face_conn, prism_conn, tet_conn, nodes, order: int, colorer=None,
                      timings: Dict = None) -> Dict[str, np.ndarray]:
    """The flattened face tables of a mesh (the keys ``afr_create`` takes).

    Args:
        face_conn: the reference's FRFaceConnectivity (or a dict with its
            fields owner_cell, neighbor_cell, owner_cube_face,
            neighbor_cube_face, area, normal, face_node_ids, is_boundary,
            face_translation).
        prism_conn: (n_prism, 6) node ids, prisms first in the cell order;
        tet_conn: (n_tet, 4) node ids; nodes: (n_nodes, 3).
        colorer: ``f(owner, neighbor, is_boundary, n_cells) -> colors``
            (default: the library's greedy coloring).
        timings: optional dict that receives the wall seconds of the host
            planning ("plan_s"), the device jobs with their transfers
            ("device_s") and the assembly with the colors ("assemble_s").
    Returns owner / neighbour cells and sides, primary flags, true normals
    and area weights, the source cells and interpolation matrices (dense,
    with the compact second-source table), colors, and the raw Newton
    coordinates and residuals (``nb_fc``, ``ow_fc``, ``nb_resid``,
    ``ow_resid``)."""
    import time

    t0 = time.perf_counter()
    pl = plan_jobs(face_conn, prism_conn, tet_conn, order)
    F, oc, nc, occ, ncc, isb = pl["F"], pl["oc"], pl["nc"], pl["occ"], pl["ncc"], pl["isb"]
    opr, npr, ms_nb, ms_ow, main_nb, main_ow = (pl[k] for k in ("opr", "npr", "ms_nb", "ms_ow", "main_nb",
                                                                 "main_ow"))
    jobs, prism_conn, tet_conn = pl["jobs"], pl["prism_conn"], pl["tet_conn"]
    nodes = np.ascontiguousarray(nodes, np.float64)
    n_prism, n_tet = prism_conn.shape[0], tet_conn.shape[0]
    n1d = order + 1
    P, S = n1d * n1d, n1d**3
    area = np.ascontiguousarray(_get(face_conn, "area"), np.float64)
    normal = np.asarray(_get(face_conn, "normal"), np.float64)
    tr = face_conn.get("face_translation") if isinstance(face_conn, dict) else getattr(face_conn, "face_translation",
                                                                                       None)
    trans = np.zeros((F, 3)) if tr is None else np.ascontiguousarray(tr, np.float64).reshape(F, 3)
    J = len(jobs["face"])
    t1 = time.perf_counter()
    mats = np.zeros((J, P, S))
    coords = np.zeros((J, P, 2))
    resid = np.zeros(J)
    if J:
        arr = {k: np.ascontiguousarray(v, np.uint32 if k == "mask" else np.int32) for k, v in jobs.items()}
        vinv_p = vandermonde_inverse("prism", order) if n_prism else None
        vinv_t = vandermonde_inverse("tet", order) if n_tet else None
        pc = np.ascontiguousarray(prism_conn, np.int32)
        tc = np.ascontiguousarray(tet_conn, np.int32)
        sps = np.ascontiguousarray(gauss_legendre(n1d)[0])
        P_D, P_I, P_U = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint32)
        pd = lambda a: None if a is None else a.ctypes.data_as(P_D)
        rc = LIB.afr_flux_point_jobs(
            order, n_prism, n_tet, nodes.shape[0], pd(nodes), pc.ctypes.data_as(P_I), tc.ctypes.data_as(P_I),
            pd(vinv_p), pd(vinv_t), pd(sps), F, pd(area), pd(trans), J,
            *[arr[k].ctypes.data_as(P_I) for k in ("face", "src_cell", "src_code", "tgt_cell", "tgt_code", "sign",
                                                     "mode")],
            arr["mask"].ctypes.data_as(P_U), pd(mats), pd(coords), pd(resid))
        _lib.check(rc)
    t2 = time.perf_counter()
    a, b, c = len(main_nb), len(main_nb) + len(main_ow), len(main_nb) + len(main_ow) + len(ms_nb)

    def dense(faces, rows):
        out = np.zeros((F, P, S))
        out[faces] = rows
        return out

    nb_src0_cell = np.full(F, -1, np.int64)
    ow_src0_cell = np.full(F, -1, np.int64)
    nb_src0_cell[main_nb] = nc[main_nb]
    ow_src0_cell[main_ow] = oc[main_ow]
    nb_src1_idx = np.full(F, -1, np.int64)
    ow_src1_idx = np.full(F, -1, np.int64)
    nb_src1_idx[ms_nb] = np.arange(len(ms_nb))
    ow_src1_idx[ms_ow] = np.arange(len(ms_ow))
    nb_fc = np.zeros((F, P, 2))
    ow_fc = np.zeros((F, P, 2))
    nb_fc[main_nb], ow_fc[main_ow] = coords[:a], coords[a:b]
    nb_resid, ow_resid = np.zeros(F), np.zeros(F)
    nb_resid[main_nb], ow_resid[main_ow] = resid[:a], resid[a:b]
    sps, w = gauss_legendre(n1d)
    wx, wy = np.meshgrid(w, w, indexing="ij")
    rel_w = (wx * wy).ravel()
    rel_w = rel_w / np.sum(rel_w)
    if colorer is None:
        colorer = _lib.greedy_face_coloring
    colors = colorer(oc, nc, isb.astype(np.uint8), n_prism + n_tet)
    if timings is not None:
        timings.update(plan_s=t1 - t0, device_s=t2 - t1, assemble_s=time.perf_counter() - t2, n_jobs=J)
    return dict(
        owner_cell=oc, neighbor_cell=nc, is_boundary=isb.astype(np.uint8),
        owner_axis=FACE_AXIS[occ], owner_side=FACE_SIDE[occ],
        neighbor_axis=np.where(isb, -1, FACE_AXIS[np.maximum(ncc, 0)]),
        neighbor_side=np.where(isb, 0.0, FACE_SIDE[np.maximum(ncc, 0)]),
        owner_is_primary=opr.astype(np.uint8), neighbor_is_primary=npr.astype(np.uint8),
        true_normal=np.repeat(normal, P, axis=0).reshape(F, P, 3),
        true_area_weight=np.outer(area, rel_w),
        nb_src0_cell=nb_src0_cell, nb_src0_mat=dense(main_nb, mats[:a]), nb_src1_idx=nb_src1_idx,
        nb_src1_cell=nc[ms_nb].astype(np.int64), nb_src1_mat=mats[b:c],
        ow_src0_cell=ow_src0_cell, ow_src0_mat=dense(main_ow, mats[a:b]), ow_src1_idx=ow_src1_idx,
        ow_src1_cell=oc[ms_ow].astype(np.int64), ow_src1_mat=mats[c:],
        colors=np.asarray(colors, np.int32),
        nb_fc=nb_fc, ow_fc=ow_fc, nb_resid=nb_resid, ow_resid=ow_resid,
    )

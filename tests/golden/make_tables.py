"""Harvest the reference-space tables the box-mesh generator needs.

Runs the reference (AutoFlowCFD, a checkout named by ``AFR_REFERENCE``,
default /root/reference) once per (cell kind, order) on a 3x3x3-hex template
box and stores, in ``autoflowcfd_b200/data/tmpl_<kind>_p<order>.npz``:

* the FR operators of ``generate_fr_operators`` (fr/operators.py:105-206) and
  the flattened-face extras (boundary extrapolation, g_left/g_right,
  distribution maps; core/fr_operators/face_kernels.py:228-351);
* the 1D Gauss-Legendre points and weights of the solution and fine grids;
* every face record of the template in relative form: owner (template hex,
  sub-cell kind), neighbour and interpolation-source cells as hex offsets +
  kind, axes / sides / primary flags, the triangle's three nodes as lattice
  offsets from the owner's hex, and indices into a de-duplicated set of
  cross-element interpolation matrices (fr/face_flux_points.py:165-236).

A 3-wide template holds one hex per topological position along each axis
(low boundary, interior, high boundary), which is all the face topology of a
hex-split box depends on: records and matrices depend on the owner's and
neighbour's sub-cell kinds, their local cube faces and the relative order of
their indices, not on the box size or the node coordinates (conforming faces
parametrise the same straight-sided patch from both sides).
``autoflowcfd_b200.boxgeom`` replays these records on boxes of any size and
recomputes all geometry from the node coordinates.

This is the recipe for committed data, not part of the package.  Run:
``AFR_REFERENCE=<checkout> NUMBA_CACHE_DIR=/tmp/nc python tests/golden/make_tables.py``.
"""

import os
import sys

import numpy as np

GOLDEN = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(GOLDEN))
HERE = os.path.join(REPO, "autoflowcfd_b200", "data")  # where the templates are written
REF = os.environ.get("AFR_REFERENCE", "/root/reference")
sys.path.insert(0, REPO)
sys.path.insert(0, GOLDEN)
sys.path.insert(0, os.path.join(REF, "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/afr_numba_cache")

from autoflowcfd_b200 import boxmesh  # noqa: E402

T = 3  # template hexes per axis


def dedupe(mats, tol=1e-10):
    """Unique matrices (within tol of the largest entry) -> (table, index)."""
    n = mats.shape[0]
    if n == 0:
        return mats[:0], np.zeros(0, np.int64)
    scale = max(np.max(np.abs(mats)), 1e-300)
    keys = np.round(mats.reshape(n, -1) / (scale * 1e-8)).astype(np.int64)
    table, index, seen = [], np.empty(n, np.int64), {}
    for i in range(n):
        k = keys[i].tobytes()
        j = seen.get(k)
        if j is not None and np.max(np.abs(table[j] - mats[i])) <= tol * scale:
            index[i] = j
            continue
        # fall back to a scan (rounding boundaries)
        found = -1
        for jj, t in enumerate(table):
            if np.max(np.abs(t - mats[i])) <= tol * scale:
                found = jj
                break
        if found < 0:
            found = len(table)
            table.append(mats[i].copy())
            seen[k] = found
        index[i] = found
    return np.stack(table), index


def harvest(kind, order):
    import make_golden as mg
    from autoflowcfd.fr.operators import gauss_legendre, generate_fr_operators
    from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry

    if kind == "prism":
        box = boxmesh.prism_box(T, T, T, (1.0, 1.0, 1.0), jitter=0.1, seed=123)
    else:
        box = boxmesh.tet_box(T, T, T, (1.0, 1.0, 1.0), jitter=0.05, seed=123, periodic=True)
    mesh = mg.ref_mesh(box, order)
    ops = generate_fr_operators(order)
    flat = get_flat_face_geometry(mesh, ops)
    fc = mesh.face_connectivity
    hexes = box.hex_index
    kinds = box.local_kind

    def rel(owner, cells):
        """(dH, kind) of cells relative to the owner's hex; kind -1 where cell < 0."""
        out = np.zeros((len(owner), 4), np.int64)
        ok = cells >= 0
        d = hexes[cells[ok]] - hexes[owner[ok]]
        if box.periodic:
            d = (d + 1) % T - 1  # wrap to {-1, 0, 1}
        out[ok, :3] = d
        out[ok, 3] = kinds[cells[ok]]
        out[~ok, 3] = -1
        return out

    own = flat.owner_cell
    order_idx = np.lexsort((np.arange(len(own)), own))  # group by owner, keep face order inside
    o = own[order_idx]
    n_t = box.n_cells
    ptr = np.zeros(n_t + 1, np.int64)
    np.add.at(ptr, o + 1, 1)
    ptr = np.cumsum(ptr)

    def src1_cells(idx, cells):
        out = np.full(len(idx), -1, np.int64)
        ok = idx >= 0
        out[ok] = cells[idx[ok]]
        return out

    P, S = flat.n_fp, flat.n_sps
    f = order_idx
    nb1c = src1_cells(flat.neighbor_src1_idx, flat.neighbor_src1_cell)
    ow1c = src1_cells(flat.owner_src1_idx, flat.owner_src1_cell)
    all_mats = [flat.neighbor_src0_mat[f], flat.owner_src0_mat[f]]
    nb1m = np.zeros((len(f), P, S))
    ok = flat.neighbor_src1_idx[f] >= 0
    nb1m[ok] = flat.neighbor_src1_mat.reshape(-1, P, S)[flat.neighbor_src1_idx[f][ok]]
    ow1m = np.zeros((len(f), P, S))
    ok = flat.owner_src1_idx[f] >= 0
    ow1m[ok] = flat.owner_src1_mat.reshape(-1, P, S)[flat.owner_src1_idx[f][ok]]
    all_mats += [nb1m, ow1m]
    stacked = np.concatenate(all_mats, axis=0)
    table, index = dedupe(stacked)
    R = len(f)
    mat_idx = index.reshape(4, R).T  # (R, 4): nb0, ow0, nb1, ow1

    # triangle nodes as lattice offsets from the owner's hex corner
    tri = box.node_ijk(fc.face_node_ids[f]) - hexes[o][:, None, :]
    out = dict(
        kind=np.array(kind), order=np.int32(order), template=np.int32(T), periodic=np.int32(box.periodic),
        cell_ptr=ptr, rec_owner_kind=kinds[o],
        rec_nb=rel(o, flat.neighbor_cell[f]),
        rec_nb_src0=rel(o, flat.neighbor_src0_cell[f]), rec_nb_src1=rel(o, nb1c[f]),
        rec_ow_src0=rel(o, flat.owner_src0_cell[f]), rec_ow_src1=rel(o, ow1c[f]),
        rec_o_axis=flat.owner_axis[f], rec_o_side=flat.owner_side[f],
        rec_n_axis=flat.neighbor_axis[f], rec_n_side=flat.neighbor_side[f],
        rec_is_boundary=flat.is_boundary[f].astype(np.uint8),
        rec_o_primary=flat.owner_is_primary[f].astype(np.uint8),
        rec_n_primary=flat.neighbor_is_primary[f].astype(np.uint8),
        rec_tri=tri.astype(np.int64), rec_mat=mat_idx, mats=table,
        boundary_extrap=flat.boundary_extrap, g_left=flat.g_left, g_right=flat.g_right,
        dist_fp_of_sp=flat.dist_fp_of_sp, dist_axis_coord_of_sp=flat.dist_axis_coord_of_sp,
    )
    out.update(mg.op_tables(ops))
    sps, w = gauss_legendre(order + 1)
    nf1 = min(2 * order, 3) + 1
    fine, wf = gauss_legendre(nf1)
    out.update(sps_1d=sps, w_1d=w, fine_1d=fine, w_fine_1d=wf)
    path = os.path.join(HERE, f"tmpl_{kind}_p{order}.npz")
    # operators the reference does not build at this order (None at P0) are left out
    out = {k: v for k, v in out.items() if v is not None}
    np.savez_compressed(path, **out)
    print(f"{path}: records={R} unique matrices={len(table)} size={os.path.getsize(path) / 1e6:.2f} MB", flush=True)


if __name__ == "__main__":
    want = sys.argv[1:] or ["prism:1", "prism:2", "prism:3", "tet:1", "tet:2", "tet:3"]
    for w in want:
        k, p = w.split(":")
        harvest(k, int(p))

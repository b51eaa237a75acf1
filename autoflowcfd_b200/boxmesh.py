"""Structured hex-box meshes split into prisms or tetrahedra.

These are the synthetic meshes the FR residual-and-update path is measured on.
Both splits follow the reference's own hex-splitting templates so the meshes
reach the reference's mesh loader unchanged:

* prisms: every (x, y) rectangle of a hex column is cut along the
  (i, j) -> (i+1, j+1) diagonal into two triangles and extruded along z, the
  wall-normal axis (the reference's channel template
  ``tests/validation/_channel_mesh.py:159-229`` with y and z swapped so that the
  no-slip wall sits at z = 0).  Cells are ordered i-major, then j, then the
  triangle, then k, so one wall-normal column of prisms is contiguous.
* tetrahedra: six tets per hex from one fixed local corner template
  (``tests/validation/_tgv_mesh.py:55-74``), which keeps opposite boundary
  planes translation images of each other so they can be paired periodically.

Node ids are ``i + (nx+1)*j + (nx+1)*(ny+1)*k`` as in the reference helpers.
Jitter moves interior nodes only (boundary planes stay flat), uniformly by
``+-jitter`` of the local spacing per axis, from a seeded generator.
"""

from dataclasses import dataclass, field
from typing import Dict, Optional, Tuple

import numpy as np

__all__ = ["BoxMesh", "prism_box", "tet_box", "PLANE_NAMES"]

PLANE_NAMES = ("x_min", "x_max", "y_min", "y_max", "z_min", "z_max")


@dataclass
class BoxMesh:
    """A hex box split into simplicial cells.

    Attributes:
        kind: "prism" or "tet".
        nodes: (n_nodes, 3) float64 coordinates.
        conn: (n_cells, 6) prism or (n_cells, 4) tet node ids, unoriented
            (the loader fixes orientation the same way the reference does).
        hex_index: (n_cells, 3) int64 (i, j, k) of the parent hex.
        local_kind: (n_cells,) int64 which sub-cell of the hex (0..1 prisms,
            0..5 tets).
        shape: (nx, ny, nz) hex counts.
        lengths: (Lx, Ly, Lz) box size.
        periodic: True when all six planes are paired periodically.
    """

    kind: str
    nodes: np.ndarray
    conn: np.ndarray
    hex_index: np.ndarray
    local_kind: np.ndarray
    shape: Tuple[int, int, int]
    lengths: Tuple[float, float, float]
    periodic: bool = False
    extras: Dict[str, object] = field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return int(self.conn.shape[0])

    def node_ijk(self, node_ids: np.ndarray) -> np.ndarray:
        """(i, j, k) lattice indices of node ids, shape (..., 3)."""
        nx, ny, _ = self.shape
        node_ids = np.asarray(node_ids, dtype=np.int64)
        i = node_ids % (nx + 1)
        j = (node_ids // (nx + 1)) % (ny + 1)
        k = node_ids // ((nx + 1) * (ny + 1))
        return np.stack([i, j, k], axis=-1)

    def plane_of_faces(self, face_node_ids: np.ndarray) -> np.ndarray:
        """Index into PLANE_NAMES of the box plane a triangle lies on, -1 if none.

        Decided from the lattice indices of its three nodes, so it holds for
        jittered and bumped meshes alike."""
        ijk = self.node_ijk(face_node_ids)  # (n,3,3)
        nx, ny, nz = self.shape
        out = np.full(ijk.shape[0], -1, dtype=np.int64)
        for code, ax, val in ((1, 0, nx), (0, 0, 0), (3, 1, ny), (2, 1, 0), (5, 2, nz), (4, 2, 0)):
            out[np.all(ijk[:, :, ax] == val, axis=1)] = code
        return out

    def plane_of_points(self, pts: np.ndarray, tol_scale: float = 1e-6) -> np.ndarray:
        """Index into PLANE_NAMES of the box plane each point lies on, -1 if none.

        Ties (edges, corners) resolve in the order z_min, z_max, y_min, y_max,
        x_min, x_max, i.e. a wall at z = 0 wins over the side planes, which is
        what the reference's face-centre classifier does for its channel
        (``tests/validation/_channel_mesh.py:42-56``).
        """
        Lx, Ly, Lz = self.lengths
        tol = tol_scale * max(Lx, Ly, Lz, 1.0)
        out = np.full(pts.shape[0], -1, dtype=np.int64)
        order = [(4, 2, 0.0), (5, 2, Lz), (2, 1, 0.0), (3, 1, Ly), (0, 0, 0.0), (1, 0, Lx)]
        for code, ax, val in reversed(order):
            hit = np.abs(pts[:, ax] - val) < tol
            out[hit] = code
        return out


def _grid_nodes(nx: int, ny: int, nz: int, lengths, jitter: float, seed: int) -> np.ndarray:
    Lx, Ly, Lz = lengths
    nx1, ny1, nz1 = nx + 1, ny + 1, nz + 1
    k, j, i = np.meshgrid(np.arange(nz1), np.arange(ny1), np.arange(nx1), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    k = k.ravel()  # node id = i + nx1*j + nx1*ny1*k is now the array position
    x = i / nx * Lx
    y = j / ny * Ly
    z = k / nz * Lz
    nodes = np.column_stack([x, y, z]).astype(np.float64)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter, jitter, size=nodes.shape)
        interior = (i > 0) & (i < nx) & (j > 0) & (j < ny) & (k > 0) & (k < nz)
        h = np.array([Lx / nx, Ly / ny, Lz / nz])
        nodes[interior] += d[interior] * h[None, :]
    return nodes


def _gid(i, j, k, nx, ny):
    return i + (nx + 1) * j + (nx + 1) * (ny + 1) * k


def prism_box(nx: int, ny: int, nz: int, lengths=(4.0, 2.0, 1.5), jitter: float = 0.0,
              seed: int = 0, bump=None) -> BoxMesh:
    """Hex box split into 2 prisms per hex, extruded along z (wall at z = 0).

    Args:
        bump: optional (height, x0, y0, sigma) Gaussian wall bump: every node
            is shifted by ``(1 - z/Lz) * h * exp(-r^2/sigma^2)`` in z.
    """
    lengths = tuple(float(v) for v in lengths)
    nodes = _grid_nodes(nx, ny, nz, lengths, jitter, seed)
    if bump is not None:
        h, x0, y0, sig = bump
        r2 = (nodes[:, 0] - x0) ** 2 + (nodes[:, 1] - y0) ** 2
        nodes[:, 2] += (1.0 - nodes[:, 2] / lengths[2]) * h * np.exp(-r2 / sig**2)
    I, J, T, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(2), np.arange(nz), indexing="ij")
    I, J, T, K = I.ravel(), J.ravel(), T.ravel(), K.ravel()
    # tri_a = (i,j),(i+1,j),(i+1,j+1); tri_b = (i,j),(i+1,j+1),(i,j+1)
    di = np.where(T[:, None] == 0, np.array([0, 1, 1])[None, :], np.array([0, 1, 0])[None, :])
    dj = np.where(T[:, None] == 0, np.array([0, 0, 1])[None, :], np.array([0, 1, 1])[None, :])
    bot = _gid(I[:, None] + di, J[:, None] + dj, K[:, None], nx, ny)
    top = _gid(I[:, None] + di, J[:, None] + dj, K[:, None] + 1, nx, ny)
    conn = np.concatenate([bot, top], axis=1).astype(np.int64)
    return BoxMesh("prism", nodes, conn, np.column_stack([I, J, K]).astype(np.int64),
                   T.astype(np.int64), (nx, ny, nz), lengths, False)


# local hex corners v0..v7 -> six tets (fixed template, independent of (i,j,k))
_HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)
_TET_TEMPLATE = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6],
                          [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]], dtype=np.int64)


def tet_box(nx: int, ny: int, nz: int, lengths=(1.0, 1.0, 1.0), jitter: float = 0.0,
            seed: int = 0, periodic: bool = True) -> BoxMesh:
    """Hex box split into 6 tets per hex; optionally triply periodic."""
    lengths = tuple(float(v) for v in lengths)
    nodes = _grid_nodes(nx, ny, nz, lengths, jitter, seed)
    I, J, K, T = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), np.arange(6), indexing="ij")
    I, J, K, T = I.ravel(), J.ravel(), K.ravel(), T.ravel()
    corners = _HEX_CORNERS[_TET_TEMPLATE[T]]  # (n,4,3)
    conn = _gid(I[:, None] + corners[:, :, 0], J[:, None] + corners[:, :, 1],
                K[:, None] + corners[:, :, 2], nx, ny).astype(np.int64)
    return BoxMesh("tet", nodes, conn, np.column_stack([I, J, K]).astype(np.int64),
                   T.astype(np.int64), (nx, ny, nz), lengths, periodic)


def signed_tet_volume(p0, p1, p2, p3):
    """Signed tet volume, vectorised over leading axes."""
    return np.einsum("...i,...i->...", np.cross(p1 - p0, p2 - p0), p3 - p0) / 6.0


def orient_cells(mesh: BoxMesh) -> np.ndarray:
    """Connectivity with the orientation fix the reference's loader applies.

    Tets with negative signed volume swap local nodes 1 and 2; prisms whose
    3-tet decomposition volume is negative swap 1<->2 and 4<->5.  Restates
    ``grid/curved_mapping/curved_mapping_orientation.py:21-31, 78-95``.
    """
    conn = mesh.conn.copy()
    p = mesh.nodes[conn]
    if mesh.kind == "tet":
        vol = signed_tet_volume(p[:, 0], p[:, 1], p[:, 2], p[:, 3])
        neg = vol < 0
        conn[neg, 1], conn[neg, 2] = mesh.conn[neg, 2], mesh.conn[neg, 1]
    else:
        v0, v1, v2, w0, w1, w2 = (p[:, i] for i in range(6))
        vol = signed_tet_volume(v0, v1, v2, w0) + signed_tet_volume(v1, v2, w0, w1) + \
            signed_tet_volume(v2, w0, w1, w2)
        neg = vol < 0
        conn[neg, 1], conn[neg, 2] = mesh.conn[neg, 2], mesh.conn[neg, 1]
        conn[neg, 4], conn[neg, 5] = mesh.conn[neg, 5], mesh.conn[neg, 4]
    return conn

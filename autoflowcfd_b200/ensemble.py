"""Batched uneven ensemble: many independent FR cases resident on one GPU.

Cases of the same order are concatenated into one mesh: cell, face, second
source, interpolation-matrix and boundary-condition indices are offset, the
operators are shared.  One set of kernel launches per RK stage then advances
every case of that order, and the steps of all order groups are replayed as
one CUDA graph.  Per-cell arithmetic does not depend on which other cells
share a launch (no cross-cell reductions, gathers stay inside a case), so each
case gets exactly the result it gets alone; per-case FP64 residual norms come
from ``afr_segment_norms``.

All cases share one molecular viscosity: the Reynolds number of a case is set
through its box length, L = Re * mu / (rho u), so a single ``mu`` serves
every Mach number of the draw.
"""

import ctypes
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import LIB, check

GAMMA = 1.4
RHO_INF = 1.225
P_INF = 101325.0
MU = 1.8e-5

# arrays of the reference's flattened tables, by the entity their first axis runs over
PER_CELL = ["det_jacs", "inv_jacs", "det_jacs_fine", "inv_jacs_fine", "cell_volumes", "wall_distance"]
PER_FACE = ["owner_side", "neighbor_side", "true_normal", "owner_axis", "neighbor_axis", "is_boundary",
            "owner_is_primary", "neighbor_is_primary", "colors", "true_area_weight", "cd_wall_face"]
FACE_CELL_IDX = ["owner_cell", "neighbor_cell", "nb_src0_cell", "ow_src0_cell"]
SRC1 = {"nb": ("nb_src1_idx", "nb_src1_cell", "nb_src1_mat_index"),
        "ow": ("ow_src1_idx", "ow_src1_cell", "ow_src1_mat_index")}
MAT0_IDX = ["nb_src0_mat_index", "ow_src0_mat_index"]
BC_ROWS = ["bc_type", "bc_noslip", "bc_wall_vel", "bc_Q", "bc_p_out"]
SHARED = ["boundary_extrap", "g_left", "g_right", "dist_fp_of_sp", "dist_axis_coord_of_sp", "n_sps", "n_fine", "order"]
OPS = ["D_3d_", "c2f_", "Dfine_", "f2c_", "filter_"]


@dataclass
class EnsembleCase:
    """One case of the draw: a jittered hex box split into prisms, wall at z = 0."""

    shape: tuple            # hex cells (nx, ny, nz)
    order: int
    mach: float
    bump: float             # Gaussian wall-bump height as a fraction of Lz
    seed: int
    lengths: tuple          # box size (m)
    jitter: float = 0.1
    bump_x: float = 0.5     # streamwise bump position as a fraction of Lx

    @property
    def velocity(self) -> float:
        return self.mach * float(np.sqrt(GAMMA * P_INF / RHO_INF))

    @property
    def n_cells(self) -> int:
        return 2 * self.shape[0] * self.shape[1] * self.shape[2]


def draw_cases(n: int, seed: int = 0, hex_cells=(2000, 64000), orders=(1, 2), mach=(0.05, 0.3),
               bump=(0.0, 0.1), reynolds: float = 1e5) -> List[EnsembleCase]:
    """Seeded draw: hex count log-uniform, order uniform over ``orders``, Mach
    and bump height uniform; box (L, L/2, L/2) with rho u L / mu = reynolds."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cells = float(np.exp(rng.uniform(np.log(hex_cells[0]), np.log(hex_cells[1]))))
        m = max(2, int(round((cells / 2.0) ** (1.0 / 3.0))))
        order = int(rng.choice(orders))
        M = float(rng.uniform(*mach))
        b = float(rng.uniform(*bump))
        u = M * float(np.sqrt(GAMMA * P_INF / RHO_INF))
        L = reynolds * MU / (RHO_INF * u)
        out.append(EnsembleCase((2 * m, m, m), order, M, b, int(rng.integers(1 << 30)), (L, L / 2, L / 2)))
    return out


def plane_config(spec: EnsembleCase) -> Dict[str, dict]:
    from .boxmesh import PLANE_NAMES

    cfg = {n: {"type": "FARFIELD", "Q_free": [RHO_INF, spec.velocity, 0.0, 0.0, P_INF]} for n in PLANE_NAMES}
    cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
    return cfg


def build_case(spec: EnsembleCase, wall_distance: bool = False) -> Dict[str, np.ndarray]:
    """Tables of one case (reference layout) from the box generator."""
    from . import boxgeom, boxmesh

    Lx, Ly, Lz = spec.lengths
    bump = (spec.bump * Lz, spec.bump_x * Lx, 0.5 * Ly, 0.25 * Lz) if spec.bump > 0 else None
    box = boxmesh.prism_box(*spec.shape, spec.lengths, jitter=spec.jitter, seed=spec.seed, bump=bump)
    return boxgeom.build_case(box, spec.order, plane_config(spec), wall_distance=wall_distance)


def uniform_state(spec: EnsembleCase, n_cells: int, n_sps: int) -> np.ndarray:
    """Free stream (FRState.initialize_uniform, core/fr_solver/state.py:50-74)."""
    u = spec.velocity
    U = np.empty((n_cells, n_sps, 5))
    U[..., 0] = RHO_INF
    U[..., 1] = RHO_INF * u
    U[..., 2] = 0.0
    U[..., 3] = 0.0
    U[..., 4] = P_INF / (GAMMA - 1.0) + 0.5 * RHO_INF * u * u
    return U


def concatenate(cases: Sequence[Dict[str, np.ndarray]]) -> Dict[str, np.ndarray]:
    """One mesh of independent cases of the same order (indices offset)."""
    if not cases:
        raise ValueError("no cases")
    order = int(cases[0]["order"])
    if any(int(c["order"]) != order for c in cases):
        raise ValueError("cases of one concatenation must share the order")
    if any(int(c["n_prism"]) != int(c["n_cells"]) for c in cases):
        raise ValueError("ensemble cases are prism meshes")
    out = {k: cases[0][k] for k in SHARED}
    for t in ("prism", "tet"):
        for k in OPS:
            if k + t in cases[0]:
                out[k + t] = cases[0][k + t]
    for k in PER_CELL + PER_FACE:
        if all(k in c and c[k] is not None for c in cases):
            out[k] = np.concatenate([c[k] for c in cases])
    cell_off = face_off = mat_off = bc_off = 0
    src1_off = {"nb": 0, "ow": 0}
    parts = {k: [] for k in FACE_CELL_IDX + MAT0_IDX + ["bc_group"] + BC_ROWS}
    for s in SRC1.values():
        for k in s:
            parts[k] = []
    tables = []
    for c in cases:
        N, F = int(c["n_cells"]), int(c["owner_cell"].shape[0])
        for k in FACE_CELL_IDX:
            a = np.asarray(c[k], np.int64)
            parts[k].append(np.where(a >= 0, a + cell_off, a))
        for k in MAT0_IDX:
            parts[k].append(np.asarray(c[k], np.int64) + mat_off)
        for side, (idx, cell, midx) in SRC1.items():
            a = np.asarray(c[idx], np.int64)
            parts[idx].append(np.where(a >= 0, a + src1_off[side], a))
            parts[cell].append(np.asarray(c[cell], np.int64) + cell_off)
            parts[midx].append(np.asarray(c[midx], np.int64) + mat_off)
            src1_off[side] += int(np.asarray(c[cell]).shape[0])
        parts["bc_group"].append(np.asarray(c["bc_group"], np.int64) + bc_off)
        for k in BC_ROWS:
            parts[k].append(np.asarray(c[k]))
        tables.append(np.asarray(c["src_mat_table"]))
        cell_off += N
        face_off += F
        mat_off += int(tables[-1].shape[0])
        bc_off += int(np.asarray(c["bc_type"]).shape[0])
    for k, v in parts.items():
        out[k] = np.concatenate(v)
    for k in MAT0_IDX + [SRC1["nb"][2], SRC1["ow"][2], "bc_group", "bc_type", "bc_noslip"]:
        out[k] = out[k].astype(np.int32)
    out["src_mat_table"] = np.concatenate(tables)
    out["n_cells"] = cell_off
    out["n_prism"] = cell_off
    return out


@dataclass
class _Group:
    order: int
    members: List[int]                 # case indices in the draw
    cell_ptr: np.ndarray               # (len(members)+1,) cell ranges inside the group
    solver: object = None


class B200Ensemble:
    """Independent cases of uneven size and order, advanced together.

    Args:
        specs: the draw (``draw_cases``).
        precision: "mixed" (default) or "fp64".
        inviscid_only: Euler instead of laminar Navier-Stokes.
        cases: prebuilt tables per spec (built from the specs when omitted).
        max_group_cells: cases of one order are split into groups of at most
            this many cells (one handle each), which bounds the transient device
            memory of a handle's set-up.
    """

    def __init__(self, specs: Sequence[EnsembleCase], precision: str = "mixed", inviscid_only: bool = False,
                 cases: Optional[Sequence[Dict[str, np.ndarray]]] = None, device="cuda:0",
                 max_group_cells: int = 2_000_000):
        from .solver import B200FRSolver

        self.specs = list(specs)
        self.device = torch.device(device)
        tables = list(cases) if cases is not None else [build_case(s) for s in self.specs]
        self.groups: List[_Group] = []
        chunks = []
        for order in sorted({s.order for s in self.specs}):
            cur, cells = [], 0
            for i in (i for i, s in enumerate(self.specs) if s.order == order):
                n = int(tables[i]["n_cells"])
                if cur and cells + n > max_group_cells:
                    chunks.append((order, cur))
                    cur, cells = [], 0
                cur.append(i)
                cells += n
            if cur:
                chunks.append((order, cur))
        for order, members in chunks:
            part = [tables[i] for i in members]
            cell_ptr = np.concatenate([[0], np.cumsum([int(c["n_cells"]) for c in part])]).astype(np.int64)
            merged = concatenate(part)
            # the handle's free stream only scales Cd/Cl
            solver = B200FRSolver(merged, turb_model_name="NONE", mu_molecular=MU, rho_inf=RHO_INF,
                                  vel_inf=self.specs[members[0]].velocity, p_inf=P_INF, inviscid_only=inviscid_only,
                                  precision=precision, device=device)
            U = np.concatenate([uniform_state(self.specs[i], int(tables[i]["n_cells"]), int(tables[i]["n_sps"]))
                                for i in members])
            solver.set_state_from_cpu(U)
            del merged, U
            self.groups.append(_Group(order, members, cell_ptr, solver))
        self.graph = None
        self.steps_done = 0

    # ---------------------------------------------------------------- running
    def step(self):
        """One SSP-RK3 step of every case (no host synchronisation)."""
        for g in self.groups:
            g.solver.step(want_norm=False)
        self.steps_done += 1

    def capture(self):
        """Capture one step of all groups as a CUDA graph (after a warm-up step)."""
        self.step()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for grp in self.groups:
                grp.solver.step(want_norm=False)
        self.graph = g
        return g

    def replay(self, n: int = 1):
        if self.graph is None:
            raise RuntimeError("capture() first")
        for _ in range(n):
            self.graph.replay()
            self.steps_done += 1

    def autotune(self) -> List[List[int]]:
        """Launch shapes per group from afr_autotune (mixed form)."""
        out = []
        from .solver import _dev_ptr, _stream

        for g in self.groups:
            ch = (ctypes.c_int32 * 3)()
            check(LIB.afr_autotune(g.solver._h, _dev_ptr(g.solver.U), None, ch, _stream()), g.solver._h)
            out.append([int(v) for v in ch])
        self.graph = None  # launch shapes changed: recapture
        return out

    # --------------------------------------------------------------- results
    def norms(self, density: bool = False) -> np.ndarray:
        """Per-case FP64 RMS residual norms of the last step (all variables, or
        the density column), in draw order."""
        from .solver import _stream

        res = np.zeros(len(self.specs))
        for g in self.groups:
            out = np.zeros(len(g.members))
            check(LIB.afr_segment_norms(g.solver._h, len(g.members), g.cell_ptr.ctypes.data_as(_lib._P_I64),
                                        1 if density else 0, out.ctypes.data_as(_lib._P_D), _stream()), g.solver._h)
            res[g.members] = out
        return res

    def status(self, clear: bool = True) -> np.ndarray:
        """Per-case device status after the last step, in draw order: 0 (AFR_OK)
        or AFR_ENONFINITE for a case whose state stopped being finite.  Cases
        share no cells, so a failed case leaves the others' results unchanged;
        ``clear`` resets each group's sticky status word so the healthy cases
        keep running.  Index or tensor-core errors of a group raise."""
        from .solver import _stream

        res = np.zeros(len(self.specs), np.int32)
        for g in self.groups:
            seg = np.zeros(len(g.members), np.int32)
            rc = LIB.afr_status(g.solver._h, len(g.members), g.cell_ptr.ctypes.data_as(_lib._P_I64),
                                seg.ctypes.data_as(_lib._P_I32), 1 if clear else 0, _stream())
            if rc not in (_lib.AFR_OK, _lib.AFR_ENONFINITE):
                check(rc, g.solver._h)
            res[g.members] = seg
        return res

    def state(self, i: int) -> torch.Tensor:
        """Device view of case i's conserved state (n_cells, n_sps, 5)."""
        for g in self.groups:
            if i in g.members:
                j = g.members.index(i)
                return g.solver.U[g.cell_ptr[j]:g.cell_ptr[j + 1]]
        raise IndexError(i)

    @property
    def n_cells(self) -> int:
        return int(sum(g.cell_ptr[-1] for g in self.groups))

    def dof_per_step(self) -> int:
        return int(sum(g.cell_ptr[-1] * g.solver.n_sps for g in self.groups)) * 5 * 3

    def cleanup(self):
        self.graph = None
        for g in self.groups:
            g.solver.cleanup()

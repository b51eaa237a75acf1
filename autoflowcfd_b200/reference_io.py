"""Drop-in from the reference solver's own objects.

The reference (AutoFlowCFD) builds a ``HighOrderMesh``, its ``FROperators``
and a ``BoundaryGhostStateProvider`` during set-up and hands them to its
residual kernels.  This module lowers exactly those objects into the flat
tables ``afr_create`` takes, and ``B200GPUFRSolver`` accepts them with the
constructor signature of the reference's ``--backend gpu`` solver
(``GPUFRSolver.__init__``, core/gpu/gpu_solver.py:51-66), so the reference
switches backends by constructing this class instead.

It runs in the reference's process: the flattened face geometry comes from
the reference's own ``get_flat_face_geometry`` (core/fr_operators/
face_kernels.py:354-369) and the boundary tagging of the force integral from
its ``tag_boundary_groups`` (grid/connectivity/face_connectivity.py), imported
when they are needed.  Paths are relative to the reference's
``src/autoflowcfd``.

Ghost providers: the reference calls an arbitrary Python callable per
boundary face (core/fr_residual/inviscid_kernel.py:288-310).  The table form
``BoundaryGhostStateProvider`` (boundary/fr_ghost_state.py:144-189) with
constant WALL / FARFIELD / INLET / OUTLET / SYMMETRY configurations lowers to
device tables; anything else -- the synthetic-eddy inlet, per-point inlet
states, other callables -- cannot run on the device and is refused with
AFR_EUNSUPPORTED.  An unknown boundary type raises ValueError, as the
reference's provider does (boundary/fr_ghost_state.py:189).
"""

from types import SimpleNamespace
from typing import Dict, Optional

import numpy as np

from . import _lib

BC_CODES = {"WALL": 0, "FARFIELD": 1, "INLET": 2, "OUTLET": 3, "SYMMETRY": 4}


def _unsupported(msg: str):
    return _lib.AfrError(_lib.AFR_EUNSUPPORTED, msg)


def lower_ghost_provider(provider, n_faces: int) -> Dict[str, np.ndarray]:
    """Device tables of a ghost-state provider: one row per group code plus a
    last row for the provider's default configuration; ``bc_group[f]`` selects
    face f's row.  ``provider is None`` gives an all-default table (meshes
    without boundary faces, e.g. triply periodic boxes)."""
    if provider is None:
        return dict(bc_group=np.full(n_faces, -1, np.int32), bc_type=np.zeros(1, np.int32),
                    bc_noslip=np.ones(1, np.int32), bc_wall_vel=np.zeros((1, 3)), bc_Q=np.zeros((1, 5)),
                    bc_p_out=np.zeros(1), bc_default=np.int32(0))
    needed = ("group_code", "code_to_config", "default_config")
    if not all(hasattr(provider, a) for a in needed):
        raise _unsupported(f"ghost provider {type(provider).__name__} is not a table-form "
                           "BoundaryGhostStateProvider; arbitrary callables cannot run on the device")
    codes = sorted(int(c) for c in provider.code_to_config)
    if codes and codes[0] < 0:
        raise ValueError("negative boundary group code")
    n = (codes[-1] + 1 if codes else 0) + 1  # last row: the default configuration
    t = np.zeros(n, np.int32)
    ns = np.ones(n, np.int32)
    wv = np.zeros((n, 3))
    Q = np.zeros((n, 5))
    po = np.zeros(n)

    def put(i, cfg):
        typ = cfg.get("type")
        if typ not in BC_CODES:
            raise ValueError(f"Unknown boundary condition type '{typ}'")
        if typ == "INLET" and cfg.get("sem") is not None:
            raise _unsupported("synthetic-eddy (SEM) inlets are time-dependent Python callables and are not "
                               "built on the device")
        t[i] = BC_CODES[typ]
        ns[i] = 1 if cfg.get("is_no_slip", True) else 0
        if cfg.get("wall_velocity") is not None:
            wv[i] = np.asarray(cfg["wall_velocity"], float).reshape(3)
        for key in ("Q_free", "Q_inlet"):
            if key in cfg:
                q = np.asarray(cfg[key], float)
                if q.shape != (5,):
                    raise _unsupported(f"{key} of shape {q.shape}: only one constant primitive state per group "
                                       "is lowered")
                Q[i] = q
        if typ == "FARFIELD" and "Q_free" not in cfg:
            raise ValueError("FARFIELD configuration without Q_free")
        if typ == "INLET" and "Q_inlet" not in cfg:
            raise ValueError("INLET configuration without Q_inlet")
        if typ == "OUTLET":
            if "p_outlet" not in cfg:
                raise ValueError("OUTLET configuration without p_outlet")
            po[i] = float(cfg["p_outlet"])

    unused = np.ones(n, bool)
    for c in codes:
        put(c, provider.code_to_config[c])
        unused[c] = False
    put(n - 1, provider.default_config)
    for i in np.flatnonzero(unused[:-1]):  # gaps in the code range: default configuration
        put(int(i), provider.default_config)
    gc = np.asarray(provider.group_code, np.int64)
    if gc.shape[0] != n_faces:
        raise ValueError(f"group_code has {gc.shape[0]} entries for {n_faces} faces")
    gc = np.where((gc < 0) | ~np.isin(gc, codes), n - 1, gc).astype(np.int32)
    return dict(bc_group=gc, bc_type=t, bc_noslip=ns, bc_wall_vel=wv, bc_Q=Q, bc_p_out=po,
                bc_default=np.int32(n - 1))


def flat_tables(flat) -> Dict[str, np.ndarray]:
    """The arrays of a ``FlatFaceGeometry`` (core/fr_operators/face_kernels.py:124-187),
    with the greedy face colors expanded to one color per face record."""
    colors = np.full(flat.n_faces, -1, np.int32)
    for c, idx in enumerate(flat.color_face_indices):
        colors[np.asarray(idx)] = c
    if np.any(colors < 0):
        raise ValueError("face coloring does not cover every face record")
    n_fp, n_sps = flat.n_fp, flat.n_sps
    return dict(
        owner_cell=flat.owner_cell, neighbor_cell=flat.neighbor_cell, is_boundary=flat.is_boundary.astype(np.uint8),
        owner_axis=flat.owner_axis, owner_side=flat.owner_side, neighbor_axis=flat.neighbor_axis,
        neighbor_side=flat.neighbor_side, owner_is_primary=flat.owner_is_primary.astype(np.uint8),
        neighbor_is_primary=flat.neighbor_is_primary.astype(np.uint8), true_normal=flat.true_normal,
        nb_src0_cell=flat.neighbor_src0_cell, nb_src0_mat=flat.neighbor_src0_mat,
        nb_src1_idx=flat.neighbor_src1_idx, nb_src1_cell=flat.neighbor_src1_cell,
        nb_src1_mat=np.asarray(flat.neighbor_src1_mat).reshape(-1, n_fp, n_sps),
        ow_src0_cell=flat.owner_src0_cell, ow_src0_mat=flat.owner_src0_mat, ow_src1_idx=flat.owner_src1_idx,
        ow_src1_cell=flat.owner_src1_cell, ow_src1_mat=np.asarray(flat.owner_src1_mat).reshape(-1, n_fp, n_sps),
        boundary_extrap=flat.boundary_extrap, g_left=flat.g_left, g_right=flat.g_right,
        dist_fp_of_sp=flat.dist_fp_of_sp, dist_axis_coord_of_sp=flat.dist_axis_coord_of_sp, colors=colors,
    )


def op_tables(ops) -> Dict[str, np.ndarray]:
    """The ``FROperators`` fields the path consumes (fr/operators.py:32-102)."""
    return dict(
        D_3d_prism=ops.D_3d_prism, D_3d_tet=ops.D_3d_tet,
        c2f_prism=ops.overint_interp_c2f_prism, c2f_tet=ops.overint_interp_c2f_tet,
        Dfine_prism=ops.overint_D_fine_prism, Dfine_tet=ops.overint_D_fine_tet,
        f2c_prism=ops.overint_restrict_f2c_prism, f2c_tet=ops.overint_restrict_f2c_tet,
        filter_prism=ops.filter_prism, filter_tet=ops.filter_tet,
    )


def _wall_face_mask(mesh) -> Optional[np.ndarray]:
    """Faces the force integral sums over: boundary faces tagged with a group
    whose mesh-level type is WALL (postprocess/fr_coefficients.py:74-79)."""
    groups = getattr(mesh, "boundary_groups", None)
    types = getattr(mesh, "boundary_bc_types", None)
    if not groups or not types:
        return None
    from autoflowcfd.grid.connectivity.face_connectivity import tag_boundary_groups

    gcode, name_to_code = tag_boundary_groups(mesh.face_connectivity, groups)
    wall_codes = [c for name, c in name_to_code.items() if types.get(name) == "WALL"]
    return np.isin(gcode, wall_codes).astype(np.uint8)


def export_case(mesh, ops, boundary_ghost_provider=None, wall_distance=None, flat=None,
                cd_wall_face=None, flux_points: str = "reference") -> Dict[str, np.ndarray]:
    """Flat tables of a reference mesh for ``afr_create``.

    Args:
        mesh: the reference's ``HighOrderMesh`` (Jacobians at solution and
            fine points, cell volumes, face flux points).
        ops: its ``FROperators``.
        boundary_ghost_provider: the solver's ``BoundaryGhostStateProvider``
            (or None for meshes without boundary faces).
        wall_distance: (n_cells, n_sps) wall distance for SST
            (``FRSolver.wall_distance``).
        flat: the mesh's ``FlatFaceGeometry``; by default taken from the
            reference's cached ``get_flat_face_geometry(mesh, ops)``.
        cd_wall_face: (n_faces,) faces of the force integral; by default from
            the mesh's WALL boundary groups.
        flux_points: "reference" takes the face tables from the mesh's own
            flux-point construction; "device" builds them on the GPU from the
            mesh's face connectivity (autoflowcfd_b200.facegeom) and the
            operators.
    """
    if flux_points not in ("reference", "device"):
        raise ValueError(f"flux_points must be 'reference' or 'device', got {flux_points!r}")
    if flux_points == "device":
        from .facegeom import flux_point_tables, operator_face_tables

        prism = mesh._fixed_prism_conn if mesh._fixed_prism_conn is not None else np.zeros((0, 6), np.int64)
        tet = mesh._fixed_tet_conn if mesh._fixed_tet_conn is not None else np.zeros((0, 4), np.int64)
        t = flux_point_tables(mesh.face_connectivity, prism, tet, mesh._node_coords, int(mesh.order))
        for k in ("nb_fc", "ow_fc", "nb_resid", "ow_resid"):
            t.pop(k)
        t.update(operator_face_tables(ops, int(mesh.order)))
        flat = SimpleNamespace(n_faces=len(t["owner_cell"]), _tables=t)
    if flat is None:
        from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry

        flat = get_flat_face_geometry(mesh, ops)
    N, S = int(mesh.n_cells), int(mesh.n_sps_per_cell)
    # order 0 has no over-integration points: the one solution point stands in
    fine = mesh.jacobians_fine if getattr(mesh, "jacobians_fine", None) is not None else mesh.jacobians
    Fn = int(mesh.n_sps_per_cell_fine) if getattr(mesh, "jacobians_fine", None) is not None else S
    out = dict(order=np.int32(mesh.order), n_cells=np.int32(N), n_prism=np.int32(mesh.n_prism_cells),
               n_sps=np.int32(S), n_fine=np.int32(Fn))
    out["det_jacs"] = np.asarray(mesh.jacobians["det_jacs"], float).reshape(N, S)
    out["inv_jacs"] = np.asarray(mesh.jacobians["inv_jacs"], float).reshape(N, S, 3, 3)
    out["det_jacs_fine"] = np.asarray(fine["det_jacs"], float).reshape(N, Fn)
    out["inv_jacs_fine"] = np.asarray(fine["inv_jacs"], float).reshape(N, Fn, 3, 3)
    out["cell_volumes"] = np.asarray(mesh.get_all_cell_volumes(), float)
    if getattr(mesh, "cell_volumes", None) is not None:
        out["fv_cell_volumes"] = np.asarray(mesh.cell_volumes, float)
    out.update(op_tables(ops))
    out.update(flat._tables if hasattr(flat, "_tables") else flat_tables(flat))
    out.update(lower_ghost_provider(boundary_ghost_provider, int(flat.n_faces)))
    taw = getattr(getattr(mesh, "face_flux_points", None), "true_area_weight", None)
    if taw is not None:
        out["true_area_weight"] = np.asarray(taw, float)
    cdw = cd_wall_face if cd_wall_face is not None else _wall_face_mask(mesh)
    if cdw is not None:
        out["cd_wall_face"] = np.asarray(cdw, np.uint8)
    if wall_distance is not None:
        out["wall_distance"] = np.asarray(wall_distance, float).reshape(N, S)
    return out


def reference_case_for_order(mesh, boundary_ghost_provider=None, cd_wall_face=None):
    """``order -> case`` over one reference ``HighOrderMesh``, for the order
    continuation of ``B200FRSolver(case_for_order=...)``: switches the mesh to
    that order (HighOrderMesh.set_order, as run_order_continuation does,
    core/utils/order_continuation.py:330-345), exports its tables with that
    order's operators (fr/operators.py generate_fr_operators) and switches the
    mesh back.  The exported ``fv_cell_volumes`` is the mesh's cell_volumes
    attribute, computed at its load order, which the reference divides the
    order-0 finite-volume residual by."""
    from autoflowcfd.fr.operators import generate_fr_operators

    def case_for_order(order: int) -> Dict[str, np.ndarray]:
        active = int(getattr(mesh, "_active_order", mesh.order))
        mesh.set_order(order)
        try:
            ops = generate_fr_operators(order)
            case = export_case(mesh, ops, boundary_ghost_provider, cd_wall_face=cd_wall_face)
        finally:
            mesh.set_order(active)
        return case

    return case_for_order


def _solver_base():
    from .solver import B200FRSolver

    return B200FRSolver


class B200GPUFRSolver(_solver_base()):
    """``GPUFRSolver`` drop-in: same constructor arguments and methods
    (core/gpu/gpu_solver.py:51-66, .step / .solve / .get_state_cpu /
    .set_state_from_cpu / .cleanup), every number computed by libafr_b200.so.

    The numerics are those of the reference's CPU path (``FRSolver.step``),
    the parity target: local time steps with the CPU path's own CFL rule
    (core/fr_solver/cfl.py:96-134), so ``cfl`` is accepted for the signature
    and must be positive; ``time_scheme`` is "ssp_rk3", "dual_time" or
    "imex_euler" (other schemes raise AFR_EUNSUPPORTED).  The state starts as
    the uniform free stream along x, as ``GPUFRSolver`` does.

    Extra keyword arguments: ``wall_distance`` (required with SST),
    ``precision`` ("fp64" or "mixed"), ``inviscid_only`` and
    ``global_dt_factor`` as in ``B200FRSolver``, and ``flat`` /
    ``cd_wall_face`` as in ``export_case``.
    """

    def __init__(self, mesh, ops, order: int = 2, n_vars: int = 5, device_id: int = 0,
                 time_scheme: str = "ssp_rk3", cfl: float = 1.0, rho_inf: float = 1.225, vel_inf: float = 33.33,
                 p_inf: float = 101325.0, mu_molecular: float = 1.8e-5, boundary_ghost_provider=None,
                 turb_model: str = "NONE", *, wall_distance=None, precision: str = "fp64",
                 inviscid_only: bool = False, global_dt_factor: float = 0.0, flat=None, cd_wall_face=None,
                 dual_time_inner_iter: int = 20):
        turb = str(turb_model).upper()
        if not cfl > 0:
            raise ValueError("cfl must be positive")
        if int(order) != int(mesh.order):
            raise ValueError(f"order {order} does not match the mesh's order {mesh.order}")
        if turb == "SST" and n_vars not in (5, 7):
            raise ValueError("SST carries 7 variables")
        if turb != "SST" and n_vars != 5:
            raise ValueError(f"n_vars {n_vars} without a turbulence model (5 expected)")
        if turb == "SST" and wall_distance is None:
            raise ValueError("SST needs wall_distance (n_cells, n_sps), e.g. FRSolver.wall_distance")
        case = export_case(mesh, ops, boundary_ghost_provider, wall_distance=wall_distance, flat=flat,
                           cd_wall_face=cd_wall_face)
        super().__init__(case, turb_model_name=turb, mu_molecular=mu_molecular, rho_inf=rho_inf, vel_inf=vel_inf,
                         p_inf=p_inf, inviscid_only=inviscid_only, global_dt_factor=global_dt_factor,
                         precision=precision, device=f"cuda:{int(device_id)}", time_scheme=time_scheme,
                         dual_time_inner_iter=dual_time_inner_iter)
        self.mesh, self.ops = mesh, ops
        self.device_id = int(device_id)
        self.boundary_ghost_provider = boundary_ghost_provider
        self.cfl = float(cfl)

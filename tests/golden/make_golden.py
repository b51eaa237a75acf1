"""Generate the golden fixtures for the FR residual-and-update path.

Runs the reference implementation (AutoFlowCFD, pure Python + Numba, read from
``/root/reference``) on small meshes from ``autoflowcfd_b200.boxmesh`` and
stores, per case, every input the path consumes (operators, Jacobians, the
flattened face tables, boundary configuration, turbulence fields, state) and
the reference's own outputs:

* inviscid and viscous residuals (``FRSolver.compute_inviscid_residual`` /
  ``compute_viscous_residual``, ``core/fr_solver/solver.py:351-432``);
* the local time step (``core/fr_solver/cfl.py:12-147``);
* the SST source / transport / point-implicit update
  (``core/fr_solver/turbulence.py:178-330``);
* the state after one and two ``FRSolver.step`` calls
  (``core/fr_solver/step.py:15-221``) and their residual norms;
* the wall force coefficients (``postprocess/fr_coefficients.py:27-152``).

Besides these single-evaluation cases it writes *trajectory* fixtures:
per-step summaries (residual norms, per-variable sums / L2 / extrema, k and
nu_t maxima) and sampled states of longer runs of the reference's
``FRSolver.step``, on meshes the tests regenerate bit-identically with
``autoflowcfd_b200.boxgeom`` (so the fixtures stay small).

The reference cannot be imported where the tests run on a GPU, so the outputs
are committed as ``tests/golden/*.npz``.  Re-run with

    AFR_REFERENCE=<reference checkout> NUMBA_CACHE_DIR=/tmp/nc \
        python tests/golden/make_golden.py [case ...]

(the reference checkout defaults to /root/reference).
"""

import copy
import os
import sys
import time
import types
from types import SimpleNamespace

import numpy as np

REF = os.environ.get("AFR_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REF, "src"))
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/afr_numba_cache")

from autoflowcfd_b200 import boxmesh  # noqa: E402
from flows import (GAMMA, FLOOR_CELLS, c1_vortex, c3_tgv, channel_state, conserved,  # noqa: E402,F401
                   plant_floor_states, tgv_state, vortex_state)
from flows import P as flows_P, RHO as flows_RHO  # noqa: E402
BC_CODES = {"WALL": 0, "FARFIELD": 1, "INLET": 2, "OUTLET": 3, "SYMMETRY": 4}


class _Nodes:
    def __init__(self, c):
        self._c = c

    def get_coordinates(self):
        return self._c


class _Cells:
    def __init__(self, conn):
        self.connectivity = conn


class _Bnd:
    def __init__(self, groups, bc_types):
        self.groups = groups
        self.bc_types = bc_types


def ref_mesh(box, order, bc_types=None):
    """Load a BoxMesh through the reference's own HighOrderMesh loader.

    ``bc_types`` maps plane names to the mesh-level boundary types the
    reference's force integration reads (``postprocess/fr_coefficients.py:74-79``)."""
    from autoflowcfd.grid.high_order.high_order_mesh import HighOrderMesh
    from autoflowcfd.grid.schema.grid_boundaries import BoundaryMap

    nodes = box.nodes.copy()
    conn = box.conn.astype(np.int32).copy()
    Lx, Ly, Lz = box.lengths
    tol = 1e-9 * max(Lx, Ly, Lz, 1.0)
    ijk = box.node_ijk(conn)  # cells touching a plane with >= 3 nodes, by lattice index
    groups = {}
    for name, ax, val in (("x_min", 0, 0), ("x_max", 0, box.shape[0]), ("y_min", 1, 0),
                          ("y_max", 1, box.shape[1]), ("z_min", 2, 0), ("z_max", 2, box.shape[2])):
        groups[name] = np.flatnonzero((ijk[:, :, ax] == val).sum(axis=1) >= 3).astype(np.int32)
    if box.periodic:
        bmap = BoundaryMap(
            groups=groups, bc_types={n: "PERIODIC" for n in groups},
            parameters={"x_min": {"paired_with": "x_max", "translation": [Lx, 0.0, 0.0]},
                        "y_min": {"paired_with": "y_max", "translation": [0.0, Ly, 0.0]},
                        "z_min": {"paired_with": "z_max", "translation": [0.0, 0.0, Lz]}})
    else:
        bmap = _Bnd(groups, dict(bc_types or {n: "FARFIELD" for n in groups}))
    if box.kind == "prism":
        vol = SimpleNamespace(cell_count=len(conn), nodes=_Nodes(nodes), cells=_Cells(np.zeros((0, 4), np.int32)),
                              prism_cells=_Cells(conn), boundaries=bmap)
    else:
        vol = SimpleNamespace(cell_count=len(conn), nodes=_Nodes(nodes), cells=_Cells(conn),
                              prism_cells=_Cells(np.zeros((0, 6), np.int32)), boundaries=bmap)
    mesh = HighOrderMesh(order=order)
    mesh.load_from_volume_mesh(vol, build_faces=True)
    return mesh


def plane_provider(mesh, box, plane_cfg):
    """Face-exact BoundaryGhostStateProvider keyed by the plane each boundary
    face centre lies on (same construction as the reference's
    ``tests/validation/_channel_mesh.py:19-66``)."""
    from autoflowcfd.boundary.fr_ghost_state import BoundaryGhostStateProvider

    fc = mesh.face_connectivity
    group_code = np.full(fc.n_faces, -1, dtype=np.int32)
    bidx = fc.get_boundary_face_indices()
    if len(bidx):
        planes = box.plane_of_faces(fc.face_node_ids[bidx])
        assert np.all(planes >= 0), "boundary face off the box planes"
        group_code[bidx] = planes
    code_to_config = {i: plane_cfg[name] for i, name in enumerate(boxmesh.PLANE_NAMES)}
    default = {"type": "FARFIELD", "Q_free": list(plane_cfg.get("_default_Q", [1.225, 0.0, 0.0, 0.0, 101325.0]))}
    return BoundaryGhostStateProvider(group_code, code_to_config, default)


def bc_tables(provider, n_faces):
    """Lower a BoundaryGhostStateProvider to plain arrays."""
    if provider is None:
        return dict(bc_group=np.full(n_faces, -1, np.int32), bc_type=np.zeros(1, np.int32),
                    bc_noslip=np.ones(1, np.int32), bc_wall_vel=np.zeros((1, 3)),
                    bc_Q=np.zeros((1, 5)), bc_p_out=np.zeros(1), bc_default=np.int32(0))
    codes = sorted(provider.code_to_config)
    n = (max(codes) + 1 if codes else 0) + 1  # last slot = default config
    t = np.zeros(n, np.int32)
    ns = np.ones(n, np.int32)
    wv = np.zeros((n, 3))
    Q = np.zeros((n, 5))
    po = np.zeros(n)

    def put(i, cfg):
        t[i] = BC_CODES[cfg["type"]]
        ns[i] = 1 if cfg.get("is_no_slip", True) else 0
        if cfg.get("wall_velocity") is not None:
            wv[i] = np.asarray(cfg["wall_velocity"], float)
        if "Q_free" in cfg:
            Q[i] = np.asarray(cfg["Q_free"], float)
        if "Q_inlet" in cfg:
            Q[i] = np.asarray(cfg["Q_inlet"], float)
        po[i] = float(cfg.get("p_outlet", 0.0))

    for c in codes:
        put(c, provider.code_to_config[c])
    put(n - 1, provider.default_config)
    gc = np.asarray(provider.group_code, np.int32).copy()
    gc[(gc < 0) | ~np.isin(gc, codes)] = n - 1
    return dict(bc_group=gc, bc_type=t, bc_noslip=ns, bc_wall_vel=wv, bc_Q=Q, bc_p_out=po,
                bc_default=np.int32(n - 1))


def flat_tables(mesh, ops):
    from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry

    f = get_flat_face_geometry(mesh, ops)
    colors = np.full(f.n_faces, -1, np.int32)
    for c, idx in enumerate(f.color_face_indices):
        colors[idx] = c
    return dict(
        owner_cell=f.owner_cell, neighbor_cell=f.neighbor_cell, is_boundary=f.is_boundary.astype(np.uint8),
        owner_axis=f.owner_axis, owner_side=f.owner_side, neighbor_axis=f.neighbor_axis,
        neighbor_side=f.neighbor_side, owner_is_primary=f.owner_is_primary.astype(np.uint8),
        neighbor_is_primary=f.neighbor_is_primary.astype(np.uint8), true_normal=f.true_normal,
        nb_src0_cell=f.neighbor_src0_cell, nb_src0_mat=f.neighbor_src0_mat, nb_src1_idx=f.neighbor_src1_idx,
        nb_src1_cell=f.neighbor_src1_cell, nb_src1_mat=f.neighbor_src1_mat.reshape(-1, f.n_fp, f.n_sps),
        ow_src0_cell=f.owner_src0_cell, ow_src0_mat=f.owner_src0_mat, ow_src1_idx=f.owner_src1_idx,
        ow_src1_cell=f.owner_src1_cell, ow_src1_mat=f.owner_src1_mat.reshape(-1, f.n_fp, f.n_sps),
        boundary_extrap=f.boundary_extrap, g_left=f.g_left, g_right=f.g_right,
        dist_fp_of_sp=f.dist_fp_of_sp, dist_axis_coord_of_sp=f.dist_axis_coord_of_sp, colors=colors,
    )


def op_tables(ops):
    return dict(
        D_3d_prism=ops.D_3d_prism, D_3d_tet=ops.D_3d_tet,
        c2f_prism=ops.overint_interp_c2f_prism, c2f_tet=ops.overint_interp_c2f_tet,
        Dfine_prism=ops.overint_D_fine_prism, Dfine_tet=ops.overint_D_fine_tet,
        f2c_prism=ops.overint_restrict_f2c_prism, f2c_tet=ops.overint_restrict_f2c_tet,
        filter_prism=ops.filter_prism, filter_tet=ops.filter_tet,
    )


def mesh_tables(mesh, solver, mesh_bc):
    """The mesh, operator, face and boundary tables of the solver's current
    order, as the device path consumes them."""
    N, S = mesh.n_cells, mesh.n_sps_per_cell
    out = dict(order=np.int32(mesh.order), n_cells=np.int32(N), n_prism=np.int32(mesh.n_prism_cells),
               n_sps=np.int32(S), n_fine=np.int32(mesh.n_sps_per_cell_fine))
    out["det_jacs"] = mesh.jacobians["det_jacs"].reshape(N, S)
    out["inv_jacs"] = mesh.jacobians["inv_jacs"].reshape(N, S, 3, 3)
    Fn = mesh.n_sps_per_cell_fine
    if mesh.jacobians_fine is None:  # order 0: no over-integration points (the inviscid flux is finite volume)
        Fn = S
        out["n_fine"] = np.int32(S)
        out["det_jacs_fine"] = out["det_jacs"].copy()
        out["inv_jacs_fine"] = out["inv_jacs"].copy()
    else:
        out["det_jacs_fine"] = mesh.jacobians_fine["det_jacs"].reshape(N, Fn)
        out["inv_jacs_fine"] = mesh.jacobians_fine["inv_jacs"].reshape(N, Fn, 3, 3)
    out["cell_volumes"] = mesh.get_all_cell_volumes()
    # the P0 finite-volume divisor: volumes computed at the mesh's load order
    out["fv_cell_volumes"] = np.asarray(mesh.cell_volumes, float)
    out["sps_coords"] = mesh.sps_coords.reshape(N, S, 3)
    out["nodes"] = mesh._node_coords
    out["conn"] = (mesh._fixed_prism_conn if mesh.n_prism_cells else mesh._fixed_tet_conn).astype(np.int64)
    out.update(op_tables(solver.ops))
    out.update(flat_tables(mesh, solver.ops))
    out.update(bc_tables(solver.boundary_ghost_provider, mesh.face_connectivity.n_faces))
    out["true_area_weight"] = np.asarray(mesh.face_flux_points.true_area_weight, float)
    if mesh_bc is not None:
        from autoflowcfd.grid.connectivity.face_connectivity import tag_boundary_groups

        gcode, name_to_code = tag_boundary_groups(mesh.face_connectivity, mesh.boundary_groups)
        wall_codes = [c for n, c in name_to_code.items() if mesh.boundary_bc_types.get(n) == "WALL"]
        out["cd_wall_face"] = np.isin(gcode, wall_codes).astype(np.uint8)
    return out


def make_case(name, box, order, turb, mu, free, plane_cfg, state_fn, inviscid_only=False,
              global_dt_factor=None, n_steps=2, turb_init=None, plant=None, tweak_flat=None,
              time_scheme="ssp_rk3", dt_step=1e-3):
    """Run the reference on one small case and store its inputs and outputs.

    ``plant(U) -> U`` edits the full start state (all n_vars columns) after
    the turbulence columns are set; ``tweak_flat(flat)`` edits the reference's
    cached ``FlatFaceGeometry`` in place before anything is evaluated, so every
    consumer of the face tables (residual kernels, transport, the stored
    tables) sees the same arrays."""
    import numba
    from autoflowcfd.core.fr_solver import FRSolver
    from autoflowcfd.core.time_integration import TimeIntegrationScheme
    from autoflowcfd.postprocess.fr_coefficients import compute_aerodynamic_coefficients_fr

    numba.set_num_threads(min(8, os.cpu_count() or 1))
    mesh_bc = None
    if plane_cfg is not None:
        mesh_bc = {n: ("WALL" if plane_cfg[n]["type"] == "WALL" and plane_cfg[n].get("is_no_slip", True)
                       else "FARFIELD") for n in boxmesh.PLANE_NAMES}
    mesh = ref_mesh(box, order, mesh_bc)
    rho_inf, u_inf, p_inf = free
    solver = FRSolver(mesh=mesh, order=order, turb_model_name=turb, time_scheme=TimeIntegrationScheme(time_scheme),
                      rho_inf=rho_inf, vel_inf=u_inf, p_inf=p_inf, mu_molecular=mu,
                      n_threads=min(8, os.cpu_count() or 1))
    solver.order_continuation_enabled = False
    if not box.periodic:
        solver.boundary_ghost_provider = plane_provider(mesh, box, plane_cfg)
    if tweak_flat is not None:
        from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry

        tweak_flat(get_flat_face_geometry(mesh, solver.ops))
    N, S = mesh.n_cells, mesh.n_sps_per_cell
    n_vars = solver.state.n_vars
    xyz = mesh.sps_coords.reshape(N, S, 3)
    U = np.zeros((N, S, n_vars))
    U[:, :, :5] = state_fn(xyz[..., 0], xyz[..., 1], xyz[..., 2])

    out = dict(meta_name=np.array(name), order=np.int32(order), n_cells=np.int32(N), n_prism=np.int32(mesh.n_prism_cells),
               n_sps=np.int32(S), n_fine=np.int32(mesh.n_sps_per_cell_fine), n_vars=np.int32(n_vars),
               turb=np.array(turb), mu=np.float64(mu), freestream=np.array(free, float),
               inviscid_only=np.int32(inviscid_only), periodic=np.int32(box.periodic),
               global_dt_factor=np.float64(global_dt_factor or 0.0),
               box_shape=np.array(box.shape), box_lengths=np.array(box.lengths), box_kind=np.array(box.kind),
               time_scheme=np.array(time_scheme), dt_step=np.float64(dt_step),
               dual_time_inner_iter=np.int32(solver.time_integrator.dual_time_steps))
    out.update(mesh_tables(mesh, solver, mesh_bc))
    Fn = int(out["n_fine"])

    if turb == "SST":
        nodes = mesh._node_coords
        wall = np.flatnonzero(np.abs(nodes[:, 2]) < 1e-12)
        solver.compute_wall_distance_field(nodes, wall)
        out["wall_distance"] = solver.wall_distance.copy()
        k0, w0, nut0 = turb_init(xyz)
        solver.turb_model.k_field = k0.copy()
        solver.turb_model.omega_field = w0.copy()
        solver.turb_model.nu_t = nut0.copy()
        rho = U[:, :, 0]
        U[:, :, 5] = rho * k0
        U[:, :, 6] = rho * w0
        out["k0"], out["omega0"], out["nu_t0"] = k0, w0, nut0
    if plant is not None:
        U = plant(U)
    out["U0"] = U.copy()

    orig_dt = solver._compute_local_time_step

    def snapshot():
        snap = dict(U=solver.state.U.copy())
        if solver.turb_model is not None:
            snap.update(k=solver.turb_model.k_field.copy(), w=solver.turb_model.omega_field.copy(),
                        nut=solver.turb_model.nu_t.copy())
        return snap

    def restore(snap):
        solver.state.U = snap["U"].copy()
        solver.state._update_primitives()
        if solver.turb_model is not None:
            solver.turb_model.k_field = snap["k"].copy()
            solver.turb_model.omega_field = snap["w"].copy()
            solver.turb_model.nu_t = snap["nut"].copy()
            if hasattr(solver.turb_model, "_last_beta_blend"):
                del solver.turb_model._last_beta_blend

    solver.state.U = U.copy()
    solver.state._update_primitives()
    s0 = snapshot()

    # --- single evaluations at the initial state ---
    out["R_inv"] = solver.compute_inviscid_residual().copy()
    out["R_visc"] = solver.compute_viscous_residual().copy()
    out["dt_local"] = orig_dt().copy()
    restore(s0)

    if turb == "SST":
        import autoflowcfd.core.turbulence.transport as tr

        captured = {}
        real = tr.compute_turbulence_transport_residual

        def spy(*a, **kw):
            r = real(*a, **kw)
            captured["tk"], captured["tw"] = r[0].copy(), r[1].copy()
            return r

        tr.compute_turbulence_transport_residual = spy
        try:
            dtl = orig_dt()
            Sk, Sw = solver.compute_turbulence_source(dtl)
        finally:
            tr.compute_turbulence_transport_residual = real
        out["sst_Sk"], out["sst_Sw"] = Sk.copy(), Sw.copy()
        out["sst_tk"], out["sst_tw"] = captured["tk"], captured["tw"]
        out["sst_k1"] = solver.turb_model.k_field.copy()
        out["sst_w1"] = solver.turb_model.omega_field.copy()
        out["sst_nut1"] = solver.turb_model.nu_t.copy()
        restore(s0)

    # --- full steps ---
    if global_dt_factor:
        solver._compute_local_time_step = lambda: np.full((N, S), global_dt_factor * float(np.min(orig_dt())))
    if inviscid_only:
        solver.compute_viscous_residual = lambda: np.zeros_like(solver.state.U)
    # count the points each clamp of enforce_positivity acts on during the steps
    import autoflowcfd.core.time_integration.base as tib

    trips = np.zeros(5, np.int64)
    real_pos = tib.enforce_positivity

    def positivity_spy(Uf, p_floor=1.0):
        rho = np.maximum(Uf[:, 0], 1e-6)
        vel = Uf[:, 1:4] / rho[:, None]
        vm = np.sqrt(np.sum(vel**2, axis=1))
        vel = np.where((vm > 1e4)[:, None], vel * (1e4 / np.maximum(vm, 1e-300))[:, None], vel)
        pp = (GAMMA - 1.0) * (Uf[:, 4] - 0.5 * rho * np.sum(vel**2, axis=1))
        trips[:] += [np.sum(Uf[:, 0] < 1e-6), np.sum(vm > 1e4), np.sum(pp < p_floor),
                     np.sum(Uf[:, 5] < 0.0) if Uf.shape[1] > 5 else 0, np.sum(Uf[:, 6] < 1e-8) if Uf.shape[1] > 6 else 0]
        return real_pos(Uf, p_floor)

    tib.enforce_positivity = positivity_spy
    norms = []
    for s in range(n_steps):
        norms.append(solver.step(dt_step))
        out[f"U_step{s + 1}"] = solver.state.U.copy()
        if solver.turb_model is not None:
            out[f"k_step{s + 1}"] = solver.turb_model.k_field.copy()
            out[f"w_step{s + 1}"] = solver.turb_model.omega_field.copy()
            out[f"nut_step{s + 1}"] = solver.turb_model.nu_t.copy()
    out["norms"] = np.array(norms)
    tib.enforce_positivity = real_pos
    out["positivity_trips"] = trips  # points clamped: rho, |u|, p, rho*k, rho*omega

    if not box.periodic and not inviscid_only:
        coef = compute_aerodynamic_coefficients_fr(solver, reference_area=1.0)
        out["cd_cl"] = np.array([coef.Cd, coef.Cl, coef.Cs], float)
    if tweak_flat is not None:
        from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry

        # the tweaked tables stayed the ones in use for the whole run
        assert np.array_equal(get_flat_face_geometry(mesh, solver.ops).true_normal, out["true_normal"])
    # operators the reference does not build at this order (None) are left out
    out = {k: v for k, v in out.items() if v is not None and not (isinstance(v, np.ndarray) and v.dtype == object)}
    for k, v in out.items():
        if isinstance(v, np.ndarray) and v.dtype.kind == "f":
            assert np.all(np.isfinite(v)), f"{name}: non-finite reference output {k}"
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: N={N} S={S} faces={len(out['owner_cell'])} colors={out['colors'].max() + 1} "
          f"norms={norms}", flush=True)
    return out


def make_continuation(name, box, order, mu, free, plane_cfg, max_iter, tol, dt=1e-3, inviscid_only=False,
                      turb="NONE"):
    """Run the reference's FRSolver.solve at ``order`` >= 2, which runs its
    order continuation (core/utils/order_continuation.py:207-425), and store
    every phase's tables (keys ``p<order>/<table>``, as that phase's mesh
    and operators give them), each step's order and residual, the state at
    the start and end of every phase and the SolverResult."""
    import numba
    from autoflowcfd.core.fr_solver import FRSolver

    numba.set_num_threads(min(8, os.cpu_count() or 1))
    mesh_bc = None
    if plane_cfg is not None:
        mesh_bc = {n: ("WALL" if plane_cfg[n]["type"] == "WALL" and plane_cfg[n].get("is_no_slip", True)
                       else "FARFIELD") for n in boxmesh.PLANE_NAMES}
    mesh = ref_mesh(box, order, mesh_bc)
    rho_inf, u_inf, p_inf = free
    solver = FRSolver(mesh=mesh, order=order, turb_model_name=turb, rho_inf=rho_inf, vel_inf=u_inf, p_inf=p_inf,
                      mu_molecular=mu, n_threads=min(8, os.cpu_count() or 1))
    assert solver.order_continuation_enabled
    if not box.periodic:
        solver.boundary_ghost_provider = plane_provider(mesh, box, plane_cfg)
    if inviscid_only:
        solver.compute_viscous_residual = lambda *a, **k: np.zeros_like(solver.state.U)
    out = dict(meta_name=np.array(name), order=np.int32(order), n_cells=np.int32(mesh.n_cells),
               n_vars=np.int32(solver.state.n_vars), turb=np.array(turb), mu=np.float64(mu),
               freestream=np.array(free, float), inviscid_only=np.int32(inviscid_only),
               periodic=np.int32(box.periodic), global_dt_factor=np.float64(0.0),
               max_iter=np.int32(max_iter), tol=np.float64(tol), dt=np.float64(dt))
    if turb == "SST":
        # wall distance at the target order's points (the continuation's P0
        # restart compresses it to cell means and each phase prolongs it)
        nodes = np.asarray(mesh._node_coords, float)
        solver.compute_wall_distance_field(nodes, np.flatnonzero(np.abs(nodes[:, 2]) < 1e-12))
        out["wall_distance"] = solver.wall_distance.copy()
    real_step = solver.step
    log_order, log_res = [], []

    def step(dt_):
        p = solver.current_order
        if f"U_start_p{p}" not in out:
            for k, v in mesh_tables(solver.mesh, solver, mesh_bc).items():
                if v is not None and not (isinstance(v, np.ndarray) and v.dtype == object):
                    out[f"p{p}/{k}"] = v
            out[f"U_start_p{p}"] = solver.state.U.copy()
            if turb == "SST":
                out[f"wall_distance_p{p}"] = np.asarray(solver.wall_distance, float).copy()
                out[f"k_start_p{p}"] = solver.turb_model.k_field.copy()
                out[f"w_start_p{p}"] = solver.turb_model.omega_field.copy()
                out[f"nut_start_p{p}"] = np.asarray(solver.turb_model.nu_t, float).copy()
        r = real_step(dt_)
        if f"p{p}/mfs_cache" not in out:
            out[f"p{p}/mfs_cache"] = np.asarray(solver._metric_flux_scale_cache, float).copy()
        log_order.append(p)
        log_res.append(r)
        out[f"U_end_p{p}"] = solver.state.U.copy()
        if turb == "SST":
            out[f"k_end_p{p}"] = solver.turb_model.k_field.copy()
            out[f"w_end_p{p}"] = solver.turb_model.omega_field.copy()
            out[f"nut_end_p{p}"] = np.asarray(solver.turb_model.nu_t, float).copy()
        return r

    solver.step = step
    res = solver.solve(max_iter=max_iter, dt=dt, tol=tol)
    out["step_order"] = np.array(log_order, np.int32)
    out["step_residual"] = np.array(log_res)
    out["result"] = np.array([float(res.converged), float(res.iterations), float(res.final_residual)])
    out["U_final"] = solver.state.U.copy()
    for k, v in out.items():
        if isinstance(v, np.ndarray) and v.dtype.kind == "f":
            assert np.all(np.isfinite(v)), f"{name}: non-finite reference output {k}"
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: N={mesh.n_cells} phases={sorted(set(log_order))} steps={len(log_res)} "
          f"result={out['result']}", flush=True)
    return out


def make_fluxpoints(name, box, order, mesh_bc=None):
    """Inputs and outputs of the reference's flux-point construction
    (fr/face_flux_points_merge.py:51-434 with fr/face_flux_points_numba.py
    and face_flux_points_ms_numba.py) on one box mesh: its FRFaceConnectivity
    and cell connectivity in, the flattened face tables and the raw Newton
    coordinates and residuals out."""
    from autoflowcfd.core.fr_operators.face_kernels import get_flat_face_geometry
    from autoflowcfd.fr.operators import generate_fr_operators

    mesh = ref_mesh(box, order, mesh_bc)
    fc = mesh.face_connectivity
    ffp = mesh.face_flux_points
    ops = generate_fr_operators(order)
    out = dict(meta_name=np.array(name), order=np.int32(order), n_cells=np.int32(mesh.n_cells),
               n_prism=np.int32(mesh.n_prism_cells), nodes=np.asarray(mesh._node_coords, float))
    out["prism_conn"] = (np.asarray(mesh._fixed_prism_conn, np.int64) if mesh._fixed_prism_conn is not None
                         else np.zeros((0, 6), np.int64))
    out["tet_conn"] = (np.asarray(mesh._fixed_tet_conn, np.int64) if mesh._fixed_tet_conn is not None
                       else np.zeros((0, 4), np.int64))
    for k in ("owner_cell", "neighbor_cell", "owner_cube_face", "neighbor_cube_face", "area", "normal",
              "face_node_ids", "is_boundary", "face_translation"):
        out["fc_" + k] = np.asarray(getattr(fc, k))
    out.update(flat_tables(mesh, ops))
    out["true_area_weight"] = np.asarray(ffp.true_area_weight, float)
    out["nb_fc"], out["ow_fc"] = np.asarray(ffp._nb_fc), np.asarray(ffp._ow_fc)
    out["nb_resid"], out["ow_resid"] = np.asarray(ffp._nb_resid), np.asarray(ffp._ow_resid)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: N={mesh.n_cells} faces={fc.n_faces} multi-source nb={int(np.sum(out['nb_src1_idx'] >= 0))} "
          f"ow={int(np.sum(out['ow_src1_idx'] >= 0))} periodic={bool(np.any(out['fc_face_translation'] != 0))}",
          flush=True)
    return out


def _summaries(U, k=None, nut=None):
    """Per-variable sum, L2, max and min of a state (and k / nu_t maxima)."""
    flat = U.reshape(-1, U.shape[-1])
    out = dict(sum=flat.sum(0), l2=np.sqrt((flat * flat).sum(0)), max=flat.max(0), min=flat.min(0),
               finite=np.int32(np.all(np.isfinite(U))))
    if k is not None:
        out.update(k_max=np.max(k), nut_max=np.max(nut), k_min=np.min(k))
    return out


def make_trajectory(name, box, order, turb, mu, free, plane_cfg, state_xyz, n_steps, *, inviscid_only=False,
                    global_dt_factor=None, turb_xyz=None, sample_steps=(), stride=1, stop_nonfinite=True):
    """Run the reference's FRSolver.step n_steps times from a start state and
    store per-step summaries plus sampled states (every ``stride``-th cell).

    ``state_xyz(xyz) -> U[..., :5]`` and ``turb_xyz(xyz) -> (k, omega, nu_t)``
    are evaluated on the reference mesh's solution points, which the
    box-mesh generator reproduces bit for bit, so a test rebuilds the same
    start state from the same formulas."""
    import numba
    from autoflowcfd.core.fr_solver import FRSolver
    from autoflowcfd.core.time_integration import TimeIntegrationScheme

    numba.set_num_threads(min(8, os.cpu_count() or 1))
    mesh_bc = None
    if plane_cfg is not None:
        mesh_bc = {n: ("WALL" if plane_cfg[n]["type"] == "WALL" and plane_cfg[n].get("is_no_slip", True)
                       else "FARFIELD") for n in boxmesh.PLANE_NAMES}
    mesh = ref_mesh(box, order, mesh_bc)
    rho_inf, u_inf, p_inf = free
    solver = FRSolver(mesh=mesh, order=order, turb_model_name=turb, time_scheme=TimeIntegrationScheme.SSP_RK3,
                      rho_inf=rho_inf, vel_inf=u_inf, p_inf=p_inf, mu_molecular=mu,
                      n_threads=min(8, os.cpu_count() or 1))
    solver.order_continuation_enabled = False
    if not box.periodic:
        solver.boundary_ghost_provider = plane_provider(mesh, box, plane_cfg)
    N, S = mesh.n_cells, mesh.n_sps_per_cell
    xyz = mesh.sps_coords.reshape(N, S, 3)
    U = np.zeros((N, S, solver.state.n_vars))
    U[:, :, :5] = state_xyz(xyz)
    out = dict(meta_name=np.array(name), order=np.int32(order), n_cells=np.int32(N), n_sps=np.int32(S),
               turb=np.array(turb), mu=np.float64(mu), freestream=np.array(free, float),
               inviscid_only=np.int32(inviscid_only), global_dt_factor=np.float64(global_dt_factor or 0.0),
               box_kind=np.array(box.kind), box_shape=np.array(box.shape), box_lengths=np.array(box.lengths),
               box_periodic=np.int32(box.periodic), stride=np.int32(stride))
    if turb == "SST":
        nodes = mesh._node_coords
        solver.compute_wall_distance_field(nodes, np.flatnonzero(np.abs(nodes[:, 2]) < 1e-12))
        k0, w0, nut0 = turb_xyz(xyz)
        solver.turb_model.k_field = k0.copy()
        solver.turb_model.omega_field = w0.copy()
        solver.turb_model.nu_t = nut0.copy()
        U[:, :, 5] = U[:, :, 0] * k0
        U[:, :, 6] = U[:, :, 0] * w0
    out["U0_sample"] = U[::stride].copy()
    solver.state.U = U.copy()
    solver.state._update_primitives()
    if global_dt_factor:
        orig_dt = solver._compute_local_time_step
        solver._compute_local_time_step = lambda: np.full((N, S), global_dt_factor * float(np.min(orig_dt())))
    if inviscid_only:
        solver.compute_viscous_residual = lambda: np.zeros_like(solver.state.U)
    rows = []
    t0 = time.time()
    for it in range(1, n_steps + 1):
        with np.errstate(all="ignore"):
            norm = solver.step(1e-3)
        tm = solver.turb_model
        row = _summaries(solver.state.U, None if tm is None else tm.k_field, None if tm is None else tm.nu_t)
        row["norm"] = norm
        rows.append(row)
        if it in sample_steps:
            out[f"U_s{it}"] = solver.state.U[::stride].copy()
            if tm is not None:
                out[f"k_s{it}"] = tm.k_field[::stride].copy()
                out[f"w_s{it}"] = tm.omega_field[::stride].copy()
                out[f"nut_s{it}"] = tm.nu_t[::stride].copy()
        print(f"{name}: step {it} norm {norm:.6e} finite {row['finite']} "
              + (f"k_max {row['k_max']:.4e} nut_max {row['nut_max']:.4e} " if tm is not None else "")
              + f"({time.time() - t0:.0f} s)", flush=True)
        if stop_nonfinite and not row["finite"]:
            break
    for key in rows[0]:
        out["step_" + key] = np.array([r[key] for r in rows])
    out["n_steps_run"] = np.int32(len(rows))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


def main(which=None):
    cases = {}

    def c_tet_p1():
        L = 1.0
        box = boxmesh.tet_box(3, 3, 3, (L, L, L), jitter=0.0, periodic=True)
        rho, p = 1.225, 101325.0
        u = 0.5 * np.sqrt(GAMMA * p / rho)
        make_case("tet_p1_vortex", box, 1, "NONE", 1.8e-5, (rho, u, p), None,
                  lambda x, y, z: vortex_state(x, y, L, L, 0.2 * L, rho, p, u),
                  inviscid_only=True, global_dt_factor=3.0)

    def c_prism_p2_sst():
        Ls = (4.0, 2.0, 1.5)
        box = boxmesh.prism_box(4, 3, 3, Ls, jitter=0.1, seed=7)
        rho, p = 1.225, 101325.0
        u = 0.1 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e6
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        k_in = 1.5 * (0.01 * u) ** 2
        w_in = rho * k_in / (10 * mu)

        def turb_init(xyz):
            rng = np.random.default_rng(3)
            N, S = xyz.shape[:2]
            pert = 1 + 0.2 * np.sin(2 * np.pi * xyz[..., 0] / Ls[0] + 0.3) * np.cos(np.pi * xyz[..., 2] / Ls[2])
            k = k_in * pert
            w = w_in * (1 + 0.3 * np.cos(2 * np.pi * xyz[..., 1] / Ls[1]))
            nut = 10 * mu / rho * (1 + 0.5 * rng.uniform(size=(N, S)))
            return k, w, nut

        make_case("prism_p2_sst", box, 2, "SST", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 11), turb_init=turb_init)

    def c_prism_p1_ns():
        Ls = (2.0, 1.0, 1.0)
        box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3))
        rho, p = 1.225, 101325.0
        u = 0.2 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e5
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
        cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
        cfg["y_min"] = {"type": "SYMMETRY"}
        cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
        make_case("prism_p1_ns", box, 1, "NONE", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 5))

    def c_tet_p3():
        L = 1.0
        box = boxmesh.tet_box(2, 2, 2, (L, L, L), jitter=0.05, seed=9, periodic=True)
        rho, p = 1.225, 101325.0
        u0 = 0.1 * np.sqrt(GAMMA * p / rho)
        make_case("tet_p3_tgv", box, 3, "NONE", 1.8e-5, (rho, 0.0, p), None,
                  lambda x, y, z: tgv_state(x, y, z, L, u0, rho, p), inviscid_only=True, global_dt_factor=3.0,
                  n_steps=1)

    def c_prism_p1_floors():
        """Start states beyond every floor and clamp of the path (values far
        from the thresholds): the AUSM+up rho >= 1e-6 / p >= 10 Pa floors
        (core/fr_operators/kernels.py:41-44) and every clamp of
        enforce_positivity (core/time_integration/positivity.py:13-45)."""
        Ls = (2.0, 1.0, 1.0)
        box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5)
        rho, p = 1.225, 101325.0
        u = 0.2 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e5
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        k_in = 1.5 * (0.01 * u) ** 2
        w_in = rho * k_in / (10 * mu)

        def turb_init(xyz):
            N, S = xyz.shape[:2]
            k = k_in * (1 + 0.2 * np.sin(2 * np.pi * xyz[..., 0] / Ls[0]))
            w = w_in * (1 + 0.3 * np.cos(2 * np.pi * xyz[..., 1] / Ls[1]))
            return k, w, k / w

        make_case("prism_p1_floors", box, 1, "SST", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 17), turb_init=turb_init,
                  plant=plant_floor_states)

    def c_tet_p1_align():
        """Face normals that disagree with the adjugate direction: on records
        f % 7 == 3 every flux point's true normal is reversed (alignment -1),
        on records f % 11 == 5 the even flux points' normals are turned by
        90 degrees (alignment ~0); both take the reference's fallback to the
        true normal (core/fr_residual/inviscid_kernel_colored.py:104-108 and
        its neighbour-side twin at :186-190)."""
        L = 1.0
        box = boxmesh.tet_box(3, 3, 3, (L, L, L), jitter=0.0, periodic=True)
        rho, p = 1.225, 101325.0
        u = 0.5 * np.sqrt(GAMMA * p / rho)

        def tweak(flat):
            tn = flat.true_normal
            F = tn.shape[0]
            rev = np.arange(F) % 7 == 3
            tn[rev] = -tn[rev]
            rot = np.flatnonzero(np.arange(F) % 11 == 5)
            for f in rot:
                for i in range(0, tn.shape[1], 2):
                    n = tn[f, i].copy()
                    e = np.array([1.0, 0.0, 0.0]) if abs(n[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
                    t = np.cross(n, e)
                    tn[f, i] = t / np.linalg.norm(t)

        make_case("tet_p1_align", box, 1, "NONE", 1.8e-5, (rho, u, p), None,
                  lambda x, y, z: vortex_state(x, y, L, L, 0.2 * L, rho, p, u),
                  inviscid_only=True, global_dt_factor=3.0, tweak_flat=tweak)

    def t_c1():
        """The small configuration at full size: 16^3 hex -> 24,576 periodic
        tets, P1, isentropic vortex, Euler, global dt 3 min(dt_local), 100 steps."""
        box = boxmesh.tet_box(16, 16, 16, (1.0, 1.0, 1.0), jitter=0.0, periodic=True)
        u = c1_vortex(np.zeros((1, 1, 3)))[1]
        make_trajectory("traj_c1_vortex", box, 1, "NONE", 1.8e-5, (flows_RHO, u, flows_P), None,
                        lambda xyz: c1_vortex(xyz)[0], 100, inviscid_only=True, global_dt_factor=3.0,
                        sample_steps=(1, 100), stride=8)

    def t_c2_sample():
        """The C2 generator on its 8 x 6 x 6-hex sample (576 prisms, P2, SST,
        the bench's start state), 20 steps: k and nu_t through the SST growth."""
        import bench

        spec = bench.SAMPLE
        box = boxmesh.prism_box(*spec["shape"], spec["lengths"], jitter=spec["jitter"], seed=spec["seed"])
        rho, u, p, mu, k0, w0 = bench.flow_conditions()

        def state(xyz):
            return bench.initial_state({"sps_coords": xyz}, spec)[0][..., :5]

        def turb(xyz):
            _, k, w, nut, _ = bench.initial_state({"sps_coords": xyz}, spec)
            return k, w, nut

        make_trajectory("traj_c2_sample", box, 2, "SST", mu, (rho, u, p), bench.plane_cfg(), state, 20,
                        turb_xyz=turb, sample_steps=(1, 6, 12), stride=1)

    def t_p3():
        """The precision-stress configuration at the oracle's size: 8^3 hex ->
        3,072 jittered periodic tets, P3, Taylor-Green at Mach 0.1, Euler,
        global dt; run until the state is non-finite (at most 12 steps)."""
        box = boxmesh.tet_box(8, 8, 8, (1.0, 1.0, 1.0), jitter=0.05, seed=7, periodic=True)
        make_trajectory("traj_p3_tgv", box, 3, "NONE", 1.8e-5, (flows_RHO, 0.0, flows_P), None,
                        lambda xyz: c3_tgv(xyz)[0], 12, inviscid_only=True, global_dt_factor=3.0,
                        sample_steps=(1,), stride=16)

    def c_prism_p1_ns_scheme(scheme, dt_step):
        Ls = (2.0, 1.0, 1.0)
        box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3))
        rho, p = 1.225, 101325.0
        u = 0.2 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e5
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
        cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
        cfg["y_min"] = {"type": "SYMMETRY"}
        cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
        make_case(f"prism_p1_ns_{scheme}", box, 1, "NONE", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 5), time_scheme=scheme, dt_step=dt_step,
                  n_steps=3)

    def c_prism_p2_sst_scheme(scheme, dt_step):
        Ls = (4.0, 2.0, 1.5)
        box = boxmesh.prism_box(4, 3, 3, Ls, jitter=0.1, seed=7)
        rho, p = 1.225, 101325.0
        u = 0.1 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e6
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        k_in = 1.5 * (0.01 * u) ** 2
        w_in = rho * k_in / (10 * mu)

        def turb_init(xyz):
            rng = np.random.default_rng(3)
            N, S = xyz.shape[:2]
            pert = 1 + 0.2 * np.sin(2 * np.pi * xyz[..., 0] / Ls[0] + 0.3) * np.cos(np.pi * xyz[..., 2] / Ls[2])
            k = k_in * pert
            w = w_in * (1 + 0.3 * np.cos(2 * np.pi * xyz[..., 1] / Ls[1]))
            nut = 10 * mu / rho * (1 + 0.5 * rng.uniform(size=(N, S)))
            return k, w, nut

        make_case(f"prism_p2_sst_{scheme}", box, 2, "SST", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 11), turb_init=turb_init,
                  time_scheme=scheme, dt_step=dt_step, n_steps=2)

    def c_prism_p0_ns():
        """Order 0 (one solution point per cell): the finite-volume inviscid flux
        (core/fr_residual/inviscid_p0.py) and the P0 viscous terms."""
        Ls = (2.0, 1.0, 1.0)
        box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3))
        rho, p = 1.225, 101325.0
        u = 0.2 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e5
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
        cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
        cfg["y_min"] = {"type": "SYMMETRY"}
        cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
        make_case("prism_p0_ns", box, 0, "NONE", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 5), n_steps=3)

    def c_prism_p0_sst():
        """Order 0 with the SST closure: the finite-volume mean flow and the
        reference's generic FR transport / source / point-implicit update at
        one point per cell (core/fr_solver/turbulence.py, core/turbulence/)."""
        Ls = (2.0, 1.0, 1.0)
        box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5)
        rho, p = 1.225, 101325.0
        u = 0.1 * np.sqrt(GAMMA * p / rho)
        mu = rho * u / 1e6
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        k_in = 1.5 * (0.01 * u) ** 2
        w_in = rho * k_in / (10 * mu)

        def turb_init(xyz):
            rng = np.random.default_rng(3)
            N, S = xyz.shape[:2]
            pert = 1 + 0.2 * np.sin(2 * np.pi * xyz[..., 0] / Ls[0] + 0.3) * np.cos(np.pi * xyz[..., 2] / Ls[2])
            k = k_in * pert
            w = w_in * (1 + 0.3 * np.cos(2 * np.pi * xyz[..., 1] / Ls[1]))
            nut = 10 * mu / rho * (1 + 0.5 * rng.uniform(size=(N, S)))
            return k, w, nut

        make_case("prism_p0_sst", box, 0, "SST", mu, (rho, u, p), cfg,
                  lambda x, y, z: channel_state(x, y, z, Ls, rho, u, p, 5), turb_init=turb_init, n_steps=3)

    def c_tet_p0_vortex():
        L = 1.0
        box = boxmesh.tet_box(3, 3, 3, (L, L, L), jitter=0.0, periodic=True)
        rho, p = 1.225, 101325.0
        u = 0.5 * np.sqrt(GAMMA * p / rho)
        make_case("tet_p0_vortex", box, 0, "NONE", 1.8e-5, (rho, u, p), None,
                  lambda x, y, z: vortex_state(x, y, L, L, 0.2 * L, rho, p, u),
                  inviscid_only=True, global_dt_factor=3.0, n_steps=3)

    def k_cont_prism_p2():
        """Order continuation P0 -> P1 -> P2 on a small wall-bump box (all five
        boundary types), a few steps per phase."""
        Ls = (1.5, 1.0, 1.0)
        box = boxmesh.prism_box(3, 2, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 0.75, 0.5, 0.3))
        rho, p = 1.225, 101325.0
        u = 0.2 * np.sqrt(GAMMA * p / rho)
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
        cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
        cfg["y_min"] = {"type": "SYMMETRY"}
        cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
        make_continuation("cont_prism_p2_ns", box, 2, rho * u / 1e5, (rho, u, p), cfg, max_iter=12, tol=1e-6)

    def k_cont_prism_p2_sst():
        """Order continuation P0 -> P1 -> P2 with the SST closure on a jittered
        box with a no-slip wall at z = 0: the P0 restart of k, omega, nu_t and
        the wall distance (cell means of the target order's field) and their
        prolongation between phases."""
        Ls = (1.5, 1.0, 1.0)
        box = boxmesh.prism_box(3, 2, 2, Ls, jitter=0.1, seed=5)
        rho, p = 1.225, 101325.0
        u = 0.1 * np.sqrt(GAMMA * p / rho)
        Qf = [rho, u, 0.0, 0.0, p]
        cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
        cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
        make_continuation("cont_prism_p2_sst", box, 2, rho * u / 1e6, (rho, u, p), cfg, max_iter=12, tol=1e-6,
                          turb="SST")

    def k_cont_tet_p2():
        """Order continuation on a periodic box from the uniform free stream:
        the residual (rounding of the free-stream preservation: ~4e-8 at P0,
        ~4e-5 at P1, ~1.5 at P2) is under every phase tolerance at its first
        step, so each phase converges at once and the run returns converged."""
        L = 1.0
        box = boxmesh.tet_box(2, 2, 2, (L, L, L), jitter=0.0, periodic=True)
        rho, p = 1.225, 101325.0
        u = 0.5 * np.sqrt(GAMMA * p / rho)
        make_continuation("cont_tet_p2_uniform", box, 2, 1.8e-5, (rho, u, p), None, max_iter=30, tol=2.0,
                          inviscid_only=True)

    def f_fluxpoints():
        wall = {n: "FARFIELD" for n in boxmesh.PLANE_NAMES}
        wall["z_min"] = "WALL"
        make_fluxpoints("fp_prism_p2", boxmesh.prism_box(4, 3, 3, (4.0, 2.0, 1.5), jitter=0.1, seed=7), 2, wall)
        make_fluxpoints("fp_prism_p3_bump", boxmesh.prism_box(3, 2, 2, (1.5, 1.0, 1.0), jitter=0.1, seed=5,
                                                              bump=(0.05, 0.75, 0.5, 0.3)), 3, wall)
        make_fluxpoints("fp_prism_p1", boxmesh.prism_box(4, 3, 2, (2.0, 1.0, 1.0), jitter=0.1, seed=5,
                                                         bump=(0.05, 1.0, 0.5, 0.3)), 1, wall)
        make_fluxpoints("fp_tet_p3", boxmesh.tet_box(2, 2, 2, (1.0, 1.0, 1.0), jitter=0.05, seed=9, periodic=True), 3)
        make_fluxpoints("fp_tet_p2", boxmesh.tet_box(3, 3, 3, (1.0, 1.0, 1.0), jitter=0.05, seed=4, periodic=True), 2)

    cases = {"tet_p1_vortex": c_tet_p1, "prism_p2_sst": c_prism_p2_sst, "prism_p1_ns": c_prism_p1_ns,
             "tet_p3_tgv": c_tet_p3, "prism_p1_floors": c_prism_p1_floors, "tet_p1_align": c_tet_p1_align,
             "traj_c1_vortex": t_c1, "traj_c2_sample": t_c2_sample, "traj_p3_tgv": t_p3,
             "prism_p1_ns_dual_time": lambda: c_prism_p1_ns_scheme("dual_time", 2e-5),
             "prism_p1_ns_imex_euler": lambda: c_prism_p1_ns_scheme("imex_euler", 1e-3),
             "prism_p2_sst_dual_time": lambda: c_prism_p2_sst_scheme("dual_time", 2e-5),
             "prism_p0_ns": c_prism_p0_ns, "prism_p0_sst": c_prism_p0_sst, "tet_p0_vortex": c_tet_p0_vortex,
             "cont_prism_p2_ns": k_cont_prism_p2, "cont_tet_p2_uniform": k_cont_tet_p2,
             "cont_prism_p2_sst": k_cont_prism_p2_sst,
             "fluxpoints": f_fluxpoints}
    for k, fn in cases.items():
        if which and k not in which:
            continue
        fn()


if __name__ == "__main__":
    main(sys.argv[1:] or None)

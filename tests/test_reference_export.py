"""The product-side exporter (autoflowcfd_b200.reference_io) lowers the
reference's own mesh, operators and ghost provider to the tables the golden
fixtures hold, and refuses what cannot run on the device.

The first test builds the reference's objects and needs the reference
checkout (AFR_REFERENCE, default /root/reference); it is skipped where the
reference is not installed.  The others need neither the reference nor a GPU.
"""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from autoflowcfd_b200 import _lib
from autoflowcfd_b200.reference_io import export_case, lower_ghost_provider
from conftest import golden_path

REF_SRC = os.path.join(os.environ.get("AFR_REFERENCE", "/root/reference"), "src")


def _reference_available():
    try:
        import importlib.util

        return os.path.isdir(os.path.join(REF_SRC, "autoflowcfd")) and importlib.util.find_spec("numba") is not None
    except Exception:
        return False


@pytest.mark.skipif(not _reference_available(), reason="the reference checkout is not installed here")
@pytest.mark.parametrize("order", [1, 0])
def test_exporter_reproduces_the_golden_tables(order):
    """prism_p1_ns / prism_p0_ns: a wall-bump box with WALL / FARFIELD / INLET /
    OUTLET / SYMMETRY / slip-wall planes, exported from the reference's
    HighOrderMesh, FROperators and BoundaryGhostStateProvider by the product
    code (order 0: no over-integration points or operators)."""
    import make_golden as mg
    from autoflowcfd.core.fr_solver import FRSolver
    from autoflowcfd_b200 import boxmesh

    g = np.load(golden_path(f"prism_p{order}_ns"))
    Ls = (2.0, 1.0, 1.0)
    box = boxmesh.prism_box(4, 3, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 1.0, 0.5, 0.3))
    rho, p = 1.225, 101325.0
    u = 0.2 * np.sqrt(1.4 * p / rho)
    Qf = [rho, u, 0.0, 0.0, p]
    cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
    cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
    cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
    cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
    cfg["y_min"] = {"type": "SYMMETRY"}
    cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
    mesh_bc = {n: ("WALL" if cfg[n]["type"] == "WALL" and cfg[n].get("is_no_slip", True) else "FARFIELD")
               for n in boxmesh.PLANE_NAMES}
    mesh = mg.ref_mesh(box, order, mesh_bc)
    solver = FRSolver(mesh=mesh, order=order, turb_model_name="NONE", rho_inf=rho, vel_inf=u, p_inf=p,
                      mu_molecular=float(g["mu"]), n_threads=1)
    provider = mg.plane_provider(mesh, box, cfg)
    case = export_case(mesh, solver.ops, provider)
    compared = 0
    for k, v in case.items():
        if k in g.files:
            assert np.array_equal(np.asarray(v), g[k]), k
            compared += 1
    assert compared >= 40
    for k in ("cd_wall_face", "true_area_weight", "colors", "bc_group", "bc_type", "nb_src0_mat"):
        assert k in case


@pytest.mark.skipif(not _reference_available(), reason="the reference checkout is not installed here")
def test_case_for_order_reproduces_the_continuation_phases():
    """reference_case_for_order over the reference's own P2 mesh gives, at
    every order, the tables the reference's order continuation used in that
    phase (cont_prism_p2_ns), including the load-order cell volumes."""
    import make_golden as mg
    from autoflowcfd_b200 import boxmesh
    from autoflowcfd_b200.reference_io import reference_case_for_order

    g = np.load(golden_path("cont_prism_p2_ns"))
    Ls = (1.5, 1.0, 1.0)
    box = boxmesh.prism_box(3, 2, 2, Ls, jitter=0.1, seed=5, bump=(0.05, 0.75, 0.5, 0.3))
    rho, p = 1.225, 101325.0
    u = 0.2 * np.sqrt(1.4 * p / rho)
    Qf = [rho, u, 0.0, 0.0, p]
    cfg = {n: {"type": "FARFIELD", "Q_free": Qf} for n in boxmesh.PLANE_NAMES}
    cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
    cfg["x_min"] = {"type": "INLET", "Q_inlet": Qf}
    cfg["x_max"] = {"type": "OUTLET", "p_outlet": p}
    cfg["y_min"] = {"type": "SYMMETRY"}
    cfg["y_max"] = {"type": "WALL", "is_no_slip": False}
    mesh_bc = {n: ("WALL" if cfg[n]["type"] == "WALL" and cfg[n].get("is_no_slip", True) else "FARFIELD")
               for n in boxmesh.PLANE_NAMES}
    mesh = mg.ref_mesh(box, 2, mesh_bc)
    case_for_order = reference_case_for_order(mesh, mg.plane_provider(mesh, box, cfg))
    for order in (0, 1, 2):
        case = case_for_order(order)
        pre = f"p{order}/"
        compared = 0
        for k, v in case.items():
            if pre + k in g.files and k != "cd_wall_face":
                assert np.array_equal(np.asarray(v), g[pre + k]), (order, k)
                compared += 1
        assert compared >= 40 and "fv_cell_volumes" in case
    assert int(mesh._active_order) == 2


def _provider(cfgs, default, n_faces=4):
    return SimpleNamespace(group_code=np.array([0, -1, 1, -1][:n_faces]), code_to_config=cfgs,
                           default_config=default)


FAR = {"type": "FARFIELD", "Q_free": [1.2, 30.0, 0.0, 0.0, 1e5]}


def test_lowering_of_a_table_provider():
    t = lower_ghost_provider(_provider({0: {"type": "WALL", "is_no_slip": False}, 1: {"type": "OUTLET",
                                                                                       "p_outlet": 9e4}}, FAR), 4)
    assert t["bc_type"].tolist() == [0, 3, 1] and t["bc_noslip"].tolist() == [0, 1, 1]
    assert t["bc_group"].tolist() == [0, 2, 1, 2] and t["bc_p_out"][1] == 9e4
    assert np.allclose(t["bc_Q"][2], FAR["Q_free"])


def test_callables_and_sem_inlets_are_refused():
    with pytest.raises(_lib.AfrError) as e:
        lower_ghost_provider(lambda f, q, n: q, 4)
    assert e.value.status == _lib.AFR_EUNSUPPORTED
    sem = {"type": "INLET", "Q_inlet": FAR["Q_free"], "sem": object()}
    with pytest.raises(_lib.AfrError) as e:
        lower_ghost_provider(_provider({0: sem}, FAR), 4)
    assert e.value.status == _lib.AFR_EUNSUPPORTED
    per_point = {"type": "INLET", "Q_inlet": np.zeros((4, 5))}
    with pytest.raises(_lib.AfrError):
        lower_ghost_provider(_provider({0: per_point}, FAR), 4)
    with pytest.raises(ValueError, match="Unknown boundary condition type"):
        lower_ghost_provider(_provider({0: {"type": "PERIODIC"}}, FAR), 4)


def test_exporter_on_stand_ins_matches_the_fixture():
    """Without the reference: stand-ins carrying a fixture's arrays go through
    the same exporter and come back as the fixture's tables."""
    import refstandins

    g = np.load(golden_path("prism_p1_ns"))
    mesh, ops, flat = refstandins.mesh_ops_flat(g)
    case = export_case(mesh, ops, refstandins.provider(g), flat=flat, cd_wall_face=g["cd_wall_face"])
    for k in ("bc_group", "bc_type", "bc_noslip", "bc_Q", "bc_p_out", "colors", "det_jacs", "inv_jacs_fine",
              "nb_src1_mat", "true_area_weight", "cd_wall_face"):
        assert np.array_equal(case[k], g[k]), k

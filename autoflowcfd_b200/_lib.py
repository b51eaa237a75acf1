"""ctypes binding of ``libafr_b200.so`` (C-ABI declared in include/afr_b200.h).

There is no fallback: if the library is missing or fails to load, importing
this module raises, so no caller can silently run anything but the CUDA path.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# AFR_B200_LIB selects another build of the same C-ABI (for example an instrumented one)
LIB_PATH = os.environ.get("AFR_B200_LIB") or os.path.join(HERE, "libafr_b200.so")

AFR_OK, AFR_EINVAL, AFR_ENOMEM, AFR_ECUDA, AFR_ENONFINITE, AFR_EUNSUPPORTED, AFR_EINDEX = range(7)
AFR_TURB_NONE, AFR_TURB_SST = 0, 1
AFR_PREC_FP64, AFR_PREC_MIXED = 0, 1

_P_D = ctypes.POINTER(ctypes.c_double)
_P_I64 = ctypes.POINTER(ctypes.c_int64)
_P_I32 = ctypes.POINTER(ctypes.c_int32)
_P_U8 = ctypes.POINTER(ctypes.c_uint8)


class AfrMeshDesc(ctypes.Structure):
    _fields_ = [
        ("n_cells", ctypes.c_int32), ("n_prism", ctypes.c_int32), ("order", ctypes.c_int32),
        ("n_sps", ctypes.c_int32), ("n_fine", ctypes.c_int32), ("n_fp", ctypes.c_int32),
        ("n_faces", ctypes.c_int32), ("n_nb_src1", ctypes.c_int32), ("n_ow_src1", ctypes.c_int32),
        ("det_jacs", _P_D), ("inv_jacs", _P_D), ("det_jacs_fine", _P_D), ("inv_jacs_fine", _P_D),
        ("cell_volumes", _P_D), ("wall_distance", _P_D),
        ("D_3d", _P_D * 2), ("c2f", _P_D * 2), ("D_fine", _P_D * 2), ("f2c", _P_D * 2), ("filter", _P_D * 2),
        ("boundary_extrap", _P_D), ("g_left", _P_D), ("g_right", _P_D),
        ("dist_fp_of_sp", _P_I64), ("dist_axis_coord_of_sp", _P_I64),
        ("owner_cell", _P_I64), ("neighbor_cell", _P_I64), ("owner_axis", _P_I64), ("neighbor_axis", _P_I64),
        ("owner_side", _P_D), ("neighbor_side", _P_D),
        ("is_boundary", _P_U8), ("owner_is_primary", _P_U8), ("neighbor_is_primary", _P_U8),
        ("true_normal", _P_D),
        ("nb_src0_cell", _P_I64), ("nb_src0_mat", _P_D),
        ("nb_src1_idx", _P_I64), ("nb_src1_cell", _P_I64), ("nb_src1_mat", _P_D),
        ("ow_src0_cell", _P_I64), ("ow_src0_mat", _P_D),
        ("ow_src1_idx", _P_I64), ("ow_src1_cell", _P_I64), ("ow_src1_mat", _P_D),
        ("colors", _P_I32),
        ("n_bc", ctypes.c_int32), ("bc_group", _P_I32), ("bc_type", _P_I32), ("bc_noslip", _P_I32),
        ("bc_wall_vel", _P_D), ("bc_Q", _P_D), ("bc_p_out", _P_D),
        ("cd_wall_face", _P_U8), ("true_area_weight", _P_D),
        ("n_src_mats", ctypes.c_int32), ("src_mat_table", _P_D),
        ("nb_src0_mat_index", _P_I32), ("nb_src1_mat_index", _P_I32),
        ("ow_src0_mat_index", _P_I32), ("ow_src1_mat_index", _P_I32),
        ("fv_cell_volumes", _P_D), ("metric_flux_scale", _P_D),
    ]


class AfrParams(ctypes.Structure):
    _fields_ = [
        ("n_vars", ctypes.c_int32), ("turb", ctypes.c_int32), ("inviscid_only", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("mu", ctypes.c_double), ("rho_inf", ctypes.c_double),
        ("vel_inf", ctypes.c_double), ("p_inf", ctypes.c_double), ("global_dt_factor", ctypes.c_double),
        ("mixed_ignore_conditioning", ctypes.c_int32),
    ]


# every symbol include/afr_b200.h declares, with its ctypes signature
SIGNATURES = {
    "afr_create": (ctypes.c_int, [ctypes.POINTER(AfrMeshDesc), ctypes.POINTER(AfrParams), ctypes.c_void_p,
                                  ctypes.POINTER(ctypes.c_void_p)]),
    "afr_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "afr_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "afr_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "afr_version": (ctypes.c_int, []),
    "afr_inviscid_residual": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "afr_viscous_residual": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "afr_local_dt": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "afr_sst_update": (ctypes.c_int, [ctypes.c_void_p] * 8),
    "afr_step": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "afr_cd_cl": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "afr_device_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "afr_step_profile": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                                                  ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]),
    "afr_rms_norm_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
    "afr_step_dual_time": (ctypes.c_int, [ctypes.c_void_p] * 6 + [ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                                                  ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                                                  ctypes.c_void_p]),
    "afr_step_imex": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "afr_residual_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "afr_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _P_I64, _P_I32, ctypes.c_int32, ctypes.c_void_p]),
    "afr_autotune": (ctypes.c_int, [ctypes.c_void_p] * 3 + [_P_I32, ctypes.c_void_p]),
    "afr_launch_shape": (ctypes.c_int, [ctypes.c_void_p, _P_I32]),
    "afr_segment_norms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, _P_I64, ctypes.c_int32, _P_D,
                                         ctypes.c_void_p]),
    "afr_tc_check": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "afr_greedy_face_coloring": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, _P_I64, _P_I64, _P_U8, _P_I32]),
    "afr_flux_point_jobs": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64, _P_D,
                                           _P_I32, _P_I32, _P_D, _P_D, _P_D, ctypes.c_int64, _P_D, _P_D,
                                           ctypes.c_int64] + [_P_I32] * 7 + [ctypes.POINTER(ctypes.c_uint32), _P_D,
                                                                             _P_D, _P_D]),
    "afr_prolong": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, _P_D,
                                   ctypes.c_void_p, ctypes.c_void_p]),
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(f"libafr_b200.so not built at {path}; run `python -m autoflowcfd_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = load()


class AfrError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"afr status {status} ({LIB.afr_status_string(status).decode()}): {msg}")
        self.status = status


def greedy_face_coloring(owner, neighbor, is_boundary, n_cells):
    """Face colors by the reference's greedy rule (C++ in libafr_b200.so)."""
    owner = np.ascontiguousarray(owner, np.int64)
    neighbor = np.ascontiguousarray(neighbor, np.int64)
    isb = np.ascontiguousarray(is_boundary, np.uint8)
    out = np.empty(owner.shape[0], np.int32)
    check(LIB.afr_greedy_face_coloring(owner.shape[0], int(n_cells), _ptr(owner, ctypes.c_int64),
                                       _ptr(neighbor, ctypes.c_int64), _ptr(isb, ctypes.c_uint8),
                                       _ptr(out, ctypes.c_int32)))
    return out


def check(status, handle=None):
    if status != AFR_OK:
        # with no handle, afr_last_error reports the last failed afr_create of this thread
        msg = LIB.afr_last_error(handle).decode()
        raise AfrError(status, msg)


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class MeshTables:
    """Host copies of the reference's flattened mesh tables, in the dtypes the
    C-ABI expects, plus the ``afr_mesh_desc`` that points into them."""

    F64 = ["det_jacs", "inv_jacs", "det_jacs_fine", "inv_jacs_fine", "cell_volumes", "boundary_extrap",
           "g_left", "g_right", "owner_side", "neighbor_side", "true_normal", "bc_wall_vel", "bc_Q", "bc_p_out"]
    MATS = ["nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"]
    I64 = ["dist_fp_of_sp", "dist_axis_coord_of_sp", "owner_cell", "neighbor_cell", "owner_axis", "neighbor_axis",
           "nb_src0_cell", "nb_src1_idx", "nb_src1_cell", "ow_src0_cell", "ow_src1_idx", "ow_src1_cell"]
    U8 = ["is_boundary", "owner_is_primary", "neighbor_is_primary"]
    I32 = ["colors", "bc_group", "bc_type", "bc_noslip"]

    def __init__(self, case):
        c = {}
        for k in self.F64:
            c[k] = np.ascontiguousarray(case[k], dtype=np.float64)
        for k in self.I64:
            c[k] = np.ascontiguousarray(case[k], dtype=np.int64)
        for k in self.U8:
            c[k] = np.ascontiguousarray(case[k], dtype=np.uint8)
        for k in self.I32:
            c[k] = np.ascontiguousarray(case[k], dtype=np.int32)
        indexed = case.get("src_mat_table") is not None
        if indexed:
            c["src_mat_table"] = np.ascontiguousarray(case["src_mat_table"], dtype=np.float64)
            for k in self.MATS:
                c[k + "_index"] = np.ascontiguousarray(case[k + "_index"], dtype=np.int32)
        else:
            for k in self.MATS:
                c[k] = np.ascontiguousarray(case[k], dtype=np.float64)
        for t in ("prism", "tet"):
            for k in ("D_3d_", "c2f_", "Dfine_", "f2c_", "filter_"):
                if k + t in case and case[k + t] is not None:
                    c[k + t] = np.ascontiguousarray(case[k + t], dtype=np.float64)
        if case.get("wall_distance") is not None:
            c["wall_distance"] = np.ascontiguousarray(case["wall_distance"], dtype=np.float64)
        for k in ("fv_cell_volumes", "metric_flux_scale"):
            if case.get(k) is not None:
                c[k] = np.ascontiguousarray(case[k], dtype=np.float64)
        if case.get("true_area_weight") is not None:
            c["true_area_weight"] = np.ascontiguousarray(case["true_area_weight"], dtype=np.float64)
            if case.get("cd_wall_face") is not None:
                c["cd_wall_face"] = np.ascontiguousarray(case["cd_wall_face"], dtype=np.uint8)
        self.c = c
        N = int(case["n_cells"])
        d = AfrMeshDesc()
        d.n_cells, d.n_prism, d.order = N, int(case["n_prism"]), int(case["order"])
        d.n_sps, d.n_fine = int(case["n_sps"]), int(case["n_fine"])
        d.n_fp = int(c["true_normal"].shape[1])
        d.n_faces = int(c["owner_cell"].shape[0])
        d.n_nb_src1 = int(c["nb_src1_cell"].shape[0])
        d.n_ow_src1 = int(c["ow_src1_cell"].shape[0])
        for k in self.F64:
            setattr(d, k, _ptr(c[k], ctypes.c_double))
        if indexed:
            d.n_src_mats = int(c["src_mat_table"].shape[0])
            d.src_mat_table = _ptr(c["src_mat_table"], ctypes.c_double)
            for k in self.MATS:
                setattr(d, k + "_index", _ptr(c[k + "_index"], ctypes.c_int32))
        else:
            for k in self.MATS:
                setattr(d, k, _ptr(c[k], ctypes.c_double))
        for k in self.I64:
            setattr(d, k, _ptr(c[k], ctypes.c_int64))
        for k in self.U8:
            setattr(d, k, _ptr(c[k], ctypes.c_uint8))
        d.colors = _ptr(c["colors"], ctypes.c_int32)
        d.bc_group = _ptr(c["bc_group"], ctypes.c_int32)
        d.bc_type = _ptr(c["bc_type"], ctypes.c_int32)
        d.bc_noslip = _ptr(c["bc_noslip"], ctypes.c_int32)
        d.n_bc = int(c["bc_type"].shape[0])
        for i, t in enumerate(("prism", "tet")):
            for k, field in (("D_3d_", "D_3d"), ("c2f_", "c2f"), ("Dfine_", "D_fine"), ("f2c_", "f2c"),
                             ("filter_", "filter")):
                arr = c.get(k + t)
                getattr(d, field)[i] = _ptr(arr, ctypes.c_double) if arr is not None else None
        d.wall_distance = _ptr(c.get("wall_distance"), ctypes.c_double)
        d.cd_wall_face = _ptr(c.get("cd_wall_face"), ctypes.c_uint8)
        d.true_area_weight = _ptr(c.get("true_area_weight"), ctypes.c_double)
        N_S = N * int(case["n_sps"])
        for k, n in (("fv_cell_volumes", N), ("metric_flux_scale", N_S)):
            if k in c and c[k].size != n:
                raise ValueError(f"{k} has {c[k].size} values, expected {n}")
            setattr(d, k, _ptr(c.get(k), ctypes.c_double))
        self.desc = d

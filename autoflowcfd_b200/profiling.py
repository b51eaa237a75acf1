"""Per-kernel device timing of one step (CUDA events recorded by the library
between its launch groups, afr_step_profile)."""

import ctypes

from ._lib import LIB, check


def step_breakdown(solver):
    """Run one step with events; returns per-kernel-group milliseconds."""
    import torch

    from .solver import _dev_ptr, _stream

    ms = (ctypes.c_double * 24)()
    nl = ctypes.c_int(0)
    check(LIB.afr_step_profile(solver._h, _dev_ptr(solver.U), _dev_ptr(solver.k), _dev_ptr(solver.omega),
                               _dev_ptr(solver.nu_t), ms, 24, ctypes.byref(nl), _stream()), solver._h)
    torch.cuda.synchronize()
    vals = [v for v in ms if v >= 0]
    sst = solver.k is not None
    names = ["local_dt"] + (["sst_point", "sst_face", "sst_update"] if sst else [])
    # per stage: pre-pass, face kernel, cell kernel (plain form) or volume
    # kernel (mixed form), update kernel (mixed form; empty in the plain form)
    for stg in range(3):
        names += [f"pre{stg}", f"face{stg}", f"cell{stg}", f"upd{stg}"]
    names += ["norm"]
    per = dict(zip(names, vals))

    def avg(key):
        xs = [per[f"{key}{i}"] for i in range(3) if f"{key}{i}" in per]
        return sum(xs) / len(xs) if xs else None

    return {"per_kernel_ms": per, "launches_per_step": int(nl.value), "k_pre_ms_per_launch": avg("pre"),
            "k_face_ms_per_launch": avg("face"), "k_cell_ms_per_launch": avg("cell"),
            "k_update_ms_per_launch": avg("upd")}

"""Checkpoint and resume of a case resident on the device.

Layout: the reference's HDF5 checkpoint (CheckpointManager.save,
core/utils/checkpoint.py:98-217, as written by write_checkpoint,
cli/solve_checkpoint_io.py:204-276): group ``metadata`` (attributes
iteration, timestamp, backend, config_hash and the solver's construction
parameters), group ``solution`` (dataset ``conserved`` = the cell-averaged
state, the full ``U_sps`` (n_cells, n_sps, n_vars) and primitive ``Q_sps``
fields), group ``convergence/history`` (``iterations``, ``residuals/<name>``).
Paths are relative to the reference's src/autoflowcfd.

h5py is not installed where this library is built or run, so the same
hierarchy is stored in one NumPy ``.npz`` archive: a dataset at HDF5 path
``a/b`` is the archive entry ``a/b``, an attribute ``x`` of group ``a`` is
the entry ``a@x``.  Converting to the reference's HDF5 file is a loop over
the entries on a machine with h5py.

Beyond the reference's fields, the archive keeps what an exact resume of the
device state needs: the SST fields ``solution/k``, ``solution/omega`` and
``solution/nu_t`` (the reference rebuilds them from their defaults) and, for
the dual-time scheme, the previous physical level ``solution/U_prev``.  A
resumed solver continues bitwise as if it had not stopped.
"""

import hashlib
import json
from datetime import datetime, timezone
from typing import Dict, Optional, Tuple

import numpy as np

GAMMA = 1.4
FORMAT = "autoflowcfd-b200 checkpoint 1 (HDF5 layout of core/utils/checkpoint.py in an npz archive)"


def _host(t) -> Optional[np.ndarray]:
    if t is None:
        return None
    if hasattr(t, "detach"):
        return t.detach().cpu().numpy()
    return np.asarray(t)


def primitives(U: np.ndarray) -> np.ndarray:
    """FRState._update_primitives (core/fr_solver/state.py:76-97): rho >= 1e-10,
    p >= 1, and k, omega >= 1e-12 from the turbulence columns."""
    rho = np.maximum(U[..., 0], 1e-10)
    u, v, w = U[..., 1] / rho, U[..., 2] / rho, U[..., 3] / rho
    ke = 0.5 * (u**2 + v**2 + w**2)
    p = np.maximum((U[..., 4] - rho * ke) * 0.4, 1.0)
    Q = np.zeros_like(U)
    Q[..., 0], Q[..., 1], Q[..., 2], Q[..., 3], Q[..., 4] = rho, u, v, w, p
    if U.shape[-1] > 5:
        Q[..., 5] = np.maximum(U[..., 5] / rho, 1e-12)
        Q[..., 6] = np.maximum(U[..., 6] / rho, 1e-12)
    return Q


def _config_hash(meta: Dict) -> str:
    """A digest of the construction parameters (CheckpointManager._compute_config_hash
    hashes the solver configuration the same way: a stable JSON dump)."""
    keys = sorted(k for k in meta if k not in ("timestamp",))
    return hashlib.sha256(json.dumps({k: meta[k] for k in keys}, default=str).encode()).hexdigest()[:16]


def save_checkpoint(solver, path: str, iteration: int, history: Optional[dict] = None,
                    metadata: Optional[dict] = None) -> str:
    """Write the solver's state (``B200FRSolver`` or any object with ``U``
    and optional ``k``, ``omega``, ``nu_t``, ``_U_prev``) to ``path``.

    ``history``: {"iterations": [...], "residuals": {name: [...]}} as the
    reference's manager takes; by default the solver's residual history."""
    U = _host(solver.U)
    meta = {
        "order": int(getattr(solver, "order", -1)),
        "turbulence_model": str(getattr(solver, "turb_model_name", "NONE")),
        "backend": "b200",
        "n_sps_per_cell": int(U.shape[1]),
        "n_vars": int(U.shape[2]),
        "precision": str(getattr(solver, "precision", "fp64")),
        "time_scheme": str(getattr(solver, "time_scheme", "ssp_rk3")),
    }
    meta.update(getattr(solver, "freestream", {}) or {})
    meta.update(metadata or {})
    out: Dict[str, np.ndarray] = {"format": np.array(FORMAT)}
    out["metadata@iteration"] = np.int64(iteration)
    out["metadata@timestamp"] = np.array(datetime.now(timezone.utc).isoformat())
    out["metadata@config_hash"] = np.array(_config_hash(meta))
    for k, v in meta.items():
        out["metadata@" + k] = np.array(v)
    out["solution/conserved"] = U.mean(axis=1)
    out["solution@shape"] = np.array(out["solution/conserved"].shape, np.int64)
    out["solution@dtype"] = np.array(str(U.dtype))
    out["solution/U_sps"] = U
    out["solution/Q_sps"] = primitives(U)
    for name, attr in (("k", "k"), ("omega", "omega"), ("nu_t", "nu_t"), ("U_prev", "_U_prev")):
        arr = _host(getattr(solver, attr, None))
        if arr is not None:
            out["solution/" + name] = arr
    if getattr(solver, "_has_prev", False):
        out["solution@has_prev"] = np.int64(1)
    hist = history
    if hist is None:
        res = list(getattr(solver, "residual_history", []))
        hist = {"iterations": list(range(1, len(res) + 1)), "residuals": {"total": res}}
    if "iterations" in hist:
        out["convergence/history/iterations"] = np.asarray(hist["iterations"], np.int32)
    for name, vals in (hist.get("residuals") or {}).items():
        out["convergence/history/residuals/" + name] = np.asarray(vals, np.float64)
    for name, vals in (hist.get("coefficients") or {}).items():
        out["convergence/history/coefficients/" + name] = np.asarray(vals, np.float64)
    if not str(path).endswith(".npz"):
        path = str(path) + ".npz"
    np.savez(path, **out)
    return str(path)


def load_checkpoint(path: str) -> Tuple[np.ndarray, dict, int, dict]:
    """(solution, history, iteration, metadata) as CheckpointManager.load
    returns them (core/utils/checkpoint_load.py); ``metadata["fields"]`` holds
    the extra solution fields (U_sps, Q_sps and, when saved, k, omega, nu_t,
    U_prev)."""
    z = np.load(path, allow_pickle=False)
    if "format" not in z.files or not str(z["format"]).startswith("autoflowcfd-b200 checkpoint"):
        raise ValueError(f"{path}: not a checkpoint written by autoflowcfd_b200.checkpoint")
    meta, fields, hist = {}, {}, {"residuals": {}, "coefficients": {}}
    for key in z.files:
        val = z[key]
        if key.startswith("metadata@"):
            meta[key[len("metadata@"):]] = val.item() if val.ndim == 0 else val
        elif key.startswith("solution/") and key != "solution/conserved":
            fields[key[len("solution/"):]] = val
        elif key == "convergence/history/iterations":
            hist["iterations"] = val.tolist()
        elif key.startswith("convergence/history/residuals/"):
            hist["residuals"][key.rsplit("/", 1)[1]] = val.tolist()
        elif key.startswith("convergence/history/coefficients/"):
            hist["coefficients"][key.rsplit("/", 1)[1]] = val.tolist()
    meta["fields"] = fields
    meta["has_prev"] = bool(z["solution@has_prev"]) if "solution@has_prev" in z.files else False
    iteration = int(meta.pop("iteration"))
    return z["solution/conserved"], hist, iteration, meta


def resume(solver, path: str) -> int:
    """Restore a solver built for the same case from a checkpoint; returns
    the checkpoint's iteration.  Refuses a state of another shape, as the
    reference's resume does (cli/solve_checkpoint_io.py:186-192)."""
    import torch

    _, hist, iteration, meta = load_checkpoint(path)
    f = meta["fields"]
    if tuple(f["U_sps"].shape) != tuple(solver.U.shape):
        raise ValueError(f"checkpoint state shape {f['U_sps'].shape} does not match the solver's "
                         f"{tuple(solver.U.shape)} (mesh or order changed)")
    solver.U.copy_(torch.from_numpy(np.ascontiguousarray(f["U_sps"])))
    for name in ("k", "omega", "nu_t"):
        dst = getattr(solver, name, None)
        if dst is not None and name in f:
            dst.copy_(torch.from_numpy(np.ascontiguousarray(f[name])))
    if "U_prev" in f and hasattr(solver, "_U_prev"):
        solver._U_prev = torch.from_numpy(np.ascontiguousarray(f["U_prev"])).to(solver.U.device)
        solver._has_prev = bool(meta.get("has_prev", False))
    if hasattr(solver, "residual_history"):
        solver.residual_history = list(hist["residuals"].get("total", []))
    return iteration

"""Host-side mirror of the reference's residual / time-step seam on one B200.

``B200FRSolver`` exposes the method surface of the reference's ``FRSolver``
residual seam (core/fr_solver/solver.py:329-446) and of the ``--backend gpu``
``GPUFRSolver`` (core/gpu/gpu_solver.py:36-453, core/gpu/gpu_solver_io.py:20-84)
with the same names, argument meaning and error behaviour, but every numeric
operation runs in ``libafr_b200.so`` on the device.  PyTorch provides device
memory and the current CUDA stream only; there is no CPU fallback.

State layouts are the reference's: U (n_cells, n_sps, n_vars) float64, k /
omega / nu_t (n_cells, n_sps) float64.
"""

import ctypes
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np
import torch

from . import _lib
from ._lib import LIB, check

GAMMA = 1.4


def _dev_ptr(t: Optional[torch.Tensor]):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("device arrays must be contiguous float64 CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _metric_flux_scale(case) -> np.ndarray:
    """(N, S) sum_m |adj(J)[m,:]| of a case's solution points
    (_get_metric_flux_scale, core/fr_solver/solver_geometry.py:18-32)."""
    N, S = int(case["n_cells"]), int(case["n_sps"])
    adj = np.asarray(case["det_jacs"], float).reshape(N, S)[..., None, None] * \
        np.asarray(case["inv_jacs"], float).reshape(N, S, 3, 3)
    return np.sum(np.linalg.norm(adj, axis=-1), axis=-1)


@dataclass
class SolverResult:
    """core/fr_solver/state.py:12-17."""

    converged: bool
    iterations: int
    final_residual: float


class B200FRSolver:
    """One FR case resident on the GPU.

    Args:
        case: mapping with the reference's flattened mesh tables, operators and
            boundary tables (the keys written by ``tests/golden/make_golden.py``
            or produced by ``autoflowcfd_b200.boxgeom``).
        turb_model_name: "SST" or "NONE" (core/fr_solver/turbulence.py:23-47).
        mu_molecular: molecular viscosity (FRSolver ``mu_molecular``).
        rho_inf, vel_inf, p_inf: free stream (FRSolver ctor).
        inviscid_only: Euler runs (the viscous residual is zero).
        global_dt_factor: > 0 selects time-accurate global stepping
            dt = factor * min(dt_local).
        precision: "fp64" (plain form, FP64 throughout) or "mixed" (operator
            contractions as BF16 hi+lo split tensor-core products with FP32
            accumulation, FP32 fluxes; FP64 state, metrics, norms and Cd/Cl).
        device: CUDA device.
        mixed_ignore_conditioning: build the mixed form even for operators
            whose row l1 norms exceed its FP32-accumulation bound (to measure
            its error there; refused by default).
        time_scheme: "ssp_rk3" (steady local time stepping), "dual_time"
            (BDF1/BDF2 physical steps by pseudo-time iteration) or
            "imex_euler" (explicit inviscid, implicit viscous), as the
            reference's TimeIntegrationScheme values
            (core/time_integration/base.py).
        dual_time_inner_iter: pseudo-time iterations per physical step
            (FRSolver ``dual_time_inner_iter``).
        case_for_order: ``order -> case`` giving the same mesh's tables at a
            lower order; with it ``solve`` runs the reference's order
            continuation for order >= 2 (FRSolver.solve,
            core/fr_solver/solver.py:270-323), P0 -> P1 -> ... -> order.
    """

    def __init__(self, case: Dict[str, np.ndarray], turb_model_name: str = "NONE", mu_molecular: float = 1.8e-5,
                 rho_inf: float = 1.225, vel_inf: float = 33.33, p_inf: float = 101325.0,
                 inviscid_only: bool = False, global_dt_factor: float = 0.0, precision: str = "fp64",
                 device="cuda:0", mixed_ignore_conditioning: bool = False, time_scheme: str = "ssp_rk3",
                 dual_time_inner_iter: int = 20, case_for_order=None):
        name = turb_model_name.upper()
        if name not in ("SST", "NONE"):
            raise ValueError(f"Unknown turbulence model: {turb_model_name}")
        self.device = torch.device(device)
        self.turb_model_name = name
        self.n_cells = int(case["n_cells"])
        self.order = int(case["order"])
        self.current_order = self.order
        self.case_for_order = case_for_order
        self.order_continuation_enabled = case_for_order is not None
        self.n_vars = 7 if name == "SST" else 5
        self.mu_molecular = float(mu_molecular)
        self.freestream = {"rho_inf": rho_inf, "vel_inf": vel_inf, "p_inf": p_inf}
        prm = _lib.AfrParams()
        prm.n_vars = self.n_vars
        prm.turb = _lib.AFR_TURB_SST if name == "SST" else _lib.AFR_TURB_NONE
        prm.inviscid_only = 1 if inviscid_only else 0
        prm.mu, prm.rho_inf, prm.vel_inf, prm.p_inf = self.mu_molecular, rho_inf, vel_inf, p_inf
        prm.global_dt_factor = float(global_dt_factor)
        scheme = str(getattr(time_scheme, "value", time_scheme)).lower()
        if scheme not in ("ssp_rk3", "dual_time", "imex_euler"):
            raise _lib.AfrError(_lib.AFR_EUNSUPPORTED, f"time scheme {time_scheme!r} is not built on the device")
        self.time_scheme = scheme
        self.dual_time_inner_iter = int(dual_time_inner_iter)
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
        self.precision = precision
        prm.precision = _lib.AFR_PREC_MIXED if precision == "mixed" else _lib.AFR_PREC_FP64
        prm.mixed_ignore_conditioning = 1 if mixed_ignore_conditioning else 0
        self._prm = prm
        self._h = None
        # the mesh's cell volumes at its load order (the order-0 finite-volume
        # divisor of an order continuation) and the metric flux scale the
        # continuation's later phases reuse
        self._fv_volumes = np.asarray(case["fv_cell_volumes"] if case.get("fv_cell_volumes") is not None
                                      else case["cell_volumes"], float)
        self._mfs_cache = None
        # SST: the wall distance at the target order's points; an order
        # continuation restarts from its cell means and prolongs them between
        # phases (core/utils/order_continuation.py:137-144, 270-275)
        self._wd_target = (np.asarray(case["wall_distance"], float)
                           if name == "SST" and case.get("wall_distance") is not None else None)
        self._wd_phase = None
        self._open(case)
        self.initialize_uniform(rho_inf, vel_inf, 0.0, 0.0, p_inf)
        self.residual_history = []

    def _open(self, case: Dict[str, np.ndarray]):
        """Create the device handle of ``case`` (tables copied to HBM) and
        fresh state fields of its size; releases the previous handle."""
        tables = _lib.MeshTables(case)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(LIB.afr_create(ctypes.byref(tables.desc), ctypes.byref(self._prm), _stream(), ctypes.byref(h)))
        self.cleanup()
        self._tables, self._h = tables, h
        self.current_order = int(case["order"])
        self.n_sps = N_S = int(case["n_sps"])
        N = self.n_cells
        self.U = torch.zeros((N, N_S, self.n_vars), dtype=torch.float64, device=self.device)
        self.k = self.omega = self.nu_t = None
        if self.turb_model_name == "SST":
            # SSTModelFR initial fields, core/turbulence/sst.py:46-49
            self.k = torch.full((N, N_S), 1e-6, dtype=torch.float64, device=self.device)
            self.omega = torch.ones((N, N_S), dtype=torch.float64, device=self.device)
            self.nu_t = torch.zeros((N, N_S), dtype=torch.float64, device=self.device)
        self._U_prev = None        # dual time: state at the previous physical level
        self._has_prev = False

    # ------------------------------------------------------ order continuation
    def _case_at(self, order: int) -> Dict[str, np.ndarray]:
        if self.case_for_order is None:
            raise ValueError("order continuation needs case_for_order (the mesh's tables at lower orders)")
        case = self.case_for_order(order)
        if int(case["order"]) != order or int(case["n_cells"]) != self.n_cells:
            raise ValueError(f"case_for_order({order}) returned order {int(case['order'])} with "
                             f"{int(case['n_cells'])} cells (expected {self.n_cells})")
        return case

    def _phase_case(self, order: int) -> Dict[str, np.ndarray]:
        """The tables of one continuation phase with the two quantities the
        reference carries over from earlier phases: the load-order cell
        volumes (its P0 finite-volume divisor, inviscid_p0.py:44-51) and the
        metric flux scale cached by the first phase, broadcast over the
        points (solver_geometry.py:18-32, cfl.py:136-146)."""
        case = dict(self._case_at(order))
        if case.get("fv_cell_volumes") is None:
            case["fv_cell_volumes"] = self._fv_volumes
        if self._mfs_cache is None:
            self._mfs_cache = _metric_flux_scale(case)
        else:
            S = int(case["n_sps"])
            c = self._mfs_cache
            case["metric_flux_scale"] = np.ascontiguousarray(
                np.broadcast_to(c, (self.n_cells, S)) if c.shape[1] in (1, S) else np.tile(c, (1, -(-S // c.shape[1])))[:, :S])
        if self._wd_phase is not None:
            case["wall_distance"] = np.ascontiguousarray(self._wd_phase)
        return case

    def _restart_at_p0(self):
        """run_order_continuation's restart (core/utils/order_continuation.py:236-288):
        the uniform free stream on a P0 handle (SST fields at their initial values)."""
        self._mfs_cache = None
        if self._wd_target is not None:
            self._wd_phase = np.tile(np.mean(self._wd_target, axis=1, keepdims=True), (1, 1))
        self._open(self._phase_case(0))
        f = self.freestream
        self.initialize_uniform(f["rho_inf"], f["vel_inf"], 0.0, 0.0, f["p_inf"])

    def _change_order(self, new_order: int, W: np.ndarray):
        """Prolong U (and k, omega, nu_t) with W (new_n_sps x old_n_sps) onto a
        handle of ``new_order``; the dual-time history is dropped
        (interpolate_to_new_order_checked, core/utils/order_continuation.py:180-205)."""
        old = {"U": self.U, "k": self.k, "omega": self.omega, "nu_t": self.nu_t}
        s_old = self.n_sps
        if self._wd_phase is not None:
            self._wd_phase = np.einsum("ab,cb->ca", np.asarray(W, dtype=np.float64), self._wd_phase)
        self._open(self._phase_case(new_order))
        Wc = np.ascontiguousarray(W, dtype=np.float64)
        if Wc.shape != (self.n_sps, s_old):
            raise ValueError(f"prolongation matrix {Wc.shape} != ({self.n_sps}, {s_old})")
        for name, src in old.items():
            dst = getattr(self, name)
            if src is None or dst is None:
                continue
            cols = src.shape[2] if src.dim() == 3 else 1
            check(LIB.afr_prolong(self._h, _dev_ptr(src.contiguous()), s_old, cols,
                                  Wc.ctypes.data_as(_lib._P_D), _dev_ptr(dst), _stream()), self._h)

    # ------------------------------------------------------------------ state
    def initialize_uniform(self, rho=1.0, u=0.0, v=0.0, w=0.0, p=1.0, k=1e-6, omega=1e-2):
        """FRState.initialize_uniform, core/fr_solver/state.py:50-74."""
        e = p / ((GAMMA - 1.0) * rho) + 0.5 * (u**2 + v**2 + w**2)
        vals = [rho, rho * u, rho * v, rho * w, rho * e]
        if self.n_vars > 5:
            vals += [rho * k, rho * omega]
        self.U[...] = torch.tensor(vals, dtype=torch.float64, device=self.device)

    def set_state_from_cpu(self, U: np.ndarray):
        """GPUFRSolver.set_state_from_cpu (core/gpu/gpu_solver_io.py:20-35)."""
        U = np.asarray(U, dtype=np.float64)
        if U.shape != tuple(self.U.shape):
            raise ValueError(f"state shape {U.shape} != {tuple(self.U.shape)}")
        self.U.copy_(torch.from_numpy(np.ascontiguousarray(U)))

    def get_state_cpu(self) -> np.ndarray:
        return self.U.cpu().numpy()

    def set_turbulence(self, k: np.ndarray, omega: np.ndarray, nu_t: np.ndarray):
        if self.k is None:
            raise ValueError("solver was built without SST")
        for dst, src in ((self.k, k), (self.omega, omega), (self.nu_t, nu_t)):
            dst.copy_(torch.from_numpy(np.ascontiguousarray(src, dtype=np.float64)))

    # -------------------------------------------------------------- residuals
    def compute_inviscid_residual(self, U_trial: Optional[torch.Tensor] = None) -> torch.Tensor:
        """FRSolver.compute_inviscid_residual (core/fr_solver/solver.py:351-400)."""
        U = self.U if U_trial is None else U_trial
        R = torch.empty_like(U)
        check(LIB.afr_inviscid_residual(self._h, _dev_ptr(U), _dev_ptr(R), _stream()), self._h)
        return R

    def compute_viscous_residual(self, U_trial: Optional[torch.Tensor] = None,
                                 mu_t_field: Optional[torch.Tensor] = None) -> torch.Tensor:
        """FRSolver.compute_viscous_residual (core/fr_solver/solver.py:402-432).

        ``mu_t_field`` here is the kinematic eddy viscosity nu_t; the library
        forms mu_t = max(rho, 1e-10) * nu_t as the reference does."""
        U = self.U if U_trial is None else U_trial
        nut = self.nu_t if mu_t_field is None else mu_t_field
        R = torch.empty_like(U)
        check(LIB.afr_viscous_residual(self._h, _dev_ptr(U), _dev_ptr(nut), _dev_ptr(R), _stream()), self._h)
        return R

    # GPUFRSolver spellings
    compute_inviscid_residual_gpu = compute_inviscid_residual
    compute_viscous_residual_gpu = compute_viscous_residual

    def _compute_local_time_step(self) -> torch.Tensor:
        """core/fr_solver/cfl.py:12-147 (global min when global_dt_factor > 0)."""
        dt = torch.empty((self.n_cells, self.n_sps), dtype=torch.float64, device=self.device)
        check(LIB.afr_local_dt(self._h, _dev_ptr(self.U), _dev_ptr(self.nu_t), _dev_ptr(dt), _stream()), self._h)
        return dt

    def compute_turbulence_source(self, dt_local: torch.Tensor, diag: bool = False):
        """core/fr_solver/turbulence.py:178-330: updates k, omega, nu_t in place;
        returns (Sk, S_omega, transport_k, transport_omega) when ``diag``."""
        if self.k is None:
            return None
        d = torch.empty((self.n_cells, self.n_sps, 4), dtype=torch.float64, device=self.device) if diag else None
        check(LIB.afr_sst_update(self._h, _dev_ptr(self.U), _dev_ptr(dt_local), _dev_ptr(self.k),
                                 _dev_ptr(self.omega), _dev_ptr(self.nu_t), _dev_ptr(d), _stream()), self._h)
        if diag:
            return d[..., 0], d[..., 1], d[..., 2], d[..., 3]
        return None

    # ------------------------------------------------------------------- step
    def step(self, dt: float = 1e-3, want_norm: bool = True) -> float:
        """FRSolver.step / GPUFRSolver.step (core/fr_solver/step.py:15-221).

        ssp_rk3: one SSP-RK3 step with local time stepping; ``dt`` is ignored,
        as in the reference's steady mode (step.py:47-58).  With ``want_norm``
        the call synchronises and raises AfrError when the step produced a
        non-finite value.  Without it nothing synchronises; a non-finite value
        is raised by the next step once the device has finished this one (or
        by ``status()``).

        dual_time: one physical step of size ``dt`` (BDF1 on the first step,
        BDF2 after); imex_euler: one IMEX Euler step with the local time step.
        Both synchronise."""
        norm = ctypes.c_double(0.0)
        if self.time_scheme == "dual_time":
            if self._U_prev is None:
                self._U_prev = torch.empty_like(self.U)
            check(LIB.afr_step_dual_time(self._h, _dev_ptr(self.U), _dev_ptr(self.k), _dev_ptr(self.omega),
                                         _dev_ptr(self.nu_t), _dev_ptr(self._U_prev), 1 if self._has_prev else 0,
                                         float(dt), self.dual_time_inner_iter, 1e-4, ctypes.byref(norm), _stream()),
                  self._h)
            self._has_prev = True
        elif self.time_scheme == "imex_euler":
            check(LIB.afr_step_imex(self._h, _dev_ptr(self.U), _dev_ptr(self.k), _dev_ptr(self.omega),
                                    _dev_ptr(self.nu_t), ctypes.byref(norm), _stream()), self._h)
        else:
            check(LIB.afr_step(self._h, _dev_ptr(self.U), _dev_ptr(self.k), _dev_ptr(self.omega),
                               _dev_ptr(self.nu_t), ctypes.byref(norm) if want_norm else None, _stream()), self._h)
            if not want_norm:
                return float("nan")
        self.residual_history.append(norm.value)
        return norm.value

    def status(self, clear: bool = False) -> int:
        """Device status after the queued work (synchronises): 0 when every
        step so far stayed finite, else raises AfrError (AFR_ENONFINITE ...).
        ``clear`` resets the sticky device status after the error is raised."""
        rc = LIB.afr_status(self._h, 0, None, None, 1 if clear else 0, _stream())
        check(rc, self._h)
        return rc

    def residual_sums(self, out: torch.Tensor) -> torch.Tensor:
        """Queue (no synchronisation, no allocation; capturable) the sums of
        squares of the last step's stage-0 dU/dt into the device tensor
        ``out`` (2 doubles): all variables, and the density column."""
        if not (out.is_cuda and out.dtype == torch.float64 and out.numel() >= 2 and out.is_contiguous()):
            raise ValueError("out must be a contiguous float64 CUDA tensor of 2 elements")
        check(LIB.afr_residual_sums(self._h, ctypes.c_void_p(out.data_ptr()), _stream()), self._h)
        return out

    def density_residual(self) -> float:
        """RMS of the density column of dU/dt at the last step (FP64), the
        quantity a steady solve's stopping rule watches."""
        ptr = np.array([0, self.n_cells], dtype=np.int64)
        out = np.zeros(1)
        check(LIB.afr_segment_norms(self._h, 1, ptr.ctypes.data_as(_lib._P_I64), 1, out.ctypes.data_as(_lib._P_D),
                                    _stream()), self._h)
        return float(out[0])

    def solve(self, max_iter: int = 1000, dt: float = 1e-3, tol: float = 1e-6, output_interval: int = 0,
              checkpoint_callback=None) -> dict:
        """GPUFRSolver.solve (core/gpu/gpu_solver.py:403-453): stops on tol or a
        non-finite norm.  With ``case_for_order`` and order >= 2 it runs the
        order continuation of FRSolver.solve instead (its SolverResult fields,
        plus the residual history)."""
        if self.order_continuation_enabled and self.order >= 2:
            from .continuation import run_order_continuation

            log = print if output_interval else None
            r = run_order_continuation(self, max_iter, dt, tol, checkpoint_callback, log)
            return {"converged": r.converged, "iterations": r.iterations, "final_residual": r.final_residual,
                    "residual_history": list(self.residual_history)}
        res = float("inf")
        it = 0
        converged = False
        for it in range(1, max_iter + 1):
            res = self.step(dt)
            if output_interval and it % output_interval == 0:
                print(f"Iteration {it}: Residual = {res:.6e}")
            if not np.isfinite(res):
                break
            if res < tol:
                converged = True
                break
        return {"converged": converged, "iterations": it, "final_residual": res,
                "residual_history": list(self.residual_history)}

    def compute_aerodynamic_coefficients(self, reference_area: float = 1.0) -> Dict[str, float]:
        """compute_aerodynamic_coefficients_fr (postprocess/fr_coefficients.py:27-152)."""
        out = (ctypes.c_double * 3)()
        check(LIB.afr_cd_cl(self._h, _dev_ptr(self.U), _dev_ptr(self.nu_t), float(reference_area), out, _stream()),
              self._h)
        return {"Cd": out[0], "Cl": out[1], "Cs": out[2]}

    def save_checkpoint(self, path: str, iteration: int, metadata: Optional[dict] = None) -> str:
        """Write the device state (U, SST fields, dual-time level n-1, residual
        history) in the reference's checkpoint layout (autoflowcfd_b200.checkpoint)."""
        from . import checkpoint

        return checkpoint.save_checkpoint(self, path, iteration, metadata=metadata)

    def resume_from_checkpoint(self, path: str) -> int:
        """Restore the device state from a checkpoint of the same case; returns its iteration."""
        from . import checkpoint

        return checkpoint.resume(self, path)

    def device_bytes(self) -> int:
        v = ctypes.c_uint64(0)
        check(LIB.afr_device_bytes(self._h, ctypes.byref(v)), self._h)
        return int(v.value)

    def autotune(self) -> list:
        """Choose the mixed form's launch shapes by timing residual evaluations
        of the current state (afr_autotune); [pre CTAs per SM, face block,
        update variant], or -1s for the plain form.  Results do not change."""
        ch = (ctypes.c_int32 * 3)()
        check(LIB.afr_autotune(self._h, _dev_ptr(self.U), _dev_ptr(self.nu_t), ch, _stream()), self._h)
        return [int(v) for v in ch]

    def launch_shape(self) -> dict:
        """Launch shapes of the mixed-form kernels (see afr_launch_shape)."""
        out = (ctypes.c_int32 * 8)()
        check(LIB.afr_launch_shape(self._h, out), self._h)
        keys = ("pre_per_sm", "pre_max_per_sm", "pre_occupancy", "vol_per_sm", "vol_occupancy", "face_block",
                "update_variant", "n_sms")
        return dict(zip(keys, (int(x) for x in out)))

    def cleanup(self):
        """GPUFRSolver.cleanup (core/gpu/gpu_solver_io.py)."""
        if getattr(self, "_h", None) is not None and self._h.value:
            LIB.afr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.cleanup()
        except Exception:
            pass

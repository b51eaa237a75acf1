"""Serving loop for steady solves on one GPU, with continuous batching.

Requests (a box case to be solved to a residual drop) arrive over time.  On
arrival a worker pool generates the request's mesh tables on the host while
the GPU keeps running the admitted requests.  A request is admitted, first
come first served, as soon as a slot is free and the free device memory
(``cudaMemGetInfo``) covers its estimated footprint plus a reserve.  Each
admitted request keeps its state resident on the device and runs on its own
CUDA stream as replays of a captured multi-step CUDA graph, so the work of all
admitted requests overlaps on the GPU.  After every slice its density residual
(the RMS of the density column of dU/dt, FP64) is read back; the request
finishes when that residual has dropped by ``drop`` relative to its first step,
at ``max_iter`` steps, or on a non-finite residual.  Its handle is then freed,
which makes room for the next admissions.

Each request's arithmetic depends only on its own handle, so its result is the
same alone and in the mix (bitwise: no cross-request reduction exists).
"""

import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from . import ensemble as E

GAMMA = 1.4


@dataclass
class SolveRequest:
    rid: int
    arrival_s: float
    spec: E.EnsembleCase


@dataclass
class SolveResult:
    rid: int
    arrival_s: float
    admitted_s: float
    finished_s: float
    iterations: int
    status: str                  # "converged", "max_iter" or "nonfinite"
    residual_drop: float         # last / first density residual
    n_cells: int
    order: int
    cd: float
    state: Optional[np.ndarray] = None

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


def poisson_requests(n: int, rate_per_s: float = 4.0, seed: int = 0, hex_cells=(8000, 200000), orders=(1, 2),
                     mach=(0.05, 0.25), bump=(0.0, 0.1), reynolds: float = 1e5) -> List[SolveRequest]:
    """Seeded Poisson stream: exponential inter-arrival times, hex count
    log-uniform, order uniform, Mach, bump height and streamwise bump position
    uniform; box length from the Reynolds number (as the ensemble draw)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        cells = float(np.exp(rng.uniform(np.log(hex_cells[0]), np.log(hex_cells[1]))))
        m = max(2, int(round((cells / 2.0) ** (1.0 / 3.0))))
        order = int(rng.choice(orders))
        M = float(rng.uniform(*mach))
        b = float(rng.uniform(*bump))
        bx = float(rng.uniform(0.25, 0.75))
        u = M * float(np.sqrt(GAMMA * E.P_INF / E.RHO_INF))
        L = reynolds * E.MU / (E.RHO_INF * u)
        spec = E.EnsembleCase((2 * m, m, m), order, M, b, int(rng.integers(1 << 30)), (L, L / 2, L / 2), bump_x=bx)
        out.append(SolveRequest(i, t, spec))
    return out


def turbulence_inflow(spec: E.EnsembleCase, intensity: float = 0.01, viscosity_ratio: float = 10.0):
    """Free-stream k and omega from turbulence intensity and viscosity ratio."""
    k = 1.5 * (intensity * spec.velocity) ** 2
    w = E.RHO_INF * k / (viscosity_ratio * E.MU)
    return k, w


@dataclass
class _Active:
    req: SolveRequest
    solver: object
    stream: torch.cuda.Stream
    graph: object
    admitted_s: float
    first: float
    iters: int = 0
    n_cells: int = 0


@dataclass
class ServingLoop:
    """Continuous-batching loop.

    Args:
        precision: "mixed" or "fp64".
        turb: "NONE" (laminar) or "SST".
        max_active: admitted requests at most.
        reserve_gb: free device memory kept after an admission.
        steps_per_slice: steps per CUDA-graph replay between residual checks.
        drop: finish when density residual <= drop * first residual.
        max_iter: finish after this many steps.
        keep_state: copy each finished request's state to the host.
    """

    precision: str = "mixed"
    turb: str = "NONE"
    max_active: int = 8
    reserve_gb: float = 8.0
    steps_per_slice: int = 10
    drop: float = 1e-6
    max_iter: int = 20000
    gen_workers: int = 2
    keep_state: bool = False
    device: str = "cuda:0"
    bytes_per_cell: Dict[int, float] = field(default_factory=lambda: {1: 16e3, 2: 48e3, 3: 96e3})

    def _estimate(self, spec: E.EnsembleCase) -> float:
        return self.bytes_per_cell.get(spec.order, 96e3) * spec.n_cells * (1.3 if self.turb == "SST" else 1.0)

    def _build(self, spec: E.EnsembleCase):
        return E.build_case(spec, wall_distance=self.turb == "SST")

    def _start(self, req: SolveRequest, case, now: float) -> _Active:
        from .solver import B200FRSolver

        stream = torch.cuda.Stream(device=self.device)
        spec = req.spec
        with torch.cuda.stream(stream):
            s = B200FRSolver(case, turb_model_name=self.turb, mu_molecular=E.MU, rho_inf=E.RHO_INF,
                             vel_inf=spec.velocity, p_inf=E.P_INF, precision=self.precision, device=self.device)
            N, S = s.n_cells, s.n_sps
            U = E.uniform_state(spec, N, S)
            if self.turb == "SST":
                k, w = turbulence_inflow(spec)
                U7 = np.zeros((N, S, 7))
                U7[..., :5] = U
                U7[..., 5], U7[..., 6] = E.RHO_INF * k, E.RHO_INF * w
                s.set_state_from_cpu(U7)
                s.set_turbulence(np.full((N, S), k), np.full((N, S), w), np.full((N, S), k / w))
            else:
                s.set_state_from_cpu(U)
            # later admissions estimate from what this handle allocated (+10 %)
            self.bytes_per_cell[spec.order] = 1.1 * (s.device_bytes() + s.U.numel() * 8) / N
            s.step(want_norm=False)              # iteration 1, eagerly
            first = s.density_residual()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                for _ in range(self.steps_per_slice):
                    s.step(want_norm=False)
        return _Active(req, s, stream, g, now, first, 1, N)

    def _finish(self, a: _Active, status: str, res: float, now: float) -> SolveResult:
        with torch.cuda.stream(a.stream):
            cd = a.solver.compute_aerodynamic_coefficients(1.0)["Cd"] if status != "nonfinite" else float("nan")
            state = a.solver.U.cpu().numpy() if self.keep_state else None
        out = SolveResult(a.req.rid, a.req.arrival_s, a.admitted_s, now, a.iters, status,
                          res / a.first if a.first > 0 else float("nan"), a.n_cells, a.req.spec.order, cd, state)
        a.graph = None
        a.solver.cleanup()
        return out

    def run(self, requests: List[SolveRequest], time_scale: float = 1.0,
            tables: Optional[Dict[int, dict]] = None) -> List[SolveResult]:
        """Serve the requests (arrival times in seconds from the start, scaled by
        time_scale).  ``tables`` may hold prebuilt mesh tables by request id."""
        torch.cuda.set_device(torch.device(self.device))
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        queue: deque = deque()
        futures = {}
        active: Dict[int, _Active] = {}
        done: List[SolveResult] = []
        pool = ThreadPoolExecutor(max_workers=self.gen_workers)
        self.peak_active = 0
        t0 = time.perf_counter()
        try:
            while pending or queue or active:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival_s * time_scale <= now:
                    r = pending.popleft()
                    queue.append(r)
                    if tables is not None and r.rid in tables:
                        futures[r.rid] = pool.submit(lambda c: c, tables[r.rid])
                    else:
                        futures[r.rid] = pool.submit(self._build, r.spec)
                while queue and len(active) < self.max_active:
                    r = queue[0]
                    if not futures[r.rid].done():
                        break
                    free, _ = torch.cuda.mem_get_info()
                    if active and free - self._estimate(r.spec) < self.reserve_gb * 1e9:
                        break
                    queue.popleft()
                    case = futures.pop(r.rid).result()
                    active[r.rid] = self._start(r, case, time.perf_counter() - t0)
                    self.peak_active = max(self.peak_active, len(active))
                    del case
                if not active:
                    time.sleep(0.002)
                    continue
                # one slice for every admitted request, issued before any check so the slices overlap
                for a in active.values():
                    with torch.cuda.stream(a.stream):
                        a.graph.replay()
                    a.iters += self.steps_per_slice
                for rid in list(active):
                    a = active[rid]
                    with torch.cuda.stream(a.stream):
                        res = a.solver.density_residual()
                    status = None
                    if not np.isfinite(res):
                        status = "nonfinite"
                    elif res <= self.drop * a.first:
                        status = "converged"
                    elif a.iters >= self.max_iter:
                        status = "max_iter"
                    if status:
                        done.append(self._finish(a, status, res, time.perf_counter() - t0))
                        del active[rid]
                        torch.cuda.empty_cache()
        finally:
            pool.shutdown(wait=True)
            for a in active.values():
                a.graph = None
                a.solver.cleanup()
        return done


def latency_summary(results: List[SolveResult], wall_s: float) -> Dict[str, float]:
    lat = np.array([r.latency_s for r in results])
    return {"completed": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "solves_per_hour": 3600.0 * len(results) / wall_s,
            "converged": int(sum(r.status == "converged" for r in results)),
            "max_iter": int(sum(r.status == "max_iter" for r in results)),
            "nonfinite": int(sum(r.status == "nonfinite" for r in results))}

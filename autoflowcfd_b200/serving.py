"""Serving loop for steady solves on one GPU, with continuous batching.

Requests (a box case to be solved to a residual drop) arrive over time.  On
arrival a worker pool generates the request's mesh tables on the host while
the GPU keeps running the admitted requests.  A request is admitted, first
come first served, as soon as a slot is free and the free device memory
(``cudaMemGetInfo``) covers its estimated footprint plus a reserve; a request
that cannot fit even on an idle device is rejected rather than tried.  Each
admitted request keeps its state resident on the device and runs on its own
CUDA stream as replays of a captured multi-step CUDA graph, so the work of all
admitted requests overlaps on the GPU.  The graph of a slice ends by copying
the slice's residual sums (``afr_residual_sums``: FP64, fixed order) into
pinned host memory and the loop polls each request's completion event: a
request whose slice is done is checked at once and, unless finished, its next
slice is issued immediately -- no request waits for the others' slices.  A
request finishes when its density residual (the RMS of the density column of
dU/dt) has dropped by ``drop`` relative to its first step, at ``max_iter``
steps, or on a non-finite residual.  Its handle is then freed, which makes
room for the next admissions.  A request whose handle cannot be created (for
example out of device memory) fails alone; the others keep running.

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
    status: str                  # "converged", "max_iter", "nonfinite", "rejected" or "error"
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
    sums: object = None          # pinned host (2,) residual sums written by the slice graph
    done: object = None          # event recorded after the last issued slice
    iters: int = 0
    n_cells: int = 0


def admission(free_bytes: float, estimate: float, reserve_bytes: float, n_active: int, max_active: int) -> str:
    """Admission decision for the queue head: "admit", "wait" (a slot or
    memory frees up when a running request finishes) or "reject" (it would
    not fit even on an idle device)."""
    if n_active >= max_active:
        return "wait"
    if free_bytes - estimate >= reserve_bytes:
        return "admit"
    return "wait" if n_active > 0 else "reject"


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
        try:
            return self._prepare(req, s, now, stream)
        except Exception:
            torch.cuda.synchronize(self.device)
            s.cleanup()
            raise

    def _prepare(self, req: SolveRequest, s, now: float, stream) -> _Active:
        spec = req.spec
        with torch.cuda.stream(stream):
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
            dev = torch.zeros(2, dtype=torch.float64, device=self.device)
            sums = torch.zeros(2, dtype=torch.float64).pin_memory()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                for _ in range(self.steps_per_slice):
                    s.step(want_norm=False)
                s.residual_sums(dev)
                sums.copy_(dev, non_blocking=True)
            s._slice_dev = dev                   # kept alive with the graph
        return _Active(req, s, stream, g, now, first, sums, None, 1, N)

    def _issue(self, a: _Active):
        with torch.cuda.stream(a.stream):
            a.graph.replay()
            a.done = torch.cuda.Event()
            a.done.record(a.stream)
        a.iters += self.steps_per_slice

    def _density(self, a: _Active) -> float:
        return float(np.sqrt(float(a.sums[1]) / (a.n_cells * a.solver.n_sps)))

    def _failed(self, req: SolveRequest, status: str, now: float) -> SolveResult:
        return SolveResult(req.rid, req.arrival_s, now, now, 0, status, float("nan"), req.spec.n_cells,
                           req.spec.order, float("nan"))

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
        self.errors: Dict[int, str] = {}
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
                while queue:
                    r = queue[0]
                    if not futures[r.rid].done():
                        break
                    free, _ = torch.cuda.mem_get_info()
                    decision = admission(free, self._estimate(r.spec), self.reserve_gb * 1e9, len(active),
                                         self.max_active)
                    if decision == "wait":
                        break
                    queue.popleft()
                    case = futures.pop(r.rid).result()
                    now = time.perf_counter() - t0
                    if decision == "reject":
                        done.append(self._failed(r, "rejected", now))
                        continue
                    try:
                        a = self._start(r, case, now)
                    except Exception as exc:  # this request alone fails (e.g. out of device memory)
                        self.errors[r.rid] = repr(exc)
                        done.append(self._failed(r, "error", time.perf_counter() - t0))
                        torch.cuda.empty_cache()
                        continue
                    finally:
                        del case
                    active[r.rid] = a
                    self._issue(a)
                    self.peak_active = max(self.peak_active, len(active))
                if not active:
                    time.sleep(0.002)
                    continue
                # every request whose slice has completed: check it, then re-issue or finish it
                progressed = False
                for rid in list(active):
                    a = active[rid]
                    if not a.done.query():
                        continue
                    progressed = True
                    res = self._density(a)
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
                    else:
                        self._issue(a)
                if not progressed:
                    time.sleep(0.0005)
        finally:
            pool.shutdown(wait=True)
            for a in active.values():
                if a.done is not None:
                    a.done.synchronize()
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

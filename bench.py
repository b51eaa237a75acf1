"""Benchmark of the FR residual-and-update path on B200.

Workload (one GPU): P2 RANS Navier-Stokes with SST k-omega and BR1 viscous
terms on 96 x 80 x 72 = 552,960 hex cells split into 1,105,920 prisms on a
[0,4] x [0,2] x [0,1.5] m box, interior nodes jittered by +-10% of the local
spacing (seeded), no-slip wall at z = 0, farfield elsewhere, free-stream Mach
0.1, Re = 1e6 per m; explicit SSP-RK3 with local time stepping.  Inputs are
synthetic (no dataset): a seeded free-stream-plus-perturbation state on a
generated mesh of the reference's own hex-splitting template.

A step is one ``afr_step`` (local dt, SST source/transport/update, three RK
stages).  metric = DOF-updates/s = n_cells * 27 SPs * 5 variables * 3 stages
per step / time.  ``value`` is the mixed-precision form (BF16 hi+lo split
tensor-core contractions, FP32 fluxes, FP64 state) timed with device-resident
inputs; the plain FP64 form runs in the same process from the same start
state (``plain_fp64``), and ``accuracy`` compares the two forms per field over
steps 1-6 (before the SST growth) and Cd.
``e2e`` times the mixed step through the C-ABI with the state in pinned host
memory, copied in and out every step.  The C2 state diverges after about 13
steps under the reference's SST closure (in both forms, as in the reference's
own algorithm), so timed steps run in segments of 8 that restart from the
seeded state outside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--small] [--form mixed|fp64|both]

Multi-GPU: the path runs one case per GPU with no inter-GPU exchange
("replicas only"); ``value`` is the sum over ranks (max-over-ranks time).
"""

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

GAMMA = 1.4
METRIC = "DOF-updates/s per RK stage at P2 vs plain FP64 GPU; HBM GB/s; serve p50/p99"
UNIT = "DOF-updates/s"
FULL = dict(shape=(96, 80, 72), lengths=(4.0, 2.0, 1.5), jitter=0.1, seed=2024, order=2)
SMALL = dict(shape=(24, 20, 18), lengths=(4.0, 2.0, 1.5), jitter=0.1, seed=2024, order=2)
SAMPLE = dict(shape=(8, 6, 6), lengths=(4.0, 2.0, 1.5), jitter=0.1, seed=2024, order=2)


def flow_conditions():
    rho, p = 1.225, 101325.0
    u = 0.1 * np.sqrt(GAMMA * p / rho)  # Mach 0.1
    mu = rho * u / 1e6  # Re = 1e6 per m
    k = 1.5 * (0.01 * u) ** 2  # turbulence intensity 1%
    w = rho * k / (10 * mu)  # viscosity ratio 10
    return rho, u, p, mu, k, w


def plane_cfg():
    from autoflowcfd_b200.boxmesh import PLANE_NAMES

    rho, u, p, *_ = flow_conditions()
    cfg = {n: {"type": "FARFIELD", "Q_free": [rho, u, 0.0, 0.0, p]} for n in PLANE_NAMES}
    cfg["z_min"] = {"type": "WALL", "is_no_slip": True}
    return cfg


def make_case(spec, colorer=None):
    """Tables of the C2 generator's box; ``colorer`` replaces the library's
    face coloring (the CPU arm passes the oracle's, so it loads no CUDA code)."""
    from autoflowcfd_b200 import boxgeom, boxmesh

    box = boxmesh.prism_box(*spec["shape"], spec["lengths"], jitter=spec["jitter"], seed=spec["seed"])
    case = boxgeom.build_case(box, spec["order"], plane_cfg(), wall_distance=True, want_sps_coords=True,
                              colorer=colorer)
    return case


def initial_state(case, spec):
    """Free stream with a wall-damped profile and a seeded smooth perturbation."""
    rho0, u0, p0, mu, k0, w0 = flow_conditions()
    xyz = case.pop("sps_coords")
    Lx, Ly, Lz = spec["lengths"]
    rng = np.random.default_rng(spec["seed"])
    ph = rng.uniform(0, 2 * np.pi, 4)
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    rho = rho0 * (1 + 0.01 * np.sin(2 * np.pi * (x / Lx + y / Ly) + ph[0]))
    u = u0 * np.tanh(6 * z / Lz + 0.3) * (1 + 0.02 * np.sin(2 * np.pi * x / Lx + ph[1]))
    v = 0.02 * u0 * np.sin(2 * np.pi * (y / Ly + z / Lz) + ph[2])
    w = 0.01 * u0 * np.sin(2 * np.pi * (x / Lx + z / Lz) + ph[3])
    p = np.full_like(x, p0)
    N, S = x.shape
    U = np.zeros((N, S, 7))
    E = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v + w * w)
    U[..., 0], U[..., 1], U[..., 2], U[..., 3], U[..., 4] = rho, rho * u, rho * v, rho * w, E
    k = np.full((N, S), k0)
    om = np.full((N, S), w0)
    nut = k / om
    U[..., 5], U[..., 6] = rho * k, rho * om
    return U, k, om, nut, mu


# algorithmic bytes per cell and RK stage of the C2 step in the reference's FP64
# layout: 3*8*7*27 (U_stage, U0, U_next) + 8*10*27 (det, adjugate) + 8*9*64
# (fine-point adjugates) + 8*3*9*R (face normals) + 8*9*27*M (interpolation
# matrices used) + 56*R (face metadata) + 8*27 (mu_t) + 8*6*27/3 (SST fields per
# step), with R = 4.04 face records and M = 7.9 used matrices per cell
C2_BYTES_PER_CELL_STAGE = 3 * 8 * 7 * 27 + 8 * 10 * 27 + 8 * 9 * 64 + 8 * 3 * 9 * 4.04 + 8 * 9 * 27 * 7.9 + 56 * 4.04 \
    + 8 * 27 + 8 * 6 * 27 / 3

# DRAM bytes per cell and launch of the mixed stage kernels, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the 76,800-prism P2 SST
# case; a full-size launch moves these times the number of cells.
MEASURED_TRAFFIC_PER_CELL = {"k_mx_pre": 8353.0, "k_mx_face": 7101.0, "k_mx_vol": 9921.0, "k_mx_update": 6126.0}


def mixed_algorithmic_bytes(case, nv=7):
    """Minimum bytes each per-stage kernel of the mixed form must move (every
    array it reads or writes once, in the layout the form stores).

    k_mx_pre: state, FP32 inverse-Jacobian rows (3 x 16 B), nu_t in; FP32
    point fields (20 per point) and face-point fields (18 per face point, 6*P
    per cell) out.
    k_mx_face: both sides' face-point fields, the slot's adjugate row (16 B),
    other-side index (1 B), true normal (24 B) per slot flux point, jumps out.
    k_mx_vol: state, FP32 point fields, FP32 adjugate rows at solution and fine
    points (3 x 16 B each), reciprocal det, metric divergence in; FP32 volume
    terms (10 per point) out.
    k_mx_update: volume terms, jumps, current and step-start state, dt,
    reciprocal det in; next state out."""
    N, S, Fn = int(case["n_cells"]), int(case["n_sps"]), int(case["n_fine"])
    P = case["true_normal"].shape[1]
    isb = case["is_boundary"].astype(bool)
    slots = int(np.sum(case["owner_is_primary"].astype(bool))) + \
        int(np.sum(~isb & case["neighbor_is_primary"].astype(bool)))
    sp = slots * P
    pre = N * S * (8 * (nv + 1) + 48) + N * S * 20 * 4 + N * 18 * 6 * P * 4
    face = sp * (2 * 18 * 4 + 16 + 1 + 24 + 10 * 4) + slots * 24
    vol = N * S * (8 * (nv + 1 + 3) + 48) + N * S * 20 * 4 + N * Fn * 48 + N * S * 10 * 4
    upd = N * S * 10 * 4 + sp * 10 * 4 + N * S * 8 * (3 * nv + 2) + slots * 4
    return {"k_mx_pre": pre, "k_mx_face": face, "k_mx_vol": vol, "k_mx_update": upd}


def algorithmic_bytes(case, nv=7):
    """Minimum bytes each per-stage kernel of the plain FP64 form must move (every array once).

    k_face: point fields of every cell (18 doubles per point), adjugates, the
    interpolation matrices of every residual slot, normals, slot metadata, and
    the jumps it writes (10 doubles per slot flux point).
    k_cell: point fields, adjugates, fine-point adjugates, det, dt, current and
    step-start state, the state it writes, and the jumps it reads."""
    N, S, Fn = int(case["n_cells"]), int(case["n_sps"]), int(case["n_fine"])
    P = case["true_normal"].shape[1]
    isb = case["is_boundary"].astype(bool)
    opr = case["owner_is_primary"].astype(bool)
    npr = case["neighbor_is_primary"].astype(bool)
    slots = int(np.sum(opr)) + int(np.sum(~isb & npr))
    mats = int(np.sum(opr & ~isb)) + int(np.sum(~isb & npr)) + \
        int(np.sum(case["nb_src1_idx"][opr & ~isb] >= 0)) + int(np.sum(case["ow_src1_idx"][~isb & npr] >= 0))
    jumps = slots * P * 10 * 8
    face = N * S * 8 * (18 + 9) + mats * P * S * 8 + slots * (P * 3 * 8 + 24) + jumps
    cell = N * S * 8 * (18 + 9 + 1 + 1 + 3 * nv) + N * Fn * 9 * 8 + jumps + slots * 4
    return {"k_face": face, "k_cell": cell}


def clocks_sampler(path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def clocks_summary(path, dev_index):
    try:
        rows = [r.split(",") for r in open(path).read().strip().splitlines()]
    except Exception:
        return None
    rows = [[c.strip() for c in r] for r in rows if len(r) >= 9 and r[0].strip() == str(dev_index)]
    if not rows:
        return None
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
    load = [s for s in sm if s > 500] or sm
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
    return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons, "samples": len(rows)}


def _blas_threads():
    try:
        from threadpoolctl import threadpool_info

        return max((int(i.get("num_threads", 1)) for i in threadpool_info() if i.get("user_api") == "blas"),
                   default=1)
    except Exception:
        return None


def _port_solver(spec):
    """The numpy restatement of the reference's step (the oracle) on a sample
    box of the C2 generator, with the oracle's own face coloring."""
    from oracle import fr_oracle as O

    case = make_case(spec, colorer=O.greedy_face_coloring)
    U, k, om, nut, mu = initial_state(case, spec)
    tab = case.pop("src_mat_table")
    for key in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        case[key] = tab[case.pop(key + "_index")]
    m = O.Mesh.from_case(case)
    return O.Solver(m, U, mu, O.TurbState(k, om, nut), case["wall_distance"]), U.shape[:2]


def cpu_baseline(spec=SAMPLE, max_seconds=25.0):
    """The reference algorithm on the host cores (the numpy oracle port), on a
    bounded sample box of the same generator; DOF-updates/s."""
    s, (N, S) = _port_solver(spec)
    s.step()  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        s.step()
        n += 1
        if time.perf_counter() - t0 > max_seconds / 2 or n >= 20:
            break
    dt = time.perf_counter() - t0
    return {"value": N * S * 5 * 3 * n / dt, "unit": UNIT, "cores": os.cpu_count(), "threads": _blas_threads(),
            "kind": "port",
            "sample": f"{N} prisms P2 SST ({spec['shape'][0]}x{spec['shape'][1]}x{spec['shape'][2]} hex), "
                      f"{n} steps, numpy restatement of the reference's FRSolver.step (the reference itself is "
                      f"Python + Numba and is not installed where the GPU runs)"}


def _repo_libraries_loaded():
    """Shared objects of this repository mapped into the process."""
    try:
        maps = open("/proc/self/maps").read().splitlines()
    except OSError:
        return []
    roots = (HERE, os.path.realpath(HERE))
    paths = {ln.split()[-1] for ln in maps if len(ln.split()) >= 6}
    return sorted(p for p in paths if ".so" in p and (p.startswith(roots) or "libafr_b200" in p))


def run_reference(args, rank, world):
    """CPU arm: the reference's algorithm (numpy restatement) on the host cores,
    rank 0 only, on a bounded sample of the C2 generator; it loads none of this
    repository's CUDA code (asserted)."""
    if rank != 0:
        return
    sample = SAMPLE
    s, (N, S) = _port_solver(sample)
    for _ in range(max(args.warmup, 1)):
        s.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step()
    dt = time.perf_counter() - t0
    loaded = _repo_libraries_loaded()
    assert not loaded, f"the CPU arm loaded repository libraries: {loaded}"
    v = N * S * 5 * 3 * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "C2 P2 RANS-SST prisms, bounded sample of the same generator "
                                   f"({sample['shape'][0]}x{sample['shape'][1]}x{sample['shape'][2]} hex -> {N} prisms)",
                       "form": "CPU"},
            "value": v, "ms_per_step": 1e3 * dt / args.steps,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "threads": _blas_threads(),
                             "kind": "port",
                             "sample": f"{N} prisms P2 SST, {args.steps} steps, numpy restatement of the "
                                       "reference's FRSolver.step"},
            "native_so_loaded": loaded,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# The C2 state diverges after about 13 steps under the reference's SST
# closure (k and omega grow from the first steps on; the mean flow follows
# once nu_t saturates), in both forms exactly as in the reference's own
# algorithm, so the timed steps run in segments that each restart from the
# seeded start state; the restarts are outside the timed region.
SEGMENT = 8
# steps after which the two forms' fields are compared (the reference's SST
# closure starts the growth of k at step 7 on this start state)
WINDOW = (1, 2, 3, 4, 5, 6)
# relative size of the seeded perturbation of the start state for the FP64
# form's own sensitivity over the window (the accuracy block's baseline)
PERTURB = 1e-9


def max_over_ranks(times_ms, dist=None, device="cpu"):
    """Per-rank device times -> the maximum over ranks (every rank gets it).
    Replicas run independent cases, so the job's time is the slowest rank's."""
    import torch

    ts = torch.tensor(list(times_ms), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(ts, op=dist.ReduceOp.MAX)
    return [float(v) for v in ts]


def replica_throughput(world, units_per_rank_step, ms_per_step):
    """Whole-job throughput of N replicas: all ranks' units over the max-over-ranks time."""
    return world * units_per_rank_step / (ms_per_step * 1e-3)


def e2e_pipelined(s, starts, steps, stream, barrier):
    """End to end through the C-ABI: every step copies its inputs (U, k,
    omega, nu_t) from pinned host memory and its result state back to pinned
    host memory.  Three device state sets rotate: while step i computes on one,
    one copy stream writes back step i-1's result from the second and another
    loads step i+1's inputs into the third, so both transfer directions run at
    once and overlap compute.  Each step starts from the same host start state
    (the C2 state diverges under long runs)."""
    import torch

    K = 3
    n = max(K, steps)
    host_in = [t.cpu().pin_memory() for t in starts]
    host_out = [[torch.empty_like(t).pin_memory() for t in host_in] for _ in range(K)]
    dev = [[torch.empty_like(t) for t in starts] for _ in range(K)]
    h2d = torch.cuda.Stream(device=starts[0].device)
    d2h = torch.cuda.Stream(device=starts[0].device)
    loaded = [torch.cuda.Event() for _ in range(K)]
    computed = [torch.cuda.Event() for _ in range(K)]
    saved = [torch.cuda.Event() for _ in range(K)]
    orig = (s.U, s.k, s.omega, s.nu_t)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h2d.wait_event(e0)
    d2h.wait_event(e0)
    with torch.cuda.stream(h2d):
        for d, h in zip(dev[0], host_in):
            d.copy_(h, non_blocking=True)
        loaded[0].record(h2d)
    for i in range(n):
        b = i % K
        if i + 1 < n:  # next inputs into the next set once its previous result is saved
            nb = (i + 1) % K
            with torch.cuda.stream(h2d):
                if i + 1 >= K:
                    h2d.wait_event(saved[nb])
                for d, h in zip(dev[nb], host_in):
                    d.copy_(h, non_blocking=True)
                loaded[nb].record(h2d)
        stream.wait_event(loaded[b])
        s.U, s.k, s.omega, s.nu_t = dev[b]
        s.step(want_norm=False)
        computed[b].record(stream)
        with torch.cuda.stream(d2h):
            d2h.wait_event(computed[b])
            for o, d in zip(host_out[b], dev[b]):
                o.copy_(d, non_blocking=True)
            saved[b].record(d2h)
    for b in range(K):
        stream.wait_event(saved[b])
    e1.record(stream)
    barrier()
    s.U, s.k, s.omega, s.nu_t = orig
    h2d_bytes = sum(t.numel() * 8 for t in host_in)
    return {"e2e_ms": e0.elapsed_time(e1) / n, "h2d": h2d_bytes, "d2h": h2d_bytes}


def run_form(s, steps, warmup, stream, barrier, want_e2e, clk_path, perturb=0.0):
    """Time one solver's steps (device-resident, restarted from the seeded
    state every SEGMENT steps), one breakdown step, and optionally the e2e
    loop; returns timings, breakdown and the fields after SEGMENT steps."""
    import torch

    from autoflowcfd_b200 import profiling

    fields = (s.U, s.k, s.omega, s.nu_t)
    starts = [t.clone() for t in fields]

    def restart():
        for d, h in zip(fields, starts):
            d.copy_(h)

    for _ in range(min(warmup, SEGMENT)):
        s.step(want_norm=False)
    restart()
    sampler = clocks_sampler(clk_path) if clk_path else None
    time.sleep(0.4 if sampler else 0.0)
    barrier()
    ms_total, done, finite = 0.0, 0, True
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    while done < steps:
        seg = min(SEGMENT, steps - done)
        restart()
        barrier()
        e0.record(stream)
        for _ in range(seg):
            s.step(want_norm=False)
        e1.record(stream)
        barrier()
        ms_total += e0.elapsed_time(e1)
        done += seg
        finite = finite and bool(torch.isfinite(s.U).all().item())
    ms = ms_total / steps
    if sampler:
        sampler.terminate()
    out = {"ms": ms, "finite": finite}
    # fields (device copies, ~2.2 GB each at full size) after the steps of the
    # accuracy window, from the start state; the window ends before the SST
    # growth of this start state (step 7)
    restart()
    out["window"] = {}
    for it in range(1, max(WINDOW) + 1):
        s.step(want_norm=False)
        if it in WINDOW:
            out["window"][it] = [t.clone() for t in (s.U, s.k, s.omega)]
    out["cd"] = s.compute_aerodynamic_coefficients(1.0)
    if perturb:
        # the same window from a start state perturbed by `perturb` (relative,
        # seeded): how far this workload itself carries a small difference
        g = torch.Generator(device=s.U.device).manual_seed(7)
        restart()
        s.U.mul_(1.0 + perturb * torch.randn(s.U.shape, generator=g, device=s.U.device, dtype=s.U.dtype))
        out["window_perturbed"] = {}
        for it in range(1, max(WINDOW) + 1):
            s.step(want_norm=False)
            if it in WINDOW:
                out["window_perturbed"][it] = [t.clone() for t in (s.U, s.k, s.omega)]
    restart()
    out["breakdown"] = profiling.step_breakdown(s)
    if want_e2e:
        out.update(e2e_pipelined(s, starts, steps, stream, barrier))
    return out


def per_field_errors(U, k, w, U_ref, k_ref, w_ref):
    """Relative L2 and max error per field of one state against a reference:
    rho, rho u, rho v, rho w, E (each momentum component relative to the
    momentum vector's size) and k, omega."""
    out = {}
    mom = U_ref[..., 1:4]
    for v, name in enumerate(("rho", "rho_u", "rho_v", "rho_w", "E")):
        d = (U[..., v] - U_ref[..., v]).double()
        ref = mom if 1 <= v <= 3 else U_ref[..., v]
        out[name] = {"l2_rel": float(d.norm() / ref.double().norm()),
                     "max_rel": float(d.abs().max() / ref.double().abs().max())}
    for name, a, b in (("k", k, k_ref), ("omega", w, w_ref)):
        d = (a - b).double()
        out[name] = {"l2_rel": float(d.norm() / b.double().norm()), "max_rel": float(d.abs().max() / b.double().abs().max())}
    return out


def run_ensemble(args):
    """C4: batched uneven ensemble (draw, build, autotune, CUDA-graph replay)."""
    import torch

    from autoflowcfd_b200 import ensemble as E

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = E.draw_cases(args.cases, seed=args.seed)
    t0 = time.perf_counter()
    cases = [E.build_case(sp) for sp in specs]
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    ens = E.B200Ensemble(specs, precision=args.form if args.form != "both" else "mixed", cases=cases)
    del cases
    t_create = time.perf_counter() - t0
    choices = ens.autotune()
    ens.capture()
    stream = torch.cuda.current_stream()
    ens.replay(max(0, args.warmup - 1))
    torch.cuda.synchronize()
    import tempfile

    clk_path = os.path.join(tempfile.gettempdir(), f"afr_bench_c4_clocks_{os.getpid()}.csv")
    sampler = clocks_sampler(clk_path)
    time.sleep(0.4 if sampler else 0.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.replay(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.terminate()
    ms = e0.elapsed_time(e1) / args.steps
    status = ens.status()
    norms = ens.norms()
    finite = all(bool(torch.isfinite(g.solver.U).all().item()) for g in ens.groups)
    n1 = sum(1 for sp in specs if sp.order == 1)
    line = {
        "metric": "DOF-updates/s, batched uneven ensemble (all cases, per RK stage)", "value": ens.dof_per_step() / (ms * 1e-3),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x2 split tensor-core contractions (f32 accumulate), f32 fluxes, f64 state" if args.form != "fp64" else "f64",
        "data": "synthetic (seeded case draw)",
        "config": {"workload": "C4 batched uneven ensemble: laminar NS Re 1e5, jittered prism boxes with wall bump",
                   "n_cases": len(specs), "cases_p1": n1, "cases_p2": len(specs) - n1, "n_cells": ens.n_cells,
                   "hex_cells_range": [2000, 64000], "mach_range": [0.05, 0.3], "launch": "one CUDA graph per step "
                   "(per order group: pre, face, volume, update launches per RK stage)",
                   "autotune_per_group": choices, "mesh_gen_s": round(t_gen, 1), "create_s": round(t_create, 1)},
        "norms": {"min": float(np.min(norms)), "max": float(np.max(norms)), "finite_cases": int(np.isfinite(norms).sum())},
        "case_status_nonfinite": int(np.sum(status != 0)),
        "state_finite": finite,
        "device_bytes": int(sum(g.solver.device_bytes() for g in ens.groups)),
    }
    clk = clocks_summary(clk_path, int(os.environ.get("LOCAL_RANK", "0")))
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)
    ens.cleanup()


C3 = dict(shape=(64, 64, 64), jitter=0.05, seed=7, order=3)


def c3_state(xyz, L=1.0):
    """Taylor-Green vortex at Mach 0.1 on the unit cube (the reference's
    tests/validation/test_tgv.py:96-112 field), SI units."""
    rho0, p0 = 1.225, 101325.0
    u0 = 0.1 * np.sqrt(GAMMA * p0 / rho0)
    k = 2 * np.pi / L
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    u = u0 * np.sin(k * x) * np.cos(k * y) * np.cos(k * z)
    v = -u0 * np.cos(k * x) * np.sin(k * y) * np.cos(k * z)
    p = p0 + rho0 * u0**2 / 16 * (np.cos(2 * k * x) + np.cos(2 * k * y)) * (np.cos(2 * k * z) + 2)
    rho = p / p0 * rho0
    U = np.stack([rho, rho * u, rho * v, np.zeros_like(rho), p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)], -1)
    return U, u0


def run_c3(args):
    """C3 precision stress at the configured size: 64^3 hex, +-5% jitter, six
    tets per hex (1,572,864 periodic tets), P3, Taylor-Green at Mach 0.1,
    Euler, SSP-RK3 with the global step 3 min(dt_local).

    The reference's P3 collapsed-tet operators make this state non-finite
    after the second step (its own FRSolver.step, committed as
    tests/golden/traj_p3_tgv.npz), so the 1000-step kinetic-energy history
    has no finite target: every timed step restarts from the start state
    (same arithmetic per step).  Reported: the plain FP64 form's throughput
    with its roofline; the kinetic energy after one step; and, with
    --mixed-opt-in, the mixed form built past its conditioning bound, its
    residual and one-step errors against the FP64 form per field."""
    import tempfile

    import torch

    from autoflowcfd_b200 import boxgeom, boxmesh, profiling
    from autoflowcfd_b200.solver import B200FRSolver

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    box = boxmesh.tet_box(*C3["shape"], (1.0, 1.0, 1.0), jitter=C3["jitter"], seed=C3["seed"], periodic=True)
    case = boxgeom.build_case(box, C3["order"], None, wall_distance=False, want_sps_coords=True)
    U, u0 = c3_state(case.pop("sps_coords"))
    t_gen = time.perf_counter() - t0
    rho0, p0 = 1.225, 101325.0
    stream = torch.cuda.current_stream()

    def make(precision, **kw):
        s = B200FRSolver(case, turb_model_name="NONE", rho_inf=rho0, vel_inf=u0, p_inf=p0, inviscid_only=True,
                         global_dt_factor=3.0, precision=precision, device=f"cuda:{local}", **kw)
        s.set_state_from_cpu(U)
        return s

    s = make("fp64")
    N, S = s.n_cells, s.n_sps
    start = s.U.clone()
    for _ in range(max(args.warmup, 1)):
        s.U.copy_(start)
        s.step(want_norm=False)
    clk_path = os.path.join(tempfile.gettempdir(), f"afr_bench_c3_clocks_{os.getpid()}.csv")
    sampler = clocks_sampler(clk_path)
    time.sleep(0.4 if sampler else 0.0)
    ms_total = 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.steps):
        s.U.copy_(start)
        torch.cuda.synchronize()
        e0.record(stream)
        s.step(want_norm=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_total += e0.elapsed_time(e1)
    if sampler:
        sampler.terminate()
    ms = ms_total / args.steps
    s.U.copy_(start)
    bd = profiling.step_breakdown(s)
    U1 = s.U.clone()

    def ke(W):
        return float((0.5 * (W[..., 1] ** 2 + W[..., 2] ** 2 + W[..., 3] ** 2) / W[..., 0]).sum())

    R64 = None
    if args.mixed_opt_in:
        s.U.copy_(start)
        R64 = s.compute_inviscid_residual()
    dev_bytes = s.device_bytes()
    s.cleanup()
    del s
    torch.cuda.empty_cache()
    alg = algorithmic_bytes(case, nv=5)
    kern_ms = {"k_face": bd["k_face_ms_per_launch"], "k_cell": bd["k_cell_ms_per_launch"]}
    per_kernel = {k: {"ms_per_launch": v, "algorithmic_bytes": alg[k], "achieved_gbs": alg[k] / (v * 1e-3) / 1e9}
                  for k, v in kern_ms.items()}
    dom = max(kern_ms, key=lambda k: kern_ms[k])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    dofs = N * S * 5 * 3
    line = {
        "metric": "DOF-updates/s, P3 precision stress (plain FP64 form)", "value": dofs / (ms * 1e-3), "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered mesh, TGV field)",
        "config": {"workload": "C3 P3 Euler TGV M0.1: 64^3 hex +-5% jitter -> 1,572,864 periodic tets",
                   "n_cells": N, "n_sps": S, "time_stepping": "SSP-RK3, global dt 3 min(dt_local)",
                   "restart_every_steps": 1, "mesh_gen_s": round(t_gen, 1),
                   "l2": "inputs larger than L2 (state %.2f GB)" % (N * S * 5 * 8 / 1e9),
                   "reference_behaviour": "non-finite after two steps with the reference's P3 tet operators "
                                          "(tests/golden/traj_p3_tgv.npz, 3,072-tet sample)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": per_kernel[dom]["achieved_gbs"], "peak": hbm_peak,
                     "unit": "GB/s", "frac": per_kernel[dom]["achieved_gbs"] / hbm_peak, "traffic": None,
                     "per_kernel": per_kernel, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "breakdown_ms_per_step": bd["per_kernel_ms"], "gpu_launches": bd["launches_per_step"] * args.steps,
        "device_bytes": dev_bytes,
        "kinetic_energy": {"start": ke(start), "after_one_step": ke(U1), "after_one_step_finite":
                           bool(torch.isfinite(U1).all().item())},
    }
    clk = clocks_summary(clk_path, local)
    if clk:
        line["clocks"] = clk
    if args.mixed_opt_in:
        sm = make("mixed", mixed_ignore_conditioning=True)
        Rm = sm.compute_inviscid_residual()
        sm.step(want_norm=False)

        def errs(a, b):
            out = {}
            d = (a - b)[..., :5].double()
            for v, name in enumerate(("rho", "rho_u", "rho_v", "rho_w", "E")):
                ref = b[..., 1:4] if 1 <= v <= 3 else b[..., v]
                out[name] = {"l2_rel": float(d[..., v].norm() / ref.double().norm()),
                             "max_rel": float(d[..., v].abs().max() / ref.double().abs().max())}
            return out

        line["mixed_opt_in"] = {
            "what": "mixed form built past its row-l1 conditioning bound (measurement only; refused by default)",
            "residual_vs_fp64": errs(Rm, R64), "state_after_one_step_vs_fp64": errs(sm.U, U1)}
        sm.cleanup()
    print(json.dumps(line), flush=True)


def p0_algorithmic_bytes(case, nv=5):
    """Minimum bytes each per-stage kernel of the order-0 path must move.

    k_p0_face: per face record its owner / neighbour / ghost-face / penalty /
    group indices, boundary flag, normal and area, the state once, and the
    flux record it writes (8 doubles).
    k_p0_cell: the flux records, the per-cell face references and slot lists,
    volume, det and dt, the current and step-start state, the state it
    writes and the two norm partials."""
    N = int(case["n_cells"])
    F = int(case["owner_cell"].shape[0])
    isb = case["is_boundary"].astype(bool)
    refs = F + int(np.sum(~isb))
    slots = int(np.sum(case["owner_is_primary"].astype(bool))) + \
        int(np.sum(~isb & case["neighbor_is_primary"].astype(bool)))
    face = F * (4 * 5 + 1 + 24 + 8) + N * nv * 8 + F * 64
    cell = F * 64 + (N + 1) * 4 * 2 + refs * 4 + slots * 4 + N * 8 * 3 + N * nv * 8 * 3 + N * 8 * 2
    return {"k_p0_face": face, "k_p0_cell": cell}


def _p0_setup(spec):
    """Order-0 case of the C2 generator's box, laminar (the order-0 path has
    no SST), with the C2 start state at the cell points."""
    rho, u, p, mu, *_ = flow_conditions()
    case = make_case(dict(spec, order=0))
    U, *_ = initial_state(case, spec)
    return case, np.ascontiguousarray(U[..., :5]), mu


def p0_cpu_baseline(spec, max_seconds=25.0):
    """The oracle's order-0 step (numpy restatement of the reference's
    finite-volume path) on a bounded sample box."""
    from oracle import fr_oracle as O

    rho, u, p, mu, *_ = flow_conditions()
    case = make_case(dict(spec, order=0), colorer=O.greedy_face_coloring)
    U, *_ = initial_state(case, spec)
    tab = case.pop("src_mat_table")
    for key in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        case[key] = tab[case.pop(key + "_index")]
    s = O.Solver(O.Mesh.from_case(case), np.ascontiguousarray(U[..., :5]), mu)
    N = s.U.shape[0]
    s.step()
    t0, n = time.perf_counter(), 0
    while n < 20 and time.perf_counter() - t0 < max_seconds / 2:
        s.step()
        n += 1
    dt = time.perf_counter() - t0
    return {"value": N * 5 * 3 * n / dt, "unit": UNIT, "cores": 1, "threads": _blas_threads(), "kind": "port",
            "sample": f"{N} prisms P0 laminar ({spec['shape'][0]}x{spec['shape'][1]}x{spec['shape'][2]} hex), "
                      f"{n} steps of the oracle's order-0 step (per-face Python loop, one core)"}


def run_p0(args):
    """Order 0 (the reference's finite-volume path, the first phase of its
    order continuation): the C2 box at P0, 1,105,920 prisms, laminar
    Navier-Stokes (wall + farfield), SSP-RK3 with local time stepping.
    DOF-updates/s = n_cells * 5 * 3 per step; inputs larger than L2 (the
    per-stage working set of face records and flux records is ~0.6 GB)."""
    import tempfile

    import torch

    from autoflowcfd_b200 import profiling
    from autoflowcfd_b200.solver import B200FRSolver

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = SMALL if args.small else FULL
    if args.shape:
        spec = dict(FULL, shape=tuple(int(x) for x in args.shape.split(",")))
    t0 = time.perf_counter()
    case, U, mu = _p0_setup(spec)
    t_gen = time.perf_counter() - t0
    rho, u, p, *_ = flow_conditions()
    s = B200FRSolver(case, mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p, device=f"cuda:{local}")
    s.set_state_from_cpu(U)
    N = s.n_cells
    stream = torch.cuda.current_stream()
    start = s.U.clone()
    for _ in range(max(args.warmup, 3)):
        s.step(want_norm=False)
    s.U.copy_(start)
    clk_path = os.path.join(tempfile.gettempdir(), f"afr_bench_p0_clocks_{os.getpid()}.csv")
    sampler = clocks_sampler(clk_path)
    time.sleep(0.4 if sampler else 0.0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.step(want_norm=False)
    e1.record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.terminate()
    ms = e0.elapsed_time(e1) / args.steps
    s.status()
    finite = bool(torch.isfinite(s.U).all().item())
    # end to end through the public API: pinned host state in and out per step
    host = torch.empty_like(s.U, device="cpu").pin_memory()
    host.copy_(start.cpu())
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        s.U.copy_(host, non_blocking=True)
        s.step(want_norm=False)
        host.copy_(s.U, non_blocking=True)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t1) * 1e3 / args.steps
    s.U.copy_(start)
    bd = profiling.step_breakdown(s)
    s.cleanup()
    alg = p0_algorithmic_bytes(case)
    kern_ms = {"k_p0_face": bd["k_face_ms_per_launch"], "k_p0_cell": bd["k_cell_ms_per_launch"]}
    per_kernel = {k: {"ms_per_launch": v, "algorithmic_bytes": alg[k], "achieved_gbs": alg[k] / (v * 1e-3) / 1e9}
                  for k, v in kern_ms.items()}
    dom = max(kern_ms, key=lambda k: kern_ms[k])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    dofs = N * 5 * 3
    nbytes = N * 5 * 8
    line = {
        "metric": "DOF-updates/s, order 0 (finite volume)", "value": dofs / (ms * 1e-3), "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered mesh, C2 state)",
        "config": {"workload": f"P0 laminar NS, C2 box {spec['shape'][0]}x{spec['shape'][1]}x{spec['shape'][2]} "
                               f"hex -> {N} prisms, wall + farfield", "n_cells": N,
                   "n_face_records": int(case["owner_cell"].shape[0]), "mesh_gen_s": round(t_gen, 1),
                   "time_stepping": "SSP-RK3, local dt", "finite_after_timed_steps": finite,
                   "l2": "inputs larger than L2 (face and flux records ~0.6 GB per stage)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": per_kernel[dom]["achieved_gbs"], "peak": hbm_peak,
                     "unit": "GB/s", "frac": per_kernel[dom]["achieved_gbs"] / hbm_peak, "traffic": None,
                     "per_kernel": per_kernel, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "breakdown_ms_per_step": bd["per_kernel_ms"], "gpu_launches": bd["launches_per_step"] * args.steps,
        "e2e": {"value": dofs / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes},
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = p0_cpu_baseline(SMALL if not args.small else SAMPLE)
    clk = clocks_summary(clk_path, local)
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)


def run_continuation(args):
    """Order continuation as FRSolver.solve runs it for P >= 2
    (core/utils/order_continuation.py:207-425): restart from the uniform free
    stream at P0, then P0 -> P1 -> P2 with max_iter // 3 steps per phase, on
    the C2 box (laminar: the order-0 path has no SST).  Reported: the solve's
    wall time through B200FRSolver.solve (handles of each order built from
    tables generated before the clock starts; device prolongation between
    phases), each phase's steps and device time per step, and the residual at
    every phase end."""
    import torch

    from autoflowcfd_b200 import boxgeom, boxmesh
    from autoflowcfd_b200.solver import B200FRSolver

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = SMALL if args.small else FULL
    rho, u, p, mu, *_ = flow_conditions()
    box = boxmesh.prism_box(*spec["shape"], spec["lengths"], jitter=spec["jitter"], seed=spec["seed"])
    t0 = time.perf_counter()
    cases = {q: boxgeom.build_case(box, q, plane_cfg()) for q in (0, 1, 2)}
    t_gen = time.perf_counter() - t0
    s = B200FRSolver(cases[2], mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p, device=f"cuda:{local}",
                     case_for_order=lambda q: cases[q])
    max_iter = args.max_iter if args.max_iter != 20000 else 3 * args.steps
    phase_ms = {0: 0.0, 1: 0.0, 2: 0.0}
    phase_steps = {0: 0, 1: 0, 2: 0}
    phase_end = {}
    stream = torch.cuda.current_stream()
    real_step = s.step
    ev = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]

    def timed_step(dt=1e-3, want_norm=True):
        ev[0].record(stream)
        r = real_step(dt, want_norm)
        ev[1].record(stream)
        torch.cuda.synchronize()
        phase_ms[s.current_order] += ev[0].elapsed_time(ev[1])
        phase_steps[s.current_order] += 1
        phase_end[s.current_order] = r
        return r

    s.step = timed_step
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    res = s.solve(max_iter=max_iter, dt=1e-3, tol=1e-12)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t1
    s.cleanup()
    N = int(cases[2]["n_cells"])
    line = {
        "metric": "order continuation P0->P1->P2 solve wall time", "value": wall, "unit": "s",
        "n_gpus": 1, "steps": int(res["iterations"]), "warmup": 0, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered mesh, uniform free stream start)",
        "config": {"workload": f"order continuation to P2, laminar NS, C2 box {spec['shape'][0]}x{spec['shape'][1]}"
                               f"x{spec['shape'][2]} hex -> {N} prisms", "max_iter": max_iter,
                   "tables_gen_s_outside_clock": round(t_gen, 1)},
        "phases": {f"P{q}": {"steps": phase_steps[q], "device_ms_per_step": phase_ms[q] / max(phase_steps[q], 1),
                             "residual_at_end": phase_end.get(q)} for q in (0, 1, 2)},
        "host_and_setup_s": wall - sum(phase_ms.values()) / 1e3,
        "converged": res["converged"],
    }
    print(json.dumps(line), flush=True)


def box_face_conn(case):
    """The FRFaceConnectivity fields of a generated box case (cube-face codes
    from the record's axis and side; areas from the area weights, which sum
    to one per face)."""
    isb = case["is_boundary"].astype(bool)
    occ = 2 * np.asarray(case["owner_axis"], np.int64) + (np.asarray(case["owner_side"]) > 0)
    ncc = np.where(isb, -1, 2 * np.asarray(case["neighbor_axis"], np.int64) + (np.asarray(case["neighbor_side"]) > 0))
    return dict(owner_cell=case["owner_cell"], neighbor_cell=case["neighbor_cell"], owner_cube_face=occ,
                neighbor_cube_face=ncc, area=case["true_area_weight"].sum(axis=1),
                normal=case["true_normal"][:, 0, :], face_node_ids=case["face_node_ids"], is_boundary=isb,
                face_translation=np.zeros((len(isb), 3)))


def run_facegeom(args):
    """Flux-point construction (set-up) on the device: the C2 generator's box
    at P2 (default 24x20x18 hex -> 17,280 prisms, the size of the reference's
    own 15.6 s mesh build; --shape for others).  Times the construction from
    face connectivity to flattened tables (host grouping, device Newton
    location and interpolation rows, assembly and colors) and compares its
    matrices with the template-replayed ones of the generator."""
    import torch

    from autoflowcfd_b200 import boxgeom, boxmesh, facegeom

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = SMALL if not args.shape else dict(FULL, shape=tuple(int(x) for x in args.shape.split(",")))

    def build(sp):
        box = boxmesh.prism_box(*sp["shape"], sp["lengths"], jitter=sp["jitter"], seed=sp["seed"])
        t0 = time.perf_counter()
        case = boxgeom.build_case(box, sp["order"], plane_cfg())
        return box, case, time.perf_counter() - t0

    # warm-up on the sample box: context creation and first-use costs
    box, case, _ = build(SAMPLE)
    facegeom.flux_point_tables(box_face_conn(case), boxmesh.orient_cells(box), np.zeros((0, 4)), box.nodes, 2)
    box, case, t_replay = build(spec)
    fc = box_face_conn(case)
    conn = boxmesh.orient_cells(box)
    runs = []
    for _ in range(max(1, min(args.steps, 3))):
        tm = {}
        t0 = time.perf_counter()
        t = facegeom.flux_point_tables(fc, conn, np.zeros((0, 4)), box.nodes, spec["order"], timings=tm)
        tm["total_s"] = time.perf_counter() - t0
        runs.append(tm)
    best = min(runs, key=lambda r: r["total_s"])
    tab = case["src_mat_table"]
    worst = 0.0
    for side in ("nb", "ow"):
        ref = tab[case[side + "_src0_mat_index"]]
        have = case[side + "_src0_cell"] >= 0
        d = np.abs(t[side + "_src0_mat"][have] - ref[have]).max() / np.abs(ref[have]).max()
        worst = max(worst, float(d))
    F = int(case["owner_cell"].shape[0])
    N = int(case["n_cells"])
    line = {
        "metric": "face flux-point construction (set-up), face records/s", "value": F / best["total_s"],
        "unit": "faces/s", "n_gpus": 1, "steps": len(runs), "warmup": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered box)",
        "config": {"workload": f"P2 prisms, C2 generator box {spec['shape'][0]}x{spec['shape'][1]}x{spec['shape'][2]} "
                               f"hex -> {N} prisms, {F} face records", "n_jobs": best["n_jobs"]},
        "seconds": {k: round(v, 4) for k, v in best.items() if k.endswith("_s")},
        "template_replay_s": round(t_replay, 3),
        "matrices_vs_template_replay_max_rel": worst,
        "reference_context": "the reference's whole mesh build of a 17,280-prism P2 mesh took 15.6 s (its own "
                             "Numba construction, measured on the survey's CPU host)",
    }
    print(json.dumps(line), flush=True)


def run_serve(args):
    """C5: serving loop (Poisson arrivals, HBM-gated admission, continuous batching)."""
    import torch

    from autoflowcfd_b200 import serving as SV
    from autoflowcfd_b200.solver import B200FRSolver

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    reqs = SV.poisson_requests(args.requests, rate_per_s=4.0, seed=args.seed)
    lp = SV.ServingLoop(precision="mixed" if args.form == "both" else args.form, turb=args.turb,
                        max_active=args.max_active, steps_per_slice=10, drop=1e-6, max_iter=args.max_iter)
    import tempfile

    clk_path = os.path.join(tempfile.gettempdir(), f"afr_bench_c5_clocks_{os.getpid()}.csv")
    sampler = clocks_sampler(clk_path)
    t0 = time.perf_counter()
    results = lp.run(reqs)
    wall = time.perf_counter() - t0
    if sampler:
        sampler.terminate()
    summary = SV.latency_summary(results, wall)
    # FP64 re-solve of 5 % of the solved requests (at least two), same number of steps, alone: the
    # smallest solved requests, which bounds the re-solve time (the FP64 form is ~5x slower)
    byid = {r.rid: r for r in results}
    solved = [i for i, q in enumerate(reqs) if byid[q.rid].status in ("converged", "max_iter")]
    solved.sort(key=lambda i: byid[reqs[i].rid].n_cells)
    pick = sorted(solved[:max(2, len(results) // 20)])
    cd_err = []
    for i in pick:
        r = byid[reqs[i].rid]
        ref = SV.ServingLoop(precision="fp64", turb=args.turb, max_active=1, steps_per_slice=10, drop=0.0,
                             max_iter=r.iterations - 1).run([SV.SolveRequest(r.rid, 0.0, reqs[i].spec)])[0]
        cd_err.append(abs(r.cd - ref.cd) / max(abs(ref.cd), 1e-300))
    cells = [r.n_cells for r in results]
    line = {
        "metric": "serving: solves/hour, p50/p99 latency (s)", "value": summary["solves_per_hour"],
        "unit": "solves/hour", "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x2 split tensor-core contractions (f32 accumulate), f32 fluxes, f64 state",
        "data": "synthetic (seeded Poisson request stream)",
        "config": {"workload": "C5 serving: Poisson 4 req/s, prism boxes 8k-200k hex, P1/P2, Mach 0.05-0.25, "
                               "parametric wall bump", "requests": len(reqs), "physics": args.turb,
                   "stop": "density residual drop 1e-6 or max_iter", "max_iter": args.max_iter,
                   "max_active": args.max_active, "admission": "free device memory (cudaMemGetInfo) minus reserve",
                   "cells_range": [int(min(cells)), int(max(cells))]},
        "latency": summary, "wall_s": wall, "peak_active": lp.peak_active, "errors": lp.errors,
        "cd_vs_fp64_resolve": {"requests": [int(reqs[i].rid) for i in pick],
                               "max_rel_err": float(max(cd_err)) if cd_err else None,
                               "mean_rel_err": float(np.mean(cd_err)) if cd_err else None},
    }
    clk = clocks_summary(clk_path, int(os.environ.get("LOCAL_RANK", "0")))
    if clk:
        line["clocks"] = clk
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--form", default="both", choices=["both", "mixed", "fp64"])
    ap.add_argument("--small", action="store_true", help="24x20x18 hex instead of 96x80x72 (profiling)")
    ap.add_argument("--shape", default=None, help="nx,ny,nz hex cells of a profiling-size box")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2",
                    choices=["c2", "c3", "ensemble", "serve", "p0", "continuation", "facegeom"])
    ap.add_argument("--mixed-opt-in", action="store_true",
                    help="c3: also build the mixed form past its conditioning bound and report its errors")
    ap.add_argument("--requests", type=int, default=32, help="serve: number of requests")
    ap.add_argument("--max-iter", type=int, default=20000, help="serve: step cap per request")
    ap.add_argument("--max-active", type=int, default=16, help="serve: admitted requests at most")
    ap.add_argument("--turb", default="NONE", choices=["NONE", "SST"], help="serve: physics of the requests")
    ap.add_argument("--cases", type=int, default=256, help="ensemble: number of cases")
    ap.add_argument("--seed", type=int, default=2024, help="ensemble: draw seed")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "ensemble":
        run_ensemble(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "c3":
        run_c3(args)
        return
    if args.workload == "p0":
        run_p0(args)
        return
    if args.workload == "continuation":
        run_continuation(args)
        return
    if args.workload == "facegeom":
        run_facegeom(args)
        return

    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from autoflowcfd_b200.solver import B200FRSolver

    spec = SMALL if args.small else FULL
    if args.shape:
        spec = dict(FULL, shape=tuple(int(x) for x in args.shape.split(",")))
    t_gen = time.perf_counter()
    case = make_case(spec)
    U, k, om, nut, mu = initial_state(case, spec)
    rho, u, p, *_ = flow_conditions()
    t_gen = time.perf_counter() - t_gen
    bytes_fp64 = algorithmic_bytes(case)
    bytes_mx = mixed_algorithmic_bytes(case)
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    import tempfile

    clk_path = os.path.join(tempfile.gettempdir(), f"afr_bench_clocks_rank{rank}_{os.getpid()}.csv")
    forms = {"both": ["mixed", "fp64"], "mixed": ["mixed"], "fp64": ["fp64"]}[args.form]
    res = {}
    for i, form in enumerate(forms):
        s = B200FRSolver(case, turb_model_name="SST", mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p,
                         precision=form, device=f"cuda:{local}")
        s.set_state_from_cpu(U)
        s.set_turbulence(k, om, nut)
        if form == "mixed":
            s.autotune()  # launch shapes only; results are the same
        N, S = s.n_cells, s.n_sps
        r = run_form(s, args.steps, args.warmup, stream, barrier, want_e2e=(i == 0), perturb=PERTURB if form == "fp64" else 0.0,
                     clk_path=clk_path if (rank == 0 and i == 0) else None)
        r["device_bytes"] = s.device_bytes()
        if form == "mixed":
            r["launch_shape"] = s.launch_shape()
        s.cleanup()
        del s
        torch.cuda.empty_cache()
        res[form] = r
    del case
    dofs_per_step = N * S * 5 * 3
    head = res[forms[0]]
    ts = max_over_ranks([head["ms"], head.get("e2e_ms", 0.0)] + [res[f]["ms"] for f in forms], dist,
                        device=f"cuda:{local}")
    ms, ms_e2e = ts[0], ts[1]
    value = replica_throughput(world, dofs_per_step, ms)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    bd = head["breakdown"]
    if forms[0] == "mixed":
        kern_ms = {"k_mx_pre": bd["k_pre_ms_per_launch"], "k_mx_face": bd["k_face_ms_per_launch"],
                   "k_mx_vol": bd["k_cell_ms_per_launch"], "k_mx_update": bd["k_update_ms_per_launch"]}
        alg = bytes_mx
    else:
        kern_ms = {"k_face": bd["k_face_ms_per_launch"], "k_cell": bd["k_cell_ms_per_launch"]}
        alg = bytes_fp64
    per_kernel = {kk: {"ms_per_launch": kern_ms[kk], "algorithmic_bytes": alg[kk],
                       "achieved_gbs": alg[kk] / (kern_ms[kk] * 1e-3) / 1e9 if kern_ms[kk] else None}
                  for kk in kern_ms}
    dom = max(kern_ms, key=lambda kk: kern_ms[kk] or 0.0)
    achieved = per_kernel[dom]["achieved_gbs"]
    mixed_head = forms[0] == "mixed"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x2 split tensor-core contractions (f32 accumulate), f32 fluxes, f64 state" if mixed_head
        else "f64",
        "data": "synthetic (seeded generated mesh and state)",
        "config": {"workload": ("C2 P2 RANS-SST: 96x80x72 hex -> 1,105,920 prisms" if spec is FULL
                                else "P2 RANS-SST %dx%dx%d hex -> %d prisms (profiling size)" % (*spec["shape"], N)),
                   "n_cells": N, "n_sps": S, "form": "mixed precision" if mixed_head else "plain FP64",
                   "time_stepping": "SSP-RK3, local dt", "parallelism": f"replicas x{world}",
                   "restart_every_steps": SEGMENT,
                   "l2": "inputs larger than L2 (state %.2f GB)" % (N * S * 7 * 8 / 1e9),
                   "mesh_gen_s": round(t_gen, 1)},
        "e2e": {"value": replica_throughput(world, dofs_per_step, ms_e2e), "unit": UNIT, "h2d_bytes_per_step": head["h2d"],
                "d2h_bytes_per_step": head["d2h"], "ms_per_step": ms_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None,
                     "traffic": (MEASURED_TRAFFIC_PER_CELL[dom] * N) if dom in MEASURED_TRAFFIC_PER_CELL else None,
                     "traffic_source": "ncu DRAM bytes per cell on 76,800 prisms, scaled to this launch",
                     "kernel": dom, "algorithmic_bytes_per_launch": alg[dom], "per_kernel": per_kernel,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        # whole step against HBM: the reference-layout algorithmic bytes per
        # cell and RK stage of the C2 configuration (every distinct array once
        # per stage in FP64: state in/out, metrics, fine-point adjugates,
        # face normals, the used interpolation matrices, face metadata, mu_t,
        # SST fields amortised over the stages)
        "step_roofline": {"bytes_per_cell_stage": C2_BYTES_PER_CELL_STAGE,
                          "achieved": C2_BYTES_PER_CELL_STAGE * N * 3 / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                          "unit": "GB/s",
                          "frac": C2_BYTES_PER_CELL_STAGE * N * 3 / (ms * 1e-3) / 1e9 / hbm_peak},
        "gpu_launches": bd.get("launches_per_step", 0) * args.steps,
        "breakdown_ms_per_step": bd.get("per_kernel_ms"),
        "device_bytes": head["device_bytes"],
        "launch_shape": res["mixed"].get("launch_shape") if "mixed" in res else None,
        "state_finite": head["finite"],
    }
    if "fp64" in res and mixed_head:
        f64 = res["fp64"]
        line["plain_fp64"] = {"value": replica_throughput(world, dofs_per_step, ts[3]), "unit": UNIT,
                              "ms_per_step": float(ts[3]),
                              "breakdown_ms_per_step": f64["breakdown"].get("per_kernel_ms"),
                              "speedup_of_mixed": float(ts[3]) / ms}
        mx = res["mixed"]
        cd64, cdmx = f64["cd"]["Cd"], mx["cd"]["Cd"]
        per_step = {str(it): per_field_errors(*mx["window"][it], *f64["window"][it]) for it in WINDOW}
        fields = list(per_step[str(WINDOW[-1])])
        worst = {f: {m: max(per_step[str(it)][f][m] for it in WINDOW) for m in ("l2_rel", "max_rel")} for f in fields}
        sens = {str(it): per_field_errors(*f64["window_perturbed"][it], *f64["window"][it]) for it in WINDOW}
        line["accuracy"] = {
            "against": f"plain FP64 form, same start state, steps {list(WINDOW)} (before the SST growth)",
            "per_field_worst_over_window": worst,
            "per_step_l2": {it: {f: v["l2_rel"] for f, v in e.items()} for it, e in per_step.items()},
            "per_step_max": {it: {f: v["max_rel"] for f, v in e.items()} for it, e in per_step.items()},
            "fp64_sensitivity": {
                "what": f"plain FP64 form from the start state times (1 + {PERTURB:g} N(0,1)) against the unperturbed run",
                "per_step_l2": {it: {f: v["l2_rel"] for f, v in e.items()} for it, e in sens.items()},
                "per_step_max": {it: {f: v["max_rel"] for f, v in e.items()} for it, e in sens.items()}},
            "field_l2_target": 1e-6, "fields_over_target": [f for f in fields if worst[f]["l2_rel"] > 1e-6],
            "Cd_fp64": cd64, "Cd_mixed": cdmx, "Cd_rel_err": abs(cdmx - cd64) / max(abs(cd64), 1e-300),
            "Cd_after_steps": WINDOW[-1]}
    clk = clocks_summary(clk_path, local) if rank == 0 else None
    if clk:
        line["clocks"] = clk
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the FR residual-and-update path on B200.

Workload (one GPU): P2 RANS Navier-Stokes with SST k-omega and BR1 viscous
terms on 96 x 80 x 72 = 552,960 hex cells split into 1,105,920 prisms on a
[0,4] x [0,2] x [0,1.5] m box, interior nodes jittered by +-10% of the local
spacing (seeded), no-slip wall at z = 0, farfield elsewhere, free-stream Mach
0.1, Re = 1e6 per m; explicit SSP-RK3 with local time stepping, plain FP64.
Inputs are synthetic (no dataset): a seeded free-stream-plus-perturbation
state on a generated mesh of the reference's own hex-splitting template.

A step is one ``afr_step`` (local dt, SST source/transport/update, three RK
stages).  metric = DOF-updates/s = n_cells * 27 SPs * 5 variables * 3 stages
per step / time.  ``value`` is timed with device-resident inputs; ``e2e``
times the same step through the C-ABI with the state in pinned host memory,
copied in and out every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--small]

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


def make_case(spec):
    from autoflowcfd_b200 import boxgeom, boxmesh

    box = boxmesh.prism_box(*spec["shape"], spec["lengths"], jitter=spec["jitter"], seed=spec["seed"])
    case = boxgeom.build_case(box, spec["order"], plane_cfg(), wall_distance=True, want_sps_coords=True)
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


def algorithmic_bytes(case, nv=7):
    """Minimum bytes each per-stage kernel must move (every array once).

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


def cpu_baseline(spec=SAMPLE, max_seconds=25.0):
    """The reference algorithm on the host cores (the numpy oracle port), on a
    bounded sample box of the same generator; DOF-updates/s."""
    from oracle import fr_oracle as O

    case = make_case(spec)
    U, k, om, nut, mu = initial_state(case, spec)
    tab = case.pop("src_mat_table")
    for key in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        case[key] = tab[case.pop(key + "_index")]
    m = O.Mesh.from_case(case)
    s = O.Solver(m, U, mu, O.TurbState(k, om, nut), case["wall_distance"])
    s.step()  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        s.step()
        n += 1
        if time.perf_counter() - t0 > max_seconds / 2 or n >= 20:
            break
    dt = time.perf_counter() - t0
    N, S = U.shape[:2]
    return {"value": N * S * 5 * 3 * n / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"{N} prisms P2 SST ({spec['shape'][0]}x{spec['shape'][1]}x{spec['shape'][2]} hex), "
                      f"{n} steps, numpy oracle (BLAS threads = host cores)"}


def run_reference(args, rank, world):
    line = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "C2 P2 RANS-SST prisms, bounded sample of the same generator", "form": "CPU"}}
    if rank != 0:
        return
    sample = SAMPLE
    from oracle import fr_oracle as O

    case = make_case(sample)
    U, k, om, nut, mu = initial_state(case, sample)
    tab = case.pop("src_mat_table")
    for key in ("nb_src0_mat", "nb_src1_mat", "ow_src0_mat", "ow_src1_mat"):
        case[key] = tab[case.pop(key + "_index")]
    m = O.Mesh.from_case(case)
    s = O.Solver(m, U, mu, O.TurbState(k, om, nut), case["wall_distance"])
    for _ in range(max(args.warmup, 1)):
        s.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step()
    dt = time.perf_counter() - t0
    N, S = U.shape[:2]
    v = N * S * 5 * 3 * args.steps / dt
    line.update(value=v, ms_per_step=1e3 * dt / args.steps,
                cpu_baseline={"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                              "sample": f"{N} prisms P2 SST, {args.steps} steps, numpy oracle"},
                e2e={"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--small", action="store_true", help="24x20x18 hex instead of 96x80x72 (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank, world)
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
    t_gen = time.perf_counter()
    case = make_case(spec)
    U, k, om, nut, mu = initial_state(case, spec)
    rho, u, p, *_ = flow_conditions()
    t_gen = time.perf_counter() - t_gen
    alg_bytes = algorithmic_bytes(case)
    s = B200FRSolver(case, turb_model_name="SST", mu_molecular=mu, rho_inf=rho, vel_inf=u, p_inf=p,
                     device=f"cuda:{local}")
    del case
    s.set_state_from_cpu(U)
    s.set_turbulence(k, om, nut)
    N, S = s.n_cells, s.n_sps
    dofs_per_step = N * S * 5 * 3
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        s.step(want_norm=False)
    U_start = s.U.clone()
    k_start, w_start, n_start = s.k.clone(), s.omega.clone(), s.nu_t.clone()
    clk_path = os.path.join(HERE, "gpurun_out", f"clocks_rank{rank}.csv")
    os.makedirs(os.path.dirname(clk_path), exist_ok=True)
    sampler = clocks_sampler(clk_path) if rank == 0 else None
    time.sleep(0.4 if sampler else 0.0)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # stage-kernel timing with events on the launching stream
    from autoflowcfd_b200 import profiling

    e0.record(stream)
    for _ in range(args.steps):
        s.step(want_norm=False)
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    # per-kernel breakdown of one step (events around each launch group)
    breakdown = profiling.step_breakdown(s)
    if sampler:
        sampler.terminate()
    # ---- e2e: state in pinned host memory, copied in/out every step ----
    hU = U_start.cpu().pin_memory()
    hk, hw, hn = k_start.cpu().pin_memory(), w_start.cpu().pin_memory(), n_start.cpu().pin_memory()
    outs = [torch.empty_like(t).pin_memory() for t in (hU, hk, hw, hn)]
    h2d = sum(t.numel() * 8 for t in (hU, hk, hw, hn))
    d2h = h2d + 8
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(max(1, args.steps // 2)):
        s.U.copy_(hU, non_blocking=True)
        s.k.copy_(hk, non_blocking=True)
        s.omega.copy_(hw, non_blocking=True)
        s.nu_t.copy_(hn, non_blocking=True)
        s.step(want_norm=True)  # the residual norm is read back every step
        for o, d in zip(outs, (s.U, s.k, s.omega, s.nu_t)):
            o.copy_(d, non_blocking=True)
    e3.record(stream)
    barrier()
    ms_e2e = e2.elapsed_time(e3) / max(1, args.steps // 2)
    finite = bool(torch.isfinite(s.U).all().item())
    # max over ranks
    ts = torch.tensor([ms, ms_e2e], dtype=torch.float64, device=s.device)
    if dist is not None:
        dist.all_reduce(ts, op=dist.ReduceOp.MAX)
    ms, ms_e2e = float(ts[0]), float(ts[1])
    value = world * dofs_per_step / (ms * 1e-3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(HERE, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    kern_ms = {"k_face": breakdown.get("k_face_ms_per_launch"), "k_cell": breakdown.get("k_cell_ms_per_launch")}
    dom = max(kern_ms, key=lambda k: kern_ms[k] or 0.0)
    per_kernel = {k: {"ms_per_launch": kern_ms[k], "algorithmic_bytes": alg_bytes[k],
                      "achieved_gbs": alg_bytes[k] / (kern_ms[k] * 1e-3) / 1e9 if kern_ms[k] else None}
                  for k in kern_ms}
    achieved = per_kernel[dom]["achieved_gbs"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generated mesh and state)",
        "config": {"workload": ("C2 P2 RANS-SST: 96x80x72 hex -> 1,105,920 prisms" if not args.small
                                else "P2 RANS-SST 24x20x18 hex -> 17,280 prisms (profiling size)"),
                   "n_cells": N, "n_sps": S, "form": "plain FP64", "time_stepping": "SSP-RK3, local dt",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (state %.2f GB)" % (
                       N * S * 7 * 8 / 1e9), "mesh_gen_s": round(t_gen, 1)},
        "e2e": {"value": world * dofs_per_step / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": (achieved / hbm_peak) if achieved else None, "traffic": None,
                     "kernel": dom, "algorithmic_bytes_per_launch": alg_bytes[dom], "per_kernel": per_kernel,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "fp64_note": "the plain FP64 form is latency / FP64-pipe bound, not HBM bound"},
        "gpu_launches": breakdown.get("launches_per_step", 0) * args.steps,
        "breakdown_ms_per_step": breakdown.get("per_kernel_ms"),
        "device_bytes": s.device_bytes(),
        "state_finite": finite,
    }
    clk = clocks_summary(clk_path, local) if rank == 0 else None
    if clk:
        line["clocks"] = clk
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.cleanup()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

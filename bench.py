#!/usr/bin/env python
"""Benchmark of the T-matrix solve hot path on B200 (one JSON line on stdout, rank 0).

Workload (default, "c2"): 2000 spheres placed by seeded random sequential addition in a ball at
volume fraction 0.20, radii lognormal (median 0.1 um, sigma_ln 0.2, clipped to [0.04, 0.25] um),
refractive index 1.6+0.005i in vacuum, wavelength 0.6 um, lmax 6 (96 coefficients per sphere,
192,000 unknowns), complex128, one plane wave (+z, TE), GMRES rtol 1e-8, block-diagonal
preconditioner on 4x4x4 spatial cells. One step = one full device GMRES solve from x0 = b.

Reported:
  value            solves/s, device-resident inputs (sum over ranks; ranks are replicas)
  e2e              solves/s through the public API with host buffers (H2D rhs, solve, D2H x)
  matvec_per_s     float64 master-operator applications per second (x - T W x)
  latency_ms       p50 / p99 of the timed solves
  mixed            complex64 inner solves in float64 refinement: solves/s and C_ext error
                   against the plain float64 solve
  roofline         the coupling contraction (contract_kernel) against the float64 pipe
  cpu_baseline     the oracle (plain-C restatement of the reference CPU matvec) on host cores,
                   row-sampled, converted to solves/s with this solve's matvec count

--impl reference times the reference's CPU algorithm (the oracle port, all host threads) on the
same workload and prints the same metric with "impl": "reference".
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "solves/s (C2: 2000 spheres, lmax 6, FP64, GMRES rtol 1e-8, 4x4x4 block-Jacobi); matvec/s"
UNIT = "solves/s"
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12  # B200: 148 SMs x 64 FP64 FMA/clk at 1965 MHz
T_NZ = {1: 20, 2: 314, 3: 1578, 4: 4904, 5: 12302, 6: 26700, 7: 52178, 8: 94160}
# Matvecs of one C2 solve on the b200 arm (float64 GMRES + block-Jacobi, rtol 1e-8), used by the
# reference arm to turn its per-matvec time into a per-solve time.
C2_MATVECS_PER_SOLVE = 63


def algorithmic_flops(n: int, lmax: int, nrhs: int = 1) -> float:
    nmax = 2 * lmax * (lmax + 2)
    return n * (n - 1) * (4 * T_NZ[lmax] + 8 * nmax * nmax * nrhs)


def workload(name: str):
    from yasf_b200.workloads import aggregate_c1, aggregate_c2, aggregate_c5

    if name == "c1":
        return aggregate_c1(seed=0), 1e-8, None
    if name == "c2":
        return aggregate_c2(seed=0), 1e-8, 4
    if name == "c5":
        return aggregate_c5(seed=0), 1e-6, 8
    raise ValueError(name)


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def cpu_matvec_seconds(agg, table, budget_s: float, threads: int) -> tuple[float, int]:
    """Oracle matvec time for the full aggregate, extrapolated from a timed row sample."""
    from oracle import restate as R

    rng = np.random.default_rng(1)
    nmax = 2 * agg.lmax * (agg.lmax + 2)
    x = rng.normal(size=agg.n * nmax) + 1j * rng.normal(size=agg.n * nmax)
    rows, spent, done = 1, 0.0, 0
    start = 0
    while spent < budget_s and done < agg.n:
        r = min(rows, agg.n - start)
        t0 = time.perf_counter()
        R.coupling_matvec_rows(agg.lmax, agg.positions, agg.k, table, x, start, start + r, threads=threads)
        dt = time.perf_counter() - t0
        spent += dt
        done += r
        start = (start + r) % agg.n
        rows = max(1, min(agg.n, int(r * 2 if dt < 0.25 * budget_s else r)))
    return spent / done * agg.n, done


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------------------------
def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from yasf_b200.numerics import cached_translation_table

    agg, _, _ = workload(args.workload)
    table = cached_translation_table(agg.lmax)
    threads = host_threads()
    per_step = max(3.0, min(30.0, 120.0 / max(1, args.steps + args.warmup)))
    times = []
    sample_rows = 0
    for i in range(args.warmup + args.steps):
        t_mv, rows = cpu_matvec_seconds(agg, table, per_step, threads)
        if i >= args.warmup:
            times.append(t_mv)
            sample_rows += rows
    t_mv = statistics.median(times)
    mv_per_solve = C2_MATVECS_PER_SOLVE if args.workload == "c2" else None
    solve_s = t_mv * (mv_per_solve or 1)
    value = 1.0 / solve_s
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": solve_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128",
        "data": "synthetic (seeded RSA aggregate)",
        "config": {"workload": agg.name, "n_spheres": agg.n, "lmax": agg.lmax,
                   "unknowns": agg.n * 2 * agg.lmax * (agg.lmax + 2), "rtol": 1e-8,
                   "parallelism": "host threads"},
        "matvec_per_s": 1.0 / t_mv,
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample_rows} receiving-sphere rows of the C-restated particle_interaction_scalar "
                      f"over {args.steps} steps, extrapolated x{agg.n}/rows per matvec; solve = "
                      f"{mv_per_solve} matvecs (the b200 solve's count, preconditioner cost excluded)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
def run_b200(args, rank: int, world: int) -> None:
    import torch

    from yasf_b200 import BlockDiagonalPreconditioner, InitialField, Numerics, Optics, Parameters
    from yasf_b200 import Particles, Simulation, Solver, _lib
    from yasf_b200.solver import MasterOperator

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _lib.load()
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811

    agg, rtol, cells = workload(args.workload)
    n = agg.n
    particles = Particles(agg.positions, agg.radii, np.full(n, agg.refractive_index))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(np.array([agg.wavelength]), np.array([1.0 + 0j]), particles, field)
    pre = None
    if cells and not args.no_precond:
        extent = agg.positions.max(axis=0) - agg.positions.min(axis=0)
        pre = BlockDiagonalPreconditioner((extent + 2.0) / cells)
    solver = Solver("gmres", tolerance=rtol, max_iter=200, restart=args.restart, preconditioner=pre)
    numerics = Numerics(lmax=agg.lmax, solver=solver)
    numerics.compute_translation_table()
    sim = Simulation(params, numerics, device=device)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    t0 = time.perf_counter()
    if pre is not None:
        pre.prepare(sim)
    torch.cuda.synchronize()
    prepare_s = time.perf_counter() - t0
    dev = sim.device_state(0)
    tmat = sim.device_tmat(0)
    op = MasterOperator(dev, tmat, "c128")
    b_host = np.ascontiguousarray(sim.right_hand_side[:, :, 0].ravel())
    b = torch.from_numpy(b_host).to(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)  # > L2 (126 MB)

    def solve_once(precision="c128"):
        x = b.clone()
        xs, info = solver.run(op, b, x, precision=precision)
        return xs, info, dict(solver.last_stats)

    for _ in range(args.warmup):
        solve_once()
    torch.cuda.synchronize()

    # ---- timed region: device-resident solves -------------------------------------------------
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.yasf_kernel_launches()
    per_ms = []
    stats = None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            x, info, stats = solve_once()
            e1.record()
            e1.synchronize()
            per_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    launches = lib.yasf_kernel_launches() - launches0
    if dist is not None:
        dist.barrier()
    total_ms = sum(per_ms)
    tot = torch.tensor([total_ms], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    max_total_ms = float(tot.item())
    value = world * args.steps / (max_total_ms / 1e3)

    # ---- cross sections of the timed solution ----------------------------------------------
    sim.scattered_field_coefficients = x.cpu().numpy().reshape(n, -1)[:, :, None]
    opt = Optics(sim)
    opt.compute_cross_sections()
    c_ext64 = float(opt.c_ext[0])
    c_sca64 = float(opt.c_sca[0])

    # ---- e2e through the public API with host buffers ----------------------------------------
    e2e_ms = []
    for i in range(max(2, min(args.steps, 5)) + 1):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xh, info_h = solver.run(op, b_host)  # H2D of b, x0 = b, device GMRES, D2H of x
        t1 = time.perf_counter()
        if i > 0:
            e2e_ms.append((t1 - t0) * 1e3)
    e2e_value = world * len(e2e_ms) / (sum(e2e_ms) / 1e3)

    # ---- matvec rate and contraction roofline -------------------------------------------------
    xv = torch.randn(dev.n, dtype=torch.complex128, device=device)
    for _ in range(3):
        dev.master(xv, tmat)
    reps = 10
    flush.zero_()
    torch.cuda.synchronize()
    m0 = torch.cuda.Event(enable_timing=True)
    m1 = torch.cuda.Event(enable_timing=True)
    m0.record()
    for _ in range(reps):
        dev.master(xv, tmat)
    m1.record()
    m1.synchronize()
    mv_ms = m0.elapsed_time(m1) / reps
    flops = algorithmic_flops(n, agg.lmax)
    achieved = flops / (mv_ms / 1e3) / 1e12
    traffic = None
    tfile = REPO / "profiles" / f"contract_{args.workload}_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("dram_bytes_per_launch")

    # ---- mixed precision (complex64 inner solves, float64 refinement) -------------------------
    mixed = None
    if not args.no_mixed:
        for _ in range(1):
            solve_once("c64")
        mixed_ms = []
        xm = None
        for _ in range(max(1, min(args.steps, 3))):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            xm, _, mst = solve_once("c64")
            e1.record()
            e1.synchronize()
            mixed_ms.append(e0.elapsed_time(e1))
        sim.scattered_field_coefficients = xm.cpu().numpy().reshape(n, -1)[:, :, None]
        om = Optics(sim)
        om.compute_cross_sections()
        mixed = {"solves_per_s": len(mixed_ms) / (sum(mixed_ms) / 1e3),
                 "c_ext_rel_err_vs_fp64": abs(float(om.c_ext[0]) - c_ext64) / abs(c_ext64),
                 "stats": mst}

    # ---- CPU baseline (oracle port, row sample) -----------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        t_mv_cpu, rows = cpu_matvec_seconds(agg, numerics.translation_ab5, args.cpu_seconds, threads)
        mv_per_solve = stats["matvecs_f64"]
        cpu = {"value": 1.0 / (t_mv_cpu * mv_per_solve), "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{rows} of {n} receiving-sphere rows of the C-restated particle_interaction_scalar, "
                         f"extrapolated to one matvec ({t_mv_cpu:.1f} s); solve = {mv_per_solve} matvecs "
                         "(this solve's count, preconditioner cost excluded)",
               "matvec_s": t_mv_cpu}

    if rank != 0:
        return
    lat = sorted(per_ms)
    nbytes = dev.n * 16
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": max_total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c128",
        "data": "synthetic (seeded RSA aggregate, no dataset)",
        "config": {"workload": agg.name, "n_spheres": n, "lmax": agg.lmax, "unknowns": dev.n,
                   "rtol": rtol, "preconditioner": f"block-Jacobi {cells}x{cells}x{cells} cells" if pre else None,
                   "restart": args.restart, "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "flushed (256 MB write) before every timed solve"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "matvec_per_s": 1e3 / mv_ms,
        "solve_stats": stats,
        "prepare_s": prepare_s,
        "c_ext": c_ext64,
        "c_sca": c_sca64,
        "mixed": mixed,
        "roofline": {"bound": "fp64", "kernel": "contract_kernel (pair side + contraction)",
                     "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / FP64_NOMINAL_TFLOPS, "traffic": traffic,
                     "flops_per_launch": flops,
                     "timing": f"CUDA events over {reps} master matvecs (source build + contraction + "
                               "reduction), {:.3f} ms each".format(mv_ms),
                     "peak_source": "nominal B200 FP64 (148 SMs x 64 FMA/clk x 2 x 1.965 GHz); "
                                    "MEASURED_PEAKS.json has no FP64 figure"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def matvec_probe(args) -> None:
    """Four coupling matvecs (the first is warm-up) on the first N spheres of the workload."""
    import torch

    from yasf_b200.device import PRECISIONS, CouplingDevice
    from yasf_b200.numerics import cached_translation_table

    agg, _, _ = workload(args.workload)
    n = min(args.matvec_probe, agg.n)
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions[:n], agg.k,
                         torch.device("cuda", 0))
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    for _ in range(4):
        y = dev.coupling(x, PRECISIONS[args.precision])
    torch.cuda.synchronize()
    print(json.dumps({"probe": agg.name, "n": n, "precision": args.precision,
                      "max_abs": float(y.abs().max())}))


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["c1", "c2", "c5"], default="c2")
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--no-precond", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--matvec-probe", type=int, default=0, metavar="N",
                    help="profiling aid: run 4 coupling matvecs on the first N spheres and exit")
    ap.add_argument("--precision", choices=["c128", "c64"], default="c128")
    args = ap.parse_args()
    if args.matvec_probe:
        matvec_probe(args)
        return
    if args.warmup < 3:
        print("bench.py: --warmup must be >= 3", file=sys.stderr)
        sys.exit(2)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_b200(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()

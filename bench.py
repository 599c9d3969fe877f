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
  batched          the mixed-precision batched form on the same aggregate: --batched-rhs incidences
                   (128 by default) in one refined solve (TF32 tensor-core inner operator), solves/s
                   and speed-up over value
  roofline         the coupling contraction (contract_kernel) against the float64 pipe
  cpu_baseline     the oracle (plain-C restatement of the reference CPU matvec) on host cores,
                   row-sampled, converted to solves/s with this solve's matvec count

Other workloads (--workload):
  c1     100 spheres, lmax 4, rtol 1e-8, no preconditioner (the reference's CPU-sized case)
  c3     the C2 aggregate with R = 128 right-hand sides (64 seeded Fibonacci directions x TE/TM):
         one step = one batched solve (TF32 tensor-core panel inner GMRES, float64 refinement to
         rtol 1e-8); value = right-hand sides solved per second; C_ext / coefficient errors
         against float64 solves of sampled columns
  serve  the serving stream (Poisson arrivals at 20 req/s; N in [50, 3000], lmax 3..8, R in
         {1, 2, 16, 64}); one step = one request of the stream's prefix (--steps requests, the
         first of the 512-request stream); warm-up = requests drawn from the same distribution
         with other seeds; value = right-hand sides solved per second over the makespan, with
         p50/p99 request latency and the C_ext error of sampled requests against float64 solves
  c5     20000 spheres, lmax 4, R = 2 (TE, TM), 8x8x8 block-Jacobi, rtol 1e-6: plain float64 and
         mixed-precision solves of both columns, phases timed separately

--impl reference times the reference's CPU algorithm (the oracle port, all host threads) on the
same workload and prints the same metric with "impl": "reference".
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

from yasf_b200.replicas import gather_records, max_over_ranks, serving_totals, shard_requests  # noqa: E402

METRIC = "solves/s (C2: 2000 spheres, lmax 6, FP64, GMRES rtol 1e-8, 4x4x4 block-Jacobi); matvec/s"
METRIC_C3 = ("solves/s (C3: 2000 spheres, lmax 6, R=128 incidences, TF32 panel inner GMRES in FP64 "
             "refinement to rtol 1e-8)")
METRIC_SERVE = "solves/s + p50/p99 latency (serving stream, mixed precision, C_ext err vs FP64 GPU)"
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
    if name == "c3":
        return aggregate_c2(seed=0), 1e-8, None
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
    from oracle.restate import reference_translation_table

    agg, _, _ = workload(args.workload)
    table = reference_translation_table(agg.lmax)  # the reference's own table (committed fixture)
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
                   "parallelism": "host threads",
                   "solve_model": "matvec time x the b200 solve's float64 matvec count; no preconditioner "
                                  "cost: the reference's own block-Jacobi prepare cannot factor cells of two "
                                  "or more spheres (yasfpy/preconditioner.py:408-423), and without it GMRES "
                                  "needs more iterations, so this understates the reference's solve time",
                   "translation_table": "the reference's own Numerics.translation_ab5 (committed fixture)"},
        "matvec_per_s": 1.0 / t_mv,
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample_rows} receiving-sphere rows of the C-restated particle_interaction_scalar "
                      f"over {args.steps} steps, extrapolated x{agg.n}/rows per matvec; solve = "
                      f"{mv_per_solve} matvecs (the b200 solve's count, preconditioner cost excluded)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_probe(args) -> None:
    """The reference's own GPU coupling matvec (Numba-CUDA CudaDenseCouplingOps,
    yasfpy/coupling/cuda_dense.py:160-448) from the unmodified copy in baseline/_ref, on the chosen
    workload's aggregate: Simulation set-up, one warm-up matvec, then the mean of three. Its stand-ins
    for pywigxjpf / refidxdb / pyperf come from oracle/stubs; its table cache goes to a temporary
    HOME. Prints one JSON line (or the reason it cannot run)."""
    import tempfile

    root = Path(__file__).resolve().parent
    out = {"probe": "reference_gpu_matvec", "workload": args.workload}
    if not (root / "baseline" / "_ref" / "yasfpy").is_dir():
        out["unavailable"] = "baseline/_ref holds no copy of the reference"
        print(json.dumps(out))
        return
    sys.path.insert(0, str(root / "baseline" / "_ref"))
    sys.path.insert(0, str(root / "oracle" / "stubs"))
    os.environ["HOME"] = tempfile.mkdtemp(prefix="yasf_ref_home_")
    try:
        from numba import cuda

        from yasfpy.initial_field import InitialField
        from yasfpy.numerics import Numerics
        from yasfpy.parameters import Parameters
        from yasfpy.particles import Particles
        from yasfpy.simulation import Simulation
        from yasfpy.solver import Solver

        out["device"] = str(cuda.get_current_device().name)
        agg, _, _ = workload(args.workload)
        particles = Particles(position=agg.positions, r=agg.radii,
                              refractive_index=np.full(agg.n, agg.refractive_index))
        field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                             polarization="TE")
        params = Parameters(wavelength=np.array([agg.wavelength]), medium_refractive_index=np.ones(1, dtype=complex),
                            particles=particles, initial_field=field)
        numerics = Numerics(lmax=agg.lmax, sampling_points_number=np.array([10]), gpu=True,
                            solver=Solver(solver_type="gmres", tolerance=1e-8, max_iter=100, restart=100),
                            coupling_backend="dense")
        numerics.compute_translation_table()
        t0 = time.perf_counter()
        sim = Simulation(params, numerics)
        out["setup_s"] = time.perf_counter() - t0
        rng = np.random.default_rng(0)
        x = rng.normal(size=agg.n * numerics.nmax) + 1j * rng.normal(size=agg.n * numerics.nmax)
        t0 = time.perf_counter()
        sim.coupling_matrix_multiply(x, idx=0)
        out["first_matvec_s"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        for _ in range(3):
            sim.coupling_matrix_multiply(x, idx=0)
        out["matvec_s"] = (time.perf_counter() - t0) / 3
    except Exception as e:  # record why the reference's GPU path cannot run here
        out["unavailable"] = f"{type(e).__name__}: {e}"
    print(json.dumps(out))


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
    max_total_ms = max_over_ranks(sum(per_ms), device)
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

    # ---- mixed-precision batched solve of the same aggregate (R incidences) ------------------
    batched = None
    if args.batched_rhs and agg.lmax <= 6 and not args.no_mixed:
        from yasf_b200.incident import plane_wave_block
        from yasf_b200.workloads import incidences

        polar, azim, pol = incidences(args.batched_rhs // 2, rotation_seed=0)
        a_blk = plane_wave_block(agg.lmax, agg.positions, agg.k, polar, azim, pol)
        A_cols = np.ascontiguousarray(np.moveaxis(a_blk, 2, 0).reshape(len(pol), -1))
        tm_host = tmat.cpu().numpy()
        B_cols = torch.from_numpy(np.ascontiguousarray(A_cols * tm_host[None, :])).to(device)
        kw = dict(rtol=rtol, restart=50, max_refine=8, inner_rtol=args.inner_rtol, inner="tf32")
        dev.batched_solve(tmat, B_cols, **kw)  # warm-up (workspace, plan set-up)
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        Xb, bst = dev.batched_solve(tmat, B_cols, **kw)
        e1.record()
        e1.synchronize()
        b_s = e0.elapsed_time(e1) / 1e3
        colres = bst.pop("column_residuals")
        errors = None
        if not args.no_column_errors:
            errors = all_column_errors(dev, tmat, A_cols, B_cols, Xb, agg.k)
        batched = {"solves_per_s": len(pol) / b_s, "speedup_vs_plain_fp64": len(pol) / b_s / value,
                   "nrhs": len(pol), "seconds": b_s, "max_fp64_relative_residual": max(colres),
                   "error_vs_fp64_all_columns": errors,
                   "stats": bst,
                   "config": f"same aggregate, {len(pol) // 2} seeded Fibonacci directions x TE/TM, TF32 "
                             f"tensor-core panel inner GMRES (inner rtol {args.inner_rtol:g}, restart 50) in float64 "
                             f"refinement to rtol {rtol}, float64 residuals by the dense multi-column "
                             "kernel from 12 columns"}
        del B_cols, Xb

    # ---- CPU baseline (oracle port, row sample) -----------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        from oracle.restate import reference_translation_table

        t_mv_cpu, rows = cpu_matvec_seconds(agg, reference_translation_table(agg.lmax), args.cpu_seconds,
                                            threads)
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
        "batched": batched,
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


# ---------------------------------------------------------------------------------------------
def cross_sections(dev, a_col, x_col, k: float) -> tuple[float, float]:
    """(C_ext, C_sca) of one solved column, on the device (optics.py formulas)."""
    c_ext = -np.real(dev.dotc(a_col, x_col)) / k**2 * np.pi
    c_sca = abs(dev.scattering_bilinear(x_col)) / k**2 * np.pi
    return float(c_ext), float(c_sca)


def all_column_errors(dev, tmat, A_cols: np.ndarray, B, X, k: float) -> dict:
    """Error of every column of a batched solution X against plain float64 GPU solutions.

    The float64 solutions come from the lockstep GMRES with the complex128 inner operator (the
    float64 dense multi-column kernel for 12 or more columns up to lmax 6, else the complex128
    coupling kernel), no preconditioner, refined to rtol 1e-10: no reduced precision anywhere.
    Reported per column: relative coefficient error (2-norm), relative C_ext and C_sca error."""
    import torch

    X64, st64 = dev.batched_solve(tmat, B, rtol=1e-10, restart=60, max_refine=4, inner_rtol=1e-10,
                                  inner="c128")
    R = X.shape[0]
    coef = (torch.linalg.vector_norm(X - X64, dim=1) / torch.linalg.vector_norm(X64, dim=1)).cpu().numpy()
    At = torch.from_numpy(np.ascontiguousarray(A_cols)).to(X.device)
    ce = (-torch.real((At.conj() * X).sum(dim=1)) / k**2 * np.pi).cpu().numpy()
    ce64 = (-torch.real((At.conj() * X64).sum(dim=1)) / k**2 * np.pi).cpu().numpy()
    cs = np.array([abs(dev.scattering_bilinear(X[c].contiguous())) for c in range(R)]) / k**2 * np.pi
    cs64 = np.array([abs(dev.scattering_bilinear(X64[c].contiguous())) for c in range(R)]) / k**2 * np.pi
    ext_err = np.abs(ce - ce64) / np.abs(ce64)
    sca_err = np.abs(cs - cs64) / np.abs(cs64)
    colres = st64.pop("column_residuals")

    def summ(v):
        return {"max": float(np.max(v)), "median": float(np.median(v)),
                "per_column": [float(f"{e:.3g}") for e in v]}

    return {"columns": R, "coef_rel_err": summ(coef), "c_ext_rel_err": summ(ext_err),
            "c_sca_rel_err": summ(sca_err),
            "fp64_reference": {"max_relative_residual": float(max(colres)), "stats": st64,
                               "how": "lockstep float64 GMRES, complex128 inner operator (float64 dense "
                                      "multi-column kernel), no preconditioner, rtol 1e-10"}}


def fp64_column(dev, tmat, b_col, rtol=1e-10):
    """Plain float64 device GMRES (no preconditioner) of one column: the float64 reference."""
    x = b_col.clone()
    st = dev.gmres(tmat, b_col, x, rtol, 100, 50)
    return x, st


def run_batched(args, rank: int, world: int) -> None:
    """C3: one batched solve of the C2 aggregate's 128 incidences per step (ranks are replicas)."""
    import torch

    from yasf_b200 import _lib
    from yasf_b200.device import CouplingDevice
    from yasf_b200.incident import plane_wave_block
    from yasf_b200.mie import mie_tmatrix_per_sphere
    from yasf_b200.numerics import cached_translation_table
    from yasf_b200.workloads import incidences

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _lib.load()
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    agg, rtol, _ = workload("c3")
    polar, azim, pol = incidences(64, rotation_seed=0)
    R = len(pol)
    tm = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
    a = plane_wave_block(agg.lmax, agg.positions, agg.k, polar, azim, pol)
    A = np.ascontiguousarray(np.moveaxis(a, 2, 0).reshape(R, -1))
    B_host = torch.from_numpy(np.ascontiguousarray(A * tm[None, :])).pin_memory()
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions, agg.k, device)
    tmat = torch.from_numpy(tm).to(device)
    B = B_host.to(device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    kw = dict(rtol=rtol, restart=args.restart_batched, max_refine=8, inner_rtol=args.inner_rtol, inner="tf32")

    for _ in range(args.warmup):
        dev.batched_solve(tmat, B, **kw)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.yasf_kernel_launches()
    per_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            X, st = dev.batched_solve(tmat, B, **kw)
            e1.record()
            e1.synchronize()
            per_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    launches = lib.yasf_kernel_launches() - launches0
    if dist is not None:
        dist.barrier()
    max_total_ms = max_over_ranks(sum(per_ms), device)
    value = world * R * args.steps / (max_total_ms / 1e3)

    # e2e: pinned host B -> device, solve, X -> host
    X_host = torch.empty_like(B_host).pin_memory()
    flush.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Bd = B_host.to(device, non_blocking=True)
    Xe, _ = dev.batched_solve(tmat, Bd, **kw)
    X_host.copy_(Xe, non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    del Bd, Xe

    # errors of every column against plain float64 GPU solutions
    errors = all_column_errors(dev, tmat, A, B, X, agg.k)
    colres = st.pop("column_residuals")

    if rank != 0:
        return
    nbytes = R * dev.n * 16
    lat = sorted(per_ms)
    line = {
        "metric": METRIC_C3, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "tf32 inner / c128 refinement",
        "data": "synthetic (seeded RSA aggregate, seeded Fibonacci incidences, no dataset)",
        "config": {"workload": agg.name + "-R128", "n_spheres": agg.n, "lmax": agg.lmax,
                   "unknowns": dev.n, "nrhs": R, "rtol": rtol, "restart": args.restart_batched,
                   "inner": f"TF32 tensor-core panel, inner_rtol {args.inner_rtol:g}", "preconditioner": None,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "flushed (256 MB write) before every timed solve"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "solve_stats": st,
        "fp64_residual_all_columns": {"max": max(colres), "median": statistics.median(colres)},
        "error_vs_fp64_all_columns": errors,
        "e2e": {"value": world * R / e2e_s, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_serve(args, rank: int, world: int) -> None:
    """Serving stream prefix; requests are dealt round-robin to ranks (replicas, no exchange)."""
    import torch

    from yasf_b200 import _lib
    from yasf_b200.device import CouplingDevice
    from yasf_b200.incident import plane_wave_block
    from yasf_b200.mie import mie_tmatrix_per_sphere
    from yasf_b200.numerics import cached_translation_table
    from yasf_b200.serve import ServeConfig, Server, summarize
    from yasf_b200.workloads import serving_requests

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _lib.load()
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
    stream = serving_requests(args.steps)
    mine = shard_requests(stream, rank, world)
    # warm-up: small requests from the same distribution (other seeds), one per lmax in use
    # at least, so that every plan and kernel variant is set up before the timed stream
    lmaxes = sorted({r.aggregate.lmax for r in mine})
    warm = []
    for i in range(max(args.warmup, len(lmaxes))):
        lm = (lmaxes[i % len(lmaxes)],) if lmaxes else (3,)
        warm += serving_requests(1, seed=7 + i, n_range=(50, 300), lmax_choices=lm, param_seed=100_000 + i)
    from yasf_b200.autotune import Autotuner

    tuner = Autotuner() if args.autotune else None
    cfg = ServeConfig(max_slots=args.slots, rtol=args.serve_rtol, tuner=tuner, group_small=not args.no_group)
    server = Server(cfg, device=device)
    server.run(warm, realtime=False)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.yasf_kernel_launches()
    with ClockSampler(local) as clk:
        results = server.run(mine, realtime=True)
    torch.cuda.synchronize()
    launches = lib.yasf_kernel_launches() - launches0
    summ = summarize(results)
    grouped = [r for r in results if r.error is None and r.stats.get("group_size", 0) >= 1]
    summ["grouped_requests"] = len(grouped)
    summ["mean_group_size"] = (sum(r.stats["group_size"] for r in grouped) / len(grouped)) if grouped else None
    summ["inner_operators"] = {k: sum(1 for r in results if r.error is None and r.stats.get("inner") == k)
                               for k in ("tf32", "c64", "c64 grouped")}
    flat = gather_records([(r.rid, r.nrhs, r.latency, r.finished, r.error) for r in results])
    tot = serving_totals(flat, min(r.arrival for r in stream))

    # C_ext of sampled requests against float64 solves (outside the timed region)
    errs = []
    for r in results[: args.error_samples]:
        if r.error is not None:
            continue
        req = next(q for q in mine if q.rid == r.rid)
        agg = req.aggregate
        dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions, agg.k, device)
        tmh = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
        a = plane_wave_block(agg.lmax, agg.positions, agg.k, req.polar[:1], req.azimuthal[:1], req.pol[:1])
        a0 = np.ascontiguousarray(a[:, :, 0].ravel())
        tmat = torch.from_numpy(tmh).to(device)
        b0 = torch.from_numpy(a0 * tmh).to(device)
        x64, st64 = fp64_column(dev, tmat, b0)
        ce64 = -np.real(np.vdot(a0, x64.cpu().numpy())) / agg.k**2 * np.pi
        errs.append({"rid": r.rid, "n": agg.n, "lmax": agg.lmax, "nrhs": r.nrhs,
                     "c_ext_rel_err": abs(r.c_ext[0] - ce64) / abs(ce64), "fp64_info": st64["info"]})
    if rank != 0:
        return
    line = {
        "metric": METRIC_SERVE, "value": tot["solves_per_s"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot["makespan_s"] * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "tf32 inner (enough columns) / c64 inner (few columns), c128 refinement",
        "data": "synthetic (seeded request stream, no dataset)",
        "config": {"workload": f"serving stream, first {args.steps} of 512 requests (Poisson 20 req/s)",
                   "requests": args.steps, "slots": args.slots, "rtol": args.serve_rtol,
                   "parallelism": "requests dealt round-robin to replicas" if world > 1 else "single GPU",
                   "l2": "inputs of a request larger than L2 for most requests; no flush between requests"},
        "latency_s": {"p50": tot["latency_p50_s"], "p99": tot["latency_p99_s"]},
        "requests_completed": tot["completed"], "requests_failed": tot["failed"],
        "rhs_solves": tot["rhs_solves"], "makespan_s": tot["makespan_s"], "rank0_summary": summ,
        "requests": [{"rid": r.rid, "n": r.n_spheres, "lmax": r.lmax, "nrhs": r.nrhs,
                      "inner": r.stats.get("inner"), "group": r.stats.get("group_size"),
                      "inner_steps": r.stats.get("inner_steps"),
                      "restart": r.stats.get("restart"),
                      "relative_residual": r.stats.get("worst_relative_residual"),
                      "admitted_s": round(r.admitted, 3),
                      "latency_s": round(r.latency, 3), "error": r.error} for r in results],
        "c_ext_error_vs_fp64": {"max": max((e["c_ext_rel_err"] for e in errs), default=None),
                                "samples": errs},
        "autotune": None if tuner is None else {
            "decisions": len(tuner.decisions()),
            "inner_chosen": {k: sum(1 for d in tuner.decisions() if d.inner == k) for k in ("tf32", "c64")}},
        "e2e": {"value": tot["solves_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "each request enters as host arrays (geometry, incidences) and returns C_ext "
                        "and the solution to the host: the serving loop is end to end"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_large(args, rank: int, world: int) -> None:
    """C5: the 20,000-sphere aggregate (lmax 4, 960,000 unknowns, R = 2 polarisations TE/TM along
    +z), block-Jacobi on 8x8x8 cells, GMRES to rtol 1e-6: plain float64 against mixed precision
    (complex64 inner GMRES in float64 refinement), each column solved on the device.

    Phases are timed separately: random sequential addition (host), preconditioner prepare
    (assembly, factorisation, finalize), each float64 solve and each mixed solve (CUDA events),
    with iteration and matvec counts. A warm-up step is one application of each operator (float64
    and complex64 master operators, preconditioner), not a solve: one C5 solve takes minutes.
    value = right-hand sides per second of the mixed form (device-resident); e2e = the same solves
    with the right-hand side copied from pinned host memory and the solution copied back inside
    the timed region."""
    import torch

    from yasf_b200 import _lib
    from yasf_b200.device import PRECISIONS, CouplingDevice, DevicePreconditioner
    from yasf_b200.incident import plane_wave_block
    from yasf_b200.mie import mie_tmatrix_per_sphere
    from yasf_b200.numerics import cached_translation_table
    from yasf_b200.preconditioner import make_particle_partition

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    lib = _lib.load()
    t0 = time.perf_counter()
    agg, rtol, cells = workload("c5")
    rsa_s = time.perf_counter() - t0
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions, agg.k, device)
    tm = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
    tmat = torch.from_numpy(tm).to(device)
    polar, azim, pol = np.zeros(2), np.zeros(2), np.array([1, 2])  # +z, TE and TM
    a_blk = plane_wave_block(agg.lmax, agg.positions, agg.k, polar, azim, pol)
    A_cols = np.ascontiguousarray(np.moveaxis(a_blk, 2, 0).reshape(2, -1))
    B_host = torch.from_numpy(np.ascontiguousarray(A_cols * tm[None, :])).pin_memory()
    B = B_host.to(device)
    extent = agg.positions.max(axis=0) - agg.positions.min(axis=0)
    blocks = make_particle_partition(agg.positions, (extent + 2.0) / cells)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pc = DevicePreconditioner(dev, blocks)
    phases = pc.prepare(tmat)
    torch.cuda.synchronize()
    prepare_s = time.perf_counter() - t0

    restart, maxiter = args.restart_large, 4
    x = torch.randn(dev.n, dtype=torch.complex128, device=device)
    for _ in range(args.warmup):
        dev.master(x, tmat, PRECISIONS["c128"])
        dev.master(x, tmat, PRECISIONS["c64"])
        pc.apply(x, PRECISIONS["c64"])
    torch.cuda.synchronize()
    del x

    def solve(col, precision, e2e=False):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        b = B_host[col].to(device, non_blocking=True) if e2e else B[col]
        e0.record()
        xs = b.clone()
        st = dev.gmres(tmat, b, xs, rtol, restart, maxiter, PRECISIONS[precision], pc)
        e1.record()
        xh = xs.cpu() if e2e else None
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        st["seconds"] = e0.elapsed_time(e1) / 1e3
        if e2e:
            st["e2e_seconds"] = wall
        return xs, xh, st

    launches0 = lib.yasf_kernel_launches()
    fp64, mixed = [], []
    with ClockSampler(local) as clk:
        for c in range(2):
            fp64.append(solve(c, "c128"))
        for c in range(2):
            mixed.append(solve(c, "c64", e2e=True))
    launches = lib.yasf_kernel_launches() - launches0

    k = agg.k
    cols = []
    for c in range(2):
        x64, xm = fp64[c][0], mixed[c][0]
        a = torch.from_numpy(A_cols[c]).to(device)
        ce64 = -np.real(dev.dotc(a, x64)) / k**2 * np.pi
        cem = -np.real(dev.dotc(a, xm)) / k**2 * np.pi
        cs64 = abs(dev.scattering_bilinear(x64)) / k**2 * np.pi
        csm = abs(dev.scattering_bilinear(xm)) / k**2 * np.pi
        cols.append({"polarisation": ["TE", "TM"][c], "c_ext_fp64": ce64, "c_sca_fp64": cs64,
                     "c_ext_rel_err_mixed": abs(cem - ce64) / abs(ce64),
                     "c_sca_rel_err_mixed": abs(csm - cs64) / abs(cs64),
                     "coef_rel_err_mixed": float(torch.linalg.vector_norm(xm - x64) / torch.linalg.vector_norm(x64)),
                     "fp64": fp64[c][2], "mixed": mixed[c][2]})
    fp64_s = sum(f[2]["seconds"] for f in fp64)
    mixed_s = sum(m[2]["seconds"] for m in mixed)
    mixed_e2e_s = sum(m[2]["e2e_seconds"] for m in mixed)
    if rank != 0:
        return
    line = {
        "metric": "solves/s (C5: 20000 spheres, lmax 4, R=2, 8x8x8 block-Jacobi, rtol 1e-6; mixed precision "
                  "vs plain FP64, C_ext err vs FP64 GPU)",
        "value": 2 / mixed_s, "unit": UNIT, "n_gpus": world, "steps": 2, "warmup": args.warmup,
        "ms_per_step": mixed_s * 1e3 / 2, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 inner / c128 refinement", "data": "synthetic (seeded RSA aggregate, no dataset)",
        "config": {"workload": agg.name + "-R2", "n_spheres": agg.n, "lmax": agg.lmax, "unknowns": dev.n,
                   "nrhs": 2, "rtol": rtol, "restart": restart,
                   "preconditioner": f"block-Jacobi {cells}x{cells}x{cells} cells ({len(blocks)} blocks)",
                   "parallelism": "single GPU",
                   "l2": "inputs (15 MB per column, 1 GB V stream, 29-58 GB of factors) larger than L2",
                   "warmup": "one application of each operator per warm-up step (not a solve)"},
        "fp64_solves_per_s": 2 / fp64_s, "mixed_speedup_vs_fp64": fp64_s / mixed_s,
        "phases_s": {"rsa_host": rsa_s, "prepare": prepare_s, "prepare_detail": phases,
                     "fp64_solves": fp64_s, "mixed_solves": mixed_s},
        "columns": cols,
        "e2e": {"value": 2 / mixed_e2e_s, "unit": UNIT, "h2d_bytes_per_step": dev.n * 16,
                "d2h_bytes_per_step": dev.n * 16},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def panel_probe(args) -> None:
    """Four panel matvecs (the first is warm-up) on the first N spheres with --nrhs columns
    (TF32 tensor-core panel, or the float64 dense multi-column kernel with --float64-panel)."""
    import torch

    from yasf_b200.device import CouplingDevice
    from yasf_b200.numerics import cached_translation_table

    agg, _, _ = workload("c2")
    n = min(args.panel_probe, agg.n)
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions[:n], agg.k,
                         torch.device("cuda", 0))
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(args.nrhs, dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    tmat = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g) * 0.1
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    apply = dev.dpanel if args.float64_panel else dev.panel
    y = apply(x, tmat)
    e0.record()
    for _ in range(3):
        y = apply(x, tmat)
    e1.record()
    e1.synchronize()
    print(json.dumps({"probe": "dpanel" if args.float64_panel else "panel", "n": n, "nrhs": args.nrhs,
                      "ms": e0.elapsed_time(e1) / 3, "max_abs": float(y.abs().max())}))


def matvec_probe(args) -> None:
    """Four coupling matvecs (the first is warm-up, the others timed) on the first N spheres."""
    import torch

    from yasf_b200.device import PRECISIONS, CouplingDevice
    from yasf_b200.numerics import cached_translation_table

    agg, _, _ = workload(args.workload)
    n = min(args.matvec_probe, agg.n)
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions[:n], agg.k,
                         torch.device("cuda", 0))
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    y = dev.coupling(x, PRECISIONS[args.precision])
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        y = dev.coupling(x, PRECISIONS[args.precision])
    e1.record()
    e1.synchronize()
    print(json.dumps({"probe": agg.name, "n": n, "precision": args.precision,
                      "ms": e0.elapsed_time(e1) / 3, "max_abs": float(y.abs().max())}))


def precond_probe(args) -> None:
    """Block-Jacobi preconditioner on the first N spheres of the C2 aggregate (4x4x4 cells of the
    aggregate's extent, as in the default bench line): prepare (assemble, batched LU, finalize),
    then one warm-up and five timed one-column complex64 applies, and one 16-column apply."""
    import torch

    from yasf_b200.device import PRECISIONS, CouplingDevice, DevicePreconditioner
    from yasf_b200.mie import mie_tmatrix_per_sphere
    from yasf_b200.numerics import cached_translation_table
    from yasf_b200.preconditioner import make_particle_partition

    agg, _, _ = workload("c2")
    n = min(args.precond_probe, agg.n)
    pos = agg.positions[:n]
    dev0 = torch.device("cuda", 0)
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), pos, agg.k, dev0)
    tmat = torch.from_numpy(mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii[:n], agg.refractive_index)).to(dev0)
    ext = agg.positions.max(axis=0) - agg.positions.min(axis=0)
    blocks = make_particle_partition(pos, (ext + 2.0) / 4)
    pc = DevicePreconditioner(dev, blocks)
    phases = pc.prepare(tmat)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(dev.n, dtype=torch.complex128, device=dev0, generator=g)
    X = torch.randn(16, dev.n, dtype=torch.complex128, device=dev0, generator=g)
    y = pc.apply(x, PRECISIONS["c64"])
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        y = pc.apply(x, PRECISIONS["c64"])
    e1.record()
    e1.synchronize()
    one = e0.elapsed_time(e1) / 5
    Y = pc.apply(X, PRECISIONS["c64"])
    e0.record()
    Y = pc.apply(X, PRECISIONS["c64"])
    e1.record()
    e1.synchronize()
    dims = [len(b) * dev.nmax for b in blocks]
    factor_bytes = sum(d * d for d in dims) * 8  # complex64 L and U, streamed once per apply
    print(json.dumps({"probe": "precond", "n": n, "blocks": len(blocks), "max_dim": max(dims),
                      "prepare_s": phases, "factor_bytes": factor_bytes, "apply_c64_ms": one,
                      "apply_c64_gbs": factor_bytes / one / 1e6, "apply_c64_16cols_ms": e0.elapsed_time(e1),
                      "finite": bool(torch.isfinite(y).all() and torch.isfinite(Y).all())}))


def farfield_probe(args) -> None:
    """Far field (E_theta, E_phi, Stokes) of the first N spheres of the C2 aggregate on 10,000
    Fibonacci sampling directions, random coefficients: one warm-up and five timed launches."""
    import torch

    from yasf_b200.device import CouplingDevice
    from yasf_b200.numerics import Numerics, cached_translation_table

    agg, _, _ = workload("c2")
    n = min(args.farfield_probe, agg.n)
    dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions[:n], agg.k,
                         torch.device("cuda", 0))
    g = torch.Generator(device="cuda").manual_seed(0)
    coef = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    _, polar, azim = Numerics.compute_fibonacci_sphere_points(10_000)
    dirs = dev.far_field_directions(polar, azim)  # setup, outside the timed launches
    dev.far_field(coef, dirs)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        dev.far_field(coef, dirs)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / 5
    cmacs = 10_000 * n * dev.nmax
    print(json.dumps({"probe": "farfield", "n": n, "directions": 10_000, "ms": ms,
                      "complex_macs": cmacs, "tflops_fp64": cmacs * 8 / ms / 1e9}))


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["c1", "c2", "c3", "serve", "c5"], default="c2")
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--no-precond", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--batched-rhs", type=int, default=128,
                    help="right-hand sides of the batched solve reported beside the plain line (0: skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--matvec-probe", type=int, default=0, metavar="N",
                    help="profiling aid: run 4 coupling matvecs on the first N spheres and exit")
    ap.add_argument("--precision", choices=["c128", "c64"], default="c128")
    ap.add_argument("--panel-probe", type=int, default=0, metavar="N",
                    help="profiling aid: run 4 TF32 panel matvecs on the first N spheres and exit")
    ap.add_argument("--nrhs", type=int, default=128, help="columns of --panel-probe")
    ap.add_argument("--reference-gpu-probe", action="store_true",
                    help="profiling aid: time the reference's own Numba-CUDA matvec (the unmodified copy in "
                         "baseline/_ref) on the workload's aggregate and exit")
    ap.add_argument("--farfield-probe", type=int, default=0, metavar="N",
                    help="profiling aid: time the far field of the first N spheres on 10,000 directions and exit")
    ap.add_argument("--precond-probe", type=int, default=0, metavar="N",
                    help="profiling aid: prepare the block-Jacobi preconditioner on the first N spheres, "
                         "time its applies and exit")
    ap.add_argument("--float64-panel", action="store_true",
                    help="--panel-probe times the float64 dense multi-column coupling instead")
    ap.add_argument("--restart-batched", type=int, default=50, help="inner GMRES cycle length (c3)")
    ap.add_argument("--restart-large", type=int, default=250, help="GMRES cycle length (c5)")
    ap.add_argument("--inner-rtol", type=float, default=2e-3,
                    help="batched solves: inner GMRES tolerance per float64 refinement step")
    ap.add_argument("--slots", type=int, default=4, help="serving slots (serve)")
    ap.add_argument("--autotune", action="store_true",
                    help="serve: choose each request's inner operator with the (lmax, N, R) autotuner "
                         "(timed inside the run) instead of the fixed rule")
    ap.add_argument("--serve-rtol", type=float, default=1e-6, help="serving refinement tolerance")
    ap.add_argument("--no-group", action="store_true",
                    help="serve: solve every request on its own (no grouped solves of small requests)")
    ap.add_argument("--error-samples", type=int, default=3, help="float64 check solves (serve)")
    ap.add_argument("--no-column-errors", action="store_true",
                    help="skip the float64 reference solves behind the batched block's per-column errors")
    args = ap.parse_args()
    if args.matvec_probe:
        matvec_probe(args)
        return
    if args.panel_probe:
        panel_probe(args)
        return
    if args.precond_probe:
        precond_probe(args)
        return
    if args.farfield_probe:
        farfield_probe(args)
        return
    if args.reference_gpu_probe:
        reference_gpu_probe(args)
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
        elif args.workload == "c3":
            run_batched(args, rank, world)
        elif args.workload == "serve":
            run_serve(args, rank, world)
        elif args.workload == "c5":
            run_large(args, rank, world)
        else:
            run_b200(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()

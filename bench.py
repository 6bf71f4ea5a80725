#!/usr/bin/env python3
"""Benchmark: CD3D Q2 on the unit cube, 32^3 cells, assembly + multigrid FGMRES solve.

Workload (the headline configuration): Q2 hexahedra on the unit cube, 32^3 cells
(274,625 DOFs, 15.8M nonzeros on the finest level), eps = 1e-2,
b = (1,1,1)/sqrt(3), c = 0, f = 1, homogeneous Dirichlet, Galerkin; FGMRES(30)
preconditioned by one V(2,2) cycle with damped Jacobi (omega 0.8), stopped at
||r|| <= 1e-10 ||r0||.  A step = assemble every multigrid level + solve.  Mesh,
patterns and transfer operators are built once before timing (the reference's
construction phase).  Synthetic, deterministic inputs (no dataset is involved).

Multigrid hierarchy: with Galerkin operators on all of 2^3 ... 32^3 the reference's
own solver does not converge for this convection-dominated problem (1000 FGMRES
iterations, residual growing).  Each arm therefore runs its best convergent setting:
ours 5 levels 2^3 ... 32^3 with SUPG coarse-grid operators (Galerkin on the finest
level, so the solution is that of the same Galerkin system) and the exact FP64 coarse
solve; the reference 3 levels 8^3 ... 32^3 Galerkin with its SSOR coarse smoother.

  value  : solves/s with every input resident in HBM (device pointers, CUDA events
           on the library's stream), the mixed form (FP32 multigrid inside FP64 FGMRES,
           solution within 1e-8 of the FP64 solution);
  e2e    : the same through the C ABI with host buffers (rhs and initial guess copied
           in, solution copied out every step);
  roofline: the FP64 CSR SpMV on the finest level (the FGMRES matvec) against the
           measured HBM copy bandwidth;
  cpu_baseline: the reference's own code (oracle/_ref/cd3d_dump, compiled from the
           reference sources) on this host, one full solve of the same workload.

Multi-GPU: replicas only -- every rank solves its own instance (weak scaling), the
time is the maximum over ranks.
"""
import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

EPS = 1e-2
B = (1 / math.sqrt(3),) * 3


def num(x):
    """A number as the reference drivers read it from argv (atof of a plain decimal)."""
    return repr(float(x))
METRIC = "CD solves/s and p50/p99 latency at 1e-8 rel. err vs FP64; assembly Mcells/s"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=32, help="cells per direction on the finest level")
    ap.add_argument("--levels", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched CD2D section")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream section")
    ap.add_argument("--batched-instances", type=int, default=4096)
    ap.add_argument("--serving-requests", type=int, default=100, help="requests per arrival rate")
    ap.add_argument("--serving-rates", default="5,10,20,40",
                    help="mean arrivals per second, swept in this order (comma separated)")
    ap.add_argument("--no-tcd", action="store_true", help="skip the time-dependent CD2D section")
    ap.add_argument("--no-cd2d", action="store_true", help="skip the CD2D plain FP64 section")
    ap.add_argument("--no-general", action="store_true", help="skip the general-path assembly section")
    ap.add_argument("--headline-only", action="store_true",
                    help="time only the mixed-form steps (warm-up and timed) and print their line: "
                         "for launch lists of the headline step; skips every other section")
    ap.add_argument("--tcd-instances", type=int, default=256)
    ap.add_argument("--tcd-steps", type=int, default=1000)
    return ap.parse_args()


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref/cd3d_dump = the reference's own sources)
# ---------------------------------------------------------------------------
DAT = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_cube.PRM
GEOFILE: {mesh}/unit_cube.GEO
MESH_TYPE: 0
UNIFORM_STEPS: {steps}
LEVELS: {levels}
ANSATZ_ORDER: 2
DISCTYPE: 1
SOLVER_TYPE: 1
SC_SOLVER_SCALAR: 16
SC_PRECONDITIONER_SCALAR: 5
SC_SMOOTHER_SCALAR: 1
SC_SMOOTH_DAMP_FACTOR_SCALAR: 0.8
SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR: 0.8
SC_PRE_SMOOTH_SCALAR: 2
SC_POST_SMOOTH_SCALAR: 2
SC_MG_CYCLE_SCALAR: 1
SC_STEP_LENGTH_CONTROL_ALL_SCALAR: 0
SC_STEP_LENGTH_CONTROL_FINE_SCALAR: 0
SC_GMRES_RESTART: 30
SC_LIN_RED_FACTOR_SCALAR: 1e-10
SC_LIN_RES_NORM_MIN_SCALAR: 0
SC_LIN_MAXIT_SCALAR: 1000
SC_VERBOSE: 0
"""


REF_LEVELS = 3  # the reference's convergent hierarchy for this problem (see module docstring)


def reference_run(n, levels, tmp, tag="0"):
    """One assemble + solve of the workload by the compiled reference; returns its timings."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cd3d_dump")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    steps = int(round(np.log2(n))) - (levels - 1)
    dat = os.path.join(tmp, f"w{tag}.dat")
    with open(dat, "w") as f:
        f.write(DAT.format(out=os.path.join(tmp, f"w{tag}.out"), mesh=os.path.join(ROOT, "oracle", "meshes"),
                           steps=steps, levels=levels))
    p = subprocess.run([exe, dat, "-", num(EPS), *map(num, B), "0", "1", "0", "1e-10"], cwd=tmp,
                       capture_output=True, text=True, check=True)
    line = [l for l in p.stdout.splitlines() if l.startswith("{")][-1]
    return json.loads(line)


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    cores = cpu_count()
    # one reference process per core, each solving the workload; memory bound ~1.5 GB each
    try:
        mem_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_AVPHYS_PAGES") / 2 ** 30
    except (ValueError, OSError):
        mem_gb = 16
    procs = max(1, min(cores, 32, int(mem_gb // 2)))
    tmp = tempfile.mkdtemp()
    try:
        # The timed part of a step is what the GPU arm times: TSystemCD3D::Assemble + Solve.
        # Every process reports its own wall-clock times of those two calls (steady_clock
        # around Assemble() and Solve() in the dump driver); the processes run concurrently,
        # so a step takes the slowest process's assemble + solve.  Mesh refinement, FE spaces
        # and matrix structures (the reference's construction phase, which the GPU arm also
        # does once before its timed region) are reported beside it, not counted.
        def step():
            ps = []
            exe = os.path.join(ROOT, "oracle", "_ref", "cd3d_dump")
            steps_ = int(round(np.log2(args.n))) - (REF_LEVELS - 1)
            for k in range(procs):
                dat = os.path.join(tmp, f"w{k}.dat")
                with open(dat, "w") as f:
                    f.write(DAT.format(out=os.path.join(tmp, f"w{k}.out"),
                                       mesh=os.path.join(ROOT, "oracle", "meshes"), steps=steps_,
                                       levels=REF_LEVELS))
                ps.append(subprocess.Popen([exe, dat, "-", num(EPS), *map(num, B), "0", "1", "0", "1e-10"],
                                           cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                           text=True))
            outs = [json.loads([l for l in p.communicate()[0].splitlines() if l.startswith("{")][-1]) for p in ps]
            timed = max(o["t_assemble"] + o["t_solve"] for o in outs)
            construct = max(o["t_mesh"] + o["t_construct"] for o in outs)
            return timed, construct, outs
        for _ in range(max(0, min(args.warmup, 1))):
            step()
        times, cons, its = [], [], []
        for _ in range(args.steps):
            dt, ct, outs = step()
            times.append(dt)
            cons.append(ct)
            its.append(outs[0]["iterations"])
        total = sum(times)
        value = procs * len(times) / total
        out = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * total / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"CD3D Q2 unit cube {args.n}^3 cells, eps 1e-2, b=(1,1,1)/sqrt(3), f=1, "
                                   f"Dirichlet 0, Galerkin; step = assembly of all levels + FGMRES(30) with "
                                   f"one V(2,2) damped-Jacobi (0.8) cycle to ||r|| <= 1e-10 ||r0||",
                       "multigrid": f"{REF_LEVELS} levels Galerkin, SSOR coarse smoother (the reference's "
                                    f"own convergent setting; its exact coarse solve needs LAPACK)",
                       "processes": procs, "fgmres_iterations": its[0],
                       "timed_region": "TSystemCD3D::Assemble + Solve per process (steady_clock in the driver), "
                                       "the slowest of the concurrent processes per step; the same calls the "
                                       "GPU arm times",
                       "construction_s_per_step": float(np.mean(cons))},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                             "sample": f"{procs} concurrent reference processes x {args.steps} steps, "
                                       f"each one assemble+solve of the workload (construction excluded)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(out), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.remove(self.path)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local):
    import ctypes as C

    import torch
    from parmoon_cmg_b200 import mesh
    from parmoon_cmg_b200.system import GALERKIN, SUPG, Context, TSystemCD3D, coeffs, solver_params

    dev = local
    torch.cuda.set_device(dev)
    ctx = Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    n0 = args.n // 2 ** (args.levels - 1)
    spaces, parents = mesh.structured_hierarchy(3, 2, n0, args.levels)
    # the finest level is Galerkin (delta unused there); on the SUPG coarse-grid operators a
    # third of the reference's default SDFEM delta gives the best preconditioner (30 -> 15
    # FGMRES iterations on this problem, the same for eps 1e-1 and at 16^3)
    co = coeffs(0, eps=EPS, b=B, f=1.0, delta0=1.0 / 3.0)
    # the public facade (TSystemCD3D mirror): Galerkin on the finest level, SUPG coarse-grid
    # operators (the preconditioner that converges for this convection-dominated problem)
    system = TSystemCD3D(spaces, parents, disctype=GALERKIN, ctx=ctx, coarse_disctype=SUPG)
    system.Init(co)
    mg, sids = system.mg, system.sids
    n = system.N_DOF
    nnz = system.nnz[-1]
    n_cells_total = sum(int(sp["n_cells"]) for sp in spaces)
    common = dict(coarse_smoother=17, stop_rule=1, red_factor=1e-10, res_norm_min=0.0)
    p64 = solver_params(precision=0, **common)
    pmix = solver_params(precision=1, **common)
    d_sol = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")

    def step(prm):
        ctx.assemble_hierarchy(mg, GALERKIN, SUPG)
        d_rhs = ctx.rhs_device(sids[-1])
        with torch.cuda.stream(stream):
            d_sol.zero_()  # initial guess 0 (= the Dirichlet data)
        info = ctx.solve_device(mg, prm, d_rhs, d_sol.data_ptr())
        if info.status != 0:
            raise RuntimeError(f"solve status {info.status}")
        return info

    if args.headline_only:
        for _ in range(args.warmup):
            step(pmix)
        torch.cuda.synchronize()
        l0 = ctx.kernel_launches
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        its = [step(pmix).iterations for _ in range(args.steps)]
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1), world)
        return {"metric": METRIC, "value": world * args.steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "headline_only": True, "fgmres_iterations": its[0],
                "gpu_launches": ctx.kernel_launches - l0}, ctx, None

    # accuracy of the mixed form against the FP64 form
    step(p64)
    torch.cuda.synchronize()
    x64 = d_sol.cpu().numpy().copy()
    step(pmix)
    torch.cuda.synchronize()
    xm = d_sol.cpu().numpy().copy()
    mixed_err = float(np.abs(xm - x64).max() / np.abs(x64).max())

    def timed(prm, steps, warmup):
        for _ in range(warmup):
            step(prm)
        torch.cuda.synchronize()
        barrier(world)
        l0 = ctx.kernel_launches
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        its = []
        for _ in range(steps):
            its.append(step(prm).iterations)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = ev0.elapsed_time(ev1)
        return max_over_ranks(ms, world), its, ctx.kernel_launches - l0

    n64 = max(2, args.steps // 2)
    with ClockSampler(dev) as clk:
        ms_mix, its_mix, launches = timed(pmix, args.steps, args.warmup)
        ms_64, its_64, _ = timed(p64, n64, 1)
    clocks = clk.summary()

    # assembly alone (all levels)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.assemble_hierarchy(mg, GALERKIN, SUPG)
    torch.cuda.synchronize()
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        ctx.assemble_hierarchy(mg, GALERKIN, SUPG)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_asm = e0.elapsed_time(e1) / reps

    # roofline: FP64 CSR SpMV on the finest level (192 MB of matrix, larger than the 126 MB L2)
    x = torch.rand(n, dtype=torch.float64, device=f"cuda:{dev}")
    y = torch.empty_like(x)
    for _ in range(3):
        ctx.check(ctx.lib.cdgpu_spmv_device(ctx.h, sids[-1], x.data_ptr(), y.data_ptr()))
    torch.cuda.synchronize()
    reps = 50
    e0.record(stream)
    for _ in range(reps):
        ctx.lib.cdgpu_spmv_device(ctx.h, sids[-1], x.data_ptr(), y.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = e0.elapsed_time(e1) / reps
    spmv_bytes = 12 * nnz + 4 * (n + 1) + 16 * n
    # the mixed form's FGMRES product on the same level: matrix-free FP64 (sum factorisation);
    # algorithmic bytes: per cell its 27 DOF numbers, T = 10 coefficients and its 27 products
    # written and read back, per row x and y, per active row its 8-wide incidence record
    for _ in range(3):
        ctx.check(ctx.lib.cdgpu_apply_fp64_device(ctx.h, sids[-1], 1, x.data_ptr(), y.data_ptr()))
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        ctx.lib.cdgpu_apply_fp64_device(ctx.h, sids[-1], 1, x.data_ptr(), y.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    mf_ms = e0.elapsed_time(e1) / reps
    n_cells_f, n_act_f = int(spaces[-1]["n_cells"]), int(spaces[-1]["n_active"])
    mf_bytes = n_cells_f * (4 * 27 + 8 * 10 + 2 * 8 * 27) + 16 * n + 32 * n_act_f
    tuning = ctx.product_tuning(sids[-1])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        hbm = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        hbm, peak_src = 6650.0, "fallback"
    achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of one launch of this kernel on this workload, from the ncu
    # capture summarised in profiles/
    traffic = None
    prof = os.path.join(ROOT, "profiles", "csr_tma_kernel_spmv_f64_cd3d_q2_32.md")
    if args.n == 32 and os.path.exists(prof):
        for line in open(prof):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = int(line.split(":")[1])

    # end to end through the public facade with host buffers: Assemble returns the
    # right-hand side to the host (drop-in behaviour), Solve copies rhs and initial guess in
    # and the solution out
    rhs_h = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    sol_h = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()

    def e2e_step():
        sol_h[:] = 0.0
        system.Assemble(sol_h, rhs_h)
        info = system.Solve(sol_h, rhs_h, pmix)
        if info.status != 0:
            raise RuntimeError(f"solve status {info.status}")

    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    e2e_val = world * args.steps / t_e2e

    value = world * args.steps / (ms_mix * 1e-3)
    fp64_value = world * n64 / (ms_64 * 1e-3)
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mix / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {
            "workload": f"CD3D Q2 unit cube {args.n}^3 cells, eps 1e-2, b=(1,1,1)/sqrt(3), f=1, "
                        f"Dirichlet 0, Galerkin; step = assembly of all {args.levels} multigrid levels "
                        f"+ FGMRES(30) with one V(2,2) damped-Jacobi (0.8) cycle to ||r|| <= 1e-10 ||r0||",
            "form": "mixed (FP32 multigrid, FP64 FGMRES, FP64 defect, FP64 exact coarse solve)",
            "multigrid": f"{args.levels} levels {n0}^3..{args.n}^3 Q2, SUPG coarse-grid operators "
                         f"(delta0 = 1/3), exact coarse solve",
            "n_dof": n, "nnz_finest": nnz, "l2": "inputs larger than L2 (finest matrix 192 MB)",
            "parallelism": f"replicas x{world}",
        },
        "mixed_rel_err_vs_fp64": mixed_err,
        "fgmres_iterations": {"mixed": its_mix[0], "fp64": its_64[0]},
        "fp64_form": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_64 / n64},
        "mixed_over_fp64": value / fp64_value,
        "assembly": {"ms_all_levels": ms_asm, "mcells_per_s": n_cells_total / (ms_asm * 1e-3) / 1e6},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "kernel": "csr_tma_kernel<SPMV, cap, stages> (finest level, the FGMRES matvec of the FP64 "
                               "form; matrix tiles streamed into shared memory by bulk copies; the mixed form "
                               "applies the operator matrix-free: roofline_mixed)",
                     "autotuner": tuning,
                     "peak_source": peak_src, "spmv_ms": spmv_ms, "algorithmic_bytes": spmv_bytes},
        "roofline_mixed": {"bound": "hbm", "achieved": mf_bytes / (mf_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                           "frac": mf_bytes / (mf_ms * 1e-3) / 1e9 / hbm,
                           "kernel": "mf64_cell27_kernel<10> + mf64_row_kernel (finest level, the FGMRES matvec of "
                                     "the mixed form: matrix-free FP64 by sum factorisation; in the solve its row "
                                     "phase is fused with the first Gram-Schmidt pass)",
                           "ms": mf_ms, "algorithmic_bytes": mf_bytes, "peak_source": peak_src},
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 16 * n,
                "d2h_bytes_per_step": 16 * n},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    return result, ctx, dict(x64=x64, xm=xm, space=spaces[-1])


def reference_accuracy(n, sols, tmp):
    """Checker of the cpu_baseline leg: the reference's own FP64 solution of the workload
    (oracle/_ref/cd3d_dump, 3 Galerkin levels, converged to ||r|| <= 1e-12 ||r0||) against the
    GPU arm's solutions at the timed stopping rule, matched through the DOF coordinates."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import refdump
    from parmoon_cmg_b200 import mesh
    exe = os.path.join(ROOT, "oracle", "_ref", "cd3d_dump")
    steps = int(round(np.log2(n))) - (REF_LEVELS - 1)
    dat = os.path.join(tmp, "acc.dat")
    with open(dat, "w") as f:
        f.write(DAT.format(out=os.path.join(tmp, "acc.out"), mesh=os.path.join(ROOT, "oracle", "meshes"),
                           steps=steps, levels=REF_LEVELS))
    out = os.path.join(tmp, "acc")
    os.makedirs(out, exist_ok=True)
    subprocess.run([exe, dat, out, num(EPS), *map(num, B), "0", "1", "0", "1e-12"], cwd=tmp,
                   capture_output=True, text=True, check=True)
    d = refdump.load_dir(out)
    L = refdump.level(d, int(d["levels"]) - 1)
    sp = sols["space"]
    nn = 2 * n + 1

    def key(X):
        k = np.rint(X * (nn - 1)).astype(np.int64)
        return k[:, 0] + nn * (k[:, 1] + nn * k[:, 2])
    kr = key(oracle.dof_coords(3, 2, L["coords"], L["global_numbers"], L["begin_index"], L["n_dof"]))
    ko = key(mesh.dof_coords(sp))
    inv = np.full(nn ** 3, -1, np.int64)
    inv[ko] = np.arange(len(ko))
    perm = inv[kr]
    if (perm < 0).any():
        raise RuntimeError("DOF coordinates of the reference and the GPU arm do not match")
    x_ref = np.empty(L["n_dof"])
    x_ref[perm] = d["solution"]
    scale = np.abs(x_ref).max()
    return {"mixed": float(np.abs(sols["xm"] - x_ref).max() / scale),
            "fp64": float(np.abs(sols["x64"] - x_ref).max() / scale),
            "reference_run": "oracle/_ref/cd3d_dump, 3 Galerkin levels, SSOR coarse smoother, "
                             f"||r|| <= 1e-12 ||r0|| ({int(d['iterations'])} FGMRES iterations)",
            "norm": "max |x - x_ref| / max |x_ref|"}


def run_batched(ctx, args):
    """Batched CD2D: independent instances (N log-uniform in [16, 256], Q1/Q2, eps
    log-uniform in [1e-6, 1e-1], random convection angle), all submitted at once and solved
    in grouped launches; solves/s = instances / wall time of submission (assembly of every
    level on the GPU) + solve.  A sample of instances is checked against a direct FP64
    solve of the same system."""
    from parmoon_cmg_b200 import workloads as W
    from parmoon_cmg_b200.serving import default_params
    from parmoon_cmg_b200.system import SUPG, Batch, coeffs
    import torch
    work = W.batched_cd2d(args.batched_instances)
    B = Batch(default_params(), ctx)
    cache = W.StructureCache(B)
    for w in work:
        cache.get(2, w["order"], w["n_used"])
    need = sum(B.instance_bytes(cache.get(2, w["order"], w["n_used"])[0]) for w in work)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    slots = []
    for w in work:
        sid, _ = cache.get(2, w["order"], w["n_used"])
        co = coeffs(0, eps=w["eps"], b=w["b"], f=1.0, poly_degree=w["order"])
        slots.append(B.submit(sid, co, SUPG))
    t_submit = time.perf_counter() - t0
    B.run(8)
    t_total = time.perf_counter() - t0
    loop_mode, loop_launches, host_its = B.loop_info()
    its, status = [], []
    for sl in slots:
        _, info = B.fetch(sl, 0)
        its.append(info.iterations)
        status.append(info.status)
    # accuracy on a seeded sample of the smaller instances
    rng = np.random.default_rng(7)
    small = [i for i, w in enumerate(work) if W.dofs(2, w["order"], w["n_used"]) <= 40000]
    sample = sorted(rng.choice(small, size=min(8, len(small)), replace=False).tolist())
    errs = []
    for i in (sample if not args.no_cpu_baseline else []):
        w = work[i]
        sid, n_dof = cache.get(2, w["order"], w["n_used"])
        x, _ = B.fetch(slots[i], n_dof)
        ref = fp64_solution(2, w["order"], w["n_used"], w["eps"], w["b"])
        errs.append(float(np.abs(x - ref).max() / np.abs(ref).max()))
    for sl in slots:
        B.release(sl)
    cpu = None if args.no_cpu_baseline else batched_cpu_baseline(work)
    return {
        "metric": "batched CD2D solves/s", "value": len(work) / t_total, "unit": "solves/s",
        "cpu_baseline": cpu,
        "instances": len(work), "wall_s": t_total, "submit_s": t_submit,
        "dofs_total": int(sum(W.dofs(2, w["order"], w["n_used"]) for w in work)),
        "device_bytes": int(need), "structures": len(cache.ids),
        "iteration_loop": {"mode": {1: "device (conditional CUDA graph)", 2: "device (conditional CUDA graph, "
                                    "no PDL in the body)", 0: "host"}.get(loop_mode, "none"),
                           "graph_launches": loop_launches, "host_iterations": host_its},
        "converged": int(sum(1 for st in status if st == 0)),
        "iterations": {"min": int(min(its)), "median": float(np.median(its)), "p99": float(np.percentile(its, 99)),
                       "max": int(max(its))},
        "rel_err_vs_fp64_direct": {"max": max(errs) if errs else None, "sample": len(errs),
                                   "reference": "the oracle's FP64 assembly of the instance, solved directly"},
        "config": "4096 instances, N log-uniform [16,256] (rounded to the hierarchy, recorded per instance), "
                  "Q1/Q2 50/50, eps 10^U(-6,-1), |b|=1 random angle, f=1, Dirichlet 0, SUPG; FGMRES(30) FP64 "
                  "with an FP32 V(2,2) multicolour-SSOR cycle, exact coarse solve, ||r|| <= 1e-10 ||r0||; "
                  "seed 20261203",
    }


def run_serving(ctx, args):
    """Serving stream: Poisson arrivals (70 % 2D / 30 % 3D, Q1/Q2, 1e3..2e6 DOFs, random
    coefficients) admitted under a 150 GB device budget into one running batch, at several
    arrival rates up to saturation (the same seeded requests, arrival times scaled).  At each
    rate a sample of finished requests (the first four of at most 40,000 DOFs) is compared with
    the FP64 solution of the same instance (checker of the cpu_baseline leg)."""
    from parmoon_cmg_b200 import workloads as W
    from parmoon_cmg_b200.serving import Server
    rates = [float(r) for r in args.serving_rates.split(",") if r.strip()]
    sweep = []
    for rate in rates:
        reqs = W.serving_stream(args.serving_requests, rate)
        srv = Server(ctx, budget_bytes=150 * 10 ** 9)
        srv.prepare(reqs)
        sample = []

        def keep(r):
            if args.no_cpu_baseline or len(sample) >= 4 or W.dofs(r["dim"], r["order"], r["n"]) > 40000:
                return False
            sample.append(r)
            return True
        srv.run(reqs, keep_solutions=keep)
        st = srv.stats()
        errs = []
        for r in sample:
            ref = fp64_solution(r["dim"], r["order"], r["n"], r["eps"], r["b"])
            errs.append(float(np.abs(r["solution"] - ref).max() / np.abs(ref).max()))
        st.update({"arrival_rate_per_s": rate, "requests": len(reqs),
                   "rel_err_vs_fp64": {"max": max(errs) if errs else None, "sample": len(errs)}})
        sweep.append(st)
    return {"metric": "serving solves/s and p50/p99 latency per arrival rate", "budget_bytes": 150 * 10 ** 9,
            "sweep": sweep,
            "config": "Poisson arrivals, 70% 2D / 30% 3D, Q1/Q2 50/50, DOFs 10^U(3, log10 2e6) mapped to the "
                      "nearest admissible mesh, eps 10^U(-6,-1), random unit b, f=1, Dirichlet 0, SUPG; "
                      f"{args.serving_requests} requests per rate, seed 20261204; error sample against the "
                      "oracle's FP64 assembly solved directly"}


BATCH_DAT = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_square.PRM
GEOFILE: {mesh}/unit_square.GEO
MESH_TYPE: 0
UNIFORM_STEPS: {steps}
LEVELS: {levels}
ANSATZ_ORDER: {order}
DISCTYPE: 2
SOLVER_TYPE: 1
SC_SOLVER_SCALAR: 16
SC_PRECONDITIONER_SCALAR: 5
SC_SMOOTHER_SCALAR: 3
SC_COARSE_SMOOTHER_SCALAR: 3
SC_SMOOTH_DAMP_FACTOR_SCALAR: 1.0
SC_SMOOTH_DAMP_FACTOR_FINE_SCALAR: 1.0
SC_PRE_SMOOTH_SCALAR: 2
SC_POST_SMOOTH_SCALAR: 2
SC_MG_CYCLE_SCALAR: 1
SC_STEP_LENGTH_CONTROL_ALL_SCALAR: 0
SC_STEP_LENGTH_CONTROL_FINE_SCALAR: 0
SC_GMRES_RESTART: 30
SC_LIN_RED_FACTOR_SCALAR: 1e-10
SC_LIN_RES_NORM_MIN_SCALAR: 0
SC_LIN_MAXIT_SCALAR: 300
SC_VERBOSE: 0
"""


def batched_cpu_baseline(work, sample_size=16):
    """cpu_baseline of the batched workload: the reference's own 2D multigrid FGMRES
    (oracle/_ref/cd2d_dump: TSystemCD2D assembly + TMultiGrid2D / TFgmresIte, lexicographic SSOR
    V(2,2), SSOR coarse smoother) on a seeded sample of the instances whose mesh the reference's
    unit-square refinement produces (N a power of two), one process per host core; solves/s =
    sample / wall time of the concurrent runs."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cd2d_dump")
    if not os.path.exists(exe):
        return {"value": None, "sample": "unavailable: oracle/_ref/cd2d_dump not built"}
    rng = np.random.default_rng(20261206)
    pick = [i for i, w in enumerate(work) if w["n0"] in (2, 4)]
    sample = sorted(rng.choice(pick, size=min(sample_size, len(pick)), replace=False).tolist())
    cores = cpu_count()
    tmp = tempfile.mkdtemp()
    try:
        cmds = []
        for k, i in enumerate(sample):
            w = work[i]
            dat = os.path.join(tmp, f"b{k}.dat")
            with open(dat, "w") as f:
                f.write(BATCH_DAT.format(out=os.path.join(tmp, f"b{k}.out"), mesh=os.path.join(ROOT, "oracle", "meshes"),
                                         steps=int(round(np.log2(w["n0"]))), levels=w["levels"], order=w["order"]))
            cmds.append([exe, dat, "-", "0", num(w["eps"]), num(w["b"][0]), num(w["b"][1]), "0", "1"])
        t0 = time.perf_counter()
        running, outs = [], []
        pending = list(cmds)
        while pending or running:
            while pending and len(running) < cores:
                running.append(subprocess.Popen(pending.pop(0), cwd=tmp, stdout=subprocess.PIPE,
                                                stderr=subprocess.DEVNULL, text=True))
            p = running.pop(0)
            outs.append(json.loads([l for l in p.communicate()[0].splitlines() if l.startswith("{")][-1]))
        wall = time.perf_counter() - t0
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    its = [o["iterations"] for o in outs]
    return {"value": len(sample) / wall, "unit": "solves/s", "cores": min(cores, len(sample)), "kind": "reference",
            "sample": f"{len(sample)} seeded instances with N a power of two (N = {sorted(set(work[i]['n_used'] for i in sample))}), "
                      f"one reference process per core, wall {wall:.1f} s including mesh and structure set-up",
            "iterations": {"median": float(np.median(its)), "max": int(max(its)),
                           "at_maxit_300": int(sum(1 for x in its if x >= 300))}}


def fp64_solution(dim, order, n, eps, b):
    """Checker of the cpu_baseline leg: the FP64 solution of one instance (unit square / cube,
    n^dim cells, SUPG with the instance's polynomial degree) from the oracle's assembly
    (oracle/cdoracle.c, pinned to the reference's fixtures), solved by a direct sparse solve."""
    import scipy.sparse as sps
    import scipy.sparse.linalg as spl
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from parmoon_cmg_b200 import mesh
    sp = mesh.structured_space(dim, order, n)
    rp, kc = oracle.pattern(sp["global_numbers"], sp["begin_index"], sp["n_dof"], sp["n_active"])
    co = oracle.coeffs(0, eps=eps, b=tuple(b), f=1.0, order_pd=order)
    ent, rhs = oracle.assemble(dim, order, 2, sp["coords"], sp["global_numbers"], sp["begin_index"],
                               sp["n_dof"], sp["n_active"], rp, kc, co)
    A = sps.csr_matrix((ent, kc, rp), shape=(sp["n_dof"],) * 2)
    return spl.spsolve(A.tocsc(), rhs)


DAT2D = """VERSION: 1
LOGFILE: logfile
OUTFILE: {out}
BNDFILE: {mesh}/unit_square.PRM
GEOFILE: {mesh}/unit_square.GEO
MESH_TYPE: 0
UNIFORM_STEPS: {steps}
LEVELS: {levels}
ANSATZ_ORDER: 1
DISCTYPE: 2
""" + DAT[DAT.index("SOLVER_TYPE"):]


def run_cd2d(ctx, args):
    """CD2D plain FP64: unit square 64 x 64 Q1, eps 1e-3, b = (1, 0.5), f = 1, Dirichlet 0,
    SUPG with the reference's delta; assemble every level + FGMRES(30) with a 5-level V(2,2)
    damped-Jacobi (0.8) cycle to the reference's relative residual 1e-10 (its own stopping
    rule), every level and the cycle in FP64.  Inputs resident on the device, CUDA events;
    the compiled reference solves the same problem on one host core."""
    import torch
    from parmoon_cmg_b200 import mesh
    from parmoon_cmg_b200.system import SUPG, TSystemCD2D, coeffs, solver_params
    spaces, parents = mesh.structured_hierarchy(2, 1, 4, 5)
    S = TSystemCD2D(spaces, parents, disctype=SUPG, ctx=ctx)
    S.Init(coeffs(0, eps=1e-3, b=(1.0, 0.5), f=1.0))
    prm = solver_params(precision=0, coarse_smoother=17, stop_rule=0, red_factor=1e-10)
    n = S.N_DOF
    d_sol = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream, device=d_sol.device)

    def step():
        ctx.assemble_hierarchy(S.mg, SUPG, SUPG)
        d_rhs = ctx.rhs_device(S.sids[-1])
        with torch.cuda.stream(stream):
            d_sol.zero_()
        info = ctx.solve_device(S.mg, prm, d_rhs, d_sol.data_ptr())
        if info.status != 0:
            raise RuntimeError(f"cd2d solve status {info.status}")
        return info
    for _ in range(max(3, args.warmup)):
        step()
    reps = 20
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        info = step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    out = {"metric": "CD2D plain FP64 solves/s", "value": 1e3 / ms, "unit": "solves/s", "ms_per_solve": ms,
           "n_dof": n, "fgmres_iterations": info.iterations, "form": "FP64 (drop-in)",
           "config": "unit square 64x64 Q1, eps 1e-3, b=(1,0.5), f=1, Dirichlet 0, SUPG (reference delta); "
                     "5 levels 4^2..64^2, FGMRES(30), V(2,2) damped Jacobi 0.8, rel. residual 1e-10"}
    exe = os.path.join(ROOT, "oracle", "_ref", "cd2d_dump")
    if not args.no_cpu_baseline and os.path.exists(exe):
        tmp = tempfile.mkdtemp()
        try:
            dat = os.path.join(tmp, "c1.dat")
            with open(dat, "w") as f:
                f.write(DAT2D.format(out=os.path.join(tmp, "c1.out"), mesh=os.path.join(ROOT, "oracle", "meshes"),
                                     steps=2, levels=5))
            times = []
            for _ in range(5):
                p = subprocess.run([exe, dat, "-", "0", "1e-3", "1.0", "0.5", "0", "1"], cwd=tmp,
                                   capture_output=True, text=True, check=True)
                t = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][-1])
                times.append(t["t_assemble"] + t["t_solve"])
            out["cpu_baseline"] = {"value": 1.0 / float(np.median(times)), "unit": "solves/s", "cores": 1,
                                   "kind": "reference", "iterations": t["iterations"],
                                   "sample": "median of 5 assemble+solve runs of the same problem by the reference"}
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "sample": f"unavailable: {e}"}
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
    return out


def run_general_assembly(ctx, args):
    """Assembly on the general path (local matrices by FP64 Gauss quadrature, as for any
    example whose BilinearCoeffs vary in space): CD3D Q2 at 32^3 cells, Galerkin, coefficients
    tabulated at the quadrature points (eps 1e-2, b = (0.5 - y, x - 0.5, 0.25), c = 0, f = 1).
    One step = the finest level's local matrices + the row gather into CSR (f64 + f32 entries,
    rhs); device time with CUDA events on the library's stream, the inputs in HBM."""
    import torch
    from parmoon_cmg_b200 import _lib, mesh
    from parmoon_cmg_b200.system import GALERKIN, coeffs
    spaces, _ = mesh.structured_hierarchy(3, 2, args.n, 1)
    sp = spaces[0]
    n_cells = len(sp["begin_index"]) - 1
    sid = ctx.upload_space(sp)
    ctx.build_pattern(sid)
    xq = ctx.quadrature_points(sid, n_cells, 3)
    tab = np.zeros(xq.shape[:-1] + (6,))
    tab[..., 0] = 1e-2
    tab[..., 1] = 0.5 - xq[..., 1]
    tab[..., 2] = xq[..., 0] - 0.5
    tab[..., 3] = 0.25
    tab[..., 5] = 1.0
    ctx.set_coeffs(sid, coeffs(_lib.COEFF_TABLE), tab)
    mg = ctx.hierarchy([sid], [None])
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", torch.cuda.current_device()))
    for _ in range(max(3, args.warmup)):
        ctx.assemble_hierarchy(mg, GALERKIN, GALERKIN)
    torch.cuda.synchronize()
    reps = 10
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ctx.assemble_hierarchy(mg, GALERKIN, GALERKIN)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nq, nbf = xq.shape[1], 27
    # algorithmic FP64 work of the local matrices: per cell, quadrature point and entry the
    # diffusion (3 + 3 products and sums), convection and reaction terms (~20 flops)
    flops = n_cells * nq * (nbf * nbf + nbf) * 20.0
    return {"metric": "general-path assembly (CD3D Q2, tabulated coefficients) cells/s",
            "value": n_cells / (ms * 1e-3), "unit": "cells/s", "ms_per_assembly": ms, "n_cells": n_cells,
            "quadrature_points": nq, "fp64_gflops_local_matrices": flops / (ms * 1e-3) / 1e9,
            "config": f"{args.n}^3 Q2 hexahedra, Galerkin, coefficient table per quadrature point, "
                      "finest level only (local matrices + CSR row gather)"}


def run_tcd(ctx, args):
    """Time-dependent CD2D: instances of 128^2 Q2 on the unit square, Crank-Nicolson with
    tau = 1e-3, rotating convection b = (0.5 - y, x - 0.5), eps log-uniform in [1e-5, 1e-2]
    (seeded), f = 0, Dirichlet 0, initial Gaussian bump (sigma 0.05 at (0.3, 0.3)).  Every
    step of every instance: right-hand side + multigrid FGMRES from the previous solution;
    one CUDA graph per step.  The mixed batch (FP32 multigrid) is compared at the final
    time with the FP64 single-instance form on instance 0."""
    import math
    import torch
    from parmoon_cmg_b200 import mesh
    from parmoon_cmg_b200 import workloads as W
    from parmoon_cmg_b200.system import Batch, TSystemTCD2D, coeffs, solver_params
    from parmoon_cmg_b200 import _lib
    tau, th = 1e-3, (0.5, 0.5, 0.5, 0.5)
    L, n0, n = W.hierarchy_shape(128)
    spaces, parents = mesh.structured_hierarchy(2, 2, n0, L)
    xy = mesh.dof_coords(spaces[-1])
    u0 = np.exp(-((xy[:, 0] - 0.3) ** 2 + (xy[:, 1] - 0.3) ** 2) / (2 * 0.05 ** 2))
    rng = np.random.default_rng(20261205)
    eps = [10.0 ** rng.uniform(-5, -2) for _ in range(args.tcd_instances)]
    prm = solver_params(smoother=1, omega=0.8, pre=2, post=2, stop_rule=1, red_factor=1e-10, restart=30, maxit=500)
    B = Batch(prm, ctx)
    sid = B.add_structure(spaces, parents)
    slots = [B.submit_tcd(sid, coeffs(_lib.COEFF_ROTATING, eps=e, f=0.0), tau, *th, u0) for e in eps]
    nd = spaces[-1]["n_dof"]
    B.tcd_step(8)  # first step: graph capture
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = []
    for _ in range(args.tcd_steps - 1):
        its.append(B.tcd_step(8))
    t_steps = time.perf_counter() - t0
    x_mixed, _ = B.fetch(slots[0], nd)
    for sl in slots:
        B.release(sl)
    # FP64 reference trajectory of instance 0 (single-instance theta-scheme system)
    S = TSystemTCD2D(spaces, parents, ctx=ctx)
    S.Init(coeffs(_lib.COEFF_ROTATING, eps=eps[0], f=0.0))
    sol = u0.copy()
    S.AssembleMRhs(sol)
    S.AssembleARhs()
    p64 = solver_params(precision=0, stop_rule=1, red_factor=1e-10, restart=30, maxit=500)
    for _ in range(args.tcd_steps):
        S.Step(sol, tau, *th, params=p64)
    err = float(np.abs(x_mixed - sol).max() / np.abs(sol).max())
    steps_timed = args.tcd_steps - 1
    return {
        "metric": "time-dependent CD2D instance-steps/s", "value": len(slots) * steps_timed / t_steps,
        "unit": "instance-steps/s", "instances": len(slots), "steps": args.tcd_steps,
        "ms_per_step_all_instances": 1e3 * t_steps / steps_timed, "n_dof_per_instance": int(nd),
        "iterations_per_step_max": {"median": float(np.median(its)), "max": int(max(its))},
        "mixed_vs_fp64_rel_err_final": err,
        "config": f"{len(slots)} x 128^2 Q2 (66,049 DOFs), Crank-Nicolson tau 1e-3, rotating b, eps 10^U(-5,-2) "
                  f"seed 20261205, f=0, Gaussian bump u0; FP32 V(2,2) Jacobi cycle in FP64 FGMRES per step, "
                  f"||r|| <= 1e-10 ||r0|| per step; one CUDA graph per step",
    }


def main():
    args = parse()
    rank, world, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world)
            return
        result, ctx, sols = run_ours(args, rank, world, local)
        if args.headline_only:
            if rank == 0:
                print(json.dumps(result), flush=True)
            ctx.close()
            return
        if not args.no_cd2d:
            result["cd2d"] = run_cd2d(ctx, args)
        if not args.no_batched:
            result["batched"] = run_batched(ctx, args)
        if not args.no_serving:
            result["serving"] = run_serving(ctx, args)
        if not args.no_tcd:
            result["tcd"] = run_tcd(ctx, args)
        if not args.no_general:
            result["general_assembly"] = run_general_assembly(ctx, args)
        if rank == 0:
            if not args.no_cpu_baseline:
                tmp = tempfile.mkdtemp()
                try:
                    t = reference_run(args.n, REF_LEVELS, tmp)
                    tt = t["t_assemble"] + t["t_solve"]
                    result["cpu_baseline"] = {
                        "value": 1.0 / tt, "unit": UNIT, "cores": 1, "kind": "reference",
                        "sample": f"one full assemble+solve of the same workload by the reference "
                                  f"(assemble {t['t_assemble']:.2f} s, solve {t['t_solve']:.2f} s, "
                                  f"{t['iterations']} FGMRES iterations), single-threaded"}
                except Exception as e:  # the product run stays valid without the baseline
                    result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                                              "sample": f"unavailable: {e}"}
                try:
                    result["rel_err_vs_reference"] = reference_accuracy(args.n, sols, tmp)
                except Exception as e:
                    result["rel_err_vs_reference"] = {"unavailable": str(e)}
                finally:
                    shutil.rmtree(tmp, ignore_errors=True)
            print(json.dumps(result), flush=True)
        ctx.close()
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the solve path: one step = FEModel.assembleStep + LinearSolver.solve of the
lidded FCBGA workload (160 x 160 x 32 elements, 8-2-8 layered substrate, ~2.07M DOF) to a
relative residual of 1e-8, with a fresh multigrid preconditioner every step (as the tool's
thermal path does) and no warm start (every step solves the same synthetic step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision mixed|fp64]

Metric: MDOF*iter/s = DOF x PCG iterations / step seconds / 1e6 (higher is better), whole
job over all ranks; the solve seconds and iterations are in the JSON line too.
`value` times device-resident inputs (device assembly + tm_solve_device); `e2e` goes through
the public host API (tm_assemble_step returning the load to the host, tm_solve with host
buffers), host<->device copies inside the timed region.
Multi-GPU: replicas only (each rank solves its own copy; the path has no exchange step).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "packaging-tm-modeling-tool_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "PCG-MG solve s & MDOF·iter/s, mixed vs FP64 GPU at ≤1e-6 warpage err; HBM GB/s"
UNIT = "MDOF·iter/s"
WORKLOAD = "lidded_c2 160x160x32 (8-2-8 layered substrate, die, TIM, Cu hat lid), 150->25 degC step, tol 1e-8"
DOMINANT = "sweep_solid"   # the level-0 z-column smoother: the largest bandwidth-bound share of the ncu launch list


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["mixed", "fp64"], help="default: mixed (c2), fp64 (c1)")
    ap.add_argument("--inplane", type=int, default=160)
    ap.add_argument("--level0", default="stencil", choices=["stencil", "mf"],
                    help="level-0 operator: the assembled 27-point stencil (default) or matrix-free cell products")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="a warm-up assemble + solve, then one assemble + solve (for ncu captures); prints no bench line")
    ap.add_argument("--workload", default="c2", choices=["c2", "c1", "screen", "c3", "tornado", "c4", "analysis"],
                    help="c2: the lidded 160x160x32 solve (the headline); c1: the plain FP64 FCBGA 48x48x20 solve; "
                         "screen: Anand screening of the 17,424 bumps of a die over three -40/125 degC cycles; "
                         "c3: the stacked-module thermal-cycle analysis (module stage, process chain, cycling branches, "
                         "bump strain tables, Anand screening at 40 load steps per cycle), about 1.2M DOF; "
                         "tornado: the 24 perturbed-material cases of the c2 package in one warm-started solve loop; "
                         "c4: 64 bump submodels of 20^3-48^3 voxels in one batch over the first history points of a "
                         "40-step -40/125 degC cycle; analysis: every step of the full thermal path of the tool's "
                         "default package at Standard (the reference's 'Full Standard analysis')")
    ap.add_argument("--c4-cells", type=int, default=64, help="c4: submodels in the batch")
    ap.add_argument("--c4-points", type=int, default=1, help="c4: history points of the timed sample")
    ap.add_argument("--c4-precond", default="line", choices=["line", "ic"], help="c4: inner-solve preconditioner")
    ap.add_argument("--sites", type=int, default=17424, help="screen: bump sites")
    a = ap.parse_args()
    a.precision_default = a.precision is None
    if a.precision is None:
        a.precision = "mixed"
    return a


def run_profile(a):
    """The smallest run of the hot path for ncu: model creation, then two steps of one assembly and
    one solve each. The first step builds what a hierarchy builds once (the launch-shape tuning, the
    captured V-cycle); the second is the step the launch list summarises (from its k_assemble on)."""
    import torch
    from tmsolve.solver import DeviceModel
    torch.cuda.set_device(0)
    pkg = make_package(a.workload, a.inplane)
    dm = DeviceModel(pkg)
    dm.set_level0(a.level0 == "mf")
    f = torch.empty(dm.ndof, dtype=torch.float64, device="cuda")
    u = torch.empty(dm.ndof, dtype=torch.float64, device="cuda")
    for key in (1, 2):
        dm.assemble_step_device(pkg.step(), f.data_ptr())
        r = dm.solve_device(f.data_ptr(), u.data_ptr(), tol=1e-8, warm=0, key=key, precision=a.precision)
    torch.cuda.synchronize()
    print(json.dumps({"profile": True, "dof": dm.ndof, "iters": r["iters"], "converged": r["converged"], "ms": r["ms"]}))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---- clocks during the timed region -------------------------------------------------------------
class Clocks:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if len(r) > 3]
        mx = max(float(r[2]) for r in rows if len(r) > 3)
        pw = [float(r[3]) for r in rows if len(r) > 3]
        load = [s for s, p in zip(sm, pw) if p > 0.5 * max(pw)] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ---- CPU: the oracle port of the reference's solve path --------------------------------------------
_CPU = {}


def make_package(workload, inplane):
    from tmsolve.packages import fcbga_c1, lidded_c2
    return fcbga_c1() if workload == "c1" else lidded_c2(n_inplane=inplane)


def cpu_init(workload, inplane):
    """Worker set-up (untimed): the package and the oracle's FEModel + LinearSolver of the workload."""
    for p in (ROOT, PKG):
        if p not in sys.path:
            sys.path.insert(0, p)
    from oracle import oracle
    pkg = make_package(workload, inplane)
    _CPU.update(pkg=pkg, om=oracle.OracleModel(pkg), key=0)


def cpu_step(_=None):
    """One step of the workload on one core, as the GPU arm's step: assembleStep + a complete
    MG-PCG solve to relres 1e-8 with a fresh multigrid set-up and no warm start."""
    om, pkg = _CPU["om"], _CPU["pkg"]
    _CPU["key"] += 1
    om.clear_warm()
    t0 = time.perf_counter()
    f = om.assemble(pkg.step())
    r = om.solve(f, tol=1e-8, key=_CPU["key"])
    dt = time.perf_counter() - t0
    return om.ndof, r["iters"], dt, r["converged"]


def reference_procs():
    n = os.cpu_count() or 1
    try:
        import psutil
        mem = psutil.virtual_memory().available / 5e9   # about 4 GB per worker on this workload
    except Exception:
        mem = 8
    return max(1, min(n, int(mem), 16))


def run_reference(a):
    """The reference is JavaScript with no engine on the image: its solve path as the C++ FP64 port
    (oracle/), each step one complete single-thread solve, the steps farmed out to a pool of worker
    processes as the tool's runSweep farms thermal-path steps (src/worker.js:111-133)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from oracle import oracle
    oracle.build()
    procs = min(reference_procs(), max(1, a.steps))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=cpu_init, initargs=(a.workload, a.inplane)) as pool:
        pool.map(cpu_step, range(max(1, min(a.warmup, procs))), chunksize=1)
        t0 = time.perf_counter()
        res = pool.map(cpu_step, range(a.steps), chunksize=1)
        dt = time.perf_counter() - t0
    n = res[0][0]
    iters = sum(r[1] for r in res)
    val = n * iters / 1e6 / dt
    conv = all(r[3] for r in res)
    sample = (f"{a.steps} steps over {procs} worker processes (one single-thread step per worker at a time, as the tool's "
              f"runSweep farms steps out); each step assembleStep + a complete MG-PCG solve of the {n}-DOF workload to "
              f"relres 1e-8 with a fresh multigrid set-up ({iters} PCG iterations summed, "
              f"{'all converged' if conv else 'NOT all converged'}, {sum(r[2] for r in res) / len(res):.1f} s per step)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * dt / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "dof": n, "precision": "fp64", "l2": "inputs larger than L2"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is JavaScript with no engine on this image; the C++ FP64 port of its solve path (oracle/) is timed"}))


# ---- GPU -----------------------------------------------------------------------------------------
def over_ranks(secs, work, device):
    """Whole-job figures of the replicas: the slowest rank's seconds and all ranks' work (MAX and
    SUM over the process group; a rank's own figures when it runs alone)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(secs), float(work)
    t = torch.tensor([secs, work], dtype=torch.float64, device=device)
    tmax = t[:1].clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    wsum = t[1:].clone()
    dist.all_reduce(wsum, op=dist.ReduceOp.SUM)
    return float(tmax), float(wsum)


def run_ours(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        from oracle import oracle
        oracle.build()
        cpu_init(a.workload, a.inplane)
        nd, it, dt, conv = cpu_step()
        _CPU.clear()
        cpu = {"value": nd * it / 1e6 / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"one step of the {nd}-DOF workload on one core: assembleStep + a complete MG-PCG solve to relres 1e-8 "
                         f"with a fresh multigrid set-up, {it} PCG iterations ({'converged' if conv else 'NOT converged'}, {dt:.1f} s)"}
    import numpy as np
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from tmsolve.packages import rms_warpage
    from tmsolve.solver import DeviceModel, launch_count
    pkg = make_package(a.workload, a.inplane)
    dm = DeviceModel(pkg)
    dm.set_level0(a.level0 == "mf")
    stream = torch.cuda.current_stream()
    dm.set_stream(stream.cuda_stream)
    n = dm.ndof
    step = pkg.step()
    f = torch.empty(n, dtype=torch.float64, device="cuda")
    u = torch.empty(n, dtype=torch.float64, device="cuda")
    u64 = torch.empty(n, dtype=torch.float64, device="cuda")
    key = [0]

    def one(precision, uu):
        key[0] += 1
        dm.assemble_step_device(step, f.data_ptr())
        return dm.solve_device(f.data_ptr(), uu.data_ptr(), tol=1e-8, warm=0, key=key[0], precision=precision)

    for _ in range(a.warmup):
        one(a.precision, u)
    # accuracy of the timed precision against the FP64 GPU solve of the same step
    r64 = one("fp64", u64)
    torch.cuda.synchronize()
    w64 = rms_warpage(pkg.mesh, u64.cpu().numpy())
    # ---- timed region (device-resident inputs)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = launch_count()
    recs = []
    with Clocks(local) as ck:
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            recs.append(one(a.precision, u))
        e1.record(stream)
        torch.cuda.synchronize()
    launches = launch_count() - l0
    ms = e0.elapsed_time(e1)
    # launch durations of the dominant kernel: events around each of its launches, in one more
    # step outside the timed region (the events would otherwise add to the step time)
    dm.time_kernel(DOMINANT)
    one(a.precision, u)
    torch.cuda.synchronize()
    kcount, kms = dm.kernel_time()
    dm.time_kernel(None)
    # and of the shell-level column sweeps (all shell levels; FP32 cycle only)
    shell = None
    if a.precision == "mixed" and not dm.level0_matrix_free:
        dm.time_kernel("sweep_shell")
        one(a.precision, u)
        torch.cuda.synchronize()
        scount, sms = dm.kernel_time()
        dm.time_kernel(None)
        sbytes, spc = dm.shell_sweep_bytes()
        if scount and spc:
            cycles = scount / spc
            shell = {"kernel": "k_sweep_shell<float> (shell-level z-column sweeps, warp per column, all levels)",
                     "bound": "latency (dependent loads per column; bandwidth figure for reference)",
                     "achieved": sbytes * cycles / (sms / 1e3) / 1e9, "unit": "GB/s",
                     "algorithmic_bytes_per_cycle": sbytes, "launches_per_cycle": spc, "launches_timed": scount,
                     "avg_launch_us": 1e3 * sms / scount}
    clocks = ck.summary()
    wmix = rms_warpage(pkg.mesh, u.cpu().numpy())
    iters = sum(r["iters"] for r in recs)
    work = n * iters / 1e6
    secs, work_all = over_ranks(ms / 1e3, work, "cuda")
    value = work_all / secs
    # ---- end to end through the host API (pinned host buffers)
    fh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    uh = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True); e3 = torch.cuda.Event(enable_timing=True)
    e2_iters = 0
    e2.record(stream)
    for _ in range(a.steps):
        key[0] += 1
        dm.assemble_step(step, out=fh)
        r = dm.solve(fh, key=key[0], tol=1e-8, warm=0, precision=a.precision, out=uh)
        e2_iters += r["iters"]
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_s = e2.elapsed_time(e3) / 1e3
    e2e_secs, e2e_work = over_ranks(e2e_s, n * e2_iters / 1e6, "cuda")
    e2e_val = e2e_work / e2e_secs
    step_bytes = sum(getattr(step, k).nbytes for k in ("layered", "D", "s0", "W", "V", "born"))
    # ---- roofline of the dominant kernel: level-0 column smoother, one colour per launch
    nn = dm.nn
    prec_bytes = 4 if a.precision == "mixed" else 8
    hbm, hbm_kind = peaks()
    mf = dm.level0_matrix_free
    avg_s = kms / kcount / 1e3 if kcount else None
    if not mf:
        # per full sweep (4 colours): operator rows 243 values + 27 neighbour ids + 18 factor values + b, x read, x write per node
        sweep_bytes = nn * (243 * prec_bytes + 27 * 4 + 18 * prec_bytes + 3 * prec_bytes * 3)
        per_launch = sweep_bytes / 4
        achieved = per_launch / avg_s / 1e9 if kcount else None
        traffic = profile_traffic(DOMINANT, a.precision)
        kname = ("k_sweep_tma (level-0 z-column smoother, one colour: position-major operator rows streamed by TMA bulk copies "
                 "through shared memory, block-tridiagonal column solves per SM run)") if a.precision == "mixed" else \
            "k_sweep_panel<double> (level-0 z-column block-tridiagonal smoother on packed column panels, one colour)"
        roof = {"kernel": kname, "bound": "hbm", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm if achieved else None, "traffic": traffic,
                "peak_kind": hbm_kind, "launches_timed": kcount, "avg_launch_us": 1e3 * kms / kcount if kcount else None,
                "algorithmic_bytes_per_launch": per_launch}
    else:
        # one colour of the matrix-free sweep (k_mf_resid + k_col_solve): per colour node the class id
        # of its 8 cells (2 B each), 18 factor values, gs/os/cd, b, x read and x write (3 values each),
        # and 8 cells x 3 rows x 24 multiply-adds
        from tmsolve.solver import device_peaks
        pk = device_peaks()
        fp32, fp64 = pk["fp32_tflops"], pk["fp64_tflops"]
        per_launch = nn / 4 * (8 * 2 + 18 * prec_bytes + 6 * 3 * prec_bytes)
        flops = nn / 4 * 1152
        achieved = per_launch / avg_s / 1e9 if kcount else None
        fpeak = 1e3 * (fp32 if prec_bytes == 4 else fp64)
        roof = {"kernel": "k_mf_resid + k_col_solve (matrix-free level-0 colour sweep: residual rows from the cell-class "
                          "table, then warp-per-column block-tridiagonal solves)",
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm if achieved else None,
                "traffic": None, "peak_kind": hbm_kind, "launches_timed": kcount,
                "avg_launch_us": 1e3 * kms / kcount if kcount else None, "algorithmic_bytes_per_launch": per_launch,
                "flops_per_launch": flops, "achieved_gflops": flops / avg_s / 1e9 if kcount else None,
                "flops_peak_gflops": fpeak, "flops_frac": flops / avg_s / 1e9 / fpeak if kcount else None,
                "flops_peak_kind": "measured FMA loop (tm_device_peaks)"}
    if shell is not None:
        shell["peak"] = hbm
        shell["frac"] = shell["achieved"] / hbm
        roof["shell_sweeps"] = shell
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 apply/smoother + f64 refinement" if a.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "dof": n, "precision": a.precision, "parallelism": f"replicas x{world}",
                       "level0": "matrix-free" if mf else "stencil",
                       "l2": "inputs larger than L2 (1.3 GB level-0 operator)"},
            "solve": {"iters_per_step": iters / a.steps, "solve_s": ms / 1e3 / a.steps, "refinements": recs[-1]["refinements"],
                      "pc_ms": recs[-1]["pcMs"], "relres": recs[-1]["relres"], "fp64_iters": r64["iters"],
                      "fp64_solve_s": r64["ms"] / 1e3, "rms_warpage_mm": wmix, "rms_warpage_rel_err_vs_fp64": abs(wmix / w64 - 1)},
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(step_bytes + 8 * n), "d2h_bytes_per_step": int(16 * n)},
            "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
        }
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def profile_traffic(kernel, precision):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, or None."""
    name = "k_sweep_tma" if precision == "mixed" else "k_sweep_panel"
    path = os.path.join(ROOT, "profiles", f"{name}_{precision}.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ---- Anand screening ------------------------------------------------------------------------------
SCREEN_METRIC = "Anand screening throughput: bump sites x time steps per second (screenJoints, FP64 return map)"
SCREEN_UNIT = "Msite-steps/s"


def screen_inputs(nsites):
    from tmsolve.anand import cycle_history, cycling_temps, synthetic_strain_table
    from tmsolve.materials import SAC305_MODULE, anand_tables
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3)      # 15-min ramps (11 degC/min) and dwells, 3 cycles
    temps = cycling_temps(-40.0, 125.0)
    table, _, _ = synthetic_strain_table(nsites, temps, die_half=12.5)
    Et, Ft = anand_tables(SAC305_MODULE)
    return hist, temps, table, Et, Ft


def run_screen(a):
    """Anand screening of one die's bumps: every site runs the whole three-cycle history (its table
    of strains at the cycling temperatures interpolated per time step, the in-plane Newton, the FP64
    return map) and reports the last cycle's dW and dE."""
    import ctypes as C
    import numpy as np
    import torch
    from oracle import oracle
    from tmsolve._lib import check, load
    from tmsolve.anand import material
    from tmsolve.materials import SAC305_MODULE, anand_params_array
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    hist, temps, table, Et, Ft = screen_inputs(a.sites)
    ns, nt, nsteps = a.sites, len(temps), len(hist["t"])
    unit_work = ns * nsteps / 1e6
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        oracle.build()
        sample = min(ns, 512)
        t0 = time.perf_counter()
        oracle.anand_screen(anand_params_array(SAC305_MODULE), Et, Ft, temps, table[:sample].ravel(), hist)
        dt = time.perf_counter() - t0
        cpu = {"value": sample * nsteps / 1e6 / dt, "unit": SCREEN_UNIT, "cores": 1, "kind": "port",
               "sample": f"the first {sample} of the {ns} sites, all {nsteps} time steps, on one core ({dt:.1f} s)"}
    torch.cuda.set_device(local)
    m, keep = material(SAC305_MODULE, Et, Ft)
    vp = lambda x: x.ctypes.data_as(C.c_void_p)
    t = np.ascontiguousarray(hist["t"]); T = np.ascontiguousarray(hist["T"])
    cyc = np.ascontiguousarray(hist["cycle"], np.int32); ph = np.ascontiguousarray(hist["phase"], np.int32)
    temps = np.ascontiguousarray(temps)
    d_table = torch.from_numpy(np.ascontiguousarray(table).ravel()).cuda()
    d_out = torch.empty(3, ns, dtype=torch.float64, device="cuda")
    L = load()

    def dev_run():
        check(L.tm_anand_screen_device(C.byref(m), ns, nt, vp(temps), C.c_void_p(d_table.data_ptr()), nsteps, vp(t), vp(T), vp(cyc),
                                       vp(ph), int(hist["cycles"]), C.c_void_p(d_out[0].data_ptr()), C.c_void_p(d_out[1].data_ptr()),
                                       C.c_void_p(d_out[2].data_ptr())))
    for _ in range(a.warmup):
        dev_run()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as ck:
        e0.record(stream)
        for _ in range(a.steps):
            dev_run()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    # end to end: the host API with host arrays (table in, dW/dE/stab out)
    hW = np.zeros(ns); hE = np.zeros(ns); hS = np.zeros(ns)
    tab = np.ascontiguousarray(table).ravel()
    e0.record(stream)
    for _ in range(a.steps):
        check(L.tm_anand_screen(C.byref(m), ns, nt, vp(temps), vp(tab), nsteps, vp(t), vp(T), vp(cyc), vp(ph), int(hist["cycles"]),
                                vp(hW), vp(hE), vp(hS)))
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / a.steps
    # accuracy against the oracle on a sample of sites
    dW = d_out[0].cpu().numpy()
    sample = np.arange(0, ns, max(1, ns // 64))
    oW, _, _ = oracle.anand_screen(anand_params_array(SAC305_MODULE), Et, Ft, temps, table[sample].ravel(), hist)
    err = float(np.max(np.abs(dW[sample] / oW - 1)))
    if rank == 0:
        print(json.dumps({
            "metric": SCREEN_METRIC, "value": unit_work / (ms / 1e3), "unit": SCREEN_UNIT, "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"Anand screening, {ns} bump sites (132 x 132 grid over a 25 mm die), SAC305 module constants, "
                                   f"3 cycles -40/125 degC, 15-min ramps and dwells, {nsteps} time steps",
                       "sites": ns, "time_steps": nsteps, "l2": "inputs smaller than L2: the kernel is bound by FP64 arithmetic"},
            "screen": {"seconds_per_screening": ms / 1e3, "reference_published_s": 15.0,
                       "dW_max_rel_err_vs_oracle_64_sites": err, "dW_mean_mj_per_mm3": float(np.nanmean(dW))},
            "e2e": {"value": unit_work / (ms_e2e / 1e3), "unit": SCREEN_UNIT, "h2d_bytes_per_step": int(tab.nbytes),
                    "d2h_bytes_per_step": int(3 * 8 * ns)},
            "cpu_baseline": cpu, "clocks": ck.summary()}))


# ---- stacked-module thermal-cycle analysis ----------------------------------------------------------
C3_METRIC = "stacked-module thermal-cycle analysis (module stage + process chain + cycling branches + bump strain tables + Anand screening)"


def run_c3(a):
    """One analysis = every step of the module's thermal path solved on the device (module stage -1,
    stage 0 from the attach temperature to 25 degC, the cycling branches through the sample
    temperatures), the bump-layer strain table at the screened die bump sites from the steps' float32
    increments, and the Anand screening of those sites over three -40/125 degC cycles at 40 load steps
    per cycle. Timed end to end (host API), device and host work included."""
    import numpy as np
    import torch
    from tmsolve import post
    from tmsolve.anand import cycle_history, cycling_temps, screen
    from tmsolve.materials import SAC305_MODULE, anand_tables
    from tmsolve.packages import module_path_steps, stacked_module
    from tmsolve.solver import DeviceModel
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    n_in = a.inplane if a.inplane != 160 else 192
    pkg = stacked_module(n_in)
    temps = cycling_temps(-40.0, 125.0)
    steps, Tb, chain, up, down = module_path_steps(pkg, temps=temps)
    sites = post.screening_sites(post.bump_field(**pkg.meta["die"]))["sites"]
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3, ramp_max_dt=10.0, dwell_steps=3)
    Et, Ft = anand_tables(SAC305_MODULE)
    bl = pkg.meta["bump_layer"]
    dm = DeviceModel(pkg)

    def analysis(key0):
        t0 = time.perf_counter()
        du, its = [], 0
        for k, st in enumerate(steps):
            r = dm.solve(dm.assemble_step(st), tol=1e-8, key=key0 + k, precision=a.precision)
            du.append(r["u"].astype(np.float32).astype(np.float64))
            its += r["iters"]
        t1 = time.perf_counter()
        table = post.site_strain_table(dm, post.ThermalPath(steps, Tb, du, chain, up, down), sites, temps, bl["zmid"], bl["part"])
        t2 = time.perf_counter()
        dW, dE, stab = screen(SAC305_MODULE, Et, Ft, temps, table, hist)
        t3 = time.perf_counter()
        return dict(solve_s=t1 - t0, table_s=t2 - t1, screen_s=t3 - t2, total_s=t3 - t0, iters=its, dW=dW)
    for w in range(a.warmup):
        analysis(1000 * (w + 1))
    torch.cuda.synchronize()
    with Clocks(local) as ck:
        runs = [analysis(100000 * (q + 1)) for q in range(a.steps)]
    tot = sum(r["total_s"] for r in runs) / a.steps
    last = runs[-1]
    n = dm.ndof
    print(json.dumps({
        "metric": C3_METRIC, "value": tot, "unit": "s per analysis", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * tot, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply/smoother + f64 refinement; f64 return map" if a.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"stacked module {n_in}x{n_in}x15 ({n} DOF), {len(steps)} path steps (module stage, "
                               f"{len(chain) - 1} chain steps, {len(up)}+{len(down)} cycling steps), {len(sites['x'])} screened bump sites, "
                               f"3 cycles -40/125 degC at 40 load steps per cycle", "dof": n, "precision": a.precision,
                   "l2": "working set larger than L2"},
        "analysis": {"solve_s": last["solve_s"], "table_s": last["table_s"], "screen_s": last["screen_s"],
                     "pcg_iters": last["iters"],
                     "solve_mdof_iter_per_s": n * last["iters"] / 1e6 / last["solve_s"] if last["iters"] else None,
                     "warm_start": "up to 20 stored solutions (WARM_START_MAX): a step whose increment is a combination of "
                                   "earlier ones is solved by the projection alone, in 0 PCG iterations",
                     "dW_mean": float(np.nanmean(last["dW"])), "dW_max": float(np.nanmax(last["dW"]))},
        "e2e": {"value": tot, "unit": "s per analysis", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "clocks": ck.summary()}))


ANALYSIS_METRIC = "full thermal-path analysis of the tool's default package (every step of buildPath solved), seconds per analysis"


def run_analysis(a):
    """The reference's 'Full Standard analysis' (its README's timing table: 611 s at 314k DOF on
    three workers): the tool's default lidded package built by the restated model-building side at
    the Standard preset (untimed, reported as build_s), then every step of its full thermal path
    (the chain, the chip-join branch, the cycling and reflow sweeps: 67 steps) assembled and solved
    through the host API from a fresh solver (no stored solutions), with the room-temperature JEITA
    warpage read at the end. Timed end to end on the host clock around device-synchronising calls."""
    import numpy as np
    import torch
    from tmsolve import post
    from tmsolve.analysis import full_path, process_package
    from tmsolve.pkgmesh import default_config
    from tmsolve.solver import DeviceModel
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    recs = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "materials_subset.json")))
    cfg = default_config()
    t0 = time.perf_counter()
    pkg = process_package(cfg, recs, "standard")
    fp = full_path(pkg, recs)
    build_s = time.perf_counter() - t0
    steps = fp["steps"]
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    dm = DeviceModel(pkg)

    def analysis():
        dm.clear_warm()
        t0 = time.perf_counter()
        u, its = np.zeros(dm.ndof), 0
        for k, (Ta, Tb, st, _) in enumerate(steps):
            r = dm.solve(dm.assemble_step(pkg.step(Ta, Tb, stage=st)), tol=1e-8, key=k, precision=a.precision)
            if not r["converged"]:
                raise RuntimeError(f"step {k} ({Ta} -> {Tb} degC) did not converge: relres {r['relres']:.2e}")
            if k in fp["chain"]:
                u += r["u"]
            its += r["iters"]
        w = post.warpage_jeita(b, lambda x, y: dm.sample_plane(u, 0, 2, x, y))
        return dict(total_s=time.perf_counter() - t0, iters=its, w=w["signed"])
    for _ in range(a.warmup):
        analysis()
    torch.cuda.synchronize()
    with Clocks(local) as ck:
        runs = [analysis() for _ in range(a.steps)]
    tot = sum(r["total_s"] for r in runs) / a.steps
    n = dm.ndof
    print(json.dumps({
        "metric": ANALYSIS_METRIC, "value": tot, "unit": "s per analysis", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * tot / len(steps), "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply/smoother + f64 refinement" if a.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"default lidded package at Standard ({n} DOF), {len(steps)} path steps, tol 1e-8, fresh solver",
                   "dof": n, "precision": a.precision, "l2": "working set larger than L2"},
        "analysis": {"build_s": build_s, "pcg_iters": runs[-1]["iters"], "rt_warpage_um": 1000 * runs[-1]["w"],
                     "reference_s": 611.0, "reference_note": "README timing table: 611 s at 314k DOF, Chromium, 3 workers"},
        "e2e": {"value": tot, "unit": "s per analysis", "h2d_bytes_per_step": 8 * n * len(steps),
                "d2h_bytes_per_step": 8 * n * len(steps)},
        "clocks": ck.summary()}))


TORNADO_METRIC = "tornado batch: base + 24 perturbed-material solves of lidded C2 (matE x6, matCTE x6 at -/+10 %), signed JEITA warpage per case"


def run_tornado(a):
    """One batch = the base case and the 24 cases of tornado_cases() on the c2 package, each assembled,
    solved to tol 1e-8 from the previous case's solution (warm start) and its JEITA warpage sampled
    (host API, end to end). The same loop with every case started from zero, as the reference's
    tornado runs its cases, is timed once beside it."""
    import torch
    from tmsolve.packages import lidded_c2
    from tmsolve.sensitivity import tornado, tornado_cases
    from tmsolve.solver import DeviceModel
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    pkg = lidded_c2(a.inplane)
    cases = tornado_cases()
    dm = DeviceModel(pkg)
    dm.set_level0(a.level0 == "mf")
    for w in range(a.warmup):
        dm.clear_warm()
        tornado(dm, cases, precision=a.precision, key=1000 * (w + 1))
    torch.cuda.synchronize()
    runs = []
    with Clocks(local) as ck:
        for q in range(a.steps):
            dm.clear_warm()
            t0 = time.perf_counter()
            res = tornado(dm, cases, precision=a.precision, key=100000 * (q + 1))
            torch.cuda.synchronize()
            runs.append((time.perf_counter() - t0, res))
    secs = sum(t for t, _ in runs) / a.steps
    res = runs[-1][1]
    # the reference's way: every case from zero (no stored solutions), the same loop otherwise
    dm.clear_warm()
    t0 = time.perf_counter()
    fresh = tornado(dm, cases, precision=a.precision, key=10000000, warm=0)
    torch.cuda.synchronize()
    cold = time.perf_counter() - t0
    cold_iters = sum(c["iters"] for c in [fresh["base"]] + fresh["cases"])
    iters = sum(c["iters"] for c in [res["base"]] + res["cases"])
    n = dm.ndof
    print(json.dumps({
        "metric": TORNADO_METRIC, "value": secs, "unit": "s per 25-solve batch", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * secs, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply/smoother + f64 refinement" if a.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"lidded_c2 {a.inplane}x{a.inplane}x32 ({n} DOF), base + 24 cases, tol 1e-8", "dof": n,
                   "precision": a.precision, "l2": "inputs larger than L2"},
        "batch": {"pcg_iters": iters, "rebuilds": sum(c["rebuilt"] for c in [res["base"]] + res["cases"]),
                  "mdof_iter_per_s": n * iters / 1e6 / secs, "base_signed_warpage_mm": res["base"]["signed"],
                  "largest_swing": max(res["swing"], key=lambda s: s["span"])},
        "cases_from_zero": {"s": cold, "pcg_iters": cold_iters, "speedup_of_warm_batch": cold / secs},
        "e2e": {"value": secs, "unit": "s per 25-solve batch", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "clocks": ck.summary()}))


C4_METRIC = "batched bump submodels (BumpSubmodel.run: B-bar voxels, Anand solder, Newton with PCG inner solves, adaptive sub-steps)"


def c4_specs(n, seed=20261203):
    """n bump cells with k x k x k voxels, k ~ U{20..48}, at sites spread over a 20 mm die (the
    joints away from the centre see more shear)."""
    import numpy as np
    from tmsolve.submodel import synthetic_spec
    rng = np.random.default_rng(seed)
    ks = rng.integers(20, 49, n)
    xy = rng.uniform(-10.0, 10.0, (n, 2))
    specs = []
    for q in range(n):
        r = float(np.hypot(*xy[q]))
        specs.append(synthetic_spec(nxy=int(ks[q]), nz=int(ks[q]), site=(float(xy[q, 0]), float(xy[q, 1])), shear=2e-6 * r,
                                    seed=seed + q))
    return specs, ks, xy


def run_c4(a):
    """The batch of --c4-cells submodels over the first --c4-points points of the 40-step cycle
    history (cycle_history with 10 degC ramp steps and 3 dwell steps), timed end to end through
    tm_submodel_run_batch. The unit of work is one voxel element through one accepted sub-step;
    the CPU baseline is the oracle's BumpSubmodel on one core for the smallest cell over the same
    points."""
    import numpy as np
    import torch
    from tmsolve.anand import cycle_history
    from tmsolve.submodel import DeviceSubmodel, run_batch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    specs, ks, xy = c4_specs(a.c4_cells)
    full = cycle_history(-40.0, 125.0, 11.0, 15.0, 1, ramp_max_dt=10.0, dwell_steps=3)
    P = min(a.c4_points + 1, len(full["t"]))
    hist = dict(t=full["t"][:P], T=full["T"][:P], cycle=full["cycle"][:P], phase=full["phase"][:P], cycles=1)
    ang = np.arctan2(xy[:, 1], xy[:, 0])
    cph, sph = np.cos(ang), np.sin(ang)

    def batch():
        models = [DeviceSubmodel(sp) for sp in specs]
        for m in models:
            m.set_precond(a.c4_precond)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        recs = run_batch(models, hist, cph, sph)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        ne = np.array([m.ne for m in models])
        for m in models:
            m.close()
        return secs, recs, ne
    for _ in range(a.warmup):
        batch()
    with Clocks(local) as ck:
        runs = [batch() for _ in range(a.steps)]
    secs = sum(r[0] for r in runs) / a.steps
    _, recs, ne = runs[-1]
    steps = np.array([r["steps"] for r in recs])
    work = float((ne * steps).sum())
    cpu = None
    if not a.no_cpu_baseline:
        import oracle.oracle as orc
        q = int(np.argmin(ks))
        t0 = time.perf_counter()
        ro = orc.OracleSubmodel(specs[q]).run(hist, float(cph[q]), float(sph[q]))
        cs = time.perf_counter() - t0
        cpu = {"value": int(ne[q]) * ro["steps"] / cs, "unit": "voxel-element sub-steps/s", "cores": 1, "kind": "port",
               "sample": f"the oracle's BumpSubmodel run of the smallest cell ({int(ks[q])}^3, {int(ne[q])} elements) over the same "
                         f"{P} history points on one core: {int(ro['steps'])} sub-steps in {cs:.1f} s"}
    print(json.dumps({
        "metric": C4_METRIC, "value": work / secs, "unit": "voxel-element sub-steps/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * secs, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(specs)} bump cells k^3 voxels, k ~ U{{20..48}} (seed 20261203, {int(ne.sum())} elements), "
                               f"first {P} points of a 40-step -40/125 degC cycle, {a.c4_precond} inner preconditioner",
                   "cells": len(specs), "elements": int(ne.sum()), "history_points": P, "precond": a.c4_precond,
                   "l2": "working set larger than L2"},
        "batch": {"s": secs, "substeps": int(steps.sum()), "max_substeps": int(steps.max()),
                  "newton_per_step_mean": float(np.mean([r["newtonPerStep"] for r in recs])),
                  "cutbacks": int(sum(r["cutbacks"] for r in recs))},
        "e2e": {"value": work / secs, "unit": "voxel-element sub-steps/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "cpu_baseline": cpu, "clocks": ck.summary()}))


def main():
    a = parse()
    if a.workload == "c4":
        run_c4(a)
        return
    if a.workload == "tornado":
        run_tornado(a)
        return
    if a.workload == "screen":
        run_screen(a)
        return
    if a.workload == "c3":
        run_c3(a)
        return
    if a.workload == "analysis":
        run_analysis(a)
        return
    if a.workload == "c1":
        global WORKLOAD
        WORKLOAD = "fcbga_c1 48x48x20 (plain FP64 linear-elastic FCBGA, 150->25 degC step), tol 1e-8"
        if a.precision_default:
            a.precision = "fp64"
    if a.profile:
        run_profile(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()

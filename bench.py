"""Benchmark of the MOSE explicit residual-and-update path on B200.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--precision exact|fp64|mixed]

Workload (one GPU): the 2-D isentropic vortex on a periodic 2048 x 2048 block,
MUSCL van Albada + HLLC, SSP-RK3, CFL 0.8, FP64; synthetic initial field of
the named shape.  A "step" is one full Explicit_Step (dt pass + 3 fused RK
stages) over the whole block.  value = cell-updates/s, one update being one
RK3 step of one cell; N GPUs run N independent replicas (weak scaling).

Precisions: value is the "fp64" path (the reference algorithm in restated
FP64 arithmetic, within 1e-12 of the reference arithmetic per step); the
reference-exact path and the mixed FP32/FP64 path are timed in the same run
under "variants"; "errors_vs_oracle" holds every precision's density error
after 100 steps against the FP64 oracle itself (run in a spawned process
beside the device-timed reports).  The line's last key, "summary", repeats
the figures a reader needs in a few hundred characters.

--impl reference times the CPU oracle (the C++/OpenMP restatement of the
reference's Fortran algorithm; the Fortran build itself cannot be compiled
without gfortran and the FLINT/ORION/FiNeR submodules) on the host cores.
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

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_CELLS_SIDE = 2048
# 8 arrays of nv = 4 doubles per cell and RK3 step: stage 1 reads P^n and
# writes P^1; stages 2 and 3 read their input and P^n and write their output
# (the fused CFL pass works on the state the last stage has just written)
BYTES_PER_CELL_STEP = 256
STAGE_BYTES_PER_CELL = (64 + 96 + 96) / 3.0   # stage 1 reads P^n, writes P^1; stages 2,3 also read P^n
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def workload_case(n=N_CELLS_SIDE, steps=100):
    from mose_b200 import cases
    return cases.isentropic_vortex(n, steps=steps, limiter="vanalbada", riemann="HLLC", cfl=0.8)


def workload_config(case, precision):
    return {"workload": f"isentropic vortex 2-D, periodic {N_CELLS_SIDE}x{N_CELLS_SIDE} block on [0,10]^2, "
                        "MUSCL van Albada + HLLC, SSP-RK3, CFL 0.8, time accurate",
            "cells": case.ncells, "precision": precision,
            "l2": "inputs larger than L2 (3 state buffers of 135 MB each, > 126 MB)"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The maximum of x over the ranks (NCCL on the GPUs, gloo on the host)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(world, cells, steps, ms):
    """Whole-job throughput: every rank advances its own replica of `cells`
    cells by `steps` steps; `ms` is the slowest rank's time."""
    return world * cells * steps / (ms / 1e3)


def fp64_ceiling(device):
    """Measured issue ceilings of FP64 FMA, IEEE division and IEEE square root
    on this GPU (mose_probe_fp64_peak, libmose_probe.so): the compute roofline of the fp64 and
    exact stage kernels, beside the HBM copy bandwidth."""
    import ctypes as C
    from mose_b200 import _lib
    lib = _lib.load_probe()
    out = np.zeros(6)
    if lib.mose_probe_fp64_peak(device, out.ctypes.data_as(C.POINTER(C.c_double))) != 0:
        return None
    return {"dfma_tflops": float(out[0]), "ddiv_g_per_s": float(out[1]), "dsqrt_g_per_s": float(out[2]),
            "method": "independent FMA / division / square-root chains per thread, 1024 threads per SM, "
                      "CUDA events around the second of two launches"}


def host_cores():
    """The host threads this process may use (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def time_oracle_build(path, case, cores, runs=5, steps_per_run=2, warmup=1):
    """One oracle build on the workload: `warmup` untimed steps, then the
    median of `runs` wall-clock runs of `steps_per_run` RK3 steps each."""
    from oracle import pyoracle
    o = pyoracle.Oracle(case, nthreads=cores, omp=True, lib_path=path)
    for _ in range(warmup):
        o.step()
    per = []
    for _ in range(runs):
        t0 = time.perf_counter()
        for _ in range(steps_per_run):
            o.step()
        per.append((time.perf_counter() - t0) / steps_per_run)
    del o
    return case.ncells / statistics.median(per), per


def cpu_baseline(runs=5, steps_per_run=2):
    """The oracle on the box's host cores, on the 2048^2 workload itself, in
    two builds made on this host: -O3 -march=native (IEEE, bit-identical to
    the serial oracle) and -O3 -march=native -ffast-math (the reference's
    RELEASE flags).  Each: one warm-up step, then the median of `runs` runs
    of `steps_per_run` steps.  The value is the faster build's."""
    import tempfile
    from oracle import pyoracle
    cores = host_cores()
    case = workload_case(N_CELLS_SIDE, steps=1)
    builds = pyoracle.build_native(tempfile.mkdtemp(prefix="mose_oracle_"))
    res = {}
    for name, path in builds.items():
        v, per = time_oracle_build(path, case, cores, runs, steps_per_run)
        res[name] = {"value": v, "ms_per_step_runs": [1e3 * x for x in per]}
    best = max(res, key=lambda k: res[k]["value"])
    return {"value": res[best]["value"], "unit": "cell-updates/s", "cores": cores, "kind": "port",
            "sample": f"the {N_CELLS_SIDE}x{N_CELLS_SIDE} workload itself: 1 warm-up step, then the median of "
                      f"{runs} runs of {steps_per_run} RK3 steps, {cores} OpenMP threads, per build; value = "
                      f"the faster build ({best}); C++/OpenMP restatement of the reference Fortran",
            "cpu_model": cpu_model(), "builds": {k: {"value": v["value"], "flags": (
                "-O3 -march=native -fopenmp -ffp-contract=off" if k == "native" else
                "-O3 -march=native -ffast-math -fomit-frame-pointer -fopenmp")} for k, v in res.items()}}


def run_reference(args):
    # the CPU arm: rank 0 alone times the oracle; no process group is needed
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import tempfile
    from oracle import pyoracle
    cores = host_cores()
    case = workload_case(N_CELLS_SIDE, steps=1)
    builds = pyoracle.build_native(tempfile.mkdtemp(prefix="mose_oracle_"))
    nwarm = max(args.warmup, 3)               # the GPU arm's warm-up count
    # each timed step is one full RK3 step of the 2048^2 block; both builds
    # run, the faster one is the arm's value; the count is bounded so the run
    # stays within minutes
    budget = 60.0
    res = {}
    for name, path in builds.items():
        o = pyoracle.Oracle(case, nthreads=cores, omp=True, lib_path=path)
        for _ in range(nwarm):
            o.step()
        t0 = time.perf_counter()
        steps = 0
        while steps < args.steps and (time.perf_counter() - t0) < budget:
            o.step()
            steps += 1
        el = time.perf_counter() - t0
        res[name] = (case.ncells * steps / el, steps, el)
        del o
    best = max(res, key=lambda k: res[k][0])
    value, steps, el = res[best]
    line = {"metric": "cell-updates/s MUSCL+HLLC RK3 FP64", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": steps, "warmup": nwarm, "ms_per_step": 1e3 * el / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(case, "fp64 (CPU oracle)"), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                             "sample": f"{steps} of the requested {args.steps} steps of the 2048^2 workload after "
                                       f"{nwarm} warm-up steps ({el:.1f} s on {cores} threads), build {best}",
                             "cpu_model": cpu_model(),
                             "builds": {k: v[0] for k, v in res.items()}},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


PRECISIONS = ("exact", "fp64", "mixed")


def precision_code(name):
    from mose_b200 import _lib
    return {"exact": _lib.PRECISION_FP64_EXACT, "fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[name]


def time_advance(s, stream, steps, world, clk=None):
    """Device time (ms, max over ranks) of `steps` graph-replayed fused steps."""
    import torch
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clk is not None:
        clk.__enter__()
    e0.record(stream)
    s.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if clk is not None:
        clk.__exit__(None, None, None)
    barrier(world)
    return max_over_ranks(e0.elapsed_time(e1), world)


def stage_roofline(s, steps, cells):
    """Per-kernel-class device times (CUDA events between launches) and the
    stage kernel's achieved HBM GB/s on the algorithmic bytes."""
    kms, kn = s.time_kernels(max(3, min(20, steps)))
    stage_ms = kms[2] / max(kn[2], 1)
    achieved = STAGE_BYTES_PER_CELL * cells / (stage_ms / 1e3) / 1e9
    return stage_ms, achieved, {"dt": kms[0] / max(1, kn[0] // 3), "ghost": kms[1] / max(1, kn[1]),
                                "stage": stage_ms}


def _oracle_density(out_path, steps, cores, n=N_CELLS_SIDE):
    """(Run in a spawned process.)  The FP64 oracle on the n x n workload
    (2048^2) for `steps` RK3 steps; saves the final interior density."""
    from mose_b200.cases import GC
    from oracle import pyoracle
    case = workload_case(n, steps=steps)
    o = pyoracle.Oracle(case, nthreads=cores, omp=True)
    for _ in range(steps):
        o.step()
    np.save(out_path, o.get_prim(1)[GC:-GC, GC:-GC, GC:-GC, 0])


def start_oracle_density(steps=100, n=N_CELLS_SIDE):
    """Starts the oracle run of _oracle_density in a fresh (spawned) process,
    so that it overlaps the device-timed reports; returns (process, path)."""
    import multiprocessing as mp
    import tempfile
    path = os.path.join(tempfile.mkdtemp(prefix="mose_oracle_"), "density.npy")
    proc = mp.get_context("spawn").Process(target=_oracle_density, args=(path, steps, host_cores(), n))
    proc.start()
    return proc, path


def errors_vs_oracle(local, proc, path, steps=100):
    """Density error of every precision against the FP64 oracle itself after
    `steps` RK3 steps of the 2048^2 workload from the same initial state: L2
    (relative, over all cells) and normwise L-infinity; for the
    reference-exact precision also whether it is bit-identical."""
    from mose_b200 import Solver
    from mose_b200.cases import GC
    proc.join()
    if proc.exitcode != 0 or not os.path.exists(path):
        return {"error": f"oracle run failed (exit code {proc.exitcode})"}
    r = np.load(path)
    case = workload_case(N_CELLS_SIDE, steps=steps)
    out = {"steps": steps, "against": "FP64 oracle (C++ restatement of the reference, OpenMP build)"}
    for name in PRECISIONS:
        s = Solver(case, precision=precision_code(name), device=local)
        s.advance(steps)
        g = s.download_prim(1)[GC:-GC, GC:-GC, GC:-GC, 0]
        s.close()
        e = {"density_l2": float(np.sqrt(((g - r) ** 2).sum() / (r ** 2).sum())),
             "density_linf": float(np.abs(g - r).max() / np.abs(r).max())}
        if name == "exact":
            e["bitwise"] = bool(np.array_equal(g, r))
        out[name] = e
    return out


def warm_up(s, stream, seconds=0.5):
    """Steps until about `seconds` of GPU time have passed: the first few
    hundred steps from the initial state run slower than the later ones, so
    the autotuner (which measures on the state it is given and restores it)
    and the timed region both start from the warmed flow."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0.0
    n = 4
    while done < seconds * 1e3:
        e0.record(stream)
        s.advance(n)
        e1.record(stream)
        e1.synchronize()
        done += e0.elapsed_time(e1)
        n = min(2 * n, 256)


def autotune(s, case):
    """The project's autotuner on a 2-D solver (work-list tiling, measured on
    this domain's warmed flow before any timing); None for 3-D, whose tiles
    and k runs are planned at setup."""
    if any(nd.shape[0] > 2 for nd in case.nodes):
        return None
    return s.autotune(steps=3)


def config_report(name, make_case, local, steps, precisions=PRECISIONS):
    """Throughput of each precision (graph-replayed steps, CUDA events) on one
    configuration, and the mixed precision's density error against the
    reference-exact path (bit-identical to the FP64 oracle) after `steps`."""
    import torch
    from mose_b200 import Solver
    from mose_b200.cases import GC
    case = make_case()
    out = {"cells": case.ncells, "blocks": len(case.nodes), "steps": steps, "limiter": case.limiter,
           "riemann": case.riemann, "cfl": case.cfl}
    dens = {}
    for prec in precisions:
        s = Solver(case, precision=precision_code(prec), device=local)
        stream = torch.cuda.ExternalStream(s.stream_handle, device=torch.device("cuda", local))
        warm_up(s, stream)
        tuned = autotune(s, case)
        ms = time_advance(s, stream, steps, 1)
        out[prec] = {"value": case.ncells * steps / (ms / 1e3), "unit": "cell-updates/s", "ms_per_step": ms / steps}
        if tuned is not None:
            out[prec]["autotune"] = tuned
        s.close()
        # error run from the initial state
        s = Solver(case, precision=precision_code(prec), device=local)
        s.advance(steps)
        dens[prec] = [s.download_prim(b)[GC:-GC, GC:-GC, GC:-GC, 0].copy() for b in range(1, len(case.nodes) + 1)]
        s.close()
    for prec in precisions:
        if prec == "exact":
            continue
        num = sum(float(((g - r) ** 2).sum()) for g, r in zip(dens[prec], dens["exact"]))
        den = sum(float((r ** 2).sum()) for r in dens["exact"])
        li = max(float(np.abs(g - r).max()) for g, r in zip(dens[prec], dens["exact"])) / \
            max(float(np.abs(r).max()) for r in dens["exact"])
        out[prec]["density_error_vs_exact"] = {"l2": float(np.sqrt(num / den)), "linf": li, "steps": steps}
    return {name: out}


def _adjoint_timing(local, case, prec, nsteps, K):
    """Device times (ms) on one context of the given precision: a plain
    graph-replayed forward of nsteps, the checkpointing forward and the
    reverse sweep (after a warm-up of each, which captures the graphs)."""
    import torch
    from mose_b200 import Solver
    from mose_b200.cases import to_ref_layout
    P0 = case.prim[0].copy()
    mach = case.extra["mach"]
    s = Solver(case, precision=precision_code(prec), device=local)
    st = torch.cuda.ExternalStream(s.stream_handle, device=torch.device("cuda", local))

    def reset():
        s.upload_prim(1, to_ref_layout(P0))
        s.set_time(0.0, 0)
        s.set_inflow_mach(mach)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        r = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    reset()
    s.advance(nsteps)                                     # warm-up (graph capture)
    reset()
    _, plain_ms = timed(lambda: s.advance(nsteps))
    reset()
    s.adjoint_forward(nsteps, K, 1, 3)
    s.adjoint_backward()                                  # warm-up (graphs, buffers)
    reset()
    J0, fwd_ms = timed(lambda: s.adjoint_forward(nsteps, K, 1, 3))
    _, bwd_ms = timed(lambda: s.adjoint_backward())
    s.close()
    return {"plain_forward_ms": plain_ms, "forward_ms": fwd_ms, "backward_ms": bwd_ms, "J_direct": J0,
            "backward_over_forward": bwd_ms / plain_ms, "gradient_over_forward": (fwd_ms + bwd_ms) / plain_ms}


def adjoint_report(local, n=512, nsteps=200, ndir=32, seed=0, precision="fp64"):
    """Configuration 5: the wall-pressure objective on the curvilinear 512^2
    channel after 200 RK3 steps (van Albada + HLLC, FP64), its gradient with
    respect to the initial state and the inflow Mach by the discrete adjoint
    with sqrt(N) checkpointing through the torch.autograd.Function, and the
    gradient against central differences (step 1e-6, and 1e-7 beside it) on
    32 seeded cell-wise random directions.  The forward runs in the fp64
    precision (the fastest FP64 forward; within rounding of the reference
    arithmetic); the cost ratios are the device times of the C ABI calls over
    a plain graph-replayed forward of the same 200 steps in the same
    precision, and beside them the same ratios in the reference-exact
    precision.  backward = the reverse sweep (segment recompute + adjoint
    steps); gradient = the checkpointing forward + the backward.  The
    objective is piecewise smooth (the limiters' cut-off where adjacent
    slopes change sign, the branches of the HLLC wave selection): a
    difference step can straddle kinks, whose share falls with the step.  The
    initial state is the uniform Mach-0.8 flow with a seeded 5 % cell-wise
    perturbation (cases.perturbed_channel): at the exactly uniform state
    every limited slope vanishes and the objective has no gradient."""
    import math
    import torch
    from mose_b200 import Solver, cases
    from mose_b200.adjoint import wall_pressure
    from mose_b200.cases import to_ref_layout
    case = cases.perturbed_channel(n, steps=nsteps, seed=seed)
    rng = np.random.default_rng(seed + 1)
    P0 = case.prim[0].copy()
    mach = case.extra["mach"]
    K = max(1, int(round(math.sqrt(nsteps))))
    times = {prec: _adjoint_timing(local, case, prec, nsteps, K) for prec in (precision, "exact")}
    s = Solver(case, precision=precision_code(precision), device=local)

    def J(P, M):
        s.upload_prim(1, to_ref_layout(P))
        s.set_time(0.0, 0)
        s.set_inflow_mach(M)
        return s.adjoint_forward(nsteps, K, 1, 3)

    p = torch.tensor(P0, requires_grad=True)
    m = torch.tensor(mach, dtype=torch.float64, requires_grad=True)
    Jt = wall_pressure(p, m, s, nsteps, K, 1, 3)
    Jt.backward()
    grad, dM = p.grad.numpy(), float(m.grad)
    h = 1e-6
    errs, errs7 = [], []
    for q in range(ndir):
        d = rng.standard_normal(P0.shape)
        d[..., 3] = 0.0                                   # w is not a state of the 2-D path
        adj = float((grad * d).sum())
        fd = (J(P0 + h * d, mach) - J(P0 - h * d, mach)) / (2 * h)
        errs.append(abs(adj - fd) / abs(fd))
        fd7 = (J(P0 + 0.1 * h * d, mach) - J(P0 - 0.1 * h * d, mach)) / (0.2 * h)
        errs7.append(abs(adj - fd7) / abs(fd7))
    fdm = (J(P0, mach + h) - J(P0, mach - h)) / (2 * h)
    s.close()
    t = times[precision]
    return {"adjoint_curvilinear_512^2_200_steps": {
        "cells": case.ncells, "steps": nsteps, "checkpoint_interval": K, "precision": precision,
        "J": float(Jt.detach()), "J_direct": t["J_direct"],
        "forward_ms": t["forward_ms"], "plain_forward_ms": t["plain_forward_ms"], "backward_ms": t["backward_ms"],
        "backward_over_fp64_forward": t["backward_over_forward"],
        "gradient_over_fp64_forward": t["gradient_over_forward"],
        "exact": times["exact"],
        "ratios": "backward = the reverse sweep (segment recompute + adjoint steps); gradient = the "
                  "checkpointing forward + the backward; each over a plain graph-replayed forward of the "
                  "same 200 steps in the same precision",
        "gradient_vs_fd": {"directions": ndir, "kind": "seeded cell-wise N(0,1) on rho, u, v, p", "step": h,
                           "max_rel_err": max(errs), "median_rel_err": float(np.median(errs)),
                           "below_1e-5": int(sum(e < 1e-5 for e in errs)),
                           "step_1e-7": {"max_rel_err": max(errs7), "median_rel_err": float(np.median(errs7)),
                                         "below_1e-5": int(sum(e < 1e-5 for e in errs7))},
                           "dJ_dmach": dM, "dJ_dmach_fd": fdm, "dJ_dmach_rel_err": abs(dM - fdm) / abs(fdm)}}}


def extra_configs(local):
    """The other benchmark configurations at their full sizes: the 64-block
    four-quadrant problem (one persistent kernel per stage over all blocks,
    graph-replayed steps) and the 3-D periodic box of 8 blocks of 128^3."""
    from mose_b200 import cases
    rep = {}
    rep.update(config_report("quadrant2d_64_blocks_ausm_minmod",
                             lambda: cases.four_quadrant(seed=0, steps=100), local, 100))
    rep.update(config_report("box3d_8x128^3_hllc_vanleer",
                             lambda: cases.periodic_box_3d(128, steps=50, seed=0), local, 50))
    rep.update(adjoint_report(local))
    rep.update(viscous_report(local))
    return rep


def viscous_report(local, n=512, steps=50):
    """The Navier-Stokes path (model 1, laminar) on the shear layer between
    walls, 2 x 2 blocks of 1024 x 512 cells on a warped mesh (2.1 M cells):
    throughput of graph-replayed steps in the reference-exact precision (the
    only one the viscous terms run in), and whether `steps` steps are bit
    for bit those of the oracle's OpenMP build on the same inputs.  mu =
    1e-4: with the case's seeded cell-wise perturbations, a viscosity of
    2e-3 at this resolution puts the heat-diffusion number (gamma / Pr times
    the momentum one the reference's VNN limit bounds) past RK3's stability
    bound, and the oracle itself stops with p < 0 in the first step."""
    import torch
    from mose_b200 import Solver, cases
    from mose_b200.cases import GC
    from oracle import pyoracle
    case = cases.shear_layer(n, nbx=2, nby=2, warp=0.05, mu=1e-4, steps=steps, seed=0)
    s = Solver(case, precision=precision_code("exact"), device=local)
    st = torch.cuda.ExternalStream(s.stream_handle, device=torch.device("cuda", local))
    s.advance(3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    s.advance(steps)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.close()
    s = Solver(case, precision=precision_code("exact"), device=local)
    s.advance(steps)
    o = pyoracle.Oracle(case, nthreads=host_cores(), omp=True)
    for _ in range(steps):
        o.step()
    same = all(np.array_equal(s.download_prim(b)[GC:-GC, GC:-GC, GC:-GC][..., [0, 1, 2, 4]],
                              o.get_prim(b)[GC:-GC, GC:-GC, GC:-GC][..., [0, 1, 2, 4]]) for b in range(1, 5))
    s.close()
    return {"navier_stokes_shear_layer_2x2_blocks_1024x512": {
        "cells": case.ncells, "steps": steps, "exact": {"value": case.ncells / (ms * 1e-3), "unit": "cell-updates/s",
                                                        "ms_per_step": ms},
        "bitwise_vs_oracle_after_steps": bool(same),
        "terms": "HLLC + van Leer convective, laminar diffusive fluxes, 302 / 301 walls, 101 / 201 connections"}}


def profile_adjoint(local, precision="fp64"):
    """The launches a profiler captures for the adjoint: the configuration-5
    channel at 512^2 with 16 steps and a checkpoint every 4, forward and
    backward once to build the graphs, then once more (forward in the given
    precision)."""
    from mose_b200 import Solver, cases
    from mose_b200.cases import to_ref_layout
    case = cases.perturbed_channel(512, steps=16)
    s = Solver(case, precision=precision_code(precision), device=local)
    for _ in range(2):
        s.upload_prim(1, to_ref_layout(case.prim[0]))
        s.set_time(0.0, 0)
        s.set_inflow_mach(case.extra["mach"])
        s.adjoint_forward(16, 4, 1, 3)
        s.adjoint_backward()
    s.close()
    return 0


# DRAM bytes per cell per stage-kernel launch, averaged over the three RK
# stages of one step (ncu dram__bytes_read.sum + dram__bytes_write.sum,
# vortex 2048^2, the benchmark's kernels).  Reads equal the algorithmic
# reads; ~45 MB of each launch's output is still in L2 when it ends, so the
# write count is below the state written.
TRAFFIC_BYTES_PER_CELL = {"fp64": 329.3e6 / 2048 ** 2, "mixed": 330.1e6 / 2048 ** 2, "exact": None}
# FP64-pipe lane slots per cell per stage of the stage kernel on the 2048^2
# vortex (ncu sm__inst_executed_pipe_fp64.sum x 32 / cells, average of the
# three RK stages of one step)
FP64_SLOTS_PER_CELL = {"fp64": 463.4, "exact": 1156.0}


def run_gpu(args):
    world, rank, local = dist_init()
    import torch
    from mose_b200 import Solver
    if args.profile_adjoint:
        return profile_adjoint(local, args.precision)
    if args.profile and args.profile_case == "quadrant":
        from mose_b200 import cases
        case = cases.four_quadrant(seed=0, steps=args.steps)
    elif args.profile and args.profile_case in ("box3d", "box3d_medium", "box3d_small"):
        from mose_b200 import cases
        # 8 x 128^3, 4 x 4 x 2 blocks of 64^3 or 8 x 64^3 cells: power-of-two
        # cells per unit length in every direction, so all run the uniform-grid kernels
        n3, nb3 = {"box3d": (128, (2, 2, 2)), "box3d_medium": (64, (4, 4, 2)),
                   "box3d_small": (64, (2, 2, 2))}[args.profile_case]
        case = cases.periodic_box_3d(n3, nb=nb3, steps=args.steps)
    else:
        case = workload_case(N_CELLS_SIDE, steps=args.steps)
    cells = case.ncells
    peak, peak_kind = peaks()
    s = Solver(case, precision=precision_code(args.precision), device=local)
    stream = torch.cuda.ExternalStream(s.stream_handle, device=torch.device("cuda", local))
    s.advance(max(args.warmup, 3))
    tuned = None
    if not args.profile:
        warm_up(s, stream)
        tuned = autotune(s, case)
    torch.cuda.synchronize()
    if args.profile:
        # the launches a profiler captures: warm-up above, then K plain steps
        for _ in range(args.steps):
            s.explicit_step()
        torch.cuda.synchronize()
        s.close()
        return 0
    # --- device-resident throughput (value) ---------------------------------
    launches0 = s.launch_count
    clk = ClockSampler(local)
    ms = time_advance(s, stream, args.steps, world, clk)
    launches = s.launch_count - launches0
    value = aggregate(world, cells, args.steps, ms)
    stage_ms, achieved, step_ms = stage_roofline(s, args.steps, cells)
    # --- end to end through the C ABI with host buffers ----------------------
    shape = (1 + 4, N_CELLS_SIDE + 4, N_CELLS_SIDE + 4, 5)
    host = torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    s.download_prim(1, host)
    n_e2e = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        s.upload_prim(1, host)
        s.explicit_step()
        s.download_prim(1, host)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = world * cells * n_e2e / e2e_s
    nbytes = int(np.prod(shape[1:])) * 8      # 2-D: the k = 1 plane of the reference array crosses the bus
    s.close()
    # --- the oracle's 100 steps run beside the device-timed reports ----------
    oracle_job = start_oracle_density() if (rank == 0 and world == 1 and not args.no_extra_configs) else None
    # --- the other precisions on the same workload ---------------------------
    variants = {}
    for name in PRECISIONS:
        if name == args.precision:
            continue
        v = Solver(case, precision=precision_code(name), device=local)
        vstream = torch.cuda.ExternalStream(v.stream_handle, device=torch.device("cuda", local))
        v.advance(3)
        warm_up(v, vstream)
        vtuned = autotune(v, case)
        vms = time_advance(v, vstream, args.steps, world)
        v_stage_ms, v_ach, v_step = stage_roofline(v, args.steps, cells)
        variants[name] = {"value": aggregate(world, cells, args.steps, vms), "ms_per_step": vms / args.steps,
                          "stage_ms": v_stage_ms, "roofline_frac": v_ach / peak, "step_kernel_ms": v_step,
                          "autotune": vtuned}
        v.close()
    # the reports beside the headline run once, on rank 0 of a one-GPU run
    extra = extra_configs(local) if oracle_job is not None else None
    errs = errors_vs_oracle(local, *oracle_job) if oracle_job is not None else None
    if rank == 0:
        line = {"metric": "cell-updates/s MUSCL+HLLC RK3 FP64", "value": value, "unit": "cell-updates/s",
                "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": dict(workload_config(case, args.precision), autotune=tuned),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak,
                             "traffic": (TRAFFIC_BYTES_PER_CELL[args.precision] * cells
                                         if TRAFFIC_BYTES_PER_CELL.get(args.precision) else None),
                             "traffic_unit": "bytes per launch (ncu, 3-stage average)",
                             "kernel": "k_stage2d (fused residual + RK stage)", "peak_kind": peak_kind,
                             "stage_ms": stage_ms, "step_kernel_ms": step_ms},
                "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": nbytes,
                        "d2h_bytes_per_step": nbytes,
                        "call": "mose_gpu_upload_prim + mose_gpu_step + mose_gpu_download_prim (pinned host)"},
                "gpu_launches": launches, "clocks": clk.summary(),
                "step_bytes_per_cell": BYTES_PER_CELL_STEP,
                "hbm_frac_whole_step": BYTES_PER_CELL_STEP * cells * args.steps / (ms / 1e3 / world) / 1e9 / peak,
                "variants": variants}
        if errs is not None:
            line["errors_vs_oracle"] = errs
        if extra is not None:
            line["configs"] = extra
        if world == 1:
            ceil = fp64_ceiling(local)
            line["fp64_ceiling"] = ceil
            slots = FP64_SLOTS_PER_CELL.get(args.precision)
            if ceil is not None and slots:
                # the stage kernel against the FP64 pipe: lane operations per
                # second over the measured FMA issue rate (2 flops per FMA)
                ach = slots * cells / (stage_ms * 1e-3) / 1e12
                pk = ceil["dfma_tflops"] / 2.0
                line["fp64_roofline"] = {"kernel": "k_stage2d", "achieved": ach, "peak": pk,
                                         "unit": "T FP64 lane-ops/s", "frac": ach / pk,
                                         "slots_per_cell_stage": slots,
                                         "slots_source": "ncu sm__inst_executed_pipe_fp64.sum x 32 / cells"}
            for name, vv in variants.items():
                sl = FP64_SLOTS_PER_CELL.get(name)
                if ceil is not None and sl and vv.get("stage_ms"):
                    vv["fp64_roofline_frac"] = (sl * cells / (vv["stage_ms"] * 1e-3) / 1e12
                                                / (ceil["dfma_tflops"] / 2.0))
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline()
        line["summary"] = summary(line, args.precision)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _g(x, digits=4):
    """x rounded to `digits` significant digits (compact report numbers)."""
    return float(f"{x:.{digits - 1}e}") if isinstance(x, (int, float)) and x == x and x != 0 else x


def summary(line, headline):
    """The figures a reader needs, in a few hundred characters: the JSON line's
    last key, so that a kept tail of the output holds them."""
    out = {headline: _g(line["value"])}
    for name, v in line.get("variants", {}).items():
        out[name] = _g(v["value"])
    out["hbm_frac"] = _g(line["roofline"]["frac"], 3)
    if "fp64_roofline" in line:
        out["fp64_pipe_frac"] = _g(line["fp64_roofline"]["frac"], 3)
    e = line.get("errors_vs_oracle") or {}
    for name in PRECISIONS:
        if isinstance(e.get(name), dict):
            out[f"{name}_rho_l2_vs_oracle"] = _g(e[name]["density_l2"], 2)
    if isinstance(e.get("exact"), dict):
        out["exact_bitwise_vs_oracle"] = e["exact"]["bitwise"]
    for cname, c in (line.get("configs") or {}).items():
        short = cname.split("_")[0]
        if "navier" in cname:
            out["navier_stokes"] = {"exact": _g(c["exact"]["value"], 3), "bitwise": c["bitwise_vs_oracle_after_steps"]}
            continue
        if "adjoint" in cname:
            out["adjoint"] = {k: _g(c[k], 3) for k in ("backward_over_fp64_forward", "gradient_over_fp64_forward")
                              if k in c}
            if "exact" in c:
                out["adjoint"]["exact_gradient_over_forward"] = _g(c["exact"]["gradient_over_forward"], 3)
            g = c.get("gradient_vs_fd", {})
            out["adjoint"]["fd_max_rel_err"] = _g(g.get("max_rel_err", float("nan")), 2)
            out["adjoint"]["fd_below_1e-5"] = g.get("below_1e-5")
            continue
        out[short] = {p: _g(c[p]["value"], 3) for p in PRECISIONS if isinstance(c.get(p), dict)}
    if "cpu_baseline" in line:
        out["cpu"] = {k: _g(v["value"], 3) for k, v in line["cpu_baseline"].get("builds", {}).items()}
    out["e2e"] = _g(line["e2e"]["value"], 3)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--precision", default="fp64", choices=list(PRECISIONS),
                    help="precision of the headline value; the others are reported under variants")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-configs", action="store_true",
                    help="skip the four-quadrant and 3-D configuration reports")
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + K fused steps (the command profiled by ncu); prints nothing")
    ap.add_argument("--profile-case", default="vortex",
                    choices=["vortex", "quadrant", "box3d", "box3d_medium", "box3d_small"],
                    help="with --profile: the 2048^2 vortex, the 64-block four-quadrant domain (seed 0), "
                         "the 3-D periodic box of 8 x 128^3, 32 x 64^3 or 8 x 64^3 cells")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="only the adjoint's forward + backward on a 16-step channel (profiled by ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark of the B200 SMAC step (CADMAS-SURF/3D VF_V1CAL + VF_F1CAL).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--case beach|flume|ensemble|unet]

Default workload (one GPU): the solitary wave on a 1:20 beach with 40
seeded porous boxes, 1024 x 128 x 128 cells (dx=dy=0.02 m, dz=0.01 m,
depth 0.6 m, amplitude 0.15 m, dt = 1e-3 s), pressure solved to a 1e-8
relative residual.  Two solvers step it from the same initial state:

  * plain: the reference's MILU-BiCGSTAB in FP64 (VF_M1BCGS, converged on
    |M^-1 r| <= 1e-8 |M^-1 b| as the reference does);
  * mixed: FP32 MILU factor and FP32 BiCGSTAB inner solves under FP64
    iterative refinement, converged on the true residual
    ||b - Ax|| <= 1e-8 ||b|| in FP64 (optionally with an initial guess:
    --guess previous|learned).

value = interior cells x steps / device time of the mixed solver's steps
(CUDA events on the library's stream); the plain run's number, the ratio,
the plain solver's roofline and the per-field error of the mixed run
against the plain one after --acc-steps steps go into `config`.  With N
GPUs every rank runs its own replica (independent instances, no data
exchange).  e2e = the mixed run through the Fortran-callable entry point
vf_step_gpu_ with the state in pinned host arrays copied in and out every
step.

--case flume: the plain FP64 wave flume with a porous breakwater, 512 x 32
x 96 cells, tolerance 1e-10, driven by the first-order stream-function
wave maker (WAVE-BC X- FUNC STREAM 1), the reference's configuration of
that run.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "multiscale-and-multiphysics-integrated-simulator-for-tsunami_b200"
METRIC = "Mcell-steps/s at 1e-8 rel residual: learned+mixed vs plain FP64 GPU; HBM %"
UNIT = "Mcell-steps/s"

# Algorithmic bytes per interior cell of each stage (each distinct array
# read or written once: 8 B per double, 4 B per int).
STAGE_BYTES = {
    "flux": 10 * 8 + 5 * 4 + 9 * 8,      # u,v,w,ANU,GL*,GG* + NF,IND*,INDC -> 9 fluxes
    "predict": 19 * 8 + 4 * 4 + 3 * 8,   # 9 fluxes,u,v,w,p,GGV,GLV,CD0,GG* + NF,IND* -> u,v,w
    "vpcoef": 10 * 8 + 5 * 4 + 8 * 8,    # u,v,w,p,F,GGV,GLV,GG* + NF,INDC,IND* -> 8 arrays
    "dcmp": 7 * 8 + 4 + 8,               # 7 coefficients + INDC -> DD
    "fwd": 7 * 8 + 8 + 8 + 8,            # 7 coefficients, DD, P -> T (SpMV fused; DD != 0 marks INDC != -1)
    "bwd": 5 * 8 + 8,                    # T, AUI, AUJ, AUK, DD -> X
}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per interior
# cell of one launch of each stage's dominant kernel, from ncu captures of
# the 256x32x96 flume with 16x16 and 8x16 blocks (the same sweep variants
# as the bench's 512x32x96, one block per SM), so the traffic per launch
# scales with the cells.
NCU_TRAFFIC_PER_CELL = {(16, 16): {"fwd": 97.4, "bwd": 52.6}, (8, 16): {"fwd": 91.0, "bwd": 50.3}}


def _load_pkg():
    import importlib.util
    if "cadmas_b200" in sys.modules:
        return sys.modules["cadmas_b200"]
    spec = importlib.util.spec_from_file_location("cadmas_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cadmas_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def combine_ranks(t_local: float, units_local: float, device=None):
    """Max of the per-rank times and sum of the per-rank work units."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return t_local, units_local
    t = torch.tensor([t_local], dtype=torch.float64, device=device)
    u = torch.tensor([units_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())


def build_case(args):
    P = _load_pkg()
    if getattr(args, "case", "flume") == "beach":
        return P.cases.solitary_beach(nx=args.beach_nx, ny=args.beach_ny, nz=args.beach_nz)
    c = P.cases.porous_flume(nx=args.nx, ny=args.ny, nz=args.nz)
    # WAVE-BC X- FUNC STREAM 1: the first-order stream-function wave, and
    # the train it would have made as the initial state
    P.cases.wave_maker(c, 0.08, 1.5, 0.5, stream=1)
    P.cases.linear_wave_initial(c, 0.08, 1.5, 0.5, phase0=c.wave["stream"].phase0)
    return c


def params_for(args):
    return dict(cgepsr=1.0e-8 if getattr(args, "case", "flume") == "beach" else 1.0e-10,
                precond_ti=args.ti, precond_tj=args.tj, precond_split=getattr(args, "split", 1),
                solver=1 if getattr(args, "solver", "fp64") == "mixed" else 0,
                warm_start={"zero": 0, "previous": 1, "learned": 2}[getattr(args, "guess", "zero")],
                mixed_eps_inner=getattr(args, "eps_inner", 1.0e-5),
                sweep_occupancy=getattr(args, "occ", 0), dot_passes=getattr(args, "dot_passes", 0))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        os.unlink(self.path)
        return out


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def cpu_baseline(case, args, max_seconds=25.0, min_steps=1, warm=1):
    """The oracle (CPU restatement, reference summation order, its solver on
    all host threads: one emulated rank per preconditioner block, plain FP64
    solver) on the same case: `warm` warm-up steps, then timed steps until
    max_seconds.  Returns Mcell-steps/s, steps, seconds and threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    sys.path.pop(0)
    prm = dict(params_for(args), solver=0, warm_start=0)
    o = pyoracle.Oracle(case, sum_mode=pyoracle.SUM_REF, **prm)
    o.init_state(True)
    for _ in range(warm):
        o.step(case.dt)
    n, t0 = 0, time.perf_counter()
    while n < min_steps or (time.perf_counter() - t0 < max_seconds and n < 50):
        o.step(case.dt)
        n += 1
    dt = time.perf_counter() - t0
    o.close()
    return case.interior_cells * n / dt / 1e6, n, dt, pyoracle.num_threads()


def run_reference(args, rank, world):
    if rank != 0:
        return
    case = build_case(args)
    budget = 150.0
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    sys.path.pop(0)
    # the reference's own solver: VF_M1BCGS in FP64 from PT = 0
    o = pyoracle.Oracle(case, sum_mode=pyoracle.SUM_REF, **dict(params_for(args), solver=0, warm_start=0))
    o.init_state(True)
    beach = args.case == "beach"
    nwarm = 0 if beach else min(args.warmup, 1)  # a beach step takes the oracle many seconds
    for _ in range(nwarm):
        o.step(case.dt)
    n, t0 = 0, time.perf_counter()
    while n < args.steps and (n == 0 or time.perf_counter() - t0 < budget):
        o.step(case.dt)
        n += 1
    dt = time.perf_counter() - t0
    v = case.interior_cells * n / dt / 1e6
    threads = pyoracle.num_threads()
    what = "beach" if beach else "flume"
    sample = (f"{n} of {args.steps} steps of the {case.ni-2}x{case.nj-2}x{case.nk-2} {what} after "
              f"{nwarm} warm-up step(s), {dt:.1f} s, oracle (plain FP64 solver, reference summation order) "
              f"on {threads} OpenMP threads (one emulated rank per preconditioner block)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
            "steps": n, "warmup": nwarm, "ms_per_step": 1e3 * dt / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(case, args),
            "solver": "plain FP64 MILU-BiCGSTAB (the reference's VF_M1BCGS) in the CPU oracle",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(case, args):
    solver = ("mixed FP32-inner/FP64-refinement" if getattr(args, "solver", "fp64") == "mixed"
              else "plain FP64")
    if getattr(args, "case", "flume") == "beach":
        # the same for both arms: the solver of a line is its "solver" key
        return {"workload": f"solitary wave on a 1:20 beach with 40 seeded porous boxes "
                            f"{case.ni-2}x{case.nj-2}x{case.nk-2} SMAC step (dt={case.dt}, pressure to a "
                            f"1e-8 relative residual, block-Jacobi MILU {args.ti}x{args.tj} columns)",
                "cells": case.interior_cells, "precond_block": [args.ti, args.tj],
                "l2": "inputs larger than L2 (about 60 arrays of 139 MB resident)"}
    if getattr(args, "guess", "zero") == "previous":
        solver += ", previous-step initial guess,"
    if getattr(args, "guess", "zero") == "learned":
        solver += (f", learned initial guess (U-Net trained on the first {args.train_steps} steps' solves, "
                   f"timed after them),")
    return {"workload": f"porous wave flume {case.ni-2}x{case.nj-2}x{case.nk-2} {solver} SMAC step "
                        f"(stream-function wave maker FUNC STREAM 1, H=0.08 T=1.5, at x=0 on a developed "
                        f"first-order wave train, "
                        f"dt={case.dt}, tol 1e-10, block-Jacobi MILU "
                        f"{args.ti}x{args.tj} columns)",
            "cells": case.interior_cells, "precond_block": [args.ti, args.tj],
            "l2": "inputs larger than L2 (about 40 arrays of 13.7 MB resident)"}


def pinned_state(P, case, torch):
    """Host state arrays in pinned memory, Fortran order."""
    ni, nj, nk, nb = case.ni, case.nj, case.nk, max(case.numb, 1)

    def buf(n, dt):
        t = torch.empty(n, dtype=dt, pin_memory=True)
        return t

    keep, arrs = [], {}
    for n in ("uu", "vv", "ww", "pp", "ff"):
        t = buf(ni * nj * nk, torch.float64)
        keep.append(t)
        arrs[n] = t.numpy().reshape((ni, nj, nk), order="F")
    for n in ("nf", "indc"):
        t = buf(ni * nj * nk, torch.int32)
        keep.append(t)
        arrs[n] = t.numpy().reshape((ni, nj, nk), order="F")
    for n in ("bcu", "bcv", "bcw", "bcp", "bcf"):
        t = buf(nb, torch.float64)
        keep.append(t)
        arrs[n] = t.numpy()
    return keep, arrs


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    P = _load_pkg()
    if rank == 0:
        P.build_library()
    if world > 1:
        dist.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    case = build_case(args)
    learned = None
    if getattr(args, "guess", "zero") == "learned":
        # train the guess on the solver's own solves of the first steps
        # (outside the timing), then time the steps after them
        import importlib
        ws = importlib.import_module(P.__name__ + ".warmstart")
        t0 = time.time()
        samples = ws.collect(case, args.train_steps, precond_ti=args.ti, precond_tj=args.tj)
        params, cscale = ws.train(samples, epochs=args.train_epochs, batch=1, lr=1.0e-3, w_mse=0.1, w_res=1.0)
        learned = {"train_steps": args.train_steps, "epochs": args.train_epochs,
                   "train_s": round(time.time() - t0, 1), "out_scale": cscale}
        del samples
    tank = P.Tank(case, **params_for(args))
    if learned is not None:
        tank.set_warm_net(params, cscale)
    tank.init_state(True)
    stream = torch.cuda.ExternalStream(tank.stream(), device=dev)
    for _ in range(args.train_steps if learned is not None else 0):
        tank.step(case.dt)
    for _ in range(args.warmup):
        tank.step(case.dt)
    tank.sync()
    l0 = P.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    iters = []
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            tank.step(case.dt)
            iters.append(tank.stats()["icgitr"])
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    launches = P.kernel_launches() - l0
    t_ms = ev0.elapsed_time(ev1)
    if world > 1:
        dist.barrier()
    clocks = clk.summary()
    # Per-stage device times from a second pass of the same number of steps
    # with an event pair around every stage (kept out of the pass above so
    # the events do not add to the step time).
    tank.stage_timers(enable=1)
    for _ in range(args.steps):
        tank.step(case.dt)
    tank.sync()
    stages = tank.stage_timers(enable=0)
    t_max, units = combine_ranks(t_ms / 1e3, case.interior_cells * args.steps, device=dev)
    value = units / t_max / 1e6
    # true relative residual of one more solve (diagnostic, outside the timing)
    relres = None
    try:
        tank2 = P.Tank(case, diag_relres=1, **params_for(args))
        tank2.set_state(tank.get_state())
        tank2.step(case.dt)
        relres = tank2.stats()["true_relres"]
        tank2.close()
    except Exception:
        relres = None
    # ---- end to end through vf_step_gpu_ with pinned host buffers
    e2e = None
    if not args.no_e2e:
        keep, arrs = pinned_state(P, case, torch)
        st = tank.get_state()
        for n in arrs:
            arrs[n][...] = st[n][: arrs[n].shape[0]] if arrs[n].ndim == 1 else st[n]
        lib = tank.lib
        hp = ctypes.c_void_p(tank.h.value)
        dtc = ctypes.c_double(case.dt)
        tnow = ctypes.c_double(st["tnow"])
        nnow = ctypes.c_int(st["nnow"])
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        argv = [ctypes.byref(hp), ctypes.byref(dtc), dp(arrs["uu"]), dp(arrs["vv"]), dp(arrs["ww"]),
                dp(arrs["pp"]), dp(arrs["ff"]), ip(arrs["nf"]), ip(arrs["indc"]), dp(arrs["bcu"]),
                dp(arrs["bcv"]), dp(arrs["bcw"]), dp(arrs["bcp"]), dp(arrs["bcf"]), ctypes.byref(tnow),
                ctypes.byref(nnow)]
        nsteps_e2e = max(1, min(args.steps, 10))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(nsteps_e2e):
            rc = lib.vf_step_gpu_(*argv)
            if rc != 0:
                raise P.CadmasError(rc, "vf_step_gpu_")
        e1.record(stream)
        e1.synchronize()
        te_max, ue = combine_ranks(e0.elapsed_time(e1) / 1e3, case.interior_cells * nsteps_e2e, device=dev)
        bytes_io = sum(a.nbytes for a in arrs.values())
        e2e = {"value": ue / te_max / 1e6, "unit": UNIT, "h2d_bytes_per_step": bytes_io,
               "d2h_bytes_per_step": bytes_io, "steps": nsteps_e2e,
               "path": "vf_step_gpu_ (pinned host state in/out every step)"}
    # ---- roofline of the dominant stage
    peak, peak_kind = measured_peak_hbm()
    dom = max((k for k in STAGE_BYTES), key=lambda k: stages[k][0])
    ms_dom, n_dom = stages[dom]
    bytes_launch = STAGE_BYTES[dom] * case.interior_cells
    achieved = bytes_launch / (ms_dom / n_dom / 1e3) / 1e9 if n_dom else 0.0
    total_ms = sum(v[0] for v in stages.values())
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (NCU_TRAFFIC_PER_CELL[(args.ti, args.tj)][dom] * case.interior_cells
                            if dom in NCU_TRAFFIC_PER_CELL.get((args.ti, args.tj), {}) else None),
                "algorithmic_bytes_per_launch": bytes_launch, "launches": n_dom,
                "avg_launch_ms": ms_dom / n_dom if n_dom else None,
                "share_of_step": ms_dom / total_ms if total_ms else None}
    if rank != 0:
        tank.close()
        return
    cpu = None
    if not args.no_cpu:
        v_cpu, n_cpu, t_cpu, thr = cpu_baseline(case, args)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{n_cpu} steps of the same flume after 1 warm-up step, {t_cpu:.1f} s, "
                         f"oracle (reference summation order) with its solver on {thr} OpenMP threads"}
    if learned is not None:
        # kept/dropped guesses, and the zero guess's iterations on the same steps
        kept, dropped = tank.warm_stats()
        z = P.Tank(case, **{**params_for(args), "warm_start": 0})
        z.init_state(True)
        for _ in range(args.train_steps + args.warmup):
            z.step(case.dt)
        zi = []
        for _ in range(args.steps):
            z.step(case.dt)
            zi.append(z.stats()["icgitr"])
        z.close()
        learned.update(kept=kept, dropped=dropped, zero_guess_mean_iters_same_steps=float(np.mean(zi)))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(case, args), "parallelism": f"replicas x{world}",
                       "mean_bicgstab_iters": float(np.mean(iters)), "true_relres": relres,
                       **({"learned_guess": learned} if learned is not None else {})},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks,
            "stage_ms_per_step": {k: v[0] / args.steps for k, v in stages.items()}}
    print(json.dumps(line), flush=True)
    tank.close()


# Algorithmic bytes per interior cell of the FP32 sweeps of the mixed
# solver (the same arrays as the FP64 ones, 4 B each).
# the mixed solver's FP32 sweeps: the fused forward sweep; the backward
# sweeps with their sums (R0 read by the one after AP, R0 and RR by the one
# after AE: 7 and 8 arrays, 7.5 on average)
STAGE_BYTES_F32 = {"fwd": 10 * 4, "bwd": 7.5 * 4}


def roofline_of(stages, cells, peak, peak_kind, bytes_table, traffic_per_cell=None):
    """Roofline object of the stage with the largest device time among the
    stages whose algorithmic bytes are known."""
    dom = max((k for k in bytes_table), key=lambda k: stages[k][0])
    ms_dom, n_dom = stages[dom]
    bytes_launch = bytes_table[dom] * cells
    achieved = bytes_launch / (ms_dom / n_dom / 1e3) / 1e9 if n_dom else 0.0
    total_ms = sum(v[0] for v in stages.values())
    tr = traffic_per_cell.get(dom) if traffic_per_cell else None
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": tr * cells if tr is not None else None,
            "algorithmic_bytes_per_launch": bytes_launch, "launches": n_dom,
            "avg_launch_ms": ms_dom / n_dom if n_dom else None,
            "share_of_step": ms_dom / total_ms if total_ms else None}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per interior
# cell of one launch of the dominant sweeps on the beach (1024x128x128,
# 16x16 tiles), from an ncu capture of a 1024x80x128 beach: the same
# layers, tile shape and sweep variants (320 tiles, two blocks per SM for
# the backward and FP32 sweeps), so the traffic per launch scales with the
# cells.  FP32 backward: the mean of the sweeps after AP (33.6) and after
# AE (38.8); the four-blocks-per-SM instances that now run them on both
# beaches issue the same bulk copies per step.
NCU_TRAFFIC_BEACH = {"fwd": 99.8, "bwd": 57.9}
NCU_TRAFFIC_BEACH_F32 = {"fwd": 49.9, "bwd": 36.2}


def field_errors(a, b, case):
    """Per-field max-abs and RMS of a - b over the interior cells, with the
    max-abs of b for scale; NF mismatches."""
    sl = (slice(1, case.ni - 1), slice(1, case.nj - 1), slice(1, case.nk - 1))
    out = {}
    for n, lab in (("ff", "F"), ("pp", "p"), ("uu", "u"), ("vv", "v"), ("ww", "w")):
        d = (a[n][sl] - b[n][sl]).ravel()
        ref = np.abs(b[n][sl]).max()
        out[lab] = {"max_abs": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d))),
                    "ref_max_abs": float(ref)}
    out["nf_mismatch_cells"] = int((a["nf"][sl] != b["nf"][sl]).sum())
    return out


def run_headline(args, rank, world, local_rank):
    """Config 2 (the solitary beach): the plain FP64 solver and the mixed
    solver (with the chosen initial guess) from the same initial state."""
    import torch
    import torch.distributed as dist
    P = _load_pkg()
    if rank == 0:
        P.build_library()
    if world > 1:
        dist.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    case = build_case(args)
    cells = case.interior_cells
    base = {k: v for k, v in params_for(args).items() if k not in ("solver", "warm_start")}
    arms = {"plain": dict(base, solver=0, warm_start=0),
            "mixed": dict(base, solver=1, warm_start={"zero": 0, "previous": 1, "learned": 2}[args.guess])}
    learned = None
    if args.guess == "learned":
        # train the guess on the solver's own solves of the first steps
        # (outside the timing)
        import importlib
        ws = importlib.import_module(P.__name__ + ".warmstart")
        t0 = time.time()
        samples = ws.collect(case, args.train_steps, precond_ti=args.ti, precond_tj=args.tj)
        wparams, cscale = ws.train(samples, epochs=args.train_epochs, batch=1, lr=1.0e-3, w_mse=0.1, w_res=1.0)
        learned = {"train_steps": args.train_steps, "epochs": args.train_epochs,
                   "train_s": round(time.time() - t0, 1), "out_scale": cscale}
        del samples
    res = {}
    tanks = {}
    for name in ("plain", "mixed"):
        tank = P.Tank(case, **arms[name])
        if name == "mixed" and learned is not None:
            tank.set_warm_net(wparams, cscale)
        tank.init_state(True)
        stream = torch.cuda.ExternalStream(tank.stream(), device=dev)
        for _ in range(args.warmup):
            tank.step(case.dt)
        tank.sync()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        iters = []
        l0 = P.kernel_launches()
        with ClockSampler(local_rank) as clk:
            ev0.record(stream)
            for _ in range(args.steps):
                tank.step(case.dt)
                iters.append(tank.stats()["icgitr"])
            ev1.record(stream)
            ev1.synchronize()
        torch.cuda.synchronize()
        launches = P.kernel_launches() - l0
        t_ms = ev0.elapsed_time(ev1)
        if world > 1:
            dist.barrier()
        t_max, units = combine_ranks(t_ms / 1e3, cells * args.steps, device=dev)
        res[name] = {"value": units / t_max / 1e6, "ms_per_step": t_max * 1e3 / args.steps,
                     "mean_iters": float(np.mean(iters)), "launches": launches, "clocks": clk.summary(),
                     "stream": stream}
        tanks[name] = tank
    # Continue both runs (untimed, per-stage event timers on) to the
    # accuracy horizon, then compare the fields.
    n_done = args.warmup + args.steps
    n_acc = max(args.acc_steps, n_done)
    stage = {}
    for name, tank in tanks.items():
        tank.stage_timers(enable=1)
        nst = 0
        while n_done + nst < n_acc or nst < min(args.steps, 5):
            tank.step(case.dt)
            nst += 1
        tank.sync()
        stage[name] = (tank.stage_timers(enable=0), nst)
    n_acc = n_done + stage["plain"][1]
    sp, sm = tanks["plain"].get_state(), tanks["mixed"].get_state()
    stp, stm = tanks["plain"].stats(), tanks["mixed"].stats()
    f0 = None
    try:
        f0 = float(np.sum(case.ff[1:-1, 1:-1, 1:-1] * case.ggv[1:-1, 1:-1, 1:-1]))
    except Exception:
        f0 = None
    acc = {"steps": n_acc, "fields_mixed_minus_plain": field_errors(sm, sp, case),
           "fsum_plain": stp["fsum"], "fsum_mixed": stm["fsum"],
           "volume_drift_rel": abs(stm["fsum"] - stp["fsum"]) / abs(stp["fsum"]) if stp["fsum"] else None,
           "mixed_last_solve_true_relres": (stm["cgxnrm"] / stm["cgbnrm"]) if stm["cgbnrm"] else None,
           "mixed_fp64_fallbacks": stm["fallbacks"]}
    if learned is not None:
        kept, dropped = tanks["mixed"].warm_stats()
        learned.update(kept=kept, dropped=dropped)
    # True residual of one plain solve from the plain run's state
    # (diagnostic outside the timing: one more handle with the check on).
    relres_plain = None
    try:
        t2 = P.Tank(case, diag_relres=1, **arms["plain"])
        t2.set_state(sp)
        t2.step(case.dt)
        relres_plain = t2.stats()["true_relres"]
        t2.close()
    except Exception:
        relres_plain = None
    tanks["plain"].close()
    # ---- e2e through vf_step_gpu_ with pinned host buffers (mixed solver)
    tank = tanks["mixed"]
    stream = res["mixed"]["stream"]
    e2e = None
    if not args.no_e2e:
        e2e = e2e_run(P, tank, case, stream, args, world, dev)
    peak, peak_kind = measured_peak_hbm()
    st_p, nst_p = stage["plain"]
    st_m, nst_m = stage["mixed"]
    roof_plain = roofline_of(st_p, cells, peak, peak_kind, STAGE_BYTES, NCU_TRAFFIC_BEACH)
    bytes_m = dict(STAGE_BYTES)
    bytes_m.update(STAGE_BYTES_F32)
    roof_mixed = roofline_of(st_m, cells, peak, peak_kind, bytes_m, NCU_TRAFFIC_BEACH_F32)
    tank.close()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu:
        v_cpu, n_cpu, t_cpu, thr = cpu_baseline(case, args, warm=0)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{n_cpu} step(s) of the same beach from its initial state, {t_cpu:.1f} s, "
                         f"oracle (reference summation order, plain FP64 solver) on {thr} OpenMP threads"}
    rp, rm = res["plain"], res["mixed"]
    guess = {"zero": "zero initial guess", "previous": "previous-step initial guess",
             "learned": "learned initial guess"}[args.guess]
    line = {"metric": METRIC, "value": rm["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": rm["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 refinement", "data": "synthetic",
            "config": workload_config(case, args),
            "solver": f"mixed FP32-inner/FP64-refinement with {guess}",
            "parallelism": f"replicas x{world}",
            "arms": {"mixed": {"value": rm["value"], "ms_per_step": rm["ms_per_step"],
                               "mean_inner_iters": rm["mean_iters"], "eps_inner_floor": args.eps_inner,
                               "roofline": roof_mixed,
                               "stage_ms_per_step": {k: v[0] / nst_m for k, v in st_m.items()}},
                     "plain_fp64": {"value": rp["value"], "ms_per_step": rp["ms_per_step"],
                                    "mean_bicgstab_iters": rp["mean_iters"], "true_relres": relres_plain,
                                    "roofline": roof_plain, "clocks": rp["clocks"],
                                    "stage_ms_per_step": {k: v[0] / nst_p for k, v in st_p.items()}}},
            "speedup_vs_plain_fp64": rm["value"] / rp["value"],
            "plain_fp64_roofline_frac": roof_plain["frac"],
            "accuracy": acc,
            **({"learned_guess": learned} if learned is not None else {}),
            "roofline": roof_mixed, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": rm["launches"],
            "clocks": rm["clocks"]}
    print(json.dumps(line), flush=True)


def e2e_run(P, tank, case, stream, args, world, dev):
    """The same steps through vf_step_gpu_ with the state in pinned host
    arrays, copied in and out every step."""
    import torch
    import torch.distributed as dist
    keep, arrs = pinned_state(P, case, torch)
    st = tank.get_state()
    for n in arrs:
        arrs[n][...] = st[n][: arrs[n].shape[0]] if arrs[n].ndim == 1 else st[n]
    lib = tank.lib
    hp = ctypes.c_void_p(tank.h.value)
    dtc = ctypes.c_double(case.dt)
    tnow = ctypes.c_double(st["tnow"])
    nnow = ctypes.c_int(st["nnow"])
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    argv = [ctypes.byref(hp), ctypes.byref(dtc), dp(arrs["uu"]), dp(arrs["vv"]), dp(arrs["ww"]),
            dp(arrs["pp"]), dp(arrs["ff"]), ip(arrs["nf"]), ip(arrs["indc"]), dp(arrs["bcu"]),
            dp(arrs["bcv"]), dp(arrs["bcw"]), dp(arrs["bcp"]), dp(arrs["bcf"]), ctypes.byref(tnow),
            ctypes.byref(nnow)]
    nsteps_e2e = max(1, min(args.steps, 10))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nsteps_e2e):
        rc = lib.vf_step_gpu_(*argv)
        if rc != 0:
            raise P.CadmasError(rc, "vf_step_gpu_")
    e1.record(stream)
    e1.synchronize()
    te_max, ue = combine_ranks(e0.elapsed_time(e1) / 1e3, case.interior_cells * nsteps_e2e, device=dev)
    bytes_io = sum(a.nbytes for a in arrs.values())
    return {"value": ue / te_max / 1e6, "unit": UNIT, "h2d_bytes_per_step": bytes_io,
            "d2h_bytes_per_step": bytes_io, "steps": nsteps_e2e,
            "path": "vf_step_gpu_ (pinned host state in/out every step)"}


def run_learned(args, rank, world, local_rank):
    """The learned initial guess on held-out grids: the network is trained
    on the solver's own (BB, PT, system) triples from the first steps of
    beaches with seeds 0..n_train-1 (the config-2 beach scaled down to a
    small grid, seeded boxes), then beaches with seeds 50.. are stepped
    with the zero guess, the previous step's solution and the learned
    guess; the line reports BiCGSTAB iterations, kept/dropped guesses and
    the device time per step of each."""
    import importlib
    import torch
    P = _load_pkg()
    P.build_library()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ws = importlib.import_module(P.__name__ + ".warmstart")
    nx, ny, nz = (int(v) for v in args.learn_grid.split("x"))
    sc = 1024 / nx

    def beach(seed):
        return P.cases.solitary_beach(nx=nx, ny=ny, nz=nz, dx=0.02 * sc, dy=0.02 * 128 / ny,
                                      dz=0.01 * 128 / nz, seed=seed, nbox=40, dt=1.0e-3 * sc)

    t0 = time.time()
    samples = []
    for sd in range(args.learn_train):
        samples += ws.collect(beach(sd), args.learn_steps, precond_ti=args.ti, precond_tj=args.tj)
    t_collect = time.time() - t0
    t0 = time.time()
    params, cscale = ws.train(samples, epochs=args.train_epochs, batch=4, lr=1.0e-3, w_mse=0.1, w_res=1.0)
    t_train = time.time() - t0
    del samples
    out = {}
    for guess, ws_mode in (("zero", 0), ("previous", 1), ("learned", 2)):
        iters, ms, kept, dropped = [], 0.0, 0, 0
        for sd in range(50, 50 + args.learn_eval):
            c = beach(sd)
            t = P.Tank(c, warm_start=ws_mode, precond_ti=args.ti, precond_tj=args.tj)
            if ws_mode == 2:
                t.set_warm_net(params, cscale)
            t.init_state(True)
            stream = torch.cuda.ExternalStream(t.stream(), device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.learn_steps):
                t.step(c.dt)
                iters.append(t.stats()["icgitr"])
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            if ws_mode == 2:
                k, d = t.warm_stats()
                kept, dropped = kept + k, dropped + d
            t.close()
        nst = args.learn_eval * args.learn_steps
        out[guess] = {"mean_iters": float(np.mean(iters)), "ms_per_step": ms / nst,
                      **({"kept": kept, "dropped": dropped, "fallback_rate": dropped / max(1, kept + dropped)}
                         if ws_mode == 2 else {})}
    if rank != 0:
        return
    z = out["zero"]["mean_iters"]
    line = {"metric": "BiCGSTAB iterations per solve on held-out beaches (learned initial guess)",
            "value": out["learned"]["mean_iters"], "unit": "iterations", "n_gpus": 1,
            "steps": args.learn_steps, "warmup": 0, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network, f64 solver", "data": "synthetic",
            "config": {"workload": f"solitary beach {nx}x{ny}x{nz} (the 1024x128x128 beach scaled to this grid), "
                                   f"train seeds 0..{args.learn_train - 1} x {args.learn_steps} steps, "
                                   f"held-out seeds 50..{49 + args.learn_eval} x {args.learn_steps} steps, "
                                   f"{args.train_epochs} epochs, tol 1e-8",
                       "collect_s": round(t_collect, 1), "train_s": round(t_train, 1)},
            "guesses": out, "gain_vs_zero": 1.0 - out["learned"]["mean_iters"] / z,
            "gain_previous_vs_zero": 1.0 - out["previous"]["mean_iters"] / z}
    print(json.dumps(line), flush=True)


def measured_peak_bf16():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
        except Exception:
            pass
    return 1590.0, "fallback"


# (cin, cout, level) of the warm-start U-Net's 3x3x3 convolutions
UNET_LAYERS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2),
               (64, 64, 2), (96, 32, 1), (32, 32, 1), (48, 16, 0), (16, 16, 0)]


def run_unet(args, rank, world, local_rank):
    """The learned guess's network alone: device time of its forward on one
    volume (the tcgen05 convolutions), FLOP/s against the bf16 peak."""
    import importlib
    P = _load_pkg()
    P.build_library()
    ws = importlib.import_module(P.__name__ + ".warmstart")
    X, Y, Z = (int(v) for v in args.unet_volume.split("x"))
    net = P.UNet(X, Y, Z, 1)
    net.set_params(ws.init_params(2))
    x = np.random.default_rng(0).normal(size=(1, Z, Y, X, 4)).astype(np.float32)
    net.forward(x)
    net.time_forward(max(1, args.warmup))
    ms = net.time_forward(args.steps)
    vox = [X * Y * Z // 8 ** lv for lv in range(3)]
    flop = sum(2 * 27 * ci * co * vox[lv] for ci, co, lv in UNET_LAYERS) + 2 * 16 * vox[0]
    tf = flop / (ms * 1e-3) / 1e12
    peak, kind = measured_peak_bf16()
    if rank == 0:
        print(json.dumps({"metric": "U-Net forward TFLOP/s (learned initial guess)", "value": tf, "unit": "TFLOP/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
                          "data": "synthetic", "config": {"workload": f"warm-start U-Net forward on a {X}x{Y}x{Z} "
                                                                      f"volume (16/32/64 channels)"},
                          "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                                       "frac": tf / peak, "peak_kind": kind, "traffic": None}}), flush=True)
    net.close()


def run_ensemble(args, rank, world, local_rank):
    """Ensemble of independent flumes of uneven size stepped side by side
    (cadmas_step_ensemble: one host thread and one stream per flume).
    value = all flumes' interior cells x steps / device time of the steps;
    the same members stepped one after another give `sequential_value`."""
    import torch
    P = _load_pkg()
    if rank == 0:
        P.build_library()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cases = P.cases.ensemble_flumes(args.members, seed=1000 * rank, scale=args.scale)
    tiles = [(args.ti, args.tj)] * len(cases)
    tune_s = None
    tune_timings = None
    if args.autotune and args.batch:
        # one block shape for the batch, timed with all members stepping
        # together (untimed here)
        import importlib
        at = importlib.import_module(P.__name__ + ".autotune")
        t0 = time.time()
        base = {k: v for k, v in params_for(args).items() if k not in ("precond_ti", "precond_tj")}
        shape, tune_timings = at.pick_batch_tiles(cases, **base)
        tiles = [shape] * len(cases)
        args.ti, args.tj = shape
        tune_s = round(time.time() - t0, 1)
    elif args.autotune:
        # block shapes per member from the tile autotuner (untimed; cached by grid size)
        import importlib
        at = importlib.import_module(P.__name__ + ".autotune")
        cache = at.TileCache()
        t0 = time.time()
        base = {k: v for k, v in params_for(args).items() if k not in ("precond_ti", "precond_tj")}
        tiles = [at.pick_tiles(c, cache=cache, **base) for c in cases]
        tune_s = round(time.time() - t0, 1)
    tanks = [P.Tank(c, **{**params_for(args), "precond_ti": ti, "precond_tj": tj}) for c, (ti, tj) in
             zip(cases, tiles)]
    for t in tanks:
        t.init_state(True)
    cells = sum(c.interior_cells for c in cases)
    streams = [torch.cuda.ExternalStream(t.stream(), device=dev) for t in tanks]

    def timed(fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        fn()
        ends = []
        for st in streams:
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            ends.append(e)
        torch.cuda.synchronize()
        return max(e0.elapsed_time(e) for e in ends)

    batch = P.Batch(tanks) if args.batch else None
    step_all = batch.step if batch is not None else (lambda: P.step_ensemble(tanks))
    for _ in range(args.warmup):
        step_all()
    l0 = P.kernel_launches()
    with ClockSampler(local_rank) as clk:
        t_par = timed(lambda: [step_all() for _ in range(args.steps)])
    launches = P.kernel_launches() - l0
    t_seq = timed(lambda: [t.step() for _ in range(args.steps) for t in tanks])
    t_max, units = combine_ranks(t_par / 1e3, cells * args.steps, device=dev)
    iters = [t.stats()["icgitr"] for t in tanks]
    if batch is not None:
        batch.close()
    # Agreement of every member with a solo plain-FP64 run of the same steps
    # from the same initial state (untimed; one solo handle at a time).
    agree = None
    if args.solver == "mixed" and not args.no_agreement:
        errs = []
        base = {k: v for k, v in params_for(args).items() if k not in ("solver", "warm_start")}
        for c, t in zip(cases, tanks):
            st = t.get_state()
            solo = P.Tank(c, **{**base, "solver": 0, "warm_start": 0, "precond_ti": args.ti, "precond_tj": args.tj})
            solo.init_state(True)
            for _ in range(int(st["nnow"])):
                solo.step()
            ref = solo.get_state()
            e = field_errors(st, ref, c)
            fs, fr = t.stats()["fsum"], solo.stats()["fsum"]
            errs.append({"p_rel": e["p"]["max_abs"] / e["p"]["ref_max_abs"], "u_max": max(e[k]["max_abs"] for k in "uvw"),
                         "F_max": e["F"]["max_abs"], "nf_mismatch": e["nf_mismatch_cells"],
                         "volume_rel": abs(fs - fr) / abs(fr)})
            solo.close()
        agree = {"steps": int(tanks[0].get_state()["nnow"]),
                 "max_p_rel": max(x["p_rel"] for x in errs), "max_u_abs": max(x["u_max"] for x in errs),
                 "max_F_abs": max(x["F_max"] for x in errs), "nf_mismatch_cells": sum(x["nf_mismatch"] for x in errs),
                 "max_volume_rel": max(x["volume_rel"] for x in errs)}
    if rank != 0:
        return
    line = {"metric": METRIC, "value": units / t_max / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_par / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement" if args.solver == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"ensemble of {args.members} independent porous wave flumes of uneven "
                                   f"size (nx U{{256..1024}}x{args.scale:g}, ny U{{16..64}}, nz U{{64..128}}, "
                                   f"wave makers, {'mixed' if args.solver == 'mixed' else 'plain FP64'} "
                                   f"SMAC step, block-Jacobi MILU "
                                   f"{('blocks chosen per grid by the tile autotuner' if not args.batch else f'{args.ti}x{args.tj} chosen by the batch autotuner') if args.autotune else f'{args.ti}x{args.tj}'})",
                       "cells": cells, "members": args.members,
                       "sizes": [[c.ni - 2, c.nj - 2, c.nk - 2] for c in cases],
                       "sequential_value": cells * args.steps / (t_seq / 1e3) / 1e6,
                       "mean_bicgstab_iters": statistics.mean(iters),
                       **({"tiles": [list(t) for t in tiles], "autotune_s": tune_s} if args.autotune else {}),
                       **({"autotune_s_per_step": tune_timings} if tune_timings else {}),
                       "parallelism": (f"{args.members} grids, one launch per solver kernel for all of them "
                                       f"(cadmas_batch_step) x{world} replicas" if args.batch else
                                       f"{args.members} streams side by side x{world} replicas")},
            "agreement_with_solo_fp64": agree,
            "gpu_launches": launches, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    for t in tanks:
        t.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--solver", choices=["fp64", "mixed"], default="fp64",
                    help="pressure solver: the reference's FP64 MILU-BiCGSTAB, or FP32 inner solves "
                         "under FP64 refinement")
    ap.add_argument("--split", type=int, choices=[1, 2], default=1,
                    help="2: each preconditioner block swept by a cluster of two thread blocks")
    ap.add_argument("--members", type=int, default=8, help="ensemble members (--case ensemble)")
    ap.add_argument("--autotune", action="store_true",
                    help="--case ensemble: preconditioner block shape per member by the tile autotuner")
    ap.add_argument("--scale", type=float, default=1.0, help="x-size factor of ensemble members")
    ap.add_argument("--batch", action="store_true",
                    help="--case ensemble with --solver mixed: the members' pressure solves together, one "
                         "launch per solver kernel (cadmas_batch_step)")
    ap.add_argument("--no-agreement", action="store_true",
                    help="--case ensemble --solver mixed: skip the members' comparison with solo FP64 runs")
    ap.add_argument("--learn-grid", default="128x32x64", help="--case learned: beach grid NXxNYxNZ")
    ap.add_argument("--learn-train", type=int, default=8, help="--case learned: training seeds")
    ap.add_argument("--learn-eval", type=int, default=3, help="--case learned: held-out seeds")
    ap.add_argument("--learn-steps", type=int, default=12, help="--case learned: steps per seed")
    ap.add_argument("--case", choices=["flume", "beach", "ensemble", "unet", "learned"], default="beach",
                    help="beach: 1024x128x128 solitary wave on a 1:20 beach with 40 porous boxes, plain "
                         "FP64 and mixed solvers (default); flume: 512x32x96 porous wave flume; "
                         "unet: the learned guess's network alone")
    ap.add_argument("--acc-steps", type=int, default=200,
                    help="--case beach: steps after which the mixed run's fields are compared with the "
                         "plain run's")
    ap.add_argument("--eps-inner", type=float, default=1.0e-2,
                    help="floor of the FP32 inner tolerance of the mixed solver (1e-2 measured best on the "
                         "beach: fewer inner iterations in all than with tighter floors)")
    ap.add_argument("--occ", type=int, choices=[0, 1, 2, 4], default=0,
                    help="thread blocks of the MILU sweeps per SM (0: the library's default)")
    ap.add_argument("--dot-passes", type=int, choices=[0, 1], default=0,
                    help="mixed solver: 0 inner products summed by the backward sweeps, 1 separate passes")
    ap.add_argument("--beach-nx", type=int, default=1024)
    ap.add_argument("--beach-ny", type=int, default=128)
    ap.add_argument("--beach-nz", type=int, default=128)
    ap.add_argument("--unet-volume", default="64x32x64", help="--case unet: XxYxZ (multiples of 4)")
    ap.add_argument("--train-steps", type=int, default=40,
                    help="--guess learned: steps whose solves train the network")
    ap.add_argument("--train-epochs", type=int, default=15, help="--guess learned: epochs over them")
    ap.add_argument("--guess", choices=["zero", "previous", "learned"], default=None,
                    help="initial guess of each pressure solve: 0 as the reference, the previous step's "
                         "solution, or the learned guess (default: previous for the mixed solver of "
                         "--case beach, zero otherwise; the plain arm of --case beach always starts "
                         "from 0 as the reference does)")
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=32)
    ap.add_argument("--nz", type=int, default=96)
    ap.add_argument("--ti", type=int, default=None,
                    help="preconditioner block columns along x (default: 8 for --case flume, 16 otherwise)")
    ap.add_argument("--tj", type=int, default=None,
                    help="preconditioner block columns along y (default: 16)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    # block shapes measured best per workload: the flume's 512x32 columns
    # make 128 blocks of 8x16 for the 148 SMs against 64 of 16x16
    if args.ti is None:
        args.ti = 8 if args.case == "flume" else 16
    if args.tj is None:
        args.tj = 16
    if args.guess is None:
        args.guess = "previous" if args.case == "beach" else "zero"
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.case == "ensemble":
            run_ensemble(args, rank, world, local_rank)
        elif args.case == "unet":
            run_unet(args, rank, world, local_rank)
        elif args.case == "learned":
            run_learned(args, rank, world, local_rank)
        elif args.case == "beach":
            run_headline(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

#!/usr/bin/env python3
"""Benchmark of the B200 pressure-Poisson projection (MultiFlow3D newsolv_mg).

One *step* = one complete projection solve (newsolv_mg.for:2-102): initial
calvel/calmas, then V-cycles + FP64 projection until the relative rmax
reaches the workload's tolerance.  Metric: Poisson solves per second.

Default workload (the multi-block FP64 configuration): a 256^3 channel split
into 2x2x2 blocks of 128^3, periodic in x and z, walls in y with tanh
wall-normal stretching (factor 2.0), velocity = seeded uniform [-1,1] noise +
4 smooth Fourier modes of amplitude 0.1, 6 multigrid levels, red-black
smoother (2 pre-, 1 post-sweeps), tolerance 1e-10 relative to the initial
rmax.  Synthetic data with the configuration's shapes and distributions.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints ONE JSON line (rank 0).  ``value`` = device-resident solves/s summed
over ranks (inputs already in HBM; every step restores p, u, v, w from a
pristine device copy first), ``e2e`` = the same through the host-array C
entry point ``mf3d_newsolv_mg`` (pinned host buffers, all host<->device
copies inside the timed call).  Multi-GPU: independent replicas (the solve
has no inter-GPU exchange), ``scaling: weak``.

``--impl reference`` times the reference's CPU path - the oracle, a literal
C++ restatement of the Fortran (the Fortran itself cannot be compiled here) -
on the host cores, one outer iteration per step, and converts to solves/s
with the iteration count the same solve takes.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "poisson_solves_per_s_fp64"
NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e, NVIDIA's DGX figure (the measured copy peak is the roofline's denominator)
UNIT = "solves/s"


def workload_config():
    return {
        "workload": "fp64 multi-block channel 2x2x2 blocks of 128^3 (256^3), tanh y-stretch 2.0, "
                    "6 levels, RB-GS(2,1), rel tol 1e-10",
        "blocks": [2, 2, 2], "block_cells": [128, 128, 128], "global_cells": [256, 256, 256],
        "ngrid": 6, "smoother": "rbgs", "irestr": 2, "iproln": 1, "tol_rel": 1e-10,
        "stretch_y": 2.0, "precision": "fp64", "bc": "periodic x,z; walls y",
        "l2": "inputs larger than L2 (level-1 arrays 268 MB, fields 1.2 GB)",
    }


def make_problem():
    from multiflow3d_b200.problems import Problem
    h = 1.0 / 256
    return Problem(2, 2, 2, 128, 128, 128, ngrid=6, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)


SEED = 2024
FOURIER = 4


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(p):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                return float(parts[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, device=None) -> float:
    """The largest of every rank's x (one all-reduce; x itself alone).
    Replicas only: ranks never exchange data, so the whole job takes as long
    as its slowest rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(steps: int, seconds: float, device=None) -> float:
    """Whole-job throughput of N independent replicas: N * steps over the
    slowest rank's time."""
    import torch.distributed as dist
    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    return world * steps / max_over_ranks(seconds, device)


def oracle_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_bridge
    lib = oracle_bridge.load()
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_set_timestamps.argtypes = [C.POINTER(C.c_double), C.c_int]
    return lib


def time_oracle_iterations(pr, n_iter: int, threads: int, lsm: int = 0, scheme: int = 3):
    """Run the oracle's newsolv_mg for n_iter outer iterations on the full
    workload; returns (seconds of the initial calvel/calmas, per-iteration
    seconds list).  lsm: variable density (densities as run_density's);
    scheme: mg_itrsch."""
    import numpy as np
    from multiflow3d_b200.abi import SolveInfo
    from multiflow3d_b200.problems import fields_struct
    orc = oracle_lib()
    orc.orc_set_threads(threads)
    blocks = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    if lsm:
        for f, dn in zip(blocks, pr.block_density(SEED + 1)):
            f["dens"] = dn
    stamps = np.zeros(n_iter + 4)
    orc.orc_set_timestamps(stamps.ctypes.data_as(C.POINTER(C.c_double)), len(stamps))
    prm = pr.params(mg_itrsch=scheme, irestr=2, iproln=1, maxcy=n_iter, eps=1e-300, lsm=lsm)
    info = SolveInfo()
    hist = np.zeros(n_iter)
    orc.orc_newsolv_mg(pr.descriptors(orc), pr.nblocks, C.byref(prm), fields_struct(blocks), 1.0, 1.0,
                       C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), n_iter)
    orc.orc_set_timestamps(None, 0)
    t_init = float(stamps[1] - stamps[0])
    iters = [float(x) for x in np.diff(stamps[1:info.iter + 2])]
    return t_init, iters


def reference_iterations():
    """Outer iterations the default workload takes to converge (the oracle
    and the GPU path agree bit for bit; recorded by oracle/count_iterations.py)."""
    p = os.path.join(ROOT, "oracle", "bench_iterations.json")
    with open(p) as f:
        return int(json.load(f)["iterations"])


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    pr = make_problem()
    threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
    n = args.warmup + args.steps
    t_init, its = time_oracle_iterations(pr, n, threads)
    timed = its[args.warmup:args.warmup + args.steps]
    t_it = sum(timed) / len(timed)
    I = reference_iterations()
    per_solve = t_init + I * t_it
    value = 1.0 / per_solve
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_it * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} timed outer iterations (after {args.warmup} warm-up) of the full "
                                   f"256^3 solve on the oracle (C++ restatement of the Fortran; blocks on "
                                   f"{threads} threads as the reference's one-rank-per-block MPI); solves/s = "
                                   f"1/(t_init {t_init:.3f}s + {I} iterations x {t_it:.3f}s)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args):
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.solver import Projection

    world, rank, local = dist_setup()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    lib = abi.load()

    pr = make_problem()
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p", "su")
    d = [{k: torch.from_numpy(f[k]).to(dev) for k in keys} for f in host]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in d]
    for f in d:
        f["su"] = None  # the final su is not requested
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-10, eps_relative=1, device=local)
    proj = Projection(pr.descriptors(lib), prm, lib)
    tuning = {g: proj.tuning(g) for g in range(1, pr.ngrid + 1)}

    def reset():
        for f, p0 in zip(d, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        reset()
        r = proj.newsolv_mg_device(d)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    iters, launches, statuses = [], 0, []
    for _ in range(args.steps):
        reset()
        r = proj.newsolv_mg_device(d)
        iters.append(r.iter)
        statuses.append(r.status)
        launches += proj.launches
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, dev)
    value = world * args.steps / (ms_max / 1e3)

    # ---- kernel timing: one more solve per kernel class, each launch of the
    # class bracketed by CUDA events on the library's stream (a solve with
    # timing on runs the outer loop from the host instead of as one graph) ----
    kernels = {}
    for name, kind in (("k_rbgs", abi.MF3D_PROF_SMOOTH_L1), ("k_calvel_calmas", abi.MF3D_PROF_CALMAS),
                       ("k_restrict", abi.MF3D_PROF_RESTRICT_L1), ("k_prolong", abi.MF3D_PROF_PROLONG_L1)):
        proj.profile(kind)
        reset()
        proj.newsolv_mg_device(d)
        kernels[name] = proj.profile_read()
    proj.profile(abi.MF3D_PROF_OFF)
    k_ms, k_n, k_bytes = kernels["k_rbgs"]

    # ---- end to end through the host-array C entry point (pinned buffers) ----
    pinned = [{k: torch.from_numpy(f[k]).pin_memory() for k in keys if k != "su"} for f in host]
    pin_p0 = [{k: f[k].clone().pin_memory() for k in ("u", "v", "w", "p")} for f in pinned]
    hfields = [{k: t.numpy() for k, t in f.items()} for f in pinned]
    for f in hfields:
        f["su"] = None
    arr = (abi.Fields * pr.nblocks)()
    dp = C.POINTER(C.c_double)
    for b, f in enumerate(hfields):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p"):
            setattr(arr[b], k, f[k].ctypes.data_as(dp))
    n_e2e = max(1, args.steps)
    e2e_s = 0.0
    for step in range(n_e2e + 1):
        for f, p0 in zip(pinned, pin_p0):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])
        barrier()
        t0 = time.perf_counter()
        r2 = proj._run(lib.mf3d_newsolv_mg, arr, 1.0, 1.0)
        t1 = time.perf_counter()
        if step > 0:  # first call allocates the library's device mirrors
            e2e_s += t1 - t0
    e2e_s = max_over_ranks(e2e_s, dev)
    e2e_value = world * n_e2e / e2e_s
    ttc = int(np.prod(pr.ttc))
    h2d = 7 * ttc * 8 * pr.nblocks
    d2h = 4 * ttc * 8 * pr.nblocks
    proj.close()

    if rank == 0:
        peak, peak_kind = measured_peaks()
        achieved = (k_bytes / (k_ms / 1e3)) / 1e9 if k_ms > 0 else None
        per_launch_bytes = k_bytes / k_n if k_n else None
        traffic = ncu_traffic("k_rbgs")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(),
            "iterations_per_solve": iters[0] if iters else None, "status": statuses[0] if statuses else None,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm",
                         "kernel": "k_rbgs<double, false> (finest-level red/black half-sweep: reads the other "
                                   "colour and rhs, writes its own colour, 12 B per cell)",
                         "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "frac_nominal": (achieved / NOMINAL_HBM_GBS) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes_per_launch": per_launch_bytes,
                         "launches": k_n, "avg_launch_ms": (k_ms / k_n) if k_n else None,
                         "other_kernels": {n: {"avg_launch_ms": v[0] / v[1] if v[1] else None,
                                               "GB/s": (v[2] / (v[0] / 1e3)) / 1e9 if v[0] > 0 else None,
                                               "frac": (v[2] / (v[0] / 1e3)) / 1e9 / peak if v[0] > 0 else None,
                                               "frac_nominal": ((v[2] / (v[0] / 1e3)) / 1e9 / NOMINAL_HBM_GBS
                                                                if v[0] > 0 else None),
                                               "launches_per_solve": v[1]}
                                           for n, v in kernels.items() if n != "k_rbgs"}},
            "clocks": clocks.summary(),
            "tuning": tuning,
        }
        if world == 1 and not args.no_cpu_baseline:
            threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
            t_init, its = time_oracle_iterations(pr, 2, threads)
            t_it = sum(its) / len(its)
            I = iters[0]
            cpu_val = 1.0 / (t_init + I * t_it)
            line["cpu_baseline"] = {
                "value": cpu_val, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": f"2 outer iterations of the same 256^3 solve on the oracle (C++ restatement of the "
                          f"reference's Fortran path, blocks on {threads} threads); solves/s = "
                          f"1/(t_init {t_init:.3f}s + {I} iterations x {t_it:.3f}s)"}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Further workloads (not the default line): mixed precision on the
# single-block 512x256x256 channel, and the batch of 64 uneven domains.
# ---------------------------------------------------------------------------
def _timed_solves(run_once, reset, steps, warmup):
    import torch
    for _ in range(warmup):
        reset()
        run_once()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    out = None
    ev0.record()
    for _ in range(steps):
        reset()
        out = run_once()
    ev1.record()
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / 1e3, out


def run_probe(args):
    """A short solve of the bench's layout at a chosen block edge, for
    profiler captures of one kernel (not a benchmark line): 2x2x2 blocks of
    n^3 with the bench's y-stretch and fields, `--probe-iters` outer
    iterations, the default launch path (MF3D_NO_GRAPH=1 launches every
    kernel on the stream, which a profiler can see)."""
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import Problem
    from multiflow3d_b200.solver import Projection
    n = args.probe_cells
    h = 1.0 / 256
    pr = Problem(2, 2, 2, n, n, n, ngrid=6 if n % 32 == 0 else 5, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)
    lib = abi.load()
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    dev = [{k: torch.from_numpy(f[k]).cuda() for k in keys} for f in host]
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=args.probe_iters, eps=1e-10, eps_relative=1, device=0)
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg_device(dev)
    torch.cuda.synchronize()
    proj.close()
    print(json.dumps({"workload": "probe", "block_cells": n, "iterations": res.iter, "status": res.status,
                      "ms_device": res.ms_device}))
    return 0


def lmr_layout(lib, n=96):
    """2x2x2 unit-cube blocks, walls around, block 0 at refinement 2 (twice
    the cells and half the spacing over the same extents, rdiv = 2); the
    others n^3.  Returns the descriptors; ngrd_gl = 6 (ngrid_input 5)."""
    import numpy as np
    from multiflow3d_b200.abi import BlockDesc
    ext = np.array([[i, i + 1, j, j + 1, k, k + 1] for k in range(2) for j in range(2) for i in range(2)],
                   dtype=np.float64).ravel()
    arr = (BlockDesc * 8)()
    fn = getattr(lib, "mf3d_build_topology", None) or getattr(lib, "orc_build_topology")
    h = 1.0 / n
    if fn(8, ext.ctypes.data_as(C.POINTER(C.c_double)), (C.c_int * 6)(*([4] * 6)), C.c_double(h), C.c_double(h),
          C.c_double(h), arr) != 0:
        raise RuntimeError("topology")
    d = arr[0]
    d.nx, d.ny, d.nz = 2 * n, 2 * n, 2 * n
    d.dx, d.dy, d.dz = h / 2, h / 2, h / 2
    return arr


def run_lmr(args):
    """The V-cycle across a 2:1 refinement interface (LMR): 2x2x2 blocks,
    one at twice the resolution (192^3 beside seven 96^3, 13.3 M cells),
    walls, 6 levels, RB-GS(2,1), FP64, mf3d_mgkcyc_device on device arrays.
    A step is one V-cycle on a seeded right-hand side.  CPU baseline: the
    oracle's mgkcyc on the same inputs, one thread per block."""
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.abi import Params
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    n, pl = 96, 2
    desc = lmr_layout(lib, n)
    prm = Params(ngrid=6, mg_itrsch=3, irestr=2, iproln=1, maxcy=1, eps=1e-8, eps_relative=1, pl=pl,
                 differencing=1, precision=0)
    shapes = [(desc[b].nz + 2 * pl, desc[b].ny + 2 * pl, desc[b].nx + 2 * pl) for b in range(8)]
    rng = np.random.default_rng(SEED)
    su_h = [rng.uniform(-1, 1, size=sh) for sh in shapes]
    su = [torch.from_numpy(a).to(dev) for a in su_h]
    pp = [torch.zeros(sh, dtype=torch.float64, device=dev) for sh in shapes]

    def timed(precision):
        prm.precision = precision
        proj = Projection(desc, prm, lib)

        def once():
            for t in pp:
                t.zero_()
            proj.mgkcyc_device(su, pp)

        for _ in range(args.warmup):
            once()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            once()
        e1.record()
        torch.cuda.synchronize()
        launches = proj.launches
        proj.close()
        prm.precision = abi.MF3D_PREC_FP64
        return e0.elapsed_time(e1) / 1e3, launches

    # the FP32 V-cycle (coarsest level in FP64) first: pp then holds its result
    sec32, _ = timed(abi.MF3D_PREC_FP32)
    pp32 = [t.cpu().numpy() for t in pp]
    sec, launches = timed(abi.MF3D_PREC_FP64)
    cells = sum(desc[b].nx * desc[b].ny * desc[b].nz for b in range(8))
    value = args.steps / sec
    line = {
        "metric": "lmr_vcycles_per_s_fp64", "value": value, "unit": "V-cycles/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"LMR 2:1: 2x2x2 unit blocks, one at {2 * n}^3 beside seven {n}^3 ({cells / 1e6:.1f} M "
                               f"cells), walls, 6 levels, RB-GS(2,1), one V-cycle (mgkcyc) per step"},
        "gpu_launches_per_step": launches,
        "fp32_vcycle": {"value": args.steps / sec32, "unit": "V-cycles/s",
                        "note": "the same V-cycle in FP32, coarsest level in FP64"},
    }
    if not args.no_cpu_baseline:
        orc = oracle_lib()
        threads = max(1, min(os.cpu_count() or 1, 8))
        orc.orc_set_threads(threads)
        odesc = lmr_layout(orc, n)
        pp_h = [np.zeros(sh) for sh in shapes]
        import oracle_bridge
        t0 = time.perf_counter()
        st = orc.orc_mgkcyc(odesc, 8, C.byref(prm), oracle_bridge.ptr_array(su_h), oracle_bridge.ptr_array(pp_h))
        t1 = time.perf_counter()
        line["cpu_baseline"] = {"value": 1.0 / (t1 - t0), "unit": "V-cycles/s", "cores": threads, "kind": "port",
                                "sample": f"one V-cycle of the same inputs on the oracle ({threads} threads)",
                                "status": st}
        line["speedup_vs_cpu"] = value * (t1 - t0)
        # the first device V-cycle equals the oracle's bit for bit
        for t in pp:
            t.zero_()
        proj2 = Projection(desc, prm, lib)
        proj2.mgkcyc_device(su, pp)
        proj2.close()
        line["bitwise_vs_oracle"] = all(np.array_equal(pp[b].cpu().numpy(), pp_h[b]) for b in range(8))
        # the FP32 V-cycle's largest deviation from the FP64 oracle, over max |pp|
        scale = max(np.abs(a).max() for a in pp_h)
        line["fp32_vcycle"]["max_err_rel_to_max_pp"] = max(np.abs(pp32[b] - pp_h[b]).max() for b in range(8)) / scale
    print(json.dumps(line), flush=True)
    return 0


def run_mixed(args):
    """Single block 512x256x256, tanh y-stretch 2.0, 7 levels, tol 1e-8: the
    FP32 V-cycle (FP64 coarsest level, FP64 outer loop) against the FP64 form
    on the same inputs; error of the mixed result against the FP64 one."""
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import Problem
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    h = 1.0 / 256
    pr = Problem(1, 1, 1, 512, 256, 256, ngrid=7, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    d = [{k: torch.from_numpy(f[k]).to(dev) for k in keys} for f in host]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in d]

    def reset():
        for f, p0 in zip(d, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    res = {}
    for name, prec in (("mixed", abi.MF3D_PREC_FP32), ("fp64", abi.MF3D_PREC_FP64)):
        prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-8, precision=prec)
        proj = Projection(pr.descriptors(lib), prm, lib)
        sec, r = _timed_solves(lambda: proj.newsolv_mg_device(d), reset, args.steps, args.warmup)
        proj.close()
        res[name] = (args.steps / sec, r, {k: d[0][k].cpu().numpy() for k in ("p", "u", "v", "w")})
    pm, pf = res["mixed"][2]["p"], res["fp64"][2]["p"]
    pm, pf = pm - pm.mean(), pf - pf.mean()
    err_p = float(np.linalg.norm(pm - pf) / np.linalg.norm(pf))
    err_uvw = max(float(np.abs(res["mixed"][2][k] - res["fp64"][2][k]).max() / np.abs(res["fp64"][2][k]).max())
                  for k in ("u", "v", "w"))
    line = {
        "metric": "poisson_solves_per_s_mixed", "value": res["mixed"][0], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32 V-cycle, f64 outer",
        "data": "synthetic",
        "config": {"workload": "mixed precision single block 512x256x256, tanh y-stretch 2.0, 7 levels, "
                               "RB-GS(2,1), rel tol 1e-8"},
        "iterations": res["mixed"][1].iter, "rel_rmax": res["mixed"][1].rmax / res["mixed"][1].rmax0,
        "fp64_same_config": {"value": res["fp64"][0], "iterations": res["fp64"][1].iter},
        "speedup_vs_fp64": res["mixed"][0] / res["fp64"][0],
        "error_vs_fp64": {"p_rel_l2_mean_free": err_p, "uvw_max_rel": err_uvw},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_density(args):
    """Variable density (the reference's L_LSM branches): 2x2x2 blocks of
    64^3 (128^3), uniform spacing, densities i.i.d. uniform in [0.5, 2],
    5 levels, RB-GS(2,1), rel tol 1e-8, FP64.  The CPU baseline is the
    oracle on the same inputs, 8 threads (one per block), timed over a
    bounded number of outer iterations and scaled to the GPU's iteration
    count (the two agree bit for bit)."""
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import Problem
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    h = 1.0 / 128
    pr = Problem(2, 2, 2, 64, 64, 64, ngrid=5, pl=2, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    dens = pr.block_density(SEED + 1)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    d = [{**{k: torch.from_numpy(f[k]).to(dev) for k in keys}, "dens": torch.from_numpy(dn).to(dev)}
         for f, dn in zip(host, dens)]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in d]

    def reset():
        for f, p0 in zip(d, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=5000, eps=1e-8, lsm=1)
    proj = Projection(pr.descriptors(lib), prm, lib)
    sec, r = _timed_solves(lambda: proj.newsolv_mg_device(d), reset, args.steps, args.warmup)
    proj.close()
    value = args.steps / sec
    line = {
        "metric": "poisson_solves_per_s_variable_density", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "variable density (L_LSM), 2x2x2 blocks of 64^3 (128^3), uniform h, density "
                               "U[0.5,2], 5 levels, RB-GS(2,1), rel tol 1e-8"},
        "iterations": r.iter, "status": r.status, "rel_rmax": r.rmax / r.rmax0,
        "ms_per_iteration": sec / args.steps * 1e3 / max(r.iter, 1),
    }
    if not args.no_cpu_baseline:
        threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
        t_init, its = time_oracle_iterations(pr, 12, threads, lsm=1)
        t_it = sum(its[2:]) / len(its[2:])
        cpu = 1.0 / (t_init + r.iter * t_it)
        line["cpu_baseline"] = {"value": cpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"10 timed outer iterations of the same solve on the oracle "
                                          f"({threads} threads), scaled to {r.iter} iterations"}
        line["speedup_vs_cpu"] = value / cpu
    print(json.dumps(line), flush=True)
    return 0


def run_linegs(args):
    """The reference's default smoother, line Gauss-Seidel with Thomas
    solves (mg_itrsch 2, control.cin), on the default workload's problem:
    2x2x2 blocks of 128^3 (256^3), tanh y-stretch 2.0, 6 levels, (2,1)
    sweeps, rel tol 1e-10, FP64.  CPU baseline: the oracle on the same
    inputs, 8 threads (one per block), a bounded number of outer iterations
    scaled to the GPU's iteration count (the two agree bit for bit)."""
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    pr = make_problem()
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    d = [{k: torch.from_numpy(f[k]).to(dev) for k in keys} for f in host]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in d]

    def reset():
        for f, p0 in zip(d, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    prm = pr.params(mg_itrsch=2, irestr=2, iproln=1, maxcy=400, eps=1e-10, eps_relative=1)
    proj = Projection(pr.descriptors(lib), prm, lib)
    sec, r = _timed_solves(lambda: proj.newsolv_mg_device(d), reset, args.steps, args.warmup)
    proj.close()
    value = args.steps / sec
    line = {
        "metric": "poisson_solves_per_s_line_gs", "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "line Gauss-Seidel (mg_itrsch 2), 2x2x2 blocks of 128^3 (256^3), tanh y-stretch "
                               "2.0, 6 levels, (2,1) sweeps, rel tol 1e-10"},
        "iterations": r.iter, "status": r.status, "rel_rmax": r.rmax / r.rmax0,
        "ms_per_iteration": sec / args.steps * 1e3 / max(r.iter, 1),
    }
    if not args.no_cpu_baseline:
        threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
        t_init, its = time_oracle_iterations(pr, 3, threads, scheme=2)
        t_it = sum(its[1:]) / len(its[1:])
        cpu = 1.0 / (t_init + r.iter * t_it)
        line["cpu_baseline"] = {"value": cpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"2 timed outer iterations of the same solve on the oracle "
                                          f"({threads} threads), scaled to {r.iter} iterations"}
        line["speedup_vs_cpu"] = value / cpu
    print(json.dumps(line), flush=True)
    return 0


def run_rungek(args):
    """The velocity predictor upstream of the projection: one Runge-Kutta
    stage of rungek_conv2nd + rungek_diff2nd (boundu/v/w included) on
    2x2x2 blocks of 128^3 (256^3), uniform spacing, periodic x and z, walls
    in y, FP64.  value: stages/s with every field resident on the device;
    GB/s counts u, v, w, uoo, voo, woo, vis read and ustar, vstar, wstar
    written once per interior cell (80 B).  CPU baseline: the oracle's
    stage on the same inputs, 8 threads (one per block)."""
    import ctypes as C
    import time
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.abi import RkFields
    from multiflow3d_b200.problems import Problem, fields_struct
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    h = 1.0 / 256
    pr = Problem(2, 2, 2, 128, 128, 128, ngrid=6, pl=2, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    rng = np.random.default_rng(SEED)
    rk = [{"uoo": f["u"] + 0.01, "voo": f["v"] - 0.01, "woo": f["w"] + 0.02,
           "vis": 1e-3 * (1.0 + rng.random(f["u"].shape))} for f in host]
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    d = [{k: torch.from_numpy(f[k]).to(dev) for k in keys} for f in host]
    drk = [{k: torch.from_numpy(r[k]).to(dev) for k in r} for r in rk]
    prm = pr.params(bounds=1, alfabc=1)
    proj = Projection(pr.descriptors(lib), prm, lib)
    fa = (abi.Fields * pr.nblocks)()
    ra = (RkFields * pr.nblocks)()
    dp = C.POINTER(C.c_double)
    for b in range(pr.nblocks):
        for k in keys:
            setattr(fa[b], k, C.cast(C.c_void_p(d[b][k].data_ptr()), dp))
        for k in ("uoo", "voo", "woo", "vis"):
            setattr(ra[b], k, C.cast(C.c_void_p(drk[b][k].data_ptr()), dp))
    dt, alfapr = 1e-3, 0.5

    def stage():
        abi.check(lib, lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfapr, 1, 0, 0.0), "mf3d_rungek_2nd_device")

    for _ in range(args.warmup):
        stage()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        stage()
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    launches = lib.mf3d_last_launch_count(proj.ctx)
    proj.close()
    cells = pr.NX * pr.NY * pr.NZ
    line = {
        "metric": "rk_stages_per_s", "value": args.steps / sec, "unit": "stages/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "velocity predictor, one RK stage (rungek_conv2nd + rungek_diff2nd + boundu/v/w), "
                               "2x2x2 blocks of 128^3 (256^3), periodic x z, walls y"},
        "GB_per_s_algorithmic": 80.0 * cells / (sec / args.steps) / 1e9, "gpu_launches_per_step": launches,
    }
    if not args.no_cpu_baseline:
        orc = oracle_lib()
        threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
        orc.orc_set_threads(threads)
        ra_h = (RkFields * pr.nblocks)()
        for b, r in enumerate(rk):
            for k in ("uoo", "voo", "woo", "vis"):
                setattr(ra_h[b], k, r[k].ctypes.data_as(dp))
        blocks = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
        t = time.perf_counter()
        orc.orc_rungek_2nd(pr.descriptors(orc), pr.nblocks, C.byref(prm), fields_struct(blocks), ra_h, dt, alfapr,
                           1, 0, 0.0)
        cpu = 1.0 / (time.perf_counter() - t)
        line["cpu_baseline"] = {"value": cpu, "unit": "stages/s", "cores": threads, "kind": "port",
                                "sample": "one stage on the same inputs on the oracle"}
        line["speedup_vs_cpu"] = line["value"] / cpu
    print(json.dumps(line), flush=True)
    return 0


def run_sip(args):
    """solver 1 (pressure_1sweep with Stone's SIP): 2x2x2 blocks of 32^3
    (64^3), periodic x and z, walls in y, 4 SIP sweeps per call, rel tol
    1e-8, FP64.  CPU baseline: the oracle on the same inputs, 8 threads,
    the whole solve."""
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.abi import SolveInfo
    from multiflow3d_b200.problems import Problem, fields_struct
    from multiflow3d_b200.solver import Projection
    lib = abi.load()
    dev = torch.device("cuda:0")
    h = 1.0 / 64
    pr = Problem(2, 2, 2, 32, 32, 32, ngrid=1, pl=1, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    d = [{k: torch.from_numpy(f[k]).to(dev) for k in keys} for f in host]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in d]

    def reset():
        for f, p0 in zip(d, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    prm = pr.params(maxcy=2000, eps=1e-8, solver=1, nswp=4)
    proj = Projection(pr.descriptors(lib), prm, lib)
    sec, r = _timed_solves(lambda: proj.newsolv_mg_device(d), reset, args.steps, args.warmup)
    proj.close()
    value = args.steps / sec
    line = {
        "metric": "poisson_solves_per_s_sip", "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "solver 1 (SIP), 2x2x2 blocks of 32^3 (64^3), periodic x z, walls y, nswp 4, "
                               "rel tol 1e-8"},
        "sip_calls": r.iter, "status": r.status,
    }
    if not args.no_cpu_baseline:
        import time
        orc = oracle_lib()
        threads = max(1, min(os.cpu_count() or 1, pr.nblocks))
        orc.orc_set_threads(threads)
        blocks = pr.block_fields(seed=SEED, fourier_modes=FOURIER)
        info = SolveInfo()
        t = time.perf_counter()
        orc.orc_newsolv_mg(pr.descriptors(orc), pr.nblocks, C.byref(prm), fields_struct(blocks), 1.0, 1.0,
                           C.byref(info), None, 0)
        cpu = 1.0 / (time.perf_counter() - t)
        line["cpu_baseline"] = {"value": cpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": "the same solve on the oracle (the SIP sweeps are serial per block)"}
        line["speedup_vs_cpu"] = value / cpu
    print(json.dumps(line), flush=True)
    return 0


def run_tecbin(args):
    """Restart files (post.for:496-548 / initial.for:689-760): decode the
    file images of the default workload's 8 blocks (ttc 132^3 each, 0.44 GB
    per file) on the device.  value: GB of file image per second with the
    images resident in HBM; e2e: the same from pinned host memory, copy
    included.  CPU baseline: the numpy restatement of the reader
    (oracle/tecbin.py) on one block."""
    import torch
    from multiflow3d_b200 import abi
    lib = abi.load()
    dev = torch.device("cuda:0")
    n, nblk = 132, args.files
    # the synthetic restart image, written by the library's own encoder
    g = torch.Generator(device=dev).manual_seed(SEED)
    fields = [torch.randn((n, n, n), dtype=torch.float64, device=dev, generator=g) for _ in range(16)]
    xyz = [(torch.arange(n, dtype=torch.float64, device=dev) - 2) / 256.0 for _ in range(3)]
    nbytes = int(lib.mf3d_tecbin_size(n, n, n))
    img0 = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    fptr = (C.c_void_p * 16)(*[t.data_ptr() for t in fields])
    assert lib.mf3d_tecbin_encode_device(n, n, n, 2, 0, -1, 0, *[C.c_void_p(t.data_ptr()) for t in xyz], fptr,
                                         C.c_void_p(img0.data_ptr()), 0) == 0
    pinned = img0.cpu().pin_memory()
    host_img = pinned.numpy().tobytes()
    info = abi.TecbinInfo()
    assert lib.mf3d_tecbin_info_of(host_img, nbytes, C.byref(info)) == 0
    imgs = [img0] + [pinned.to(dev) for _ in range(nblk - 1)]
    outs = [torch.empty((n, n, n), dtype=torch.float64, device=dev) for _ in range(16)]
    ptrs = (C.c_void_p * 16)(*[o.data_ptr() for o in outs])

    def decode(img):
        st = lib.mf3d_tecbin_decode_device(C.c_void_p(img.data_ptr()), C.byref(info), ptrs, 0)
        assert st == 0, abi.last_error(lib)

    for _ in range(args.warmup):
        for img in imgs:
            decode(img)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        for img in imgs:
            decode(img)
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3 / args.steps
    value = nblk * nbytes / sec / 1e9
    # end to end: pinned host image -> device -> fields
    stage = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        for _b in range(nblk):
            stage.copy_(pinned, non_blocking=True)
            decode(stage)
    e1.record()
    torch.cuda.synchronize()
    sec_e2e = e0.elapsed_time(e1) / 1e3 / args.steps
    # algorithmic bytes of one decode: the image read, 16 of the 19 doubles written
    alg = nbytes + 16 * n ** 3 * 8
    peak, peak_src = measured_peaks()
    line = {
        "metric": "tecbin_decode_gb_per_s", "value": value, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "dtype": "u32 words / f64",
        "data": "synthetic",
        "config": {"workload": f"{nblk} restart files of ttc {n}^3 (pl 2), {nbytes / 1e9:.3f} GB each, decoded "
                               "into the 16 fields the reader keeps"},
        "e2e": {"value": nblk * nbytes / sec_e2e / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nblk * nbytes,
                "d2h_bytes_per_step": 0},
        "roofline": {"bound": "hbm", "achieved": alg * nblk / sec / 1e9, "peak": peak, "peak_source": peak_src,
                     "unit": "GB/s", "frac": alg * nblk / sec / 1e9 / peak, "traffic": None},
    }
    if not args.no_cpu_baseline:
        import time
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import tecbin as orc_tb
        t = time.perf_counter()
        orc_tb.read(host_img)
        cpu = nbytes / (time.perf_counter() - t) / 1e9
        line["cpu_baseline"] = {"value": cpu, "unit": "GB/s", "cores": 1, "kind": "port",
                                "sample": "numpy restatement of the reader (oracle/tecbin.py) on one file"}
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """64 independent domains (edges log-uniform in [32,192], multiples of 8,
    periodic/wall per axis), tol 1e-8: one mixed-precision batch context
    against the same batch in FP64 and against plain FP64 solves one at a
    time (one context per domain)."""
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import domain_problem, domain_desc, random_batch
    from multiflow3d_b200.solver import Batch
    lib = abi.load()
    dev = torch.device("cuda:0")
    doms = [domain_problem(nx, ny, nz, bc, lib.mf3d_max_levels(nx, ny, nz))
            for nx, ny, nz, bc in random_batch(64, SEED)]
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    fields = [{k: torch.from_numpy(v).to(dev) for k, v in pr.block_fields(seed=SEED + i)[0].items() if k in keys}
              for i, pr in enumerate(doms)]
    pristine = [{k: f[k].clone() for k in ("u", "v", "w", "p")} for f in fields]

    def reset():
        for f, p0 in zip(fields, pristine):
            for k in ("u", "v", "w", "p"):
                f[k].copy_(p0[k])

    out = {}
    for name, prec in (("mixed", abi.MF3D_PREC_FP32), ("fp64", abi.MF3D_PREC_FP64)):
        prm = doms[0].params(mg_itrsch=3, maxcy=300, eps=1e-8, precision=prec)
        prm.ngrid = 1
        b = Batch([domain_desc(pr) for pr in doms], prm, lib)
        sec, r = _timed_solves(lambda: b.solve_device(fields), reset, args.steps, args.warmup)
        b.close()
        rs, st = r
        out[name] = (len(doms) * args.steps / sec, sum(x.status == 0 for x in rs), max(x.iter for x in rs))
    # plain FP64, one domain at a time
    prm = doms[0].params(mg_itrsch=3, maxcy=300, eps=1e-8, precision=abi.MF3D_PREC_FP64)
    prm.ngrid = 1
    solo = [Batch([domain_desc(pr)], prm, lib) for pr in doms]

    def one_at_a_time():
        for b, f in zip(solo, fields):
            b.solve_device([f])

    sec, _ = _timed_solves(one_at_a_time, reset, args.steps, args.warmup)
    for b in solo:
        b.close()
    plain = len(doms) * args.steps / sec
    line = {
        "metric": "poisson_solves_per_s_batched", "value": out["mixed"][0], "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32 V-cycle, f64 outer",
        "data": "synthetic",
        "config": {"workload": "64 domains, edges log-uniform in [32,192] (multiples of 8), periodic/wall per "
                               "axis, max levels per domain, RB-GS(2,1), rel tol 1e-8, one batch context"},
        "converged": out["mixed"][1], "max_iterations": out["mixed"][2],
        "fp64_batch": {"value": out["fp64"][0], "converged": out["fp64"][1]},
        "plain_fp64_one_at_a_time": {"value": plain},
        "speedup_vs_plain": out["mixed"][0] / plain,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_served(args):
    """Poisson arrivals at each rate of --rates: sizes as the batched
    workload plus 10 % 384^3 requests, mixed precision at 1e-8, admission
    capped at 150 GB of resident hierarchies.  Per rate, --requests requests;
    latency = completion - submission on the server's clock.  Baseline:
    plain FP64 solves one at a time, run over the same arrival trace and
    measured (each request starts at its arrival or when the one before it
    ends, whichever is later)."""
    import numpy as np
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import domain_problem, domain_desc, random_batch, WALL, PERIODIC
    from multiflow3d_b200.solver import Server, Batch
    lib = abi.load()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(SEED)
    small = [domain_problem(nx, ny, nz, bc, lib.mf3d_max_levels(nx, ny, nz))
             for nx, ny, nz, bc in random_batch(64, SEED)]
    large = [domain_problem(384, 384, 384, bc, lib.mf3d_max_levels(384, 384, 384))
             for bc in ((PERIODIC, WALL, PERIODIC), (WALL, WALL, WALL))]
    templates = small + large
    ro = ("ustar", "vstar", "wstar")
    rw = ("u", "v", "w", "p")
    tmpl = []
    for i, pr in enumerate(templates):
        f = pr.block_fields(seed=SEED + 1000 + i)[0]
        tmpl.append({k: torch.from_numpy(f[k]).to(dev) for k in ro + rw})

    def fresh(i):
        t = tmpl[i]
        d = {k: t[k] for k in ro}
        for k in rw:
            d[k] = t[k].clone()
        return d

    def draw(n):
        big = rng.random(n) < 0.10
        return [int(len(small) + rng.integers(0, len(large))) if b else int(rng.integers(0, len(small))) for b in big]

    prm = small[0].params(mg_itrsch=3, maxcy=400, eps=1e-8, precision=abi.MF3D_PREC_FP32)
    # baseline: plain FP64 solves one at a time, one warm context per domain
    # shape (graphs captured before the timed runs)
    p64 = small[0].params(mg_itrsch=3, maxcy=400, eps=1e-8, precision=abi.MF3D_PREC_FP64)
    p64.ngrid = 1
    solo = []
    for i, pr in enumerate(templates):
        b = Batch([domain_desc(pr)], p64, lib)
        b.solve_device([fresh(i)])  # warm-up (graph capture)
        solo.append(b)
    torch.cuda.synchronize()

    def fifo(arrivals, kinds):
        """The trace served by the baseline, measured: each request waits for
        its arrival and for the one before it, then runs alone."""
        lat = []
        t0 = time.perf_counter()
        for a, kind in zip(arrivals, kinds):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            f = fresh(kind)
            torch.cuda.synchronize()
            solo[kind].solve_device([f])
            torch.cuda.synchronize()
            lat.append(time.perf_counter() - t0 - a)
        return np.array(lat), time.perf_counter() - t0
    rates = [float(x) for x in args.rates.split(",")]
    traces = []
    for lam in rates:
        kinds = draw(args.requests)
        gaps = rng.exponential(1.0 / lam, size=args.requests)
        traces.append((lam, kinds, np.cumsum(gaps) - gaps[0]))
    # the baseline first, over every trace; its contexts are freed before the
    # server runs, so the two never hold device memory at once
    base = [fifo(arrivals, kinds) for _, kinds, arrivals in traces]
    for b in solo:
        b.close()
    solo.clear()
    torch.cuda.synchronize()
    field_bytes = [sum(tmpl[i][k].numel() * 8 for k in rw) for i in range(len(templates))]
    held_cap = 48e9  # the caller's own copies of u, v, w, p of the requests in flight
    results = []
    for (lam, kinds, arrivals), (lb, span_b) in zip(traces, base):
        srv = Server(prm, mem_cap_bytes=150e9, max_resident=512, lib=lib)
        # warm the server's kernels with one small request
        w0 = fresh(0)
        torch.cuda.synchronize()
        w = srv.submit(domain_desc(templates[0]), w0)
        while srv.poll(w, wait_ms=50)[0] == abi.MF3D_PENDING:
            pass
        held, tickets, kind_of, done = {}, [], {}, {}
        held_bytes = 0.0

        def reap(wait_ms):
            """Collect the finished requests; sleep wait_ms when none was."""
            nonlocal held_bytes
            got = False
            for t in list(held):
                st, info = srv.poll(t, wait_ms=0)
                if st != abi.MF3D_PENDING:
                    done[t] = (st, info)
                    held.pop(t)
                    held_bytes -= field_bytes[kind_of[t]]
                    got = True
            if not got:
                time.sleep(wait_ms / 1e3)
        t0 = time.perf_counter()
        s0 = srv.clock()
        for a, kind in zip(arrivals, kinds):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            # back-pressure on the caller's copies: the request still counts
            # from its arrival
            while held and held_bytes + field_bytes[kind] > held_cap:
                reap(1)
            f = fresh(kind)
            torch.cuda.current_stream().synchronize()  # the server's streams do not order after ours
            t = srv.submit(domain_desc(templates[kind]), f)
            held[t] = f
            held_bytes += field_bytes[kind]
            kind_of[t] = kind
            tickets.append((t, s0 + a))
        while held:
            reap(2)
        stats = srv.stats()
        prof = srv.profile()
        srv.close()
        lat = np.array([done[t][1].t_done - arr for t, arr in tickets])
        t_first = min(arr for _, arr in tickets)
        t_last = max(done[t][1].t_done for t, _ in tickets)
        ok = sum(done[t][0] == abi.MF3D_OK for t, _ in tickets)
        results.append({
            "rate_per_s": lam, "requests": len(tickets), "large": int(sum(k >= len(small) for k in kinds)),
            "converged": int(ok), "throughput": len(tickets) / (t_last - t_first),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "cycles": stats["cycles"], "worker_s": prof,
            "plain_fp64_fifo": {"throughput": len(tickets) / span_b, "p50_s": float(np.percentile(lb, 50)),
                                "p99_s": float(np.percentile(lb, 99))},
        })
    line = {
        "metric": "served_solves_per_s", "value": results[-1]["throughput"], "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32 V-cycle, f64 outer", "data": "synthetic",
        "config": {"workload": "Poisson arrivals; sizes as the batched workload plus 10% 384^3; mixed precision "
                               "tol 1e-8; admission cap 150 GB; continuous batching (one outer iteration per cycle)"},
        "rates": results,
        "baseline_note": "plain FP64 one-at-a-time, measured: the same arrival trace run request by request "
                         "(each waits for its arrival and for the one before it) on warm FP64 contexts; "
                         "latencies of both from the request's arrival",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mf3d", choices=["mf3d", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="multiblock",
                    choices=["multiblock", "mixed", "batched", "served", "density", "tecbin", "sip", "linegs",
                             "rungek", "probe", "lmr"],
                    help="multiblock: the default FP64 line; mixed / batched / served / density: the further "
                         "workloads (1 GPU)")
    ap.add_argument("--rates", default="50,200,800", help="served: arrival rates per second")
    ap.add_argument("--requests", type=int, default=1000, help="served: requests per rate")
    ap.add_argument("--files", type=int, default=8, help="tecbin: restart files decoded per step")
    ap.add_argument("--probe-cells", type=int, default=96, help="probe: block edge of the 2x2x2 layout")
    ap.add_argument("--probe-iters", type=int, default=3, help="probe: outer iterations")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "probe":
        return run_probe(args)
    if args.workload == "lmr":
        return run_lmr(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "served":
        return run_served(args)
    if args.workload == "density":
        return run_density(args)
    if args.workload == "tecbin":
        return run_tecbin(args)
    if args.workload == "sip":
        return run_sip(args)
    if args.workload == "linegs":
        return run_linegs(args)
    if args.workload == "rungek":
        return run_rungek(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())

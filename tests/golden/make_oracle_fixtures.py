"""Writes tests/golden/oracle_fullsize.json: the oracle's results on the
benchmark configurations at their full sizes, for the GPU parity tests that
the oracle is too slow to run inline (tests/test_gpu_fullsize.py).

Test infrastructure: runs the CPU oracle (oracle/_build/liboracle.so, the
literal restatement of newsolv_mg.for:2-102 and mgsolver.for) on the same
seeded inputs the benchmark uses, and records per case

  - ``status``, ``iterations``, ``rmax0`` and the raw per-iteration rmax
    history (newsolv_mg.for:23-56 computes one rmax per outer iteration);
    Python's float repr round-trips, so the JSON values are the oracle's bits;
  - ``p_sha256``: SHA-256 of the final pressure's interior, assembled into one
    global (NZ, NY, NX) float64 C-order array (``Problem.gather``), so that a
    GPU pressure with the same digest is the oracle's pressure bit for bit;
  - ``p_norm`` and ``p_samples`` (8 fixed cells), readable spot values.

Cases:
  config2_stretched  2x2x2 blocks of 128^3, tanh y-stretch 2.0, 6 levels, tol 1e-10
  config2_uniform    the same without stretching (the reference's own grid)
  config3_fp64       one block of 512x256x256, stretched, 7 levels, tol 1e-8
  config4_batch      the benchmark's 64 domains (edges log-uniform in
                     [32, 192], multiples of 8), tol 1e-8, maxcy 300, each
                     domain solved alone

    python tests/golden/make_oracle_fixtures.py [case ...]   # about 15 minutes on 8 cores

Existing cases in the file are kept unless named on the command line.
"""
import ctypes as C
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "oracle_fullsize.json")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

SAMPLE_FRACS = [(0.1, 0.2, 0.3), (0.5, 0.5, 0.5), (0.9, 0.05, 0.7), (0.0, 0.0, 0.0),
                (0.99, 0.99, 0.99), (0.25, 0.75, 0.5), (0.6, 0.01, 0.2), (0.33, 0.66, 0.99)]


def p_digest(pg: np.ndarray) -> dict:
    """Digest of a global interior pressure (NZ, NY, NX), float64."""
    a = np.ascontiguousarray(pg, dtype=np.float64)
    nz, ny, nx = a.shape
    samples = []
    for fz, fy, fx in SAMPLE_FRACS:
        k, j, i = min(int(fz * nz), nz - 1), min(int(fy * ny), ny - 1), min(int(fx * nx), nx - 1)
        samples.append([k, j, i, float(a[k, j, i])])
    return {"p_sha256": hashlib.sha256(a.tobytes()).hexdigest(), "p_norm": float(np.linalg.norm(a)),
            "p_samples": samples}


def solve(pr, prm, seed, fourier, threads):
    import oracle_bridge
    from multiflow3d_b200.abi import SolveInfo
    from multiflow3d_b200.problems import fields_struct
    orc = oracle_bridge.load()
    orc.orc_set_threads.argtypes = [C.c_int]
    orc.orc_set_threads(threads)
    blocks = pr.block_fields(seed=seed, fourier_modes=fourier)
    info = SolveInfo()
    hist = np.zeros(prm.maxcy)
    t0 = time.time()
    st = orc.orc_newsolv_mg(pr.descriptors(orc), pr.nblocks, C.byref(prm), fields_struct(blocks), 1.0, 1.0,
                            C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), prm.maxcy)
    out = {"status": int(st), "iterations": int(info.iter), "rmax0": float(info.rmax0), "rmax": float(info.rmax),
           "history": [float(x) for x in hist[:info.iter]], "seconds": round(time.time() - t0, 1)}
    out.update(p_digest(pr.gather(blocks, "p")))
    return out


def case_config2(stretch):
    import bench
    from multiflow3d_b200.problems import Problem
    h = 1.0 / 256
    pr = Problem(2, 2, 2, 128, 128, 128, ngrid=6, pl=2, stretch_y=stretch, dx=h, dy=h, dz=h)
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-10, eps_relative=1)
    r = solve(pr, prm, bench.SEED, bench.FOURIER, 8)
    r["config"] = (f"2x2x2 blocks of 128^3 (256^3), {'tanh y-stretch 2.0' if stretch else 'uniform'}, 6 levels, "
                   f"RB-GS(2,1), rel tol 1e-10, seed {bench.SEED}, {bench.FOURIER} Fourier modes")
    return r


def case_config3():
    import bench
    from multiflow3d_b200.problems import Problem
    h = 1.0 / 256
    pr = Problem(1, 1, 1, 512, 256, 256, ngrid=7, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-8)
    r = solve(pr, prm, bench.SEED, bench.FOURIER, 1)
    r["config"] = (f"one block of 512x256x256, tanh y-stretch 2.0, 7 levels, RB-GS(2,1), rel tol 1e-8, "
                   f"seed {bench.SEED}, {bench.FOURIER} Fourier modes, FP64")
    return r


def batch_domains():
    import bench
    from multiflow3d_b200 import abi
    from multiflow3d_b200.problems import domain_problem, random_batch
    lib = abi.load()
    return [domain_problem(nx, ny, nz, bc, lib.mf3d_max_levels(nx, ny, nz))
            for nx, ny, nz, bc in random_batch(64, bench.SEED)]


def _batch_one(i):
    import bench
    pr = batch_domains()[i]
    prm = pr.params(mg_itrsch=3, maxcy=300, eps=1e-8)
    r = solve(pr, prm, bench.SEED + i, 0, 1)
    r["shape"] = [pr.nx, pr.ny, pr.nz]
    r["bc"] = [pr.bc[0], pr.bc[2], pr.bc[4]]
    r["ngrid"] = pr.ngrid
    return r


def case_config4():
    import bench
    n = len(batch_domains())
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        doms = pool.map(_batch_one, range(n), chunksize=1)
    return {"config": f"64 domains from random_batch(64, {bench.SEED}) (edges log-uniform in [32,192], multiples "
                      f"of 8, periodic/wall per axis, max levels), fields seed {bench.SEED}+i, RB-GS(2,1), "
                      f"rel tol 1e-8, maxcy 300, FP64, each domain alone",
            "domains": doms}


CASES = {
    "config2_stretched": lambda: case_config2(2.0),
    "config2_uniform": lambda: case_config2(0.0),
    "config3_fp64": case_config3,
    "config4_batch": case_config4,
}


def main():
    names = sys.argv[1:] or list(CASES)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names:
        t0 = time.time()
        data[name] = CASES[name]()
        print(name, f"{time.time() - t0:.0f}s", flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=0)


if __name__ == "__main__":
    main()

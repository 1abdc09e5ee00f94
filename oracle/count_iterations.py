"""Test infrastructure: records how many outer iterations the benchmark's
default workload takes to converge on the oracle, for bench.py's reference
arm (which times a bounded number of iterations and scales by this count).

    python oracle/count_iterations.py      # writes oracle/bench_iterations.json

The GPU path reproduces the oracle's iterates bit for bit, so the count is
the same on both; bench.py's GPU arm reports its own count alongside.
"""
import ctypes as C
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def main():
    import bench
    from multiflow3d_b200.abi import SolveInfo
    from multiflow3d_b200.problems import fields_struct
    orc = bench.oracle_lib()
    pr = bench.make_problem()
    orc.orc_set_threads(max(1, min(os.cpu_count() or 1, pr.nblocks)))
    blocks = pr.block_fields(seed=bench.SEED, fourier_modes=bench.FOURIER)
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=1000, eps=1e-10, eps_relative=1)
    info = SolveInfo()
    hist = np.zeros(prm.maxcy)
    t0 = time.time()
    st = orc.orc_newsolv_mg(pr.descriptors(orc), pr.nblocks, C.byref(prm), fields_struct(blocks), 1.0, 1.0,
                            C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), prm.maxcy)
    out = {"iterations": int(info.iter), "status": int(st), "rmax0": info.rmax0, "rmax": info.rmax,
           "workload": bench.workload_config()["workload"], "seconds": round(time.time() - t0, 1),
           "rel_history": [float(x) for x in hist[:info.iter] / info.rmax0]}
    with open(os.path.join(ROOT, "oracle", "bench_iterations.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out["iterations"], out["status"], out["seconds"])


if __name__ == "__main__":
    main()

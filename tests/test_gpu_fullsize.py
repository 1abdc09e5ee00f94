"""The benchmark configurations at their full sizes.

Parity against the oracle: tests/golden/oracle_fullsize.json holds the
oracle's results on exactly these inputs (written by
tests/golden/make_oracle_fixtures.py, which runs the oracle for minutes):
per case the iteration count, the raw per-iteration rmax history
(newsolv_mg.for:23-56) and a SHA-256 digest of the final pressure.  The GPU
FP64 solves must reproduce all three bit for bit:
- the 256^3 multi-block solve, tanh-stretched (the benchmark's workload) and
  uniform (the grid the reference itself supports);
- the 512x256x256 single block in FP64, against which the mixed-precision
  solve of the same inputs is then measured (the FP64 oracle, via the
  digest-equal GPU pressure): relative L2 of p (mean removed) <= 1e-8;
- the 64-domain batch (edges log-uniform in [32, 192]), every domain; the
  mixed-precision batch then within 1e-8 of it per domain.

Size-independent properties as well: the final rmax the solve reports
equals max |div(u) * volume| recomputed from the returned u, v, w with plain
FP64 tensor arithmetic in calmas' operation order (press.for:46-62), bit for
bit, and the 1024^3 single block converges with the same bitwise check."""
import json
import os
import sys

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.problems import Problem, domain_desc
from multiflow3d_b200.solver import Projection, Batch

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
from make_oracle_fixtures import p_digest  # noqa: E402

MIXED_BAR = 1e-8  # relative L2 of p (mean removed) of a mixed-precision solve against the FP64 oracle


def fixture(name):
    with open(os.path.join(GOLDEN, "oracle_fullsize.json")) as f:
        data = json.load(f)
    if name not in data:
        pytest.fail(f"oracle fixture {name} missing: run tests/golden/make_oracle_fixtures.py {name}")
    return data[name]


def assert_matches_fixture(fx, status, iters, history, p_global):
    assert status == fx["status"], (status, fx["status"])
    assert iters == fx["iterations"], (iters, fx["iterations"])
    assert np.array_equal(np.asarray(history), np.asarray(fx["history"])), "rmax history differs from the oracle"
    dg = p_digest(p_global)
    for (k, j, i, v), (_, _, _, vr) in zip(dg["p_samples"], fx["p_samples"]):
        assert v == vr, ((k, j, i), v, vr)
    assert dg["p_sha256"] == fx["p_sha256"], "pressure differs from the oracle"


def rel_mean_free(a, b):
    a = a - a.mean()
    b = b - b.mean()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def recomputed_rmax(pr, dev, cuda):
    """max |fact*hx*hy*hz| over every interior cell, fact = (u(i)-u(i-1))/hx
    + (v(j)-v(j-1))/hy + (w(k)-w(k-1))/hz from the returned fields."""
    import torch
    pl, nx, ny, nz = pr.pl, pr.nx, pr.ny, pr.nz
    best = torch.zeros((), dtype=torch.float64, device=cuda)
    for b, f in enumerate(dev):
        hyb = pr.block_widths_y(b)
        W = 1 << (pr.ngrid - 1)
        hy = torch.from_numpy(np.ascontiguousarray(hyb[W:W + ny])).to(cuda).view(1, ny, 1) if hyb is not None \
            else torch.full((1, ny, 1), pr.dy, dtype=torch.float64, device=cuda)
        K, J, I = slice(pl, pl + nz), slice(pl, pl + ny), slice(pl, pl + nx)
        u, v, w = f["u"], f["v"], f["w"]
        du = u[K, J, I] - u[K, J, pl - 1:pl + nx - 1]
        dv = v[K, J, I] - v[K, pl - 1:pl + ny - 1, I]
        dw = w[K, J, I] - w[pl - 1:pl + nz - 1, J, I]
        fact = du / pr.dx + dv / hy + dw / pr.dz
        best = torch.maximum(best, (fact * pr.dx * hy * pr.dz).abs().max())
    return float(best.item())


def _solve_256cube(lib, cuda, stretch):
    import torch
    sys.path.insert(0, ROOT)
    import bench
    h = 1.0 / 256
    pr = Problem(2, 2, 2, 128, 128, 128, ngrid=6, pl=2, stretch_y=stretch, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=bench.SEED, fourier_modes=bench.FOURIER)
    dev = [{k: torch.from_numpy(f[k]).to(cuda) for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p")}
           for f in host]
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-10)
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg_device(dev)
    proj.close()
    return pr, dev, res


def test_fp64_multiblock_256cube(lib, cuda):
    """The benchmark's workload (config 2, tanh-stretched): bit for bit the
    oracle's 91 iterations, rmax history and pressure."""
    pr, dev, res = _solve_256cube(lib, cuda, 2.0)
    assert res.status == 0 and res.rmax < 1e-10 * res.rmax0
    assert recomputed_rmax(pr, dev, cuda) == res.rmax
    pg = pr.gather([{"p": f["p"].cpu().numpy()} for f in dev], "p")
    assert_matches_fixture(fixture("config2_stretched"), res.status, res.iter, res.history, pg)
    # the history the benchmark's reference arm scales by (oracle/bench_iterations.json)
    with open(os.path.join(ROOT, "oracle", "bench_iterations.json")) as f:
        bi = json.load(f)
    assert res.iter == bi["iterations"]
    assert np.array_equal(res.history / res.rmax0, np.asarray(bi["rel_history"]))


def test_fp64_multiblock_256cube_uniform(lib, cuda):
    """Config 2 on the uniform grid, the variant the reference itself can
    express (localparameters.for:245-247): the parity gate at full size."""
    pr, dev, res = _solve_256cube(lib, cuda, 0.0)
    assert res.status == 0 and res.rmax < 1e-10 * res.rmax0
    pg = pr.gather([{"p": f["p"].cpu().numpy()} for f in dev], "p")
    assert_matches_fixture(fixture("config2_uniform"), res.status, res.iter, res.history, pg)


def test_mixed_precision_512x256x256(lib, cuda):
    """Config 3: the FP64 solve equals the oracle bit for bit; the mixed
    solve (FP32 V-cycle, FP64 coarsest level and outer loop) of the same
    inputs reaches the same relative rmax and lies within 1e-8 of it."""
    import torch
    sys.path.insert(0, ROOT)
    import bench
    h = 1.0 / 256
    pr = Problem(1, 1, 1, 512, 256, 256, ngrid=7, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=bench.SEED, fourier_modes=bench.FOURIER)
    out = {}
    for name, prec in (("fp64", abi.MF3D_PREC_FP64), ("mixed", abi.MF3D_PREC_FP32)):
        dev = [{k: torch.from_numpy(f[k]).to(cuda) for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p")}
               for f in host]
        proj = Projection(pr.descriptors(lib), pr.params(maxcy=400, eps=1e-8, precision=prec), lib)
        res = proj.newsolv_mg_device(dev)
        proj.close()
        assert res.status == 0 and res.rmax < 1e-8 * res.rmax0
        assert recomputed_rmax(pr, dev, cuda) == res.rmax
        out[name] = (res, pr.interior(dev[0]["p"].cpu().numpy()),
                     {k: dev[0][k].cpu().numpy() for k in ("u", "v", "w")})
        del dev
    res64, p64, _ = out["fp64"]
    assert_matches_fixture(fixture("config3_fp64"), res64.status, res64.iter, res64.history, p64)
    err = rel_mean_free(out["mixed"][1], p64)
    assert err <= MIXED_BAR, err
    for k in ("u", "v", "w"):
        a, b = out["mixed"][2][k], out["fp64"][2][k]
        assert np.abs(a - b).max() <= MIXED_BAR * np.abs(b).max()


def test_batch_config4_matches_oracle(lib, cuda):
    """Config 4: the benchmark's 64 domains (edges log-uniform in [32, 192],
    multiples of 8, periodic/wall per axis, the most levels each allows) in
    one FP64 batch context: every domain's status, iterations, rmax history
    and pressure equal the oracle's solo solve.  The mixed-precision batch
    of the same domains then lies within 1e-8 of it per converged domain."""
    import torch
    sys.path.insert(0, ROOT)
    import bench
    from make_oracle_fixtures import batch_domains
    fx = fixture("config4_batch")["domains"]
    doms = batch_domains()
    assert [[d.nx, d.ny, d.nz] for d in doms] == [x["shape"] for x in fx]
    keys = ("ustar", "vstar", "wstar", "u", "v", "w", "p")
    host = [pr.block_fields(seed=bench.SEED + i)[0] for i, pr in enumerate(doms)]
    ps = {}
    for name, prec in (("fp64", abi.MF3D_PREC_FP64), ("mixed", abi.MF3D_PREC_FP32)):
        fields = [{k: torch.from_numpy(h[k]).to(cuda) for k in keys} for h in host]
        prm = doms[0].params(mg_itrsch=3, maxcy=300, eps=1e-8, precision=prec)
        prm.ngrid = 1
        b = Batch([domain_desc(pr) for pr in doms], prm, lib)
        res, st = b.solve_device(fields)
        b.close()
        assert st >= 0
        ps[name] = (res, [pr.interior(f["p"].cpu().numpy()) for pr, f in zip(doms, fields)])
    res64, p64 = ps["fp64"]
    for d in range(len(doms)):
        assert_matches_fixture(fx[d], res64[d].status, res64[d].iter, res64[d].history, p64[d])
    resm, pm = ps["mixed"]
    for d in range(len(doms)):
        if res64[d].status != 0:
            continue
        assert resm[d].status == 0 and resm[d].rmax < 1e-8 * resm[d].rmax0, d
        assert rel_mean_free(pm[d], p64[d]) <= MIXED_BAR, d


def test_fp64_1024cube_single_block(lib, cuda):
    """The largest single block this layout holds in one GPU's memory with
    room to spare: 1024^3 cells (ttc 1028^3, 1.09 G elements per field;
    about 80 GB for the seven fields and the multigrid hierarchy), FP64,
    8 levels, periodic x and z, walls in y, tol 1e-8.  Inputs are made on
    the device (uniform random face velocities, mean removed, zero normal
    velocity on the walls).  The reported rmax is recomputed bit for bit from
    the returned velocities, slab by slab."""
    import torch
    n, pl = 1024, 2
    pr = Problem(1, 1, 1, n, n, n, ngrid=8, pl=pl, dx=1 / n, dy=1 / n, dz=1 / n)
    t = n + 2 * pl
    g = torch.Generator(device=cuda).manual_seed(11)
    f = {}
    for k in ("ustar", "vstar", "wstar"):
        a = torch.rand((t, t, t), dtype=torch.float64, device=cuda, generator=g).mul_(2).sub_(1)
        a.sub_(a[pl:pl + n, pl:pl + n, pl:pl + n].mean())
        f[k] = a
    f["vstar"][:, pl - 1, :] = 0.0
    f["vstar"][:, pl + n - 1, :] = 0.0
    for k in ("u", "v", "w"):
        f[k] = f[k + "star"].clone()
    f["p"] = torch.zeros((t, t, t), dtype=torch.float64, device=cuda)
    proj = Projection(pr.descriptors(lib), pr.params(maxcy=400, eps=1e-8), lib)
    res = proj.newsolv_mg_device([f])
    proj.close()
    assert res.status == 0 and res.rmax < 1e-8 * res.rmax0
    del f["ustar"], f["vstar"], f["wstar"], f["p"]
    h = 1.0 / n
    best = 0.0
    for k0 in range(pl, pl + n, 128):
        K = slice(k0, k0 + 128)
        J, I = slice(pl, pl + n), slice(pl, pl + n)
        u, v, w = f["u"], f["v"], f["w"]
        fact = ((u[K, J, I] - u[K, J, pl - 1:pl + n - 1]) / h + (v[K, J, I] - v[K, pl - 1:pl + n - 1, I]) / h +
                (w[K, J, I] - w[k0 - 1:k0 + 127, J, I]) / h)
        best = max(best, float((fact * h * h * h).abs().max().item()))
        del fact
    assert best == res.rmax

"""The benchmark configurations at full size, checked through properties
that do not need the oracle (which would take minutes there): the final
rmax the solve reports equals max |div(u) * volume| recomputed from the
returned u, v, w with plain FP64 tensor arithmetic in calmas' operation
order (press.for:46-62), bit for bit; the solve converged to the
tolerance; and the mixed-precision solve of the 512x256x256 channel lands
within 1e-8 of the FP64 one."""
import os
import sys

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.problems import Problem
from multiflow3d_b200.solver import Projection

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def test_fp64_multiblock_256cube(lib, cuda):
    import torch
    sys.path.insert(0, ROOT)
    import bench
    pr = bench.make_problem()
    host = pr.block_fields(seed=bench.SEED, fourier_modes=bench.FOURIER)
    dev = [{k: torch.from_numpy(f[k]).to(cuda) for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p")}
           for f in host]
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, maxcy=400, eps=1e-10)
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg_device(dev)
    proj.close()
    assert res.status == 0 and res.rmax < 1e-10 * res.rmax0
    assert np.all(np.diff(res.history[:5]) < 0)
    assert recomputed_rmax(pr, dev, cuda) == res.rmax


def test_mixed_precision_512x256x256(lib, cuda):
    import torch
    h = 1.0 / 256
    pr = Problem(1, 1, 1, 512, 256, 256, ngrid=7, pl=2, stretch_y=2.0, dx=h, dy=h, dz=h)
    host = pr.block_fields(seed=5, fourier_modes=4)
    out = {}
    for name, prec in (("fp64", abi.MF3D_PREC_FP64), ("mixed", abi.MF3D_PREC_FP32)):
        dev = [{k: torch.from_numpy(f[k]).to(cuda) for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p")}
               for f in host]
        proj = Projection(pr.descriptors(lib), pr.params(maxcy=400, eps=1e-8, precision=prec), lib)
        res = proj.newsolv_mg_device(dev)
        proj.close()
        assert res.status == 0
        assert recomputed_rmax(pr, dev, cuda) == res.rmax
        p = dev[0]["p"][2:-2, 2:-2, 2:-2]
        out[name] = p - p.mean()
    err = float((out["mixed"] - out["fp64"]).norm() / out["fp64"].norm())
    assert err < 1e-8, err


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

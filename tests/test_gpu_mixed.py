"""Mixed precision: the V-cycle in FP32 (coarsest level in FP64) inside the
FP64 defect-correction loop.  The outer residual, p += pp and the velocity
projection stay FP64, so the solve reaches the same relative rmax as the
FP64 path and its result matches the FP64 oracle to far below the solver
tolerance.  Bars, stated per case: the same stopping rule (rel rmax < tol),
at most 2 more outer iterations than the oracle, and relative L2 of p (mean
removed: these problems have a floating constant) and max relative error of
u, v, w at most 1e-9."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.abi import SolveInfo
from multiflow3d_b200.problems import Problem, fields_struct, domain_problem, domain_desc, random_batch, WALL, PERIODIC
from multiflow3d_b200.solver import Projection, Batch

pytestmark = pytest.mark.gpu

ERR_BAR = 1e-9


def rel_mean_free(a, b):
    a = a - a.mean()
    b = b - b.mean()
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def oracle_solve(oracle, pr, prm, seed):
    ref = pr.block_fields(seed=seed, fourier_modes=4)
    info = SolveInfo()
    hist = np.zeros(prm.maxcy)
    st = oracle.orc_newsolv_mg(pr.descriptors(oracle), pr.nblocks, C.byref(prm), fields_struct(ref), 1.0, 1.0,
                               C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), prm.maxcy)
    assert st == 0
    return ref, info


CASES = [
    ("config 1: 64x32x32, 4 levels", Problem(1, 1, 1, 64, 32, 32, ngrid=4, pl=2), 1e-8),
    ("2x2x2 blocks of 16^3, stretched", Problem(2, 2, 2, 16, 16, 16, ngrid=4, pl=2, stretch_y=2.0,
                                              dx=1 / 32, dy=1 / 32, dz=1 / 32), 1e-8),
    ("2x1x1 blocks of 32x16x16, walls", Problem(2, 1, 1, 32, 16, 16, bc=(WALL,) * 6, ngrid=3, pl=1), 1e-10),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_mixed_matches_fp64_oracle(lib, oracle, cuda, case):
    import torch
    _, pr, tol = case
    ref, info = oracle_solve(oracle, pr, pr.params(mg_itrsch=3, maxcy=300, eps=tol), seed=5)
    prm = pr.params(mg_itrsch=3, maxcy=300, eps=tol, precision=abi.MF3D_PREC_FP32)
    blocks = pr.block_fields(seed=5, fourier_modes=4)
    dev = [{k: torch.from_numpy(v).to(cuda) for k, v in f.items()} for f in blocks]
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg_device(dev)
    proj.close()
    got = [{k: v.cpu().numpy() for k, v in f.items()} for f in dev]
    assert res.status == 0 and res.rmax < tol * res.rmax0
    assert res.iter <= info.iter + 2
    assert rel_mean_free(pr.gather(got, "p"), pr.gather(ref, "p")) <= ERR_BAR
    for k in ("u", "v", "w"):
        g, r = pr.gather(got, k), pr.gather(ref, k)
        assert np.abs(g - r).max() <= ERR_BAR * np.abs(r).max()


SMOOTHER_CASES = [
    ("line GS, 2x1x1 blocks of 64^3 (8-CTA clusters at level 1)", 2,
     Problem(2, 1, 1, 64, 64, 64, ngrid=4, pl=2, stretch_y=2.0), 1e-8),
    ("line GS, config 1: 64x32x32", 2, Problem(1, 1, 1, 64, 32, 32, ngrid=4, pl=2), 1e-8),
    ("lex GS, 2x1x1 blocks of 32x32x64 (8-CTA clusters at level 1)", 1,
     Problem(2, 1, 1, 32, 32, 64, bc=(WALL,) * 6, ngrid=3, pl=1), 1e-8),
]


@pytest.mark.parametrize("case", SMOOTHER_CASES, ids=[c[0] for c in SMOOTHER_CASES])
def test_mixed_other_smoothers(lib, oracle, cuda, case):
    """The FP32 line and lexicographic relaxations (mgsolver.for:403-545),
    clustered and not, against the FP64 oracle with the same smoother, to
    the bars above."""
    import torch
    _, sch, pr, tol = case
    ref, info = oracle_solve(oracle, pr, pr.params(mg_itrsch=sch, maxcy=300, eps=tol), seed=6)
    prm = pr.params(mg_itrsch=sch, maxcy=300, eps=tol, precision=abi.MF3D_PREC_FP32)
    blocks = pr.block_fields(seed=6, fourier_modes=4)
    dev = [{k: torch.from_numpy(v).to(cuda) for k, v in f.items()} for f in blocks]
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg_device(dev)
    proj.close()
    got = [{k: v.cpu().numpy() for k, v in f.items()} for f in dev]
    assert res.status == 0 and res.rmax < tol * res.rmax0
    assert res.iter <= info.iter + 2
    assert rel_mean_free(pr.gather(got, "p"), pr.gather(ref, "p")) <= ERR_BAR
    for k in ("u", "v", "w"):
        g, r = pr.gather(got, k), pr.gather(ref, k)
        assert np.abs(g - r).max() <= ERR_BAR * np.abs(r).max()


@pytest.mark.parametrize("same_depth", [True, False])
def test_mixed_batch(lib, cuda, same_depth):
    """A batch in mixed precision (FP64 coarsest level only when every domain
    bottoms out on the same level) converges like the FP64 batch."""
    import torch
    if same_depth:
        shapes = [(32, 32, 32, (PERIODIC, WALL, PERIODIC)), (64, 32, 32, (WALL, WALL, WALL)),
                  (32, 64, 32, (PERIODIC, PERIODIC, PERIODIC)), (48, 32, 64, (WALL, PERIODIC, WALL))]
        doms = [domain_problem(nx, ny, nz, bc, 3) for nx, ny, nz, bc in shapes]
    else:
        doms = [domain_problem(nx, ny, nz, bc, lib.mf3d_max_levels(nx, ny, nz))
                for nx, ny, nz, bc in random_batch(6, 4, lo=16, hi=64)]
    out = {}
    for prec in (abi.MF3D_PREC_FP64, abi.MF3D_PREC_FP32):
        prm = doms[0].params(mg_itrsch=3, maxcy=200, eps=1e-8, precision=prec)
        prm.ngrid = 1
        b = Batch([domain_desc(pr) for pr in doms], prm, lib)
        fields = [{k: torch.from_numpy(v).to(cuda) for k, v in pr.block_fields(seed=30 + d)[0].items()}
                  for d, pr in enumerate(doms)]
        res, st = b.solve_device(fields)
        b.close()
        out[prec] = (res, [f["p"].cpu().numpy() for f in fields])
    r64, p64 = out[abi.MF3D_PREC_FP64]
    r32, p32 = out[abi.MF3D_PREC_FP32]
    for d, pr in enumerate(doms):
        assert r32[d].status == r64[d].status
        if r64[d].status == 0:
            assert r32[d].iter <= r64[d].iter + 2
            assert rel_mean_free(pr.interior(p32[d]), pr.interior(p64[d])) <= 1e-7

"""The velocity predictor (one Runge-Kutta stage of rungek_conv2nd and
rungek_diff2nd; with differencing = 2 rungek_conv4th and rungek_diff4th;
with 3 rungek_convWENO and rungek_diff2nd) on the GPU against the oracle,
FP64, bit for bit: ustar,
vstar, wstar over their faces and the u, v, w ghosts that boundu/v/w
refresh on the way, for periodic, wall, symmetry, inflow and outflow
faces, both stages' alfabc, and the pressure forcing."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.abi import RkFields
from multiflow3d_b200.problems import Problem, PERIODIC, WALL
from multiflow3d_b200.solver import Projection
from test_gpu_edges import face_mask
from test_rungek import rk_inputs, orc_rk

pytestmark = pytest.mark.gpu
P, W, S = PERIODIC, WALL, 3

CASES = {
    "2x2x1 periodic x y, walls z, first stage, forcing": (
        lambda: Problem(2, 2, 1, 16, 16, 8, bc=(P, P, P, P, W, W), ngrid=2, pl=2), 1, 1, 1),
    "2x1x2 inflow / outflow x, walls y, periodic z, first stage": (
        lambda: Problem(2, 1, 2, 16, 8, 16, bc=(1, 2, W, W, P, P), ngrid=2, pl=3), 2, 1, 0),
    "2x1x1 inflow / convective outflow x, walls y, periodic z, first stage": (
        lambda: Problem(2, 1, 1, 16, 8, 8, bc=(1, 21, W, W, P, P), ngrid=2, pl=2), 1, 1, 0),
    "1 block, walls and symmetry, later stage": (
        lambda: Problem(1, 1, 1, 16, 12, 8, bc=(W, W, S, S, W, W), ngrid=2, pl=2), 1, 0, 0),
}


def dev(t, cuda):
    import torch
    return torch.from_numpy(t.copy()).to(cuda)


CASES4 = {
    "4th order, 2x2x1 periodic x y, walls z, first stage, forcing": (
        lambda: Problem(2, 2, 1, 16, 16, 8, bc=(P, P, P, P, W, W), ngrid=2, pl=3), 1, 1, 1),
    "4th order, 2x1x2 inflow / outflow x, walls y, periodic z, first stage": (
        lambda: Problem(2, 1, 2, 16, 8, 16, bc=(1, 2, W, W, P, P), ngrid=2, pl=3), 2, 1, 0),
    "4th order, 1 block, walls and symmetry, later stage": (
        lambda: Problem(1, 1, 1, 16, 12, 8, bc=(W, W, S, S, W, W), ngrid=2, pl=4), 1, 0, 0),
}


CASESW = {
    "WENO, 2x2x1 periodic x y, walls z, first stage, forcing": (
        lambda: Problem(2, 2, 1, 16, 16, 8, bc=(P, P, P, P, W, W), ngrid=2, pl=4), 2, 1, 1),
    "WENO, 2x1x2 inflow / outflow x, walls y, periodic z, later stage": (
        lambda: Problem(2, 1, 2, 16, 8, 16, bc=(1, 2, W, W, P, P), ngrid=2, pl=4), 2, 0, 0),
}


@pytest.mark.parametrize("case", sorted(CASES) + sorted(CASES4) + sorted(CASESW))
def test_predictor_matches_oracle(lib, oracle, cuda, case):
    import torch
    differencing = 2 if case in CASES4 else 3 if case in CASESW else 1
    make, pl_ex, alfabc, pforce = (CASES4 if differencing == 2 else CASESW if differencing == 3 else CASES)[case]
    pr = make()
    blocks, rk = rk_inputs(pr, 21)
    dt, alfapr, forcn, ubulk = 0.0137, 0.5, 0.31, 0.6
    gpu = [{k: dev(v, cuda) for k, v in f.items()} for f in blocks]
    grk = [{k: dev(v, cuda) for k, v in r.items()} for r in rk]
    assert orc_rk(oracle, pr, blocks, rk, dt, alfapr, alfabc=alfabc, pforce=pforce, forcn=forcn,
                  pl_ex=pl_ex, ubulk=ubulk, differencing=differencing) == 0
    # the context's alfabc is the projection's own (its final boundu/v/w);
    # the stage's comes with each predictor call
    prm = pr.params(pl_ex=pl_ex, bounds=1, alfabc=0, ubulk=ubulk, differencing=differencing)
    proj = Projection(pr.descriptors(lib), prm, lib)
    fa = (abi.Fields * pr.nblocks)()
    ra = (RkFields * pr.nblocks)()
    dp = C.POINTER(C.c_double)
    for b in range(pr.nblocks):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p"):
            setattr(fa[b], k, C.cast(C.c_void_p(gpu[b][k].data_ptr()), dp))
        for k in ("uoo", "voo", "woo", "vis"):
            setattr(ra[b], k, C.cast(C.c_void_p(grk[b][k].data_ptr()), dp))
    st = lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfapr, alfabc, pforce, forcn)
    proj.close()
    assert st == 0, abi.last_error(lib)
    torch.cuda.synchronize()
    pl = pr.pl
    inner = (slice(pl, pl + pr.nz), slice(pl, pl + pr.ny), slice(pl, pl + pr.nx))
    for b in range(pr.nblocks):
        got = {k: v.cpu().numpy() for k, v in gpu[b].items()}
        for k in ("ustar", "vstar", "wstar"):
            assert np.array_equal(got[k][inner], blocks[b][k][inner]), (b, k)
        for k in ("u", "v", "w"):
            m = face_mask(got[k].shape, pl, pl_ex)
            assert np.array_equal(got[k][m], blocks[b][k][m]), (b, k)


def test_predictor_refusals(lib, cuda):
    """Without bounds = 1, or on a stretched grid, the call is refused before any device work."""
    pr = Problem(1, 1, 1, 8, 8, 8, ngrid=1, pl=1)
    proj = Projection(pr.descriptors(lib), pr.params(), lib)
    st = lib.mf3d_rungek_2nd_device(proj.ctx, (abi.Fields * 1)(), (RkFields * 1)(), 0.1, 1.0, 1, 0, 0.0)
    proj.close()
    assert st == abi.MF3D_E_UNSUPPORTED


def test_two_stages_with_calvel_between(lib, oracle, cuda):
    """The reference's stage loop (flosol.for:151-172) with kuttacond = 2:
    predictor (alfabc 1), calvel, predictor (alfabc 0) - mf3d_rungek_2nd_device,
    mf3d_calvel_device, mf3d_rungek_2nd_device on one context against the
    oracle's rungek_2nd, calvel, rungek_2nd."""
    import torch
    from multiflow3d_b200.problems import fields_struct
    pr = Problem(2, 1, 2, 16, 12, 16, bc=(1, 2, W, W, P, P), ngrid=2, pl=2)
    pl_ex, ubulk, dt = 1, 0.4, 0.011
    alfark = (0.5, 1.0)
    blocks, rk = rk_inputs(pr, 23)
    gpu = [{k: dev(v, cuda) for k, v in f.items()} for f in blocks]
    grk = [{k: dev(v, cuda) for k, v in r.items()} for r in rk]
    # oracle
    assert orc_rk(oracle, pr, blocks, rk, dt, alfark[0], alfabc=1, pl_ex=pl_ex, ubulk=ubulk) == 0
    prm_o = pr.params(pl_ex=pl_ex, bounds=1, alfabc=1, ubulk=ubulk)
    assert oracle.orc_calvel(pr.descriptors(oracle), pr.nblocks, C.byref(prm_o), fields_struct(blocks),
                             dt, alfark[0]) == 0
    assert orc_rk(oracle, pr, blocks, rk, dt, alfark[1], alfabc=0, pl_ex=pl_ex, ubulk=ubulk) == 0
    # device
    proj = Projection(pr.descriptors(lib), pr.params(pl_ex=pl_ex, bounds=1, alfabc=1, ubulk=ubulk), lib)
    fa = (abi.Fields * pr.nblocks)()
    ra = (RkFields * pr.nblocks)()
    dp = C.POINTER(C.c_double)
    for b in range(pr.nblocks):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p"):
            setattr(fa[b], k, C.cast(C.c_void_p(gpu[b][k].data_ptr()), dp))
        for k in ("uoo", "voo", "woo", "vis"):
            setattr(ra[b], k, C.cast(C.c_void_p(grk[b][k].data_ptr()), dp))
    assert lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfark[0], 1, 0, 0.0) == 0, abi.last_error(lib)
    assert lib.mf3d_calvel_device(proj.ctx, fa, dt, alfark[0]) == 0, abi.last_error(lib)
    assert lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfark[1], 0, 0, 0.0) == 0, abi.last_error(lib)
    proj.close()
    torch.cuda.synchronize()
    pl = pr.pl
    inner = (slice(pl, pl + pr.nz), slice(pl, pl + pr.ny), slice(pl, pl + pr.nx))
    for b in range(pr.nblocks):
        got = {k: v.cpu().numpy() for k, v in gpu[b].items()}
        for k in ("ustar", "vstar", "wstar"):
            assert np.array_equal(got[k][inner], blocks[b][k][inner]), (b, k)
        for k in ("u", "v", "w"):
            m = face_mask(got[k].shape, pl, pl_ex)
            assert np.array_equal(got[k][m], blocks[b][k][m]), (b, k)


def test_stage_loop_reads_block_edge_ghosts(lib, oracle, cuda):
    """2x2x1 blocks with walls outside: the interior block edges along z join
    four blocks.  The u predictor reads v(i+1,j-1,k) and w(i+1,j,k-1)
    (rungek.for:336-343), which at a block's outer i-edge are the (x,y) and
    (x,z) edge ghosts that calvel's exchange(2), (3) fill from the edge
    neighbour (exchange.for:2231-2397).  Stage (alfabc 1) -> calvel ->
    stage (alfabc 0) on the device against the oracle: ustar, vstar, wstar,
    u, v, w bit for bit on every cell."""
    import torch
    from multiflow3d_b200.problems import fields_struct
    pr = Problem(2, 2, 1, 16, 16, 8, bc=(W,) * 6, ngrid=2, pl=2)
    pl_ex, dt = 1, 0.013
    alfark = (0.5, 1.0)
    blocks, rk = rk_inputs(pr, 37)
    gpu = [{k: dev(v, cuda) for k, v in f.items()} for f in blocks]
    grk = [{k: dev(v, cuda) for k, v in r.items()} for r in rk]
    assert orc_rk(oracle, pr, blocks, rk, dt, alfark[0], alfabc=1, pl_ex=pl_ex) == 0
    prm_o = pr.params(pl_ex=pl_ex, bounds=1, alfabc=1)
    assert oracle.orc_calvel(pr.descriptors(oracle), pr.nblocks, C.byref(prm_o), fields_struct(blocks),
                             dt, alfark[0]) == 0
    assert orc_rk(oracle, pr, blocks, rk, dt, alfark[1], alfabc=0, pl_ex=pl_ex) == 0
    proj = Projection(pr.descriptors(lib), pr.params(pl_ex=pl_ex, bounds=1, alfabc=1), lib)
    fa = (abi.Fields * pr.nblocks)()
    ra = (RkFields * pr.nblocks)()
    dp = C.POINTER(C.c_double)
    for b in range(pr.nblocks):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p"):
            setattr(fa[b], k, C.cast(C.c_void_p(gpu[b][k].data_ptr()), dp))
        for k in ("uoo", "voo", "woo", "vis"):
            setattr(ra[b], k, C.cast(C.c_void_p(grk[b][k].data_ptr()), dp))
    assert lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfark[0], 1, 0, 0.0) == 0, abi.last_error(lib)
    assert lib.mf3d_calvel_device(proj.ctx, fa, dt, alfark[0]) == 0, abi.last_error(lib)
    assert lib.mf3d_rungek_2nd_device(proj.ctx, fa, ra, dt, alfark[1], 0, 0, 0.0) == 0, abi.last_error(lib)
    proj.close()
    torch.cuda.synchronize()
    pl = pr.pl
    for b in range(pr.nblocks):
        got = {k: v.cpu().numpy() for k, v in gpu[b].items()}
        for k in ("ustar", "vstar", "wstar", "u", "v", "w"):
            diff = np.argwhere(got[k] != blocks[b][k])
            assert diff.size == 0, (b, k, len(diff), diff[:4].tolist())

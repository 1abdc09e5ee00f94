"""Variable density (the reference's L_LSM branches) on the GPU against the
oracle, FP64, bit for bit: per-solve coefficients from the density field
(mgsolver.for:69-203), density-weighted calvel (press.for:152-190), the
volume-scaled rhs sup (press.for:51-53), for the three smoothers, several
block layouts and boundary sets, a non-trivial time step, and the host
entry point."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.problems import Problem, PERIODIC, WALL
from multiflow3d_b200.solver import Projection
from test_gpu_edges import run_both, assert_same, face_mask

pytestmark = pytest.mark.gpu
P, W = PERIODIC, WALL


def density_blocks(pr, seed):
    blocks = pr.block_fields(seed=seed, fourier_modes=2)
    for f, d in zip(blocks, pr.block_density(seed + 1)):
        f["dens"] = d
    return blocks


LAYOUTS = {
    "one block": lambda: Problem(1, 1, 1, 16, 16, 16, ngrid=3, pl=1),
    "2x2x1 periodic x y": lambda: Problem(2, 2, 1, 16, 16, 8, bc=(P, P, P, P, W, W), ngrid=3, pl=2),
    "2x1x2 walls": lambda: Problem(2, 1, 2, 16, 8, 16, bc=(W,) * 6, ngrid=3, pl=2),
}


@pytest.mark.parametrize("scheme", [1, 2, 3])
@pytest.mark.parametrize("layout", sorted(LAYOUTS))
def test_variable_density_matches_oracle(lib, oracle, cuda, scheme, layout):
    pr = LAYOUTS[layout]()
    prm = pr.params(mg_itrsch=scheme, maxcy=60, eps=1e-9, lsm=1, pl_ex=pr.pl - 1)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    density_blocks(pr, 5))
    assert_same(o, g, pr.pl, pr.pl - 1)


def test_variable_density_converged_with_time_step(lib, oracle, cuda):
    """A converged solve (hundreds of outer iterations: the reference's
    variable-density coarse levels keep the fine spacings) with dt and
    alfapr that are not powers of two, and differencing = 3 (WENO convection,
    which the reference requires with L_LSM)."""
    pr = Problem(2, 1, 1, 16, 16, 16, ngrid=4, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=1500, eps=1e-10, lsm=1, differencing=3)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    density_blocks(pr, 8), dt=0.37, alfapr=1.3)
    assert o[0] == 0
    assert_same(o, g, pr.pl)


def test_variable_density_host_entry_point(lib, oracle, cuda):
    """mf3d_newsolv_mg on host arrays (dens mirrored with the other fields)
    equals the oracle."""
    pr = Problem(2, 1, 1, 16, 8, 8, ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, lsm=1)
    blocks = density_blocks(pr, 14)
    o, _ = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    host = [{k: v.copy() for k, v in f.items()} for f in blocks]
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg(host)
    proj.close()
    st, info, hist, ref = o
    assert res.status == st and res.iter == info.iter and np.array_equal(res.history, hist)
    for b in range(pr.nblocks):
        for k in ("p", "u", "v", "w"):
            m = face_mask(ref[b][k].shape, pr.pl, 0)
            assert np.array_equal(host[b][k][m], ref[b][k][m]), (b, k)


def test_variable_density_single_vcycle_rejected(lib, cuda):
    """The variable-density coefficients come from a solve's density field:
    a lone V-cycle on such a context is refused."""
    import torch
    pr = Problem(1, 1, 1, 8, 8, 8, ngrid=2, pl=1)
    proj = Projection(pr.descriptors(lib), pr.params(lsm=1), lib)
    t = torch.zeros(pr.ttc, dtype=torch.float64, device=cuda)
    su = (C.POINTER(C.c_double) * 1)(C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)))
    pp = (C.POINTER(C.c_double) * 1)(C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)))
    assert lib.mf3d_mgkcyc_device(proj.ctx, su, pp) == abi.MF3D_E_UNSUPPORTED
    proj.close()

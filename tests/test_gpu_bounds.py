"""boundu/boundv/boundw after the loop (newsolv_mg.for:86-88; `bounds`) on
the GPU against the oracle, FP64, bit for bit.  With at most one periodic
axis every cell of u, v, w matches: the final exchange(1..3) with its full
periodic planes, then the periodic copy and the inflow / outflow / wall /
symmetry faces of the three components.  With two periodic axes the corner cells of the
reference carry values from earlier iterations' exchanges, which the device
path does not replay; there interior and face ghosts are compared."""
import numpy as np
import pytest

from multiflow3d_b200.problems import Problem, PERIODIC, WALL
from test_gpu_edges import run_both, assert_same, face_mask

pytestmark = pytest.mark.gpu
P, W, S = PERIODIC, WALL, 3

ONE_PERIODIC_AXIS = {
    "1 block, periodic x, walls y, symmetry z": (lambda: Problem(1, 1, 1, 16, 16, 16, bc=(P, P, W, W, S, S),
                                                                 ngrid=3, pl=2), 1),
    "2x1x1 periodic partners in x, walls": (lambda: Problem(2, 1, 1, 16, 8, 8, bc=(P, P, W, W, W, W),
                                                            ngrid=3, pl=2), 1),
    "2x2x1 walls and symmetry, no periodic": (lambda: Problem(2, 2, 1, 16, 16, 8, bc=(W, W, S, S, W, W),
                                                              ngrid=3, pl=3), 2),
    "1x2x2 periodic partners in z, symmetry x, walls y": (lambda: Problem(1, 2, 2, 8, 16, 16, bc=(S, S, W, W, P, P),
                                                                          ngrid=3, pl=2), 0),
}


def assert_all_cells(o, g, pl, pl_ex):
    assert_same(o, g, pl, pl_ex)
    ref, got = o[3], g[1]
    for b in range(len(ref)):
        for k in ("u", "v", "w"):
            assert np.array_equal(got[b][k], ref[b][k]), (b, k)


@pytest.mark.parametrize("layout", sorted(ONE_PERIODIC_AXIS))
def test_bounds_every_cell(lib, oracle, cuda, layout):
    make, pl_ex = ONE_PERIODIC_AXIS[layout]
    pr = make()
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=pl_ex, bounds=1)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=31, fourier_modes=2))
    assert_all_cells(o, g, pr.pl, pl_ex)


def test_bounds_two_periodic_axes(lib, oracle, cuda):
    pr = Problem(2, 1, 2, 16, 8, 16, bc=(P, P, W, W, P, P), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=1, bounds=1)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=32, fourier_modes=2))
    assert_same(o, g, pr.pl, 1)


def test_bounds_with_variable_density(lib, oracle, cuda):
    pr = Problem(2, 1, 1, 16, 8, 8, bc=(P, P, W, W, S, S), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=2, maxcy=30, eps=1e-9, pl_ex=1, bounds=1, lsm=1)
    blocks = pr.block_fields(seed=33, fourier_modes=2)
    for f, d in zip(blocks, pr.block_density(34)):
        f["dens"] = d
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    assert_all_cells(o, g, pr.pl, 1)


INFLOW_OUTFLOW = {
    "1 block, inflow west, outflow east, walls y, periodic z":
        (lambda: Problem(1, 1, 1, 16, 16, 16, bc=(1, 2, W, W, P, P), ngrid=3, pl=2), 1, 1),
    "2x1x2, inflow west and bottom, outflow east, symmetry y, wall top":
        (lambda: Problem(2, 1, 2, 16, 8, 16, bc=(1, 2, S, S, 1, W), ngrid=3, pl=3), 2, 1),
    "2x1x1, outflow skipped (alfabc 0)":
        (lambda: Problem(2, 1, 1, 16, 8, 8, bc=(1, 2, W, W, S, S), ngrid=3, pl=2), 1, 0),
}


@pytest.mark.parametrize("layout", sorted(INFLOW_OUTFLOW))
def test_bounds_inflow_outflow_every_cell(lib, oracle, cuda, layout):
    """Codes 1 (inflow: ubulk on the west, 1.1 for w on the bottom) and 2
    (outflow: copy of the last face when alfabc = 1), bounds.for:42-53,
    136-170 and the matching branches of boundv/boundw."""
    make, pl_ex, alfabc = INFLOW_OUTFLOW[layout]
    pr = make()
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=pl_ex, bounds=1, alfabc=alfabc, ubulk=0.7)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=35, fourier_modes=2))
    assert_all_cells(o, g, pr.pl, pl_ex)

"""Line and lexicographic Gauss-Seidel (mg_itrsch 2 and 1) at the block
sizes where the device splits each block over a cluster of CTAs.  Line
Gauss-Seidel (mg_itrsch 2, mgsolver.for:430-545) at the block sizes
where the device sweeps each block's line diagonals with a cluster of CTAs
(lines of 64 cells and more: the slices of a diagonal meet at CTA borders,
where a line reads its neighbour line from another CTA's results) against
the oracle, FP64, bit for bit; and under variable density (per-cell
coefficients) at a size that uses a cluster too."""
import numpy as np
import pytest

from multiflow3d_b200.problems import Problem, PERIODIC, WALL
from test_gpu_edges import run_both, assert_same

pytestmark = pytest.mark.gpu
P, W = PERIODIC, WALL

LAYOUTS = {
    "2x1x1 blocks of 64^3, stretched y": (lambda: Problem(2, 1, 1, 64, 64, 64, ngrid=3, pl=2, stretch_y=2.0), 3),
    "1 block of 128x64x96, walls": (lambda: Problem(1, 1, 1, 128, 64, 96, bc=(W,) * 6, ngrid=3, pl=1), 2),
    # 512-cell lines: a CTA's 64 lines of a diagonal no longer fit in shared
    # memory at once and are staged in groups of 7
    "1 block of 512x64x64, periodic x": (
        lambda: Problem(1, 1, 1, 512, 64, 64, bc=(P, P, W, W, W, W), ngrid=3, pl=1), 2),
    "2x2x1 blocks of 128x128x32, periodic x y": (
        lambda: Problem(2, 2, 1, 128, 128, 32, bc=(P, P, P, P, W, W), ngrid=4, pl=2), 2),
}


@pytest.mark.parametrize("layout", sorted(LAYOUTS))
def test_line_gs_clustered_matches_oracle(lib, oracle, cuda, layout):
    make, maxcy = LAYOUTS[layout]
    pr = make()
    prm = pr.params(mg_itrsch=2, maxcy=maxcy, eps=1e-12)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=41, fourier_modes=2))
    assert_same(o, g, pr.pl)


def test_line_gs_clustered_variable_density(lib, oracle, cuda):
    pr = Problem(2, 1, 1, 64, 64, 32, ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=2, maxcy=2, eps=1e-12, lsm=1)
    blocks = pr.block_fields(seed=42, fourier_modes=2)
    for f, d in zip(blocks, pr.block_density(43)):
        f["dens"] = d
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    assert_same(o, g, pr.pl)


LEX_LAYOUTS = {
    "2x1x1 blocks of 64^3, stretched y": lambda: Problem(2, 1, 1, 64, 64, 64, ngrid=3, pl=2, stretch_y=2.0),
    "1 block of 96x64x128, walls": lambda: Problem(1, 1, 1, 96, 64, 128, bc=(W,) * 6, ngrid=3, pl=1),
}


@pytest.mark.parametrize("layout", sorted(LEX_LAYOUTS))
def test_lex_gs_clustered_matches_oracle(lib, oracle, cuda, layout):
    """Lexicographic Gauss-Seidel (mg_itrsch 1, mgsolver.for:403-428) where
    each block's hyperplanes are split over a cluster of CTAs by k (64 and
    more planes): a slice's first plane reads the previous CTA's results."""
    pr = LEX_LAYOUTS[layout]()
    prm = pr.params(mg_itrsch=1, maxcy=2, eps=1e-12)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=44, fourier_modes=2))
    assert_same(o, g, pr.pl)

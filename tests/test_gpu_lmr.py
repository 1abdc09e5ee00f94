"""GPU parity of the V-cycle across LMR 2:1 refinement interfaces.

mf3d_mgkcyc_device on layouts whose blocks differ in refinement (rdiv 1
and 2) against the oracle's mgkcyc: the levels past a block's own last
(injection and whole-array correction, mgsolver.for:714-727, 806-818) and
the fine/coarse exchangepp branches; also a chain of rdiv 1, 2 and 4, whose
finest block halves its refinement on its extra levels.  FP64 bit for bit on pp's interior
and first ghost layer; FP32 (coarsest level in FP64) within a stated bar.  The ring entries of a fine block's face buffer are
0 on both sides; the L-shaped layout, where the V-cycle reads them, also
shows the cells that do not depend on them (the oracle run with another
ring value).
"""
import ctypes as C

import numpy as np
import pytest

import oracle_bridge as ob
from lmr_layouts import LmrLayout
from multiflow3d_b200.problems import PERIODIC, WALL
from multiflow3d_b200.solver import Projection

pytestmark = pytest.mark.gpu

ALL_WALLS = (WALL,) * 6

LAYOUTS = [
    dict(px=2, py=1, pz=1, n=8, refine=[1], bc=ALL_WALLS),
    dict(px=2, py=2, pz=2, n=8, refine=[0], bc=ALL_WALLS),
    dict(px=2, py=2, pz=2, n=8, refine=[3, 4], bc=ALL_WALLS),
    dict(px=3, py=2, pz=1, n=8, refine=[1, 4], bc=(WALL, WALL, PERIODIC, PERIODIC, WALL, WALL)),
    dict(px=2, py=2, pz=1, n=8, refine=[0], bc=ALL_WALLS, drop=((1, 1, 0),)),
    dict(px=2, py=1, pz=1, n=32, refine=[0], bc=ALL_WALLS),
    dict(px=3, py=1, pz=1, n=8, refine={1: 2, 2: 4}, bc=ALL_WALLS),  # rdiv 1 | 2 | 4
]


def run_pair(lib, oracle, cuda, L, scheme, seed=42, ring=0.0, precision=0):
    import torch
    prm = L.params(mg_itrsch=scheme)
    rng = np.random.default_rng(seed)
    su = [rng.uniform(-1, 1, size=L.ttc(b)) for b in range(L.nblocks)]
    pp_ref = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
    oracle.orc_set_lmr_ring.argtypes = [C.c_double]
    oracle.orc_set_lmr_ring(ring)
    try:
        assert oracle.orc_mgkcyc(L.descriptors(oracle), L.nblocks, C.byref(prm), ob.ptr_array(su),
                                 ob.ptr_array(pp_ref)) == 0
    finally:
        oracle.orc_set_lmr_ring(0.0)
    proj = Projection(L.descriptors(lib), L.params(mg_itrsch=scheme, precision=precision), lib)
    su_d = [torch.from_numpy(a).to(cuda) for a in su]
    pp_d = [torch.zeros(L.ttc(b), dtype=torch.float64, device=cuda) for b in range(L.nblocks)]
    proj.mgkcyc_device(su_d, pp_d)
    launches = proj.launches
    proj.close()
    pl = L.pl
    got, ref = [], []
    for b in range(L.nblocks):
        nx, ny, nz = L.cells(b)
        s = (slice(pl - 1, pl + nz + 1), slice(pl - 1, pl + ny + 1), slice(pl - 1, pl + nx + 1))
        got.append(pp_d[b].cpu().numpy()[s])
        ref.append(pp_ref[b][s])
    return got, ref, launches


@pytest.mark.parametrize("scheme", [3, 1, 2])
@pytest.mark.parametrize("lay", LAYOUTS, ids=lambda d: f"{d['px']}x{d['py']}x{d['pz']}-n{d['n']}-ref"
                         + "-".join(map(str, d['refine'])) + ("-L" if d.get("drop") else ""))
def test_lmr_vcycle_bitwise(lib, oracle, cuda, lay, scheme):
    L = LmrLayout(lay["px"], lay["py"], lay["pz"], lay["n"], lay["refine"], lay["bc"], 3, drop=lay.get("drop", ()))
    got, ref, launches = run_pair(lib, oracle, cuda, L, scheme)
    assert launches > 0
    for b in range(L.nblocks):
        assert np.array_equal(got[b], ref[b]), f"block {b}: max diff {np.abs(got[b] - ref[b]).max()}"


def test_lmr_ring_independent_cells(lib, oracle, cuda):
    """On the L-shaped layout with the refined block at the re-entrant edge,
    the V-cycle reads the ring entries: the device equals the oracle with
    ring 0 on every cell, and the cells where the oracle with ring 1e3
    agrees (those that do not depend on the ring) are most of the domain."""
    L = LmrLayout(2, 2, 1, 8, [0], ALL_WALLS, 3, drop=((1, 1, 0),))
    got, ref, _ = run_pair(lib, oracle, cuda, L, 3)
    _, ref2, _ = run_pair(lib, oracle, cuda, L, 3, ring=1.0e3)
    dep = tot = 0
    for b in range(L.nblocks):
        assert np.array_equal(got[b], ref[b])
        same = ref[b] == ref2[b]
        assert np.array_equal(got[b][same], ref2[b][same])
        dep += int((~same).sum())
        tot += same.size
    assert 0 < dep < tot // 2


def test_lmr_refusals(lib, cuda):
    """The outer loop refuses an LMR context (its field exchanges at
    refinement interfaces are not restated)."""
    import torch
    L = LmrLayout(2, 1, 1, 8, [1], ALL_WALLS, 3)
    proj = Projection(L.descriptors(lib), L.params(), lib)
    fields = [{k: torch.zeros(L.ttc(b), dtype=torch.float64, device=cuda)
               for k in ("u", "v", "w", "p", "pp", "su", "ustar", "vstar", "wstar")} for b in range(L.nblocks)]
    with pytest.raises(RuntimeError, match="LMR"):
        proj.newsolv_mg_device(fields)
    proj.close()


FP32_BAR = 2e-5


@pytest.mark.parametrize("scheme", [3, 1, 2])
@pytest.mark.parametrize("lay", LAYOUTS, ids=lambda d: f"{d['px']}x{d['py']}x{d['pz']}-n{d['n']}-ref"
                         + "-".join(map(str, d['refine'])) + ("-L" if d.get("drop") else ""))
def test_lmr_vcycle_fp32(lib, oracle, cuda, lay, scheme):
    """The FP32 V-cycle (coarsest level in FP64) on the LMR layouts against
    the FP64 oracle: pp within FP32_BAR of the largest |pp| on every block,
    cells of levels past a block's own and across refinement interfaces
    included."""
    from multiflow3d_b200 import abi
    L = LmrLayout(lay["px"], lay["py"], lay["pz"], lay["n"], lay["refine"], lay["bc"], 3, drop=lay.get("drop", ()))
    got, ref, launches = run_pair(lib, oracle, cuda, L, scheme, precision=abi.MF3D_PREC_FP32)
    assert launches > 0
    scale = max(np.abs(r).max() for r in ref)
    assert scale > 0
    for b in range(L.nblocks):
        err = np.abs(got[b] - ref[b]).max()
        assert err <= FP32_BAR * scale, f"block {b}: {err / scale:.3e} of max |pp|"
    assert any(not np.array_equal(g, r) for g, r in zip(got, ref))  # the FP32 path ran: its rounding shows


def test_lmr_vcycle_random_layouts(lib, oracle, cuda):
    """The V-cycle on 12 seeded random LMR layouts (grids with a block left
    out, periodic axes, random refined sets), the three smoothers in turn:
    pp bit-identical to the oracle."""
    from lmr_layouts import random_layouts
    for q, L in enumerate(random_layouts(4242, 12)):
        got, ref, _ = run_pair(lib, oracle, cuda, L, (3, 1, 2)[q % 3], seed=q)
        for b in range(L.nblocks):
            assert np.array_equal(got[b], ref[b]), (L.pos, L.refine, L.bc, b)


@pytest.mark.parametrize("pl", [1, 3])
def test_lmr_vcycle_ghost_widths(lib, oracle, cuda, pl):
    """su and pp with 1 and 3 ghost layers (the ttc layout the V-cycle reads
    and writes): pp bit-identical to the oracle."""
    L = LmrLayout(2, 2, 1, 8, [0, 3], ALL_WALLS, 3, pl=pl)
    got, ref, _ = run_pair(lib, oracle, cuda, L, 3, seed=pl)
    for b in range(L.nblocks):
        assert np.array_equal(got[b], ref[b])


def test_lmr_vcycle_fp32_random_layouts(lib, oracle, cuda):
    """The FP32 V-cycle on the 12 seeded random LMR layouts, the three
    smoothers in turn: pp within FP32_BAR of max |pp| of the FP64 oracle."""
    from lmr_layouts import random_layouts
    from multiflow3d_b200 import abi
    for q, L in enumerate(random_layouts(4242, 12)):
        got, ref, _ = run_pair(lib, oracle, cuda, L, (3, 1, 2)[q % 3], seed=q, precision=abi.MF3D_PREC_FP32)
        scale = max(np.abs(r).max() for r in ref)
        for b in range(L.nblocks):
            assert np.abs(got[b] - ref[b]).max() <= FP32_BAR * scale, (L.pos, L.refine, L.bc, b)

"""LMR 2:1 refinement interfaces in the oracle's V-cycle (CPU only).

The oracle restates the multigrid half of the reference's LMR: the
per-block level clamping (localparameters.for:26-75; mgsolver.for:27-31,
388-392, 670-678, 790-798) and the fine/coarse cases of exchangepp
(exchangepp.for:43-4763).  The reference cannot run here, so its formulas
are pinned by known answers:

- a linear field is reproduced exactly (to rounding) by every interpolation
  the exchange performs across a refinement interface - the coarse side's
  8-cell averages, the fine side's corner and edge blends (but for an
  edge's two end cells, which blend the sender's ghost beyond the edge's
  end: a mirror at a wall), and the fine side's face extrapolation
  (recv + 3 phi_1 - phi_2)/4 along the face normal;
- repeated V-cycles converge on a compatible right-hand side, for all three
  smoothers.

The ring of a fine block's face buffer (the entries no coarse sender
writes) holds g_lmr_ring; which cells depend on it is measured by changing
it.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_bridge as ob
from lmr_layouts import LmrLayout
from multiflow3d_b200.problems import PERIODIC, WALL

ALL_WALLS = (WALL,) * 6


@pytest.fixture(scope="module")
def orc():
    lib = ob.load()
    lib.orc_set_lmr_ring.argtypes = [C.c_double]
    return lib


def level_dims(L, b, g):
    """Interior cells of block b on level g: clamped to the block's own
    last level (ngrid_input + log2(rdiv) levels)."""
    gl = min(g, L.own_levels(b))
    return tuple(n >> (gl - 1) for n in L.cells(b)), gl


def centres(L, b, g):
    """Cell-centre coordinates (x, y, z) of block b's ghost-inclusive level-g
    array, shaped (nz+2, ny+2, nx+2)."""
    (nx, ny, nz), gl = level_dims(L, b, g)
    h = L.h / L.rdiv.get(b, 1) * 2 ** (gl - 1)
    o = L.origin(b)
    ax = [o[a] + (np.arange(n + 2) - 0.5) * h for a, n in enumerate((nx, ny, nz))]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return x, y, z


def rdv(L, b, g):
    """rdv(dom, g) (localparameters.for:47-57): rdiv on the levels every
    block has, halving on the block's extra levels, 1 below its own."""
    r = L.rdiv.get(b, 1)
    for lev in range(1, g + 1):
        if lev > L.own_levels(b):
            return 1
        if lev > L.ngrid_in:
            r //= 2
    return r


def interface_cells(L, desc, b, g, fine_normal_axis=None):
    """Ghost cells of block b on level g that an LMR formula writes and a
    linear field must reproduce: the plane interior of each face whose
    neighbour has another rdv (a finer receiver's faces only along
    `fine_normal_axis`), and the interior of each edge and the corner cell
    toward a neighbour of another rdv."""
    (nx, ny, nz), _ = level_dims(L, b, g)
    d = desc[b]
    me = rdv(L, b, g)
    pos = {desc[q].id: q for q in range(L.nblocks)}
    mask = np.zeros((nz + 2, ny + 2, nx + 2), dtype=bool)
    faces = [(d.iprev, 0, 0), (d.inext, 0, nx + 1), (d.jprev, 1, 0), (d.jnext, 1, ny + 1), (d.kprev, 2, 0),
             (d.knext, 2, nz + 1)]
    for nb, ax, at in faces:
        if nb < 0 or rdv(L, pos[nb], g) == me:
            continue
        if me > rdv(L, pos[nb], g) and ax != fine_normal_axis:
            continue
        sl = [slice(1, nz + 1), slice(1, ny + 1), slice(1, nx + 1)]
        sl[2 - ax] = at
        mask[tuple(sl)] = True
    dirs_p = [(-1, -1), (-1, +1), (+1, +1), (+1, -1)]
    dirs_n = [(+1, +1), (+1, -1), (-1, -1), (-1, +1)]
    for q in range(4):
        for nb, (ex, ey), ez in ((d.corprev[q], dirs_p[q], -1), (d.cornext[q], dirs_n[q], +1)):
            if nb >= 0 and rdv(L, pos[nb], g) != me:
                mask[0 if ez < 0 else nz + 1, 0 if ey < 0 else ny + 1, 0 if ex < 0 else nx + 1] = True
    edp = [(-1, 0, -1), (0, +1, -1), (+1, 0, -1), (0, -1, -1), (-1, -1, 0), (-1, +1, 0)]
    edn = [(+1, 0, +1), (0, -1, +1), (-1, 0, +1), (0, +1, +1), (+1, +1, 0), (+1, -1, 0)]
    n3 = (nx, ny, nz)
    for q in range(6):
        for nb, e in ((d.edgprev[q], edp[q]), (d.edgnext[q], edn[q])):
            if nb < 0 or rdv(L, pos[nb], g) == me:
                continue
            # a finer receiver's two end cells blend the coarse sender's
            # ghost beyond the edge's end, a mirror where that end is a wall
            end = 1 if me > rdv(L, pos[nb], g) else 0
            sl = []
            for a in range(3):
                sl.append(slice(1 + end, n3[a] + 1 - end) if e[a] == 0 else (0 if e[a] < 0 else n3[a] + 1))
            mask[sl[2], sl[1], sl[0]] = True
    return mask


LAYOUTS = [
    dict(px=2, py=1, pz=1, refine=[1]),
    dict(px=2, py=2, pz=2, refine=[0]),
    dict(px=2, py=2, pz=2, refine=[7]),
    dict(px=2, py=2, pz=1, refine=[1, 2]),
    dict(px=3, py=1, pz=1, refine={1: 2, 2: 4}),
]


@pytest.mark.parametrize("lay", LAYOUTS)
def test_lmr_exchange_reproduces_linear_fields(orc, lay):
    L = LmrLayout(lay["px"], lay["py"], lay["pz"], 8, lay["refine"], ALL_WALLS, 3)
    desc = L.descriptors(orc)
    checked = 0
    for g in range(1, L.ngrid):  # the levels on which the refinements differ
        for axis in range(3):
            coef = np.zeros(3)
            coef[axis] = 1.0 + axis
            fi, exact = [], []
            for b in range(L.nblocks):
                x, y, z = centres(L, b, g)
                f = 0.25 + coef[0] * x + coef[1] * y + coef[2] * z
                exact.append(f)
                fi.append(np.ascontiguousarray(f.copy()))
            assert orc.orc_exchangepp(desc, L.nblocks, L.ngrid, g, ob.ptr_array(fi)) == 0
            for b in range(L.nblocks):
                m = interface_cells(L, desc, b, g, fine_normal_axis=axis)
                checked += int(m.sum())
                err = np.abs(fi[b][m] - exact[b][m]).max() if m.any() else 0.0
                assert err < 1e-12, f"level {g}, axis {axis}, block {b}: error {err}"
    assert checked > 0


def residual(orc, L, desc, su, p):
    """su - A p on level 1, the ghosts from mgbound + exchangepp."""
    pl = L.pl
    lv, out = [], []
    for b in range(L.nblocks):
        nx, ny, nz = L.cells(b)
        lv.append(np.ascontiguousarray(p[b][pl - 1:pl + nz + 1, pl - 1:pl + ny + 1, pl - 1:pl + nx + 1]))
        out.append(np.zeros_like(lv[-1]))
    assert orc.orc_exchangepp(desc, L.nblocks, L.ngrid, 1, ob.ptr_array(lv)) == 0
    assert orc.orc_apply_operator(desc, L.nblocks, L.ngrid, 1, ob.ptr_array(lv), ob.ptr_array(out)) == 0
    r = []
    for b in range(L.nblocks):
        nx, ny, nz = L.cells(b)
        r.append(su[b][pl:pl + nz, pl:pl + ny, pl:pl + nx] - out[b][1:-1, 1:-1, 1:-1])
    return r


def vcycle(orc, L, desc, su, scheme=3):
    prm = L.params(mg_itrsch=scheme)
    pp = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
    st = orc.orc_mgkcyc(desc, L.nblocks, C.byref(prm), ob.ptr_array(su), ob.ptr_array(pp))
    assert st == 0, orc.orc_last_error()
    return pp


@pytest.mark.parametrize("scheme", [3, 1, 2])
@pytest.mark.parametrize("lay", [dict(px=2, py=1, pz=1, refine=[1]), dict(px=2, py=2, pz=1, refine=[0, 3])])
def test_lmr_vcycles_converge(orc, lay, scheme):
    """V-cycles as a stationary iteration p += V(su - A p) on su = A p*:
    the residual falls by at least 1e4 in 10 cycles."""
    L = LmrLayout(lay["px"], lay["py"], lay["pz"], 8, lay["refine"], ALL_WALLS, 3)
    desc = L.descriptors(orc)
    rng = np.random.default_rng(5)
    pl = L.pl
    zero = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
    pstar = [rng.uniform(-1, 1, size=L.ttc(b)) for b in range(L.nblocks)]
    r = residual(orc, L, desc, zero, pstar)
    su = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
    for b in range(L.nblocks):
        nx, ny, nz = L.cells(b)
        su[b][pl:pl + nz, pl:pl + ny, pl:pl + nx] = -r[b]
    p = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
    norms = []
    for _ in range(11):
        r = residual(orc, L, desc, su, p)
        norms.append(max(np.abs(x).max() for x in r))
        rr = [np.zeros(L.ttc(b)) for b in range(L.nblocks)]
        for b in range(L.nblocks):
            nx, ny, nz = L.cells(b)
            rr[b][pl:pl + nz, pl:pl + ny, pl:pl + nx] = r[b]
        e = vcycle(orc, L, desc, rr, scheme)
        p = [p[b] + e[b] for b in range(L.nblocks)]
    assert norms[-1] < 1e-4 * norms[0], norms


def ring_dependent(orc, L, desc, su, scheme=3):
    """Cells of pp (interior and first ghost layer) that change with the
    value of the ring entries."""
    orc.orc_set_lmr_ring(0.0)
    a = vcycle(orc, L, desc, su, scheme)
    orc.orc_set_lmr_ring(1.0e3)
    try:
        c = vcycle(orc, L, desc, su, scheme)
    finally:
        orc.orc_set_lmr_ring(0.0)
    pl = L.pl
    out = []
    for b in range(L.nblocks):
        nx, ny, nz = L.cells(b)
        s = (slice(pl - 1, pl + nz + 1), slice(pl - 1, pl + ny + 1), slice(pl - 1, pl + nx + 1))
        out.append(a[b][s] != c[b][s])
    return out


def test_lmr_ring_entries(orc):
    """With walls or same-level neighbours around the refined blocks, the
    ring entries are overwritten before anything reads them (by mgbound, a
    later sync_dir's face or an edge copy), so no cell depends on them.  A
    fine block at the re-entrant edge of an L-shaped domain keeps an edge
    ghost from its second LMR face, and the V-cycle reads it."""
    rng = np.random.default_rng(3)
    for lay in (dict(px=2, py=1, pz=1, refine=[1]), dict(px=2, py=2, pz=2, refine=[0]),
                dict(px=2, py=2, pz=1, refine=[0, 3]), dict(px=2, py=2, pz=1, refine=[1], drop=((1, 1, 0),))):
        L = LmrLayout(lay["px"], lay["py"], lay["pz"], 8, lay["refine"], ALL_WALLS, 3, drop=lay.get("drop", ()))
        desc = L.descriptors(orc)
        su = [rng.uniform(-1, 1, size=L.ttc(b)) for b in range(L.nblocks)]
        assert not any(m.any() for m in ring_dependent(orc, L, desc, su)), lay
    L = LmrLayout(2, 2, 1, 8, [0], ALL_WALLS, 3, drop=((1, 1, 0),))
    desc = L.descriptors(orc)
    su = [rng.uniform(-1, 1, size=L.ttc(b)) for b in range(L.nblocks)]
    assert any(m.any() for m in ring_dependent(orc, L, desc, su))


def test_lmr_refusals(orc):
    """The oracle refuses what it does not restate: LMR in the outer loop
    (its field exchanges at refinement interfaces), periodic partners of
    different refinement, neighbours more than 2:1 apart."""
    from multiflow3d_b200.abi import Fields, SolveInfo
    L = LmrLayout(2, 1, 1, 8, [1], ALL_WALLS, 3)
    desc = L.descriptors(orc)
    prm = L.params()
    info = SolveInfo()
    hist = np.zeros(4)
    assert orc.orc_newsolv_mg(desc, L.nblocks, C.byref(prm), (Fields * L.nblocks)(), 1.0, 1.0, C.byref(info),
                              hist.ctypes.data_as(C.POINTER(C.c_double)), 4) == -6
    Lp = LmrLayout(2, 1, 1, 8, [1], (PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), 3)
    descp = Lp.descriptors(orc)
    su = [np.zeros(Lp.ttc(b)) for b in range(Lp.nblocks)]
    pp = [np.zeros(Lp.ttc(b)) for b in range(Lp.nblocks)]
    assert orc.orc_mgkcyc(descp, Lp.nblocks, C.byref(Lp.params()), ob.ptr_array(su), ob.ptr_array(pp)) != 0
    # rdiv 4 next to rdiv 1
    L4 = LmrLayout(2, 1, 1, 8, [1], ALL_WALLS, 3)
    d4 = L4.descriptors(orc)
    d4[1].nx, d4[1].ny, d4[1].nz = 32, 32, 32
    d4[1].dx = d4[1].dy = d4[1].dz = 1.0 / 32
    prm4 = L4.params()
    prm4.ngrid = 5
    su = [np.zeros((8 + 4,) * 3), np.zeros((32 + 4,) * 3)]
    pp = [np.zeros_like(a) for a in su]
    assert orc.orc_mgkcyc(d4, 2, C.byref(prm4), ob.ptr_array(su), ob.ptr_array(pp)) != 0


HOST_LAYOUTS = [
    dict(px=2, py=1, pz=1, refine=[1], bc=ALL_WALLS),
    dict(px=2, py=2, pz=2, refine=[0], bc=ALL_WALLS),
    dict(px=2, py=2, pz=2, refine=[3, 4], bc=ALL_WALLS),
    dict(px=2, py=2, pz=1, refine=[0], bc=ALL_WALLS, drop=((1, 1, 0),)),
    dict(px=3, py=2, pz=1, refine=[1, 4], bc=(WALL, WALL, PERIODIC, PERIODIC, WALL, WALL)),
    dict(px=3, py=1, pz=1, refine={1: 2, 2: 4}, bc=ALL_WALLS),  # rdiv 1 | 2 | 4
]


@pytest.mark.parametrize("lay", HOST_LAYOUTS)
def test_library_lmr_refresh_matches_oracle(lib, orc, lay):
    """The library's halo refresh (its LMR program evaluated on the host with
    the device kernels' arithmetic, mf3d_halo_refresh_host) against the
    oracle's mgbound + exchangepp, bit for bit, on every level of LMR
    layouts - walls, an L-shaped domain (the ring entries read as 0 on both
    sides), periodic partners of equal refinement."""
    L = LmrLayout(lay["px"], lay["py"], lay["pz"], 8, lay["refine"], lay["bc"], 3, drop=lay.get("drop", ()))
    dl, do = L.descriptors(lib), L.descriptors(orc)
    rng = np.random.default_rng(11)
    for g in range(1, L.ngrid + 1):
        a = []
        for b in range(L.nblocks):
            (nx, ny, nz), _ = level_dims(L, b, g)
            a.append(rng.uniform(-1, 1, size=(nz + 2, ny + 2, nx + 2)))
        mine = [np.ascontiguousarray(x.copy()) for x in a]
        ref = [np.ascontiguousarray(x.copy()) for x in a]
        assert lib.mf3d_halo_refresh_host(dl, L.nblocks, L.ngrid, g, ob.ptr_array(mine)) == 0
        assert orc.orc_exchangepp(do, L.nblocks, L.ngrid, g, ob.ptr_array(ref)) == 0
        for b in range(L.nblocks):
            assert np.array_equal(mine[b], ref[b]), f"level {g} block {b}: {np.argwhere(mine[b] != ref[b])[:5]}"


def test_library_lmr_plan_refusals(lib):
    """mf3d_create checks an LMR layout before it touches the device
    (alloc_dom.for:12-230 and the restated scope): lsm, periodic partners
    of different refinement, neighbours more than 2:1 apart, and spacings
    that are not powers of two of one another are refused with no GPU."""
    ctx = C.c_void_p()
    L = LmrLayout(2, 1, 1, 8, [1], ALL_WALLS, 3)
    d = L.descriptors(lib)
    p = L.params()
    p.lsm = 1
    assert lib.mf3d_create(d, L.nblocks, C.byref(p), C.byref(ctx)) == -6  # MF3D_E_UNSUPPORTED
    assert b"LMR" in lib.mf3d_last_error()
    Lp = LmrLayout(2, 1, 1, 8, [1], (PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), 3)
    assert lib.mf3d_create(Lp.descriptors(lib), Lp.nblocks, C.byref(Lp.params()), C.byref(ctx)) == -1  # INVALID
    assert b"periodic" in lib.mf3d_last_error()
    L4 = LmrLayout(2, 1, 1, 8, {1: 4}, ALL_WALLS, 3)
    assert lib.mf3d_create(L4.descriptors(lib), L4.nblocks, C.byref(L4.params()), C.byref(ctx)) == -1
    assert b"rdiv" in lib.mf3d_last_error()
    d3 = L.descriptors(lib)
    d3[1].dx = d3[1].dy = d3[1].dz = 1.0 / 24  # a ratio of 3
    d3[1].nx = d3[1].ny = d3[1].nz = 24
    assert lib.mf3d_create(d3, 2, C.byref(L.params()), C.byref(ctx)) == -1


def test_library_lmr_refresh_random_layouts(lib, orc):
    """The library's LMR refresh against the oracle's on every level of 16
    seeded random layouts (grids with a block left out, periodic axes,
    random refined sets), bit for bit."""
    from lmr_layouts import random_layouts
    rng = np.random.default_rng(7)
    for L in random_layouts(2024, 16):
        dl, do = L.descriptors(lib), L.descriptors(orc)
        for g in range(1, L.ngrid + 1):
            a = []
            for b in range(L.nblocks):
                (nx, ny, nz), _ = level_dims(L, b, g)
                a.append(rng.uniform(-1, 1, size=(nz + 2, ny + 2, nx + 2)))
            mine = [np.ascontiguousarray(x.copy()) for x in a]
            ref = [np.ascontiguousarray(x.copy()) for x in a]
            assert lib.mf3d_halo_refresh_host(dl, L.nblocks, L.ngrid, g, ob.ptr_array(mine)) == 0
            assert orc.orc_exchangepp(do, L.nblocks, L.ngrid, g, ob.ptr_array(ref)) == 0
            for b in range(L.nblocks):
                assert np.array_equal(mine[b], ref[b]), (L.pos, L.refine, L.bc, g, b)

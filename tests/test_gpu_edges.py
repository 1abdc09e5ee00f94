"""Edge cases against the oracle, FP64, bit for bit: iteration limits of 0,
1 and 2, a zero right-hand side, a time step that is not a power of two, a
single level with odd sizes (the plain-load calvel/calmas and odd rows in
the sweep), ragged blocks (two blocks of different lengths) and the ghost
layers of u, v, w that the final exchange(1..3) refreshes."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.abi import SolveInfo, BlockDesc
from multiflow3d_b200.problems import Problem, fields_struct, PERIODIC, WALL
from multiflow3d_b200.solver import Projection

pytestmark = pytest.mark.gpu


def run_both(lib, oracle, cuda, desc_lib, desc_orc, nb, prm, blocks, dt=1.0, alfapr=1.0, prepare=None):
    """The same solve on the oracle (host arrays) and on the GPU (device
    arrays); returns (oracle status, info, history, blocks), (GPU result, blocks).
    `prepare(proj)` runs on the GPU context before its solve."""
    import torch
    ref = [{k: v.copy() for k, v in f.items()} for f in blocks]
    info = SolveInfo()
    cap = max(prm.maxcy, 1)
    hist = np.zeros(cap)
    st = oracle.orc_newsolv_mg(desc_orc, nb, C.byref(prm), fields_struct(ref), dt, alfapr, C.byref(info),
                               hist.ctypes.data_as(C.POINTER(C.c_double)), cap)
    assert st >= 0, st
    dev = [{k: torch.from_numpy(v.copy()).to(cuda) for k, v in f.items()} for f in blocks]
    proj = Projection(desc_lib, prm, lib)
    if prepare is not None:
        prepare(proj)
    res = proj.newsolv_mg_device(dev, dt=dt, alfapr=alfapr)
    proj.close()
    got = [{k: v.cpu().numpy() for k, v in f.items()} for f in dev]
    return (st, info, hist[:info.iter], ref), (res, got)


def face_mask(shape, pl, nly):
    """Interior cells plus ghost layers 0..nly of the six faces over the
    interior tangential range: what the projection defines.  Ghost edges and
    corners (and deeper layers) are left as the caller gave them."""
    nz, ny, nx = (n - 2 * pl for n in shape)
    m = np.zeros(shape, dtype=bool)
    I, J, K = slice(pl, pl + nx), slice(pl, pl + ny), slice(pl, pl + nz)
    m[K, J, I] = True
    for ly in range(nly + 1):
        m[K, J, pl - 1 - ly] = m[K, J, pl + nx + ly] = True
        m[K, pl - 1 - ly, I] = m[K, pl + ny + ly, I] = True
        m[pl - 1 - ly, J, I] = m[pl + nz + ly, J, I] = True
    return m


def assert_same(o, g, pl, pl_ex=0, every_cell=True):
    """Status, iterations, history and rmax0 equal; p, u, v, w bit for bit
    on every cell - interior and every ghost that p = p + pp, exchange(1..4)
    (periodic planes, faces, the corner and edge neighbours' ghosts) and
    pbound write, and the ghosts they leave as given (an mf3d_create
    context).  every_cell=False: p on the interior and its first ghost
    layer, u, v, w on the interior and face ghost layers 0..pl_ex."""
    st, info, hist, ref = o
    res, got = g
    assert res.status == st and res.iter == info.iter
    assert np.array_equal(res.history, hist)
    assert res.rmax0 == info.rmax0
    for b in range(len(ref)):
        for k in ("p", "u", "v", "w"):
            if every_cell:
                diff = np.argwhere(got[b][k] != ref[b][k])
                assert diff.size == 0, (b, k, len(diff), diff[:4].tolist())
            else:
                m = face_mask(ref[b][k].shape, pl, 0 if k == "p" else pl_ex)
                assert np.array_equal(got[b][k][m], ref[b][k][m]), (b, k)


@pytest.mark.parametrize("maxcy", [0, 1, 2])
def test_iteration_limits(lib, oracle, cuda, maxcy):
    pr = Problem(2, 1, 1, 16, 8, 8, ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=maxcy, eps=1e-12)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=4, fourier_modes=2))
    assert_same(o, g, pr.pl)


def test_zero_rhs(lib, oracle, cuda):
    """Zero velocity: rmax0 = 0, the relative threshold is 0 and no
    iteration can pass it; both run to maxcy and report it."""
    pr = Problem(1, 2, 1, 8, 8, 16, ngrid=3, pl=1)
    prm = pr.params(mg_itrsch=3, maxcy=5, eps=1e-8)
    blocks = pr.block_fields(seed=1)
    for f in blocks:
        for k in ("ustar", "vstar", "wstar", "u", "v", "w"):
            f[k][...] = 0.0
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    assert_same(o, g, pr.pl)
    assert g[0].rmax0 == 0.0


def test_time_step_not_a_power_of_two(lib, oracle, cuda):
    pr = Problem(2, 2, 1, 16, 16, 8, ngrid=3, pl=2, stretch_y=1.5, dx=1 / 32, dy=1 / 32, dz=1 / 16)
    prm = pr.params(mg_itrsch=3, maxcy=80, eps=1e-10)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=9, fourier_modes=3), dt=0.37, alfapr=1.3)
    assert_same(o, g, pr.pl)


@pytest.mark.parametrize("scheme", [1, 2, 3])
def test_single_level_odd_sizes(lib, oracle, cuda, scheme):
    pr = Problem(1, 1, 1, 7, 5, 3, bc=(PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), ngrid=1, pl=1,
                 dx=0.1, dy=0.2, dz=0.3)
    prm = pr.params(mg_itrsch=scheme, maxcy=40, eps=1e-6)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=6))
    assert_same(o, g, pr.pl)


def ragged_blocks(lib_or_orc, nxs, ny, nz, h, pl, bc, seed):
    """Blocks side by side along x with lengths nxs; descriptors from the
    neighbour search of `lib_or_orc` and seeded fields cut from one global
    velocity (walls: zero normal velocity)."""
    NX = sum(nxs)
    x0 = np.concatenate([[0], np.cumsum(nxs)])
    ext = np.array([[x0[b] * h, x0[b + 1] * h, 0.0, ny * h, 0.0, nz * h] for b in range(len(nxs))])
    arr = (BlockDesc * len(nxs))()
    fn = getattr(lib_or_orc, "mf3d_build_topology", None) or getattr(lib_or_orc, "orc_build_topology")
    e = np.ascontiguousarray(ext.ravel())
    assert fn(len(nxs), e.ctypes.data_as(C.POINTER(C.c_double)), (C.c_int * 6)(*bc), h, h, h, arr) == 0
    rng = np.random.default_rng(seed)
    shape = (nz + 2 * pl, ny + 2 * pl, NX + 2 * pl)
    g = {k: rng.uniform(-1, 1, size=shape) for k in ("ustar", "vstar", "wstar")}
    # periodic x: ghost columns hold the wrapped values
    for k in g:
        g[k][:, :, :pl] = g[k][:, :, NX:NX + pl]
        g[k][:, :, NX + pl:] = g[k][:, :, pl:2 * pl]
    g["vstar"][:, pl - 1, :] = 0.0
    g["vstar"][:, pl + ny - 1, :] = 0.0
    g["wstar"][pl - 1, :, :] = 0.0
    g["wstar"][pl + nz - 1, :, :] = 0.0
    blocks = []
    for b in range(len(nxs)):
        sl = (slice(None), slice(None), slice(x0[b], x0[b + 1] + 2 * pl))
        f = {k: np.ascontiguousarray(g[k][sl]) for k in g}
        f["p"] = np.zeros_like(f["ustar"])
        f["u"], f["v"], f["w"] = f["ustar"].copy(), f["vstar"].copy(), f["wstar"].copy()
        f["su"] = np.zeros_like(f["p"])
        blocks.append(f)
    return arr, blocks


def test_ragged_blocks(lib, oracle, cuda):
    """Two blocks of 16 and 32 cells along a periodic x (walls in y, z)."""
    bc = (PERIODIC, PERIODIC, WALL, WALL, WALL, WALL)
    dl, blocks = ragged_blocks(lib, [16, 32], 16, 8, 1 / 32, 2, bc, seed=12)
    do, _ = ragged_blocks(oracle, [16, 32], 16, 8, 1 / 32, 2, bc, seed=12)
    prm = abi.Params(ngrid=3, mg_itrsch=3, irestr=2, iproln=1, maxcy=100, eps=1e-10, eps_relative=1, pl=2,
                     differencing=1, precision=abi.MF3D_PREC_FP64, device=0)
    o, g = run_both(lib, oracle, cuda, dl, do, 2, prm, blocks)
    assert_same(o, g, 2)


@pytest.mark.parametrize("pl,pl_ex", [(2, 1), (3, 2), (3, 0)])
def test_velocity_ghost_layers(lib, oracle, cuda, pl, pl_ex):
    """The final exchange(1..3) refreshes ghost layers 0..pl_ex of u, v, w on
    inter-block and periodic faces (2x2x1 blocks, periodic x and y)."""
    pr = Problem(2, 2, 1, 16, 16, 8, bc=(PERIODIC, PERIODIC, PERIODIC, PERIODIC, WALL, WALL), ngrid=3, pl=pl)
    prm = pr.params(mg_itrsch=3, maxcy=30, eps=1e-9, pl_ex=pl_ex)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=17, fourier_modes=2))
    assert_same(o, g, pl, pl_ex)


def test_poisoned_allocations(lib, oracle, cuda, monkeypatch):
    """Every new device allocation filled with NaN bytes (MF3D_POISON_ALLOC):
    the FP64 solves of all three smoothers still equal the oracle, and an
    FP32 V-cycle gives the same bits as without poisoning - no kernel reads
    library memory that nothing wrote, which a pool block reused from an
    earlier context would otherwise hand over with stale data."""
    import torch
    pr = Problem(2, 2, 1, 16, 16, 8, ngrid=3, pl=2, stretch_y=1.5, dx=1 / 32, dy=1 / 32, dz=1 / 16)
    blocks = pr.block_fields(seed=23, fourier_modes=2)

    def fp32_solve():
        dev = [{k: torch.from_numpy(v.copy()).to(cuda) for k, v in f.items()} for f in blocks]
        proj = Projection(pr.descriptors(lib), pr.params(mg_itrsch=3, maxcy=40, eps=1e-8,
                                                         precision=abi.MF3D_PREC_FP32), lib)
        res = proj.newsolv_mg_device(dev)
        proj.close()
        return res, [{k: v.cpu().numpy() for k, v in f.items()} for f in dev]

    clean = fp32_solve()
    monkeypatch.setenv("MF3D_POISON_ALLOC", "1")
    for scheme in (1, 2, 3):
        prm = pr.params(mg_itrsch=scheme, maxcy=40, eps=1e-10, pl_ex=1)
        o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
        assert_same(o, g, pr.pl, 1)
    poisoned = fp32_solve()
    assert np.array_equal(poisoned[0].history, clean[0].history)
    for b in range(pr.nblocks):
        for k in ("p", "u", "v", "w"):
            m = face_mask(blocks[b][k].shape, pr.pl, 0)
            assert np.array_equal(poisoned[1][b][k][m], clean[1][b][k][m]), (b, k)


@pytest.mark.parametrize("pl,pl_ex,layout", [(2, 0, "2x2x1 periodic x y"), (2, 1, "2x2x1 periodic x y"),
                                             (3, 2, "2x1x2 walls"), (2, 1, "1 block, walls")])
def test_fourth_order_calmas(lib, oracle, cuda, pl, pl_ex, layout):
    """differencing = 2: calmas' 4th-order divergence (press.for:13-35) on
    the velocities of calvel and its exchange(1..3), every outer iteration;
    u(i-2) and u(i+1) at the block faces are the exchanged layers where
    pl_ex reaches them, else the caller's ghost values.  The whole solve -
    rmax history, p, u, v, w - bit-identical to the oracle."""
    if layout.startswith("2x2x1"):
        pr = Problem(2, 2, 1, 16, 16, 8, bc=(PERIODIC, PERIODIC, PERIODIC, PERIODIC, WALL, WALL), ngrid=3, pl=pl)
    elif layout.startswith("2x1x2"):
        pr = Problem(2, 1, 2, 16, 8, 16, bc=(WALL,) * 6, ngrid=3, pl=pl)
    else:
        pr = Problem(1, 1, 1, 32, 16, 16, bc=(WALL,) * 6, ngrid=3, pl=pl)
    # the 2nd-order multigrid preconditions a 4th-order divergence: the
    # iteration contracts slowly, so a few iterations and the status as is
    prm = pr.params(mg_itrsch=3, maxcy=12, eps=1e-9, pl_ex=pl_ex, differencing=2)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm,
                    pr.block_fields(seed=23, fourier_modes=2))
    assert o[0] in (0, 1), o[0]
    assert_same(o, g, pl, pl_ex)


def test_fourth_order_calmas_host_entry(lib, oracle, cuda):
    """The host-array entry point with differencing = 2: u, v, w reach the
    device before the first calmas (which reads their ghost faces)."""
    pr = Problem(2, 1, 1, 16, 16, 16, bc=(PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=12, eps=1e-9, pl_ex=1, differencing=2)
    blocks = pr.block_fields(seed=29, fourier_modes=2)
    o, _ = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    host = [{k: v.copy() for k, v in f.items()} for f in blocks]
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg(host)
    proj.close()
    assert_same(o, (res, host), 2, 1)


@pytest.mark.parametrize("layout", ["2x2x2 walls", "3x2x1 periodic x", "2x2x2 periodic"])
def test_corner_and_edge_ghosts(lib, oracle, cuda, layout):
    """Every ghost cell of p, u, v, w after the projection, corner and edge
    ghosts included: exchange_smlvl unpacks (pl+1)^3 corner cubes and
    (pl+1)^2 edge bars from the corner and edge neighbours
    (exchange.for:671-1201, 2120-2397) before the faces, and pbound writes
    whole ghost-inclusive planes; the library replays that sequence as a copy
    map, the oracle literally."""
    if layout == "2x2x2 walls":
        pr = Problem(2, 2, 2, 16, 8, 8, bc=(WALL,) * 6, ngrid=3, pl=2)
    elif layout == "3x2x1 periodic x":
        pr = Problem(3, 2, 1, 8, 8, 16, bc=(PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), ngrid=3, pl=3)
    else:
        pr = Problem(2, 2, 2, 8, 8, 8, bc=(PERIODIC,) * 6, ngrid=3, pl=2)
    pl_ex = 1
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=pl_ex)
    blocks = pr.block_fields(seed=31, fourier_modes=2, p_random=True)
    rng = np.random.default_rng(5)
    for f in blocks:  # every ghost starts distinct, so a missed or extra copy shows
        for k in ("u", "v", "w"):
            f[k] += 1e-3 * rng.standard_normal(f[k].shape)
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    assert_same(o, g, pr.pl, pl_ex)


@pytest.mark.parametrize("layout", ["2x2x2 blocks of 32^3, 4 levels", "2x1x1 blocks of 64x32x32, 5 levels, no cluster"])
def test_middle_level_launch_matches_launch_path(lib, oracle, cuda, layout, monkeypatch):
    """The middle levels as one cooperative launch per direction
    (k_mid_cycle, MF3D_MID_CYCLE=1) against the launch-per-phase path and
    the oracle: bit for bit.  Without the coarse cluster launch
    (MF3D_COARSE_CLUSTER=0) the middle launch runs down to the coarsest
    level."""
    if layout.startswith("2x2x2"):
        pr = Problem(2, 2, 2, 32, 32, 32, ngrid=4, pl=2, stretch_y=1.5, dx=1 / 64, dy=1 / 64, dz=1 / 64)
    else:
        monkeypatch.setenv("MF3D_COARSE_CLUSTER", "0")
        pr = Problem(2, 1, 1, 64, 32, 32, ngrid=5, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=60, eps=1e-10)
    blocks = pr.block_fields(seed=44, fourier_modes=2)
    monkeypatch.setenv("MF3D_MID_CYCLE", "1")
    o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    assert_same(o, g, pr.pl)
    monkeypatch.setenv("MF3D_MID_CYCLE", "0")
    o2, g2 = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks)
    for b in range(pr.nblocks):
        for k in ("p", "u", "v", "w"):
            assert np.array_equal(g[1][b][k], g2[1][b][k]), (b, k)

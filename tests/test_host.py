"""CPU-only checks of the native library's host logic (no GPU needed):
the C ABI loads and exports every symbol of include/mf3d.h, the neighbour
search matches the oracle's restatement of alloc_dom.for, and the halo copy
map reproduces the oracle's literal exchangepp + mgbound + exchbc_mgpp."""
import ctypes as C
import itertools
import os
import re

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.problems import Problem, PERIODIC, WALL
import oracle_bridge as ob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "mf3d.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|double|const char \*)\s*\*?\s*(mf3d_\w+)\s*\(", txt, re.M)))


def test_exports_every_header_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 10
    assert set(syms) == set(abi.EXPORTED_SYMBOLS)
    for s in syms:
        assert hasattr(lib, s), s
    assert lib.mf3d_abi_version() == 1
    assert lib.mf3d_status_string(abi.MF3D_NOT_CONVERGED) == b"not converged"


def test_ctypes_struct_sizes_match_header(lib):
    # a descriptor round-trips through the library's topology builder
    pr = Problem(2, 1, 1, 8, 8, 8)
    d = pr.descriptors(lib)
    assert d[0].inext == 1 and d[1].iprev == 0
    assert d[0].nx == 8 and d[1].xsl == pytest.approx(8 * pr.dx)


FIELDS = [f for f, _ in abi.BlockDesc._fields_ if f not in ("hx", "hy", "hz")]
LAYOUTS = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (2, 2, 2), (3, 2, 1), (1, 1, 3)]
BCS = list(itertools.product([PERIODIC, WALL], repeat=3))


@pytest.mark.parametrize("layout", LAYOUTS)
def test_topology_matches_oracle(lib, oracle, layout):
    for bcs in BCS:
        bc = (bcs[0], bcs[0], bcs[1], bcs[1], bcs[2], bcs[2])
        pr = Problem(*layout, 8, 6, 4, bc=bc, ngrid=2)
        d1, d2 = pr.descriptors(lib), pr.descriptors(oracle)
        for b in range(pr.nblocks):
            for f in FIELDS:
                a, c = getattr(d1[b], f), getattr(d2[b], f)
                if hasattr(a, "__len__"):
                    a, c = list(a), list(c)
                assert a == c, (layout, bc, b, f)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_halo_map_matches_oracle_exchangepp(lib, oracle, layout):
    """Applying the library's (dst, src) copy map to random level data equals
    the oracle's sequence exchangepp -> mgbound -> exchbc_mgpp, bit for bit,
    for every periodic/wall combination and two levels."""
    for bcs in BCS:
        bc = (bcs[0], bcs[0], bcs[1], bcs[1], bcs[2], bcs[2])
        pr = Problem(*layout, 8, 6, 4, bc=bc, ngrid=2)
        d1, d2 = pr.descriptors(lib), pr.descriptors(oracle)
        for level in (1, 2):
            shape = ((pr.nz >> (level - 1)) + 2, (pr.ny >> (level - 1)) + 2, (pr.nx >> (level - 1)) + 2)
            rng = np.random.default_rng(level)
            arrs = [rng.standard_normal(shape) for _ in range(pr.nblocks)]
            ref = [a.copy() for a in arrs]
            assert oracle.orc_exchangepp(d2, pr.nblocks, pr.ngrid, level, ob.ptr_array(ref)) == 0
            n = lib.mf3d_halo_map(d1, pr.nblocks, pr.ngrid, level, None, None)
            dst = (C.c_longlong * n)()
            src = (C.c_longlong * n)()
            assert lib.mf3d_halo_map(d1, pr.nblocks, pr.ngrid, level, dst, src) == n
            flat = np.concatenate([a.ravel() for a in arrs])
            out = flat.copy()
            out[np.array(dst[:], dtype=np.int64)] = flat[np.array(src[:], dtype=np.int64)]
            assert np.array_equal(out, np.concatenate([a.ravel() for a in ref])), (layout, bc, level)


FX_CASES = [((2, 2, 2), (WALL,) * 6, 2, 0), ((2, 2, 2), (WALL,) * 6, 3, 2), ((2, 2, 1), (PERIODIC,) * 4 + (WALL,) * 2, 2, 1),
            ((3, 2, 2), (PERIODIC, PERIODIC, WALL, WALL, PERIODIC, PERIODIC), 2, 1),
            ((1, 1, 1), (PERIODIC,) * 6, 2, 1), ((2, 1, 1), (WALL,) * 6, 1, 0),
            ((2, 2, 2), (PERIODIC,) * 6, 1, 0)]


@pytest.mark.parametrize("layout,bc,pl,pl_ex", FX_CASES)
def test_field_exchange_map_matches_oracle(lib, oracle, layout, bc, pl, pl_ex):
    """The library's copy map of exchange(op) - exchange_bc on periodic faces,
    exchange_smlvl with its corner cubes, edge bars and faces
    (exchange.for:343-2498), and pbound after exchange(4) - applied to
    random fields equals the oracle's literal sequence on every cell of u, v,
    w and p, bit for bit."""
    from multiflow3d_b200.problems import fields_struct
    pr = Problem(*layout, 8, 6, 4, bc=bc, ngrid=2, pl=pl)
    d1, d2 = pr.descriptors(lib), pr.descriptors(oracle)
    prm = pr.params(pl_ex=pl_ex)
    rng = np.random.default_rng(pl * 10 + pl_ex)
    for op, key in ((1, "u"), (2, "v"), (3, "w"), (4, "p")):
        blocks = pr.block_fields(seed=3)
        for f in blocks:
            f[key][...] = rng.standard_normal(f[key].shape)
        flat = np.concatenate([f[key].ravel() for f in blocks])
        assert oracle.orc_exchange(d2, pr.nblocks, C.byref(prm), fields_struct(blocks), op) == 0
        n = lib.mf3d_field_exchange_map(d1, pr.nblocks, pl, pl_ex, op, None, None)
        assert n > 0
        dst = (C.c_longlong * n)()
        src = (C.c_longlong * n)()
        assert lib.mf3d_field_exchange_map(d1, pr.nblocks, pl, pl_ex, op, dst, src) == n
        out = flat.copy()
        out[np.array(dst[:], dtype=np.int64)] = flat[np.array(src[:], dtype=np.int64)]
        assert np.array_equal(out, np.concatenate([f[key].ravel() for f in blocks])), (op, key)


def test_create_rejects_bad_config_without_gpu(lib):
    """Divisibility rule of localparameters.for:201-206 is checked before any
    device work."""
    pr = Problem(1, 1, 1, 12, 8, 8, ngrid=4)
    ctx = C.c_void_p()
    st = lib.mf3d_create(pr.descriptors(lib), 1, C.byref(pr.params()), C.byref(ctx))
    assert st == abi.MF3D_E_INVALID
    assert b"not correct for mgsolver" in lib.mf3d_last_error()
    prm = pr.params()
    prm.mg_itrsch = 7
    assert lib.mf3d_create(pr.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_INVALID
    prm = Problem(1, 1, 1, 8, 8, 8, ngrid=2).params()
    prm.differencing = 2  # the 4th-order divergence reads u(i-2): pl = 1 has no such ghost
    assert lib.mf3d_create(Problem(1, 1, 1, 8, 8, 8, ngrid=2).descriptors(lib), 1, C.byref(prm),
                           C.byref(ctx)) == abi.MF3D_E_INVALID
    assert b"pl >= 2" in lib.mf3d_last_error()
    pst = Problem(1, 1, 1, 8, 8, 8, ngrid=2, pl=2, stretch_y=2.0)
    prm = pst.params(differencing=2)  # 4th order on a stretched grid: no reference definition
    assert lib.mf3d_create(pst.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_UNSUPPORTED
    prm.differencing = 4
    assert lib.mf3d_create(Problem(1, 1, 1, 8, 8, 8, ngrid=2).descriptors(lib), 1, C.byref(prm),
                           C.byref(ctx)) == abi.MF3D_E_INVALID


def test_create_rejects_bad_pl_ex_without_gpu(lib, oracle):
    """pl_ex (extra ghost planes of u, v, w refreshed by the final
    exchange(1..3)) must lie in 0..pl-1, and every block edge must exceed it;
    the library and the oracle reject the same configurations."""
    ctx = C.c_void_p()
    pr = Problem(1, 1, 1, 8, 8, 8, ngrid=2, pl=2)
    for pl_ex in (-1, 2):
        prm = pr.params(pl_ex=pl_ex)
        assert lib.mf3d_create(pr.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_INVALID
        assert b"pl_ex" in lib.mf3d_last_error()
    small = Problem(1, 1, 1, 8, 2, 8, ngrid=1, pl=3)
    prm = small.params(pl_ex=2)
    assert lib.mf3d_create(small.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_INVALID
    assert b"pl_ex" in lib.mf3d_last_error()
    blocks = small.block_fields(seed=1)
    from multiflow3d_b200.abi import SolveInfo
    from multiflow3d_b200.problems import fields_struct
    st = oracle.orc_newsolv_mg(small.descriptors(oracle), 1, C.byref(prm), fields_struct(blocks), 1.0, 1.0,
                               C.byref(SolveInfo()), None, 0)
    assert st == abi.MF3D_E_INVALID


def test_bounds_face_codes_refused_without_gpu(lib):
    """bounds = 1 refuses, before any device work, the face codes whose
    boundu/v/w branch needs data the library does not hold, and a power-law
    inlet on a stretched grid (the profile reads uniform cell centres).  The
    convective outflow (21) and the file inlets (7, 8) are checked at the
    solve, once their inputs can have been handed over."""
    ctx = C.c_void_p()
    for bc, kw, stretch in (((12, 2, WALL, WALL, WALL, WALL), {}, 2.0),
                            ((1, 2, WALL, WALL, 66, WALL), {}, 0.0), ((1, 2, WALL, WALL, WALL, WALL), {"lsm": 1}, 0.0)):
        pr = Problem(1, 1, 1, 8, 8, 8, bc=bc, ngrid=2, pl=1, stretch_y=stretch)
        prm = pr.params(bounds=1, **kw)
        assert lib.mf3d_create(pr.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_UNSUPPORTED, bc
        assert b"bounds" in lib.mf3d_last_error()


def test_variable_density_limits_without_gpu(lib):
    """lsm (the reference's L_LSM) runs in FP64 on uniform blocks through
    mf3d_create only; the other combinations are refused before any device
    work."""
    ctx = C.c_void_p()
    pr = Problem(1, 1, 1, 8, 8, 8, ngrid=2, pl=1)
    prm = pr.params(lsm=1, precision=abi.MF3D_PREC_FP32)
    assert lib.mf3d_create(pr.descriptors(lib), 1, C.byref(prm), C.byref(ctx)) == abi.MF3D_E_UNSUPPORTED
    st = Problem(1, 1, 1, 8, 8, 8, ngrid=2, pl=1, stretch_y=2.0)
    assert lib.mf3d_create(st.descriptors(lib), 1, C.byref(st.params(lsm=1)), C.byref(ctx)) == abi.MF3D_E_UNSUPPORTED
    dom = (abi.DomainDesc * 1)()
    dom[0].nx = dom[0].ny = dom[0].nz = 8
    dom[0].dx = dom[0].dy = dom[0].dz = 1 / 8
    assert lib.mf3d_batch_create(dom, 1, C.byref(pr.params(lsm=1)), C.byref(ctx)) == abi.MF3D_E_UNSUPPORTED
    srv = C.c_void_p()
    assert lib.mf3d_server_create(C.byref(pr.params(lsm=1)), 1e9, 4, C.byref(srv)) == abi.MF3D_E_UNSUPPORTED


def test_topology_rejects_fractional_extent(lib):
    ext = np.array([0.0, 1.05, 0.0, 1.0, 0.0, 1.0])
    bc6 = (C.c_int * 6)(5, 5, 4, 4, 5, 5)
    out = (abi.BlockDesc * 1)()
    st = lib.mf3d_build_topology(1, ext.ctypes.data_as(C.POINTER(C.c_double)), bc6, 0.1, 0.1, 0.1, out)
    assert st == abi.MF3D_E_INVALID

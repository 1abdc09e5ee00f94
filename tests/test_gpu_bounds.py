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


INLETS = {
    "code 12: 1/7 power law in y and z": (12, 0),
    "code 13: 1/7 power law in y": (13, 0),
    "code 7: inlet file values": (7, 0),
    "code 8: SEM fluctuations on ubulk": (8, 0),
    "code 8: SEM fluctuations on the power law (UPROF_SEM 12)": (8, 12),
}


def inlet_values(pr, desc, code, seed):
    """Random inlet-file contents for every block with a west inlet face."""
    from multiflow3d_b200.solver import inlet_counts
    rng = np.random.default_rng(seed)
    vals = {}
    for b in range(pr.nblocks):
        if desc[b].iprev < 0:
            vals[desc[b].id] = rng.uniform(-1.0, 1.0, sum(inlet_counts(desc[b], code)))
    return vals


@pytest.mark.parametrize("case", sorted(INLETS))
def test_bounds_inlets_every_cell(lib, oracle, cuda, case):
    """The west inlets of boundu (bounds.for:55-135): file values (7), SEM
    fluctuations (8), the power-law profiles (12, 13), each on every ghost
    layer 0..pl_ex, with v = w = 0 for code 12 (:374-377, 662-665); every
    cell of u, v, w against the oracle."""
    import ctypes as C
    code, uprof = INLETS[case]
    pr = Problem(2, 2, 1, 16, 16, 8, bc=(code, 2, W, W, S, S), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    desc_l, desc_o = pr.descriptors(lib), pr.descriptors(oracle)
    vals = inlet_values(pr, desc_l, code, 36) if code in (7, 8) else {}
    for i, v in vals.items():
        assert oracle.orc_set_inlet(i, code, uprof, v.ctypes.data_as(C.POINTER(C.c_double)), v.size) == 0
    try:
        o, g = run_both(lib, oracle, cuda, desc_l, desc_o, pr.nblocks, prm, pr.block_fields(seed=37, fourier_modes=2),
                        prepare=lambda proj: [proj.set_inlet(i, code, v, uprof) for i, v in vals.items()])
    finally:
        oracle.orc_clear_inlets()
    assert_all_cells(o, g, pr.pl, 1)
    # the inlet is in place: u on the west ghost layers differs from the input
    west = [b for b in range(pr.nblocks) if desc_l[b].iprev < 0]
    assert west and all(np.any(g[1][b]["u"][:, :, pr.pl - 1] != 0.0) for b in west)


def test_bounds_inlet_needs_values(lib, cuda):
    """A code-7 inlet with no values: the solve refuses (the reference would
    fail to open its file)."""
    import torch
    from multiflow3d_b200 import abi
    from multiflow3d_b200.solver import Projection
    pr = Problem(1, 1, 1, 16, 8, 8, bc=(7, 2, W, W, S, S), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=5, eps=1e-9, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    proj = Projection(pr.descriptors(lib), prm, lib)
    dev = [{k: torch.from_numpy(v).to(cuda) for k, v in f.items()} for f in pr.block_fields(seed=38)]
    with pytest.raises(RuntimeError):
        proj.newsolv_mg_device(dev)
    with pytest.raises(RuntimeError):  # the wrong count
        proj.set_inlet(0, 7, np.zeros(3))
    from multiflow3d_b200.solver import inlet_counts
    proj.set_inlet(0, 7, np.zeros(sum(inlet_counts(pr.descriptors(lib)[0], 7))))
    assert proj.newsolv_mg_device(dev).status in (abi.MF3D_OK, abi.MF3D_NOT_CONVERGED)
    proj.close()


def test_bounds_convective_outflow_every_cell(lib, oracle, cuda):
    """East code 21 with alfabc = 1 after the solve: the bound old
    velocities (mf3d_bind_old_velocity) give every east ghost layer of u, v,
    w (bounds.for:141-170, 449-474, 743-768) with the solve's dt and alfapr;
    every cell against the oracle."""
    import ctypes as C
    import torch
    from oracle_bridge import _dp
    pr = Problem(2, 1, 2, 16, 8, 8, bc=(1, 21, W, W, S, S), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=40, eps=1e-9, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    blocks = pr.block_fields(seed=39, fourier_modes=2)
    rng = np.random.default_rng(40)
    oo = [{k: rng.uniform(-1, 1, f["u"].shape) for k in ("uoo", "voo", "woo")} for f in blocks]
    ptrs = [(_dp * pr.nblocks)(*[o[k].ctypes.data_as(_dp) for o in oo]) for k in ("uoo", "voo", "woo")]
    dev_oo = [{k: torch.from_numpy(v).to(cuda) for k, v in o.items()} for o in oo]
    oracle.orc_bind_old_velocity(pr.nblocks, *ptrs)
    try:
        o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks,
                        dt=0.37, alfapr=1.3, prepare=lambda proj: proj.bind_old_velocity(dev_oo))
    finally:
        oracle.orc_bind_old_velocity(0, None, None, None)
    assert_all_cells(o, g, pr.pl, 1)


def test_bounds_convective_outflow_needs_old_velocities(lib, cuda):
    import torch
    from multiflow3d_b200.solver import Projection
    pr = Problem(1, 1, 1, 16, 8, 8, bc=(1, 21, W, W, S, S), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, maxcy=5, eps=1e-9, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    proj = Projection(pr.descriptors(lib), prm, lib)
    dev = [{k: torch.from_numpy(v).to(cuda) for k, v in f.items()} for f in pr.block_fields(seed=41)]
    with pytest.raises(RuntimeError):
        proj.newsolv_mg_device(dev)
    oo = [{k: torch.zeros_like(f["u"]) for k in ("uoo", "voo", "woo")} for f in dev]
    proj.bind_old_velocity(oo)
    proj.newsolv_mg_device(dev)
    proj.bind_old_velocity(None)
    with pytest.raises(RuntimeError):
        proj.newsolv_mg_device(dev)
    proj.close()


WALL_LAWS = {
    "61 smooth log law on the bottom, 62 rough on the top": ((4, 4, W, W, 61, 62), 1.0e-3),
    "63 and 64 power laws on south and north, 65 on the west": ((65, 4, 63, 64, S, S), 0.0),
}


def _wall_fields(pr, seed):
    rng = np.random.default_rng(seed)
    out = []
    for f in pr.block_fields(seed=seed, fourier_modes=2):
        for k in ("u", "v", "w", "ustar", "vstar", "wstar"):
            f[k] = f[k] + rng.uniform(0.5, 1.5, f[k].shape)  # a mean flow along every axis
        out.append(f)
    return out


def assert_close_velocities(o, g, rtol=1e-12):
    """p bit for bit; u, v, w to rounding (the wall laws take CUDA's sqrt,
    log and pow against libm's)."""
    st, info, hist, ref = o
    res, got = g
    assert res.status == st and res.iter == info.iter and np.array_equal(res.history, hist)
    for b in range(len(ref)):
        assert np.array_equal(got[b]["p"], ref[b]["p"]), b
        for k in ("u", "v", "w"):
            np.testing.assert_allclose(got[b][k], ref[b][k], rtol=rtol, atol=1e-15, err_msg=f"{b} {k}")


@pytest.mark.parametrize("case", sorted(WALL_LAWS))
def test_bounds_wall_functions(lib, oracle, cuda, case):
    """The wall functions of boundu/v/w after the solve (codes 61-65:
    log_law.for, wall_function.for, bounds.for:187-206 and the matching
    branches): against the oracle, two consecutive solves on one context so
    the kept wall stresses carry over."""
    bc, fric = WALL_LAWS[case]
    pr = Problem(2, 1, 1, 16, 8, 8, bc=bc, ngrid=3, pl=2, dx=0.01, dy=0.01, dz=0.01)
    prm = pr.params(mg_itrsch=3, maxcy=30, eps=1e-9, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    re = 5.0e4
    oracle.orc_set_wall_model(re, fric)
    try:
        blocks = _wall_fields(pr, 42)
        o, g = run_both(lib, oracle, cuda, pr.descriptors(lib), pr.descriptors(oracle), pr.nblocks, prm, blocks,
                        dt=0.02, prepare=lambda proj: proj.set_wall_model(re, fric))
    finally:
        oracle.orc_set_wall_model(0.0, 0.0)
    assert_close_velocities(o, g)
    # the laws changed the first cells: the bounds without them differ
    plain = Problem(2, 1, 1, 16, 8, 8, bc=tuple(4 if c >= 61 else c for c in bc), ngrid=3, pl=2,
                    dx=0.01, dy=0.01, dz=0.01)
    o2, g2 = run_both(lib, oracle, cuda, plain.descriptors(lib), plain.descriptors(oracle), plain.nblocks, prm,
                      _wall_fields(pr, 42), dt=0.02)
    assert any(not np.array_equal(g[1][b]["u"], g2[1][b]["u"]) for b in range(pr.nblocks))


def test_bounds_device_with_wall_functions(lib, oracle, cuda):
    """mf3d_bounds_device against orc_bounds, twice in a row (the second
    reads the wall stresses the first kept), codes 61 and 64 with inflow and
    outflow faces."""
    import ctypes as C
    import torch
    from multiflow3d_b200.problems import fields_struct
    from multiflow3d_b200.solver import Projection
    pr = Problem(1, 2, 1, 16, 8, 16, bc=(1, 2, 61, 64, S, S), ngrid=2, pl=2, dx=0.01, dy=0.01, dz=0.01)
    prm = pr.params(pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
    host = _wall_fields(pr, 43)
    dev = [{k: torch.from_numpy(v.copy()).to(cuda) for k, v in f.items()} for f in host]
    proj = Projection(pr.descriptors(lib), prm, lib)
    proj.set_wall_model(3.0e4, 0.0)
    oracle.orc_set_wall_model(3.0e4, 0.0)
    try:
        for _ in range(2):
            assert oracle.orc_bounds(pr.descriptors(oracle), pr.nblocks, C.byref(prm), fields_struct(host), 0.02,
                                     1.0, 1) == 0
            proj.bounds_device(dev, dt=0.02, alfapr=1.0, alfabc=1)
    finally:
        oracle.orc_set_wall_model(0.0, 0.0)
        proj.close()
    for b in range(pr.nblocks):
        for k in ("u", "v", "w"):
            np.testing.assert_allclose(dev[b][k].cpu().numpy(), host[b][k], rtol=1e-12, atol=1e-15, err_msg=f"{b} {k}")

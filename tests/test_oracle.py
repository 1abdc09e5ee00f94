"""Known-answer tests that pin the CPU oracle.

The reference (Fortran 90 + MPI) ships no tests, golden vectors or fixtures
and cannot be compiled in this container, so the oracle is pinned by
analytic identities of the discrete problem it restates:

* discrete eigenfunctions of the 7-point operator (cosines on periodic and
  Neumann axes) are reproduced by the full projection newsolv_mg;
* an independent direct solve (FFT on periodic axes, DCT-II on Neumann
  axes) of A p = div(u*)/dt agrees with the converged multigrid pressure;
* A is symmetric and annihilates constants (the nullspace of the
  all-periodic/Neumann problem);
* the converged solution does not depend on the block decomposition;
* the three smoothers converge to the same solution.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.fft as sfft

from multiflow3d_b200.problems import Problem, fields_struct, PERIODIC, WALL
from multiflow3d_b200.abi import SolveInfo
import oracle_bridge as ob


def solve(oracle, pr, blocks, **kw):
    prm = pr.params(**kw)
    hist = np.zeros(max(prm.maxcy, 1))
    info = SolveInfo()
    st = oracle.orc_newsolv_mg(pr.descriptors(oracle), pr.nblocks, C.byref(prm), fields_struct(blocks),
                               1.0, 1.0, C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), len(hist))
    return st, info, hist[:info.iter]


def divergence(pr, blocks):
    """div(u*) on the global grid, from the block fields (interior faces)."""
    NX, NY, NZ, pl = pr.NX, pr.NY, pr.NZ, pr.pl
    us = np.zeros((NZ, NY, NX + 1))
    vs = np.zeros((NZ, NY + 1, NX))
    ws = np.zeros((NZ + 1, NY, NX))
    for b, f in enumerate(blocks):
        bx, by, bz = pr.block_pos(b)
        sz, sy, sx = slice(bz * pr.nz, (bz + 1) * pr.nz), slice(by * pr.ny, (by + 1) * pr.ny), slice(bx * pr.nx, (bx + 1) * pr.nx)
        inner = (slice(pl, pl + pr.nz), slice(pl, pl + pr.ny), slice(pl - 1, pl + pr.nx))
        us[sz, sy, bx * pr.nx:(bx + 1) * pr.nx + 1] = f["u"][inner]
        inner = (slice(pl, pl + pr.nz), slice(pl - 1, pl + pr.ny), slice(pl, pl + pr.nx))
        vs[sz, by * pr.ny:(by + 1) * pr.ny + 1, sx] = f["v"][inner]
        inner = (slice(pl - 1, pl + pr.nz), slice(pl, pl + pr.ny), slice(pl, pl + pr.nx))
        ws[bz * pr.nz:(bz + 1) * pr.nz + 1, sy, sx] = f["w"][inner]
    return (np.diff(us, axis=2) / pr.dx + np.diff(vs, axis=1) / pr.dy + np.diff(ws, axis=0) / pr.dz)


def direct_solve(pr, f):
    """Exact solution of the discrete A p = f, mean zero (FFT / DCT-II)."""
    axes = [(0, pr.NZ, pr.dz, pr.bc[4] == PERIODIC), (1, pr.NY, pr.dy, pr.bc[2] == PERIODIC),
            (2, pr.NX, pr.dx, pr.bc[0] == PERIODIC)]
    F = f.astype(np.complex128)
    lam = np.zeros(f.shape)
    for ax, n, h, per in axes:
        if per:
            F = np.fft.fft(F, axis=ax)
            theta = 2 * np.pi * np.arange(n) / n
        else:
            F = sfft.dct(F.real, type=2, axis=ax, norm="ortho") + 1j * sfft.dct(F.imag, type=2, axis=ax, norm="ortho")
            theta = np.pi * np.arange(n) / n
        shape = [1, 1, 1]
        shape[ax] = n
        lam = lam + ((2 * np.cos(theta) - 2) / h ** 2).reshape(shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        P = np.where(np.abs(lam) > 1e-12, F / lam, 0.0)
    for ax, n, h, per in reversed(axes):
        if per:
            P = np.fft.ifft(P, axis=ax)
        else:
            P = sfft.idct(P.real, type=2, axis=ax, norm="ortho") + 1j * sfft.idct(P.imag, type=2, axis=ax, norm="ortho")
    return P.real


def demean(a):
    return a - a.mean()


@pytest.mark.parametrize("scheme", [1, 2, 3])
def test_config1_matches_direct_solve(oracle, scheme):
    """Config 1 (64x32x32, periodic x,z, walls y): the converged oracle
    pressure solves the discrete Poisson problem exactly."""
    pr = Problem(1, 1, 1, 64, 32, 32, ngrid=4)
    blocks = pr.block_fields(seed=2)
    f = divergence(pr, blocks)  # dt = 1
    st, info, hist = solve(oracle, pr, blocks, mg_itrsch=scheme, maxcy=200, eps=1e-12)
    assert st == 0, (st, info.iter)
    assert hist[-1] < 1e-12 * info.rmax0
    p = demean(pr.gather(blocks, "p"))
    pex = demean(direct_solve(pr, f))
    assert np.linalg.norm(p - pex) / np.linalg.norm(pex) < 1e-9
    # the projected velocity is divergence-free to the tolerance
    assert np.abs(divergence(pr, blocks)).max() * pr.dx * pr.dy * pr.dz < 1e-12 * info.rmax0 * 10


@pytest.mark.parametrize("bc", [
    (PERIODIC, PERIODIC, WALL, WALL, PERIODIC, PERIODIC),
    (WALL, WALL, WALL, WALL, WALL, WALL),
    (PERIODIC, PERIODIC, PERIODIC, PERIODIC, PERIODIC, PERIODIC),
])
def test_eigenfunction_known_answer(oracle, bc):
    """u* = dt * G(phi_e) for a discrete eigenfunction phi_e of A: the
    projection must return p = phi_e + const and u = 0."""
    pr = Problem(2, 1, 2, 16, 16, 8, bc=bc, ngrid=4, pl=2)
    z = (np.arange(pr.NZ + 2 * pr.pl) - pr.pl + 0.5)
    y = (np.arange(pr.NY + 2 * pr.pl) - pr.pl + 0.5)
    x = (np.arange(pr.NX + 2 * pr.pl) - pr.pl + 0.5)

    def mode(c, n, per, m):
        return np.cos((2 if per else 1) * np.pi * m * c / n)

    phi = (mode(z, pr.NZ, bc[4] == PERIODIC, 1)[:, None, None] * mode(y, pr.NY, bc[2] == PERIODIC, 2)[None, :, None]
           * mode(x, pr.NX, bc[0] == PERIODIC, 1)[None, None, :])
    # face gradients of phi (zero on wall faces, as boundu/v/w leave them)
    gu = np.zeros_like(phi); gv = np.zeros_like(phi); gw = np.zeros_like(phi)
    gu[:, :, :-1] = np.diff(phi, axis=2) / pr.dx
    gv[:, :-1, :] = np.diff(phi, axis=1) / pr.dy
    gw[:-1, :, :] = np.diff(phi, axis=0) / pr.dz
    blocks = pr.block_fields(seed=0)
    pl = pr.pl
    for b, f in enumerate(blocks):
        bx, by, bz = pr.block_pos(b)
        sl = (slice(bz * pr.nz, bz * pr.nz + pr.nz + 2 * pl), slice(by * pr.ny, by * pr.ny + pr.ny + 2 * pl),
              slice(bx * pr.nx, bx * pr.nx + pr.nx + 2 * pl))
        for k, g in (("ustar", gu), ("vstar", gv), ("wstar", gw)):
            f[k][...] = g[sl]
        if bx == 0 and bc[0] != PERIODIC: f["ustar"][:, :, pl - 1] = 0
        if bx == pr.px - 1 and bc[1] != PERIODIC: f["ustar"][:, :, pl + pr.nx - 1] = 0
        if by == 0 and bc[2] != PERIODIC: f["vstar"][:, pl - 1, :] = 0
        if by == pr.py - 1 and bc[3] != PERIODIC: f["vstar"][:, pl + pr.ny - 1, :] = 0
        if bz == 0 and bc[4] != PERIODIC: f["wstar"][pl - 1, :, :] = 0
        if bz == pr.pz - 1 and bc[5] != PERIODIC: f["wstar"][pl + pr.nz - 1, :, :] = 0
        for a, s in (("u", "ustar"), ("v", "vstar"), ("w", "wstar")):
            f[a][...] = f[s]
    st, info, hist = solve(oracle, pr, blocks, mg_itrsch=3, maxcy=300, eps=1e-13)
    assert st == 0
    p = demean(pr.gather(blocks, "p"))
    pe = demean(phi[pl:pl + pr.NZ, pl:pl + pr.NY, pl:pl + pr.NX])
    assert np.linalg.norm(p - pe) / np.linalg.norm(pe) < 1e-10
    for k in ("u", "v", "w"):
        assert np.abs(pr.gather(blocks, k)).max() < 1e-9


def _ghosted(pr, level, rng):
    shape = ((pr.nz >> (level - 1)) + 2, (pr.ny >> (level - 1)) + 2, (pr.nx >> (level - 1)) + 2)
    return [rng.standard_normal(shape) for _ in range(pr.nblocks)]


@pytest.mark.parametrize("layout", [(1, 1, 1), (2, 2, 1)])
def test_operator_symmetric_and_constant_nullspace(oracle, layout):
    pr = Problem(*layout, 8, 8, 8, bc=(PERIODIC, PERIODIC, WALL, WALL, PERIODIC, PERIODIC), ngrid=2)
    desc = pr.descriptors(oracle)
    rng = np.random.default_rng(0)
    for level in (1, 2):
        u = _ghosted(pr, level, rng)
        v = _ghosted(pr, level, rng)
        for a in (u, v):
            assert oracle.orc_exchangepp(desc, pr.nblocks, pr.ngrid, level, ob.ptr_array(a)) == 0
        Au = [np.zeros_like(a) for a in u]
        Av = [np.zeros_like(a) for a in v]
        oracle.orc_apply_operator(desc, pr.nblocks, pr.ngrid, level, ob.ptr_array(u), ob.ptr_array(Au))
        oracle.orc_apply_operator(desc, pr.nblocks, pr.ngrid, level, ob.ptr_array(v), ob.ptr_array(Av))
        s = lambda a: a[1:-1, 1:-1, 1:-1]
        lhs = sum(np.sum(s(x) * s(y)) for x, y in zip(Au, v))
        rhs = sum(np.sum(s(x) * s(y)) for x, y in zip(u, Av))
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0) * 1e3
        const = [np.full_like(a, 3.25) for a in u]
        Ac = [np.zeros_like(a) for a in u]
        oracle.orc_apply_operator(desc, pr.nblocks, pr.ngrid, level, ob.ptr_array(const), ob.ptr_array(Ac))
        assert max(np.abs(s(a)).max() for a in Ac) < 1e-9


def test_vcycle_zero_rhs_gives_zero(oracle):
    pr = Problem(2, 1, 1, 8, 8, 8, ngrid=3, pl=1)
    prm = pr.params()
    su = [np.zeros(pr.ttc) for _ in range(pr.nblocks)]
    pp = [np.full(pr.ttc, 7.0) for _ in range(pr.nblocks)]
    assert oracle.orc_mgkcyc(pr.descriptors(oracle), pr.nblocks, C.byref(prm), ob.ptr_array(su), ob.ptr_array(pp)) == 0
    for a in pp:
        assert np.all(a[:pr.nz + 2, :pr.ny + 2, :pr.nx + 2] == 0.0)


def test_decomposition_invariance(oracle):
    """The same global problem split 1x1x1 and 2x2x2 converges to the same
    pressure (the iterates differ: ghosts are exchanged once per sweep)."""
    sols = []
    for lay in ((1, 1, 1), (2, 2, 2)):
        n = (32 // lay[0], 16 // lay[1], 16 // lay[2])
        pr = Problem(*lay, *n, ngrid=3)
        blocks = pr.block_fields(seed=9)
        st, info, _ = solve(oracle, pr, blocks, mg_itrsch=3, maxcy=300, eps=1e-12)
        assert st == 0
        sols.append(demean(pr.gather(blocks, "p")))
    assert np.linalg.norm(sols[0] - sols[1]) / np.linalg.norm(sols[0]) < 1e-9


def test_not_converged_and_diverged_status(oracle):
    pr = Problem(1, 1, 1, 16, 8, 8, ngrid=2)
    blocks = pr.block_fields(seed=1)
    st, info, hist = solve(oracle, pr, blocks, mg_itrsch=3, maxcy=2, eps=1e-14)
    assert st == 1 and info.iter == 2 and len(hist) == 2
    blocks = pr.block_fields(seed=1)
    for f in blocks:
        for k in ("ustar", "vstar", "wstar", "u", "v", "w"):
            f[k] *= 1e6
    st, info, _ = solve(oracle, pr, blocks, mg_itrsch=3, maxcy=1, eps=1e-14)
    assert st == 2  # rmax > 100 after the loop (newsolv_mg.for:64)


@pytest.mark.parametrize("pl,pl_ex", [(1, 0), (2, 1), (3, 2)])
def test_velocity_ghost_layers_wrap(oracle, pl, pl_ex):
    """One block, periodic in x and y: after the projection, ghost layer ly
    (0..pl_ex) of u, v, w holds the interior value ly planes inside the
    opposite face (exchange_bc.for:147-178), and deeper layers are untouched."""
    pr = Problem(1, 1, 1, 8, 8, 8, bc=(PERIODIC, PERIODIC, PERIODIC, PERIODIC, WALL, WALL), ngrid=2, pl=pl)
    blocks = pr.block_fields(seed=5)
    given = {k: blocks[0][k].copy() for k in ("u", "v", "w")}
    info = SolveInfo()
    st = oracle.orc_newsolv_mg(pr.descriptors(oracle), 1, C.byref(pr.params(maxcy=3, pl_ex=pl_ex)),
                               fields_struct(blocks), 1.0, 1.0, C.byref(info), None, 0)
    assert st >= 0
    n = 8
    K = J = I = slice(pl, pl + n)
    for k in ("u", "v", "w"):
        a = blocks[0][k]
        for ly in range(pl):
            lo, hi = pl - 1 - ly, pl + n + ly
            if ly <= pl_ex:
                assert np.array_equal(a[K, J, lo], a[K, J, pl + n - 1 - ly])
                assert np.array_equal(a[K, J, hi], a[K, J, pl + ly])
                assert np.array_equal(a[K, lo, I], a[K, pl + n - 1 - ly, I])
                assert np.array_equal(a[K, hi, I], a[K, pl + ly, I])
            else:
                assert np.array_equal(a[K, J, lo], given[k][K, J, lo])
                assert np.array_equal(a[K, lo, I], given[k][K, lo, I])


@pytest.mark.parametrize("rho", [1.0, 2.5])
def test_variable_density_constant_rho_known_answer(oracle, rho):
    """L_LSM with a constant density rho solves div(grad p / rho) = div(u*)/dt:
    the converged pressure is rho times the uniform-density one (up to the
    floating constant) and the projected velocities are the same.  Pins the
    scaling of the L_LSM coefficients (mgsolver.for:120-182), of calvel
    (press.for:152-190) and of the rhs sup (press.for:51-53)."""
    pr = Problem(2, 1, 1, 16, 16, 16, ngrid=3, pl=1)
    a = pr.block_fields(seed=3)
    b = [{k: v.copy() for k, v in f.items()} for f in a]
    for f, d in zip(b, pr.block_density(0, const=rho)):
        f["dens"] = d
    st_a, info_a, _ = solve(oracle, pr, a, maxcy=400, eps=1e-12)
    st_b, info_b, _ = solve(oracle, pr, b, maxcy=400, eps=1e-12, lsm=1)
    assert st_a == 0 and st_b == 0
    assert info_b.rmax0 == info_a.rmax0
    pa, pb = demean(pr.gather(a, "p")), demean(pr.gather(b, "p"))
    assert np.abs(pb - rho * pa).max() <= 1e-9 * np.abs(rho * pa).max()
    for k in ("u", "v", "w"):
        assert np.abs(pr.gather(b, k) - pr.gather(a, k)).max() <= 1e-10


def test_variable_density_projection_is_divergence_free(oracle):
    """A random density field in [0.5, 2]: the converged projection leaves
    u, v, w discretely divergence-free to the stopping tolerance."""
    pr = Problem(2, 2, 1, 16, 16, 8, ngrid=3, pl=2)
    blocks = pr.block_fields(seed=11, fourier_modes=2)
    for f, d in zip(blocks, pr.block_density(7)):
        f["dens"] = d
    div0 = np.abs(divergence(pr, blocks)).max()
    st, info, hist = solve(oracle, pr, blocks, maxcy=2000, eps=1e-11, lsm=1)
    assert st == 0
    assert np.abs(divergence(pr, blocks)).max() <= 1e-9 * div0


def test_weno_differencing_takes_the_second_order_divergence(oracle):
    """L_LSM runs with differencing = 3 (WENO convection, initial.for:133-135);
    calmas branches only on differencing = 2 (press.for:13-35), so 3 gives
    the same projection as 1, bit for bit, and 2 is refused."""
    pr = Problem(2, 1, 1, 16, 8, 8, ngrid=3, pl=2)
    runs = []
    for d in (1, 3):
        blocks = pr.block_fields(seed=4, fourier_modes=2)
        for f, r in zip(blocks, pr.block_density(5)):
            f["dens"] = r
        st, info, hist = solve(oracle, pr, blocks, maxcy=30, eps=1e-9, lsm=1, differencing=d)
        assert st in (0, 1)
        runs.append((info.rmax, hist, blocks))
    assert runs[0][0] == runs[1][0] and np.array_equal(runs[0][1], runs[1][1])
    for a, b in zip(runs[0][2], runs[1][2]):
        for k in ("p", "u", "v", "w", "su"):
            assert np.array_equal(a[k], b[k])
    blocks = pr.block_fields(seed=4)
    for f, r in zip(blocks, pr.block_density(5)):
        f["dens"] = r
    assert solve(oracle, pr, blocks, maxcy=2, differencing=2, lsm=1)[0] == -1  # L_LSM needs WENO
    assert solve(oracle, pr, blocks, maxcy=2, differencing=4)[0] == -1


@pytest.mark.parametrize("layout", ["1 block, walls", "2x2x1 blocks, walls"])
def test_fourth_order_divergence_known_answer(oracle, layout):
    """calmas' 4th-order branch (press.for:13-35) is exact for cubic face
    velocities: with u = f(x), v = g(y), w = q(z) cubic on every face
    (ghosts included) and p = 0, the initial calvel leaves u = ustar and the
    exchange hands over the same polynomial, so su = f'(x) + g'(y) + q'(z)
    at the cell centres and rmax0 = max |su * dx*dy*dz|.  The 2nd-order
    branch misses the cubic term (its error h^2/24 times the third
    derivative is visible).  A pl = 1 layout, with no second ghost face, is
    refused."""
    h = 1.0 / 16
    if layout.startswith("1"):
        pr = Problem(1, 1, 1, 16, 8, 8, bc=(WALL,) * 6, ngrid=2, pl=2, dx=h, dy=h, dz=h)
    else:
        pr = Problem(2, 2, 1, 8, 8, 8, bc=(WALL,) * 6, ngrid=2, pl=2, dx=h, dy=h, dz=h)
    f = lambda x: 0.3 + 1.7 * x - 2.1 * x ** 2 + 3.3 * x ** 3
    g = lambda y: -0.4 + 0.9 * y + 1.1 * y ** 2 - 0.7 * y ** 3
    q = lambda z: 0.2 - 1.3 * z + 0.5 * z ** 2 + 2.9 * z ** 3
    df = lambda x: 1.7 - 4.2 * x + 9.9 * x ** 2
    dg = lambda y: 0.9 + 2.2 * y - 2.1 * y ** 2
    dq = lambda z: -1.3 + 1.0 * z + 8.7 * z ** 2

    def fields():
        out = []
        for b in range(pr.nblocks):
            bx, by, bz = pr.block_pos(b)
            # u(i) sits on the face between cells i and i+1: x = (global cell index + 1) * h
            xi = (bx * pr.nx + np.arange(-pr.pl, pr.nx + pr.pl) + 1) * h
            yj = (by * pr.ny + np.arange(-pr.pl, pr.ny + pr.pl) + 1) * h
            zk = (bz * pr.nz + np.arange(-pr.pl, pr.nz + pr.pl) + 1) * h
            shp = pr.ttc
            us = np.broadcast_to(f(xi)[None, None, :], shp).copy()
            vs = np.broadcast_to(g(yj)[None, :, None], shp).copy()
            ws = np.broadcast_to(q(zk)[:, None, None], shp).copy()
            out.append({"ustar": us, "vstar": vs, "wstar": ws, "u": us.copy(), "v": vs.copy(), "w": ws.copy(),
                        "p": np.zeros(shp), "su": np.zeros(shp)})
        return out

    blocks = fields()
    st, info, _ = solve(oracle, pr, blocks, maxcy=0, differencing=2)
    assert st in (0, 1), st
    worst = 0.0
    for b, fb in enumerate(blocks):
        bx, by, bz = pr.block_pos(b)
        xc = (bx * pr.nx + np.arange(pr.nx) + 0.5) * h
        yc = (by * pr.ny + np.arange(pr.ny) + 0.5) * h
        zc = (bz * pr.nz + np.arange(pr.nz) + 0.5) * h
        exact = dq(zc)[:, None, None] + dg(yc)[None, :, None] + df(xc)[None, None, :]
        got = pr.interior(fb["su"])
        assert np.abs(got - exact).max() <= 1e-10 * np.abs(exact).max()
        worst = max(worst, float(np.abs(got * h ** 3).max()))
    assert abs(info.rmax0 - worst) <= 1e-14 * worst
    # the 2nd-order branch on the same faces misses the cubic term
    blocks2 = fields()
    solve(oracle, pr, blocks2, maxcy=0, differencing=1)
    assert np.abs(pr.interior(blocks2[0]["su"]) - pr.interior(blocks[0]["su"])).max() > 1e-4
    # pl = 1 has no u(isp-2)
    pr1 = Problem(1, 1, 1, 16, 8, 8, bc=(WALL,) * 6, ngrid=2, pl=1)
    assert solve(oracle, pr1, pr1.block_fields(seed=1), maxcy=1, differencing=2)[0] == -1


def test_bounds_known_answers(oracle):
    """boundu/boundv/boundw after the loop (bounds: periodic x, walls in y,
    symmetry in z, two ghost layers): a wall mirrors the tangential
    components with a sign change and zeroes the normal one, a symmetry face
    mirrors without it, and the periodic planes wrap."""
    SYM = 3
    n, pl = 8, 2
    pr = Problem(1, 1, 1, n, n, n, bc=(PERIODIC, PERIODIC, WALL, WALL, SYM, SYM), ngrid=2, pl=pl)
    blocks = pr.block_fields(seed=19)
    st, info, _ = solve(oracle, pr, blocks, maxcy=6, eps=1e-12, pl_ex=1, bounds=1)
    assert st >= 0
    u, v, w = (blocks[0][k] for k in ("u", "v", "w"))
    I = slice(pl - 1, pl + n + 1)          # x range widened by one (u, v, w: x periodic)
    Ki = slice(pl, pl + n)                 # interior z
    Ji = slice(pl, pl + n)
    for ly in range(2):
        lo, hi = pl - 1 - ly, pl + n + ly
        # y walls: tangential -mirror, normal 0 (v stops one face short of the north wall)
        for a in (u, w):
            assert np.array_equal(a[Ki, lo, I], -a[Ki, pl + ly, I])
            assert np.array_equal(a[Ki, hi, I], -a[Ki, pl + n - 1 - ly, I])
        assert not v[Ki, lo, I].any() and not v[Ki, pl + n - 1 + ly, I].any()
        # z symmetry: tangential +mirror, normal 0
        for a in (u, v):
            assert np.array_equal(a[lo, Ji, I], a[pl + ly, Ji, I])
            assert np.array_equal(a[hi, Ji, I], a[pl + n - 1 - ly, Ji, I])
        assert not w[lo, Ji, I].any() and not w[pl + n - 1 + ly, Ji, I].any()
    for a in (u, v, w):  # periodic x: full first ghost planes wrap
        assert np.array_equal(a[:, :, pl - 1], a[:, :, pl + n - 1])
        assert np.array_equal(a[:, :, pl + n], a[:, :, pl])


def test_bounds_inflow_outflow_known_answers(oracle):
    """Inflow (code 1) on the west and the bottom, outflow (code 2) on the
    east with alfabc = 1: the west ghost layers hold u = ubulk, v = w = 0
    (bounds.for:42-53, 374-377, 662-665), the bottom ones u = v = 0 and
    w = 1.1 (226-229, 536-539, 873-876), and every east ghost layer copies
    the last face ie (136-170, 444-470): u's ie is one face short of the
    boundary, v's and w's is the last cell."""
    SYM, INF, OUT = 3, 1, 2
    n, pl = 8, 3
    pr = Problem(1, 1, 1, n, n, n, bc=(INF, OUT, WALL, WALL, INF, SYM), ngrid=2, pl=pl)
    blocks = pr.block_fields(seed=23)
    st, info, _ = solve(oracle, pr, blocks, maxcy=6, eps=1e-12, pl_ex=2, bounds=1, alfabc=1, ubulk=0.7)
    assert st >= 0
    u, v, w = (blocks[0][k] for k in ("u", "v", "w"))
    Ji, Ki, Ii = slice(pl, pl + n), slice(pl, pl + n), slice(pl, pl + n)
    for ly in range(3):
        west = pl - 1 - ly
        assert (u[Ki, Ji, west] == 0.7).all()
        assert not v[Ki, Ji, west].any() and not w[Ki, Ji, west].any()
        bottom = pl - 1 - ly
        assert not u[bottom, Ji, Ii].any() and not v[bottom, Ji, Ii].any()
        assert (w[bottom, Ji, Ii] == 1.1).all()
        assert np.array_equal(u[Ki, Ji, pl + n - 1 + ly], u[Ki, Ji, pl + n - 2])
        for a in (v, w):
            assert np.array_equal(a[Ki, Ji, pl + n + ly], a[Ki, Ji, pl + n - 1])
    # alfabc = 0: the outflow branch is skipped, the east ghosts keep what calvel's exchange left
    b2 = pr.block_fields(seed=23)
    solve(oracle, pr, b2, maxcy=6, eps=1e-12, pl_ex=2, bounds=1, alfabc=0, ubulk=0.7)
    assert not np.array_equal(b2[0]["v"][Ki, Ji, pl + n + 1], b2[0]["v"][Ki, Ji, pl + n - 1])


@pytest.mark.parametrize("bc,kw,expect", [
    ((7, 2, WALL, WALL, WALL, WALL), {}, -1),               # inflow slices: no file values given
    ((12, 2, WALL, WALL, WALL, WALL), {}, 0),               # power-law inlet
    ((13, 2, WALL, WALL, WALL, WALL), {}, 0),
    ((1, 21, WALL, WALL, WALL, WALL), {"alfabc": 1}, -6),   # convective outflow reads uoo
    ((1, 21, WALL, WALL, WALL, WALL), {"alfabc": 0}, 0),    # ... unless alfabc skips it
    ((1, 2, WALL, WALL, 61, WALL), {}, -6),                 # wall function
    ((1, 2, WALL, WALL, WALL, WALL), {"lsm": 1}, -6),       # phi-gated inflow under L_LSM
    ((4, 4, 1, 2, 44, 6), {"alfabc": 1}, 0),                # codes without a branch on those faces
])
def test_bounds_face_codes(oracle, bc, kw, expect):
    """The face codes whose boundu/v/w branch reads data outside the
    projection are refused (MF3D_E_UNSUPPORTED), an inlet file that was never
    given is invalid; every other code runs, and one without a branch for its
    face writes nothing there."""
    pr = Problem(1, 1, 1, 8, 8, 8, bc=bc, ngrid=2, pl=1)
    blocks = pr.block_fields(seed=1)
    if kw.get("lsm"):
        for f, d in zip(blocks, pr.block_density(2)):
            f["dens"] = d
    st, _, _ = solve(oracle, pr, blocks, maxcy=2, bounds=1, **kw)
    assert (st >= 0) if expect == 0 else (st == expect)


def power_law(ubulk, yc, zc, H, Z, code):
    """bounds.for:105-135 in numpy: the 1/7 law of the distance to the
    nearer y wall, times the same law in z for code 12."""
    a = np.where(yc < H / 2, ubulk * (1.0 + 1.0 / 7.0) * np.abs(2 * yc / H) ** (1.0 / 7.0),
                 ubulk * (1.0 + 1.0 / 7.0) * np.abs(2 * (H - yc) / H) ** (1.0 / 7.0))
    if code == 12:
        a = a[None, :] * (1.0 + 1.0 / 7.0) * (np.abs(zc / Z) ** (1.0 / 7.0))[:, None]
    else:
        a = np.broadcast_to(a[None, :], (len(zc), len(yc)))
    return a


@pytest.mark.parametrize("code", [12, 13])
def test_bounds_power_law_inlet_known_answer(oracle, code):
    """Codes 12 and 13 put the 1/7 power-law profile on every west ghost
    layer of u (bounds.for:105-135; cell centres xc = x - dx/2 from the
    running sum x(i) = x(i-1) + dx, initial.for:341-365) and, for 12,
    v = w = 0 there; 13 leaves v and w."""
    n, pl, ubulk = 8, 2, 0.7
    pr = Problem(1, 1, 1, 2 * n, n, n, bc=(code, 2, WALL, WALL, WALL, WALL), ngrid=2, pl=pl,
                 dx=0.05, dy=0.1, dz=0.125)
    blocks = pr.block_fields(seed=24)
    before = {k: blocks[0][k].copy() for k in ("v", "w")}
    st, _, _ = solve(oracle, pr, blocks, maxcy=4, eps=1e-12, pl_ex=1, bounds=1, alfabc=1, ubulk=ubulk)
    assert st >= 0
    d = pr.descriptors(oracle)[0]
    y = np.cumsum(np.concatenate([[d.ysl + (1 - pl) * d.dy], np.full(n + 2 * pl - 1, d.dy)]))
    z = np.cumsum(np.concatenate([[d.zsl + (1 - pl) * d.dz], np.full(n + 2 * pl - 1, d.dz)]))
    yc, zc = y - 0.5 * d.dy, z - 0.5 * d.dz
    # js..je, ks..ke: the wall faces after the west one (S, N, B, T) mirror
    # into the ghost rows js-1, je+1, ks-1, ke+1 of the same layer
    rows = slice(pl, pl + n)
    want = power_law(ubulk, yc[rows], zc[rows], d.yel - d.ysl, d.zel - d.zsl, code)
    u = blocks[0]["u"]
    for ly in range(2):
        np.testing.assert_allclose(u[rows, rows, pl - 1 - ly], want, rtol=1e-15, atol=0)  # numpy and libm pow
        if code == 12:
            assert not blocks[0]["v"][rows, rows, pl - 1 - ly].any()
    if code == 13:  # the v and w west ghosts are left as calvel's exchange left them
        assert not np.array_equal(blocks[0]["v"][:, :, pl - 1], 0 * before["v"][:, :, pl - 1])


def test_bounds_inlet_files(oracle, tmp_path):
    """Codes 7 and 8 take the inlet file's values (bounds.for:55-103,
    397-438, 686-730): 7 one value per line, u's over its rows js-1..je+1 and
    planes ks-1..ke+1, then v's and w's over theirs (v one row short at the
    north wall, w one plane short at the top wall); 8 u = ubulk plus the first
    column of the SEM file (after two header lines), v and w the second and
    third, over rows js-1..je and planes ks-1..ke only.  The files are
    written in the reference's formats and read back with read_inlet_file."""
    from multiflow3d_b200.solver import read_inlet_file, inlet_values, inlet_counts
    n, pl, ubulk = 8, 2, 0.7
    rng = np.random.default_rng(3)
    for code in (7, 8):
        pr = Problem(1, 1, 1, 2 * n, n, n, bc=(code, 2, WALL, WALL, WALL, WALL), ngrid=2, pl=pl)
        d = pr.descriptors(oracle)[0]
        nu, nv, nw = inlet_counts(d, code)
        if code == 7:
            vals = rng.uniform(-1, 1, nu + nv + nw)
            path = tmp_path / "Inlet_000_00001.dat"
            path.write_text("".join(f"  {x:.17E}\n" for x in vals))
        else:
            cols = rng.uniform(-1, 1, (max(nu, nv, nw), 3))
            path = tmp_path / "Inlet_0000_000001.dat"
            path.write_text("header one\nheader two\n" + "".join(f" {a:.17E} {b:.17E} {c:.17E}\n" for a, b, c in cols))
        got = inlet_values(d, code, read_inlet_file(str(path), code))
        blocks = pr.block_fields(seed=25)
        assert oracle.orc_set_inlet(0, code, 0, got.ctypes.data_as(C.POINTER(C.c_double)), got.size) == 0
        try:
            st, _, _ = solve(oracle, pr, blocks, maxcy=3, eps=1e-12, pl_ex=1, bounds=1, alfabc=1, ubulk=ubulk)
        finally:
            oracle.orc_clear_inlets()
        assert st >= 0
        # rows js..je, planes ks..ke (the wall faces mirror into the ghost rows)
        I = slice(pl, pl + n)
        Iv, Iw = slice(pl, pl + n - 1), slice(pl, pl + n - 1)
        for ly in range(2):
            x = pl - 1 - ly
            if code == 7:
                u_plane = got[:nu].reshape(n + 2, n + 2)
                v_plane = got[nu:nu + nv].reshape(n + 2, n + 1)
                w_plane = got[nu + nv:].reshape(n + 1, n + 2)
                assert np.array_equal(blocks[0]["u"][I, I, x], u_plane[1:n + 1, 1:n + 1])
                assert np.array_equal(blocks[0]["v"][I, Iv, x], v_plane[1:n + 1, 1:n])
                assert np.array_equal(blocks[0]["w"][Iw, I, x], w_plane[1:n, 1:n + 1])
            else:
                assert np.array_equal(blocks[0]["u"][I, I, x], ubulk + got[:nu].reshape(n + 1, n + 1)[1:, 1:])
                assert np.array_equal(blocks[0]["v"][I, Iv, x], got[nu:nu + nv].reshape(n + 1, n)[1:, 1:])
                assert np.array_equal(blocks[0]["w"][Iw, I, x], got[nu + nv:].reshape(n, n + 1)[1:, 1:])


def test_bounds_convective_outflow_in_the_solve(oracle):
    """East code 21 with alfabc = 1 at the end of the solve (bounds.for:
    141-170, 449-474, 743-768): every east ghost layer of u, v, w is
    oo(ie+1+ly) - dt*alfapr*(oo(ie+1+ly) - oo(ie))/dx from the bound old
    velocities, with the solve's dt and alfapr; with nothing bound the face
    is refused."""
    n, pl, dt, alfapr = 8, 2, 0.37, 1.3
    pr = Problem(1, 1, 1, 2 * n, n, n, bc=(1, 21, WALL, WALL, WALL, WALL), ngrid=2, pl=pl)
    blocks = pr.block_fields(seed=26)
    rng = np.random.default_rng(27)
    oo = {k: rng.uniform(-1, 1, blocks[0]["u"].shape) for k in ("uoo", "voo", "woo")}
    ptrs = [(ob._dp * 1)(oo[k].ctypes.data_as(ob._dp)) for k in ("uoo", "voo", "woo")]
    oracle.orc_bind_old_velocity(1, *ptrs)
    try:
        prm = pr.params(maxcy=4, eps=1e-12, pl_ex=1, bounds=1, alfabc=1, ubulk=0.7)
        hist = np.zeros(4)
        info = SolveInfo()
        st = oracle.orc_newsolv_mg(pr.descriptors(oracle), 1, C.byref(prm), fields_struct(blocks), dt, alfapr,
                                   C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), 4)
    finally:
        oracle.orc_bind_old_velocity(0, None, None, None)
    assert st >= 0
    J, K = slice(pl, pl + n), slice(pl, pl + n)
    for k, ie in (("u", pl + 2 * n - 2), ("v", pl + 2 * n - 1), ("w", pl + 2 * n - 1)):
        o = oo[k + "oo"]
        Jc = slice(pl, pl + n - 1) if k == "v" else J  # v's last face is a wall face
        Kc = slice(pl, pl + n - 1) if k == "w" else K
        for ly in range(2):
            g = ie + 1 + ly
            want = o[Kc, Jc, g] - dt * alfapr * (o[Kc, Jc, g] - o[Kc, Jc, ie]) / pr.dx
            assert np.array_equal(blocks[0][k][Kc, Jc, g], want), (k, ly)
    st, _, _ = solve(oracle, pr, pr.block_fields(seed=26), maxcy=2, bounds=1, alfabc=1)
    assert st == -6


def smooth_wall_tau2(vtan, delta, re):
    """log_law.for:47-75 in numpy (smooth wall, code 61): tau2 of the log law
    where y+ >= 11.067, else the kept value (0 at the start)."""
    rrey, kappa, E = 1.0 / re, 0.41, 9.0
    out = np.zeros_like(vtan)
    for idx, vt in np.ndenumerate(vtan):
        ustar, conv, it = 1.0, 1.0, 0
        while conv > 1e-3 and it < 10:
            it += 1
            old = ustar
            yplus = max(1.0000001, delta * ustar / rrey)
            ustar = vt * kappa / np.log(E * yplus)
            conv = abs((ustar - old) / ustar)
        assert it < 10
        if yplus >= 11.067:
            out[idx] = ustar * ustar / vt
    return out


def test_bounds_wall_function_known_answer(oracle):
    """Code 61 on the bottom face (boundu, bounds.for:260-283, with
    log_law(5), log_law.for:206-254): on the interior face cells u(i,j,ks)
    += sign(tau2*u/dx, -u)*alfapr*dt and u(i,j,ks-1) = -u(i,j,ks), tau2 from
    the smooth-wall log law of the first cell layer; the normal component w
    is 0 on every ghost layer; without Re the code is refused."""
    from multiflow3d_b200.problems import fields_struct
    n, pl, dt, alfapr, re = 8, 2, 0.05, 1.0, 2.0e4
    pr = Problem(1, 1, 1, n, n, n, bc=(WALL, WALL, WALL, WALL, 61, WALL), ngrid=2, pl=pl, dx=0.1, dy=0.1, dz=0.1)
    rng = np.random.default_rng(28)
    shape = (n + 2 * pl,) * 3
    f = {k: rng.uniform(0.5, 1.5, shape) for k in ("u", "v", "w")}
    f.update({k: np.zeros(shape) for k in ("ustar", "vstar", "wstar", "p", "su")})
    before = {k: f[k].copy() for k in ("u", "v", "w")}
    prm = pr.params(pl_ex=1, bounds=1)
    assert oracle.orc_bounds(pr.descriptors(oracle), 1, C.byref(prm), fields_struct([f]), dt, alfapr, 1) == -6
    oracle.orc_set_wall_model(re, 0.0)
    try:
        assert oracle.orc_bounds(pr.descriptors(oracle), 1, C.byref(prm), fields_struct([f]), dt, alfapr, 1) == 0
    finally:
        oracle.orc_set_wall_model(0.0, 0.0)
    u0, v0, w0 = before["u"], before["v"], before["w"]
    ks = pl  # 0-based first interior plane
    # i = isp+1 .. iep-1 (the law reads u(i-1) inside; u(iep) is the east
    # wall face, zeroed by boundu's east branch first), j = jsp+1 .. jep
    I, Im = slice(pl + 1, pl + n - 1), slice(pl, pl + n - 2)
    J, Jm = slice(pl + 1, pl + n), slice(pl, pl + n - 1)
    uc = 0.5 * (u0[ks, J, I] + u0[ks, J, Im])
    vc = 0.5 * (v0[ks, J, I] + v0[ks, Jm, I])
    wc = 0.5 * (w0[ks, J, I] + w0[ks - 1, J, I])
    vtan = np.sqrt(np.abs(uc * uc + vc * vc + wc * wc - wc * wc + 1e-30))
    tau2 = smooth_wall_tau2(vtan, 0.1, re)
    assert (tau2 > 0).any()
    uu = u0[ks, J, I]
    fw = np.copysign(np.abs(tau2 * uu / 0.1), -uu)
    want = uu + fw * alfapr * dt
    np.testing.assert_allclose(f["u"][ks, J, I], want, rtol=1e-14, atol=0)
    assert np.array_equal(f["u"][ks - 1, J, I], -f["u"][ks, J, I])
    for ly in range(2):
        assert not f["w"][ks - 1 - ly, pl:pl + n, pl:pl + n].any()

"""The velocity predictor upstream of the projection: one Runge-Kutta stage
of rungek_conv2nd (rungek.for:314-412) and rungek_diff2nd (:584-779).  The
oracle's restatement is pinned here against an independent numpy
evaluation of the same expressions (the same IEEE operations in the same
order, hence bit for bit) and against the identity at dt = 0; the GPU
parity tests are in test_gpu_rungek.py."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200.abi import RkFields
from multiflow3d_b200.problems import Problem, fields_struct, PERIODIC, WALL
import oracle_bridge as ob

P, W = PERIODIC, WALL


def rk_inputs(pr, seed):
    """u, v, w, ustar.. and p as the projection's tests build them, plus
    start-of-step velocities and a positive viscosity field (ttc layout)."""
    rng = np.random.default_rng(seed)
    blocks = pr.block_fields(seed=seed, fourier_modes=2)
    rk = []
    for f in blocks:
        shp = f["u"].shape
        rk.append({"uoo": f["u"] + 0.1 * rng.standard_normal(shp), "voo": f["v"] + 0.1 * rng.standard_normal(shp),
                   "woo": f["w"] + 0.1 * rng.standard_normal(shp), "vis": 1e-3 * (1.0 + rng.random(shp))})
    return blocks, rk


def rk_struct(rk):
    arr = (RkFields * len(rk))()
    for b, f in enumerate(rk):
        for k in ("uoo", "voo", "woo", "vis"):
            setattr(arr[b], k, f[k].ctypes.data_as(C.POINTER(C.c_double)))
    return arr


def orc_rk(oracle, pr, blocks, rk, dt, alfapr, alfabc=1, pforce=0, forcn=0.0, **kw):
    prm = pr.params(pl_ex=kw.get("pl_ex", 0), alfabc=alfabc, ubulk=kw.get("ubulk", 0.0),
                    differencing=kw.get("differencing", 1))
    return oracle.orc_rungek_2nd(pr.descriptors(oracle), pr.nblocks, C.byref(prm), fields_struct(blocks),
                                 rk_struct(rk), dt, alfapr, alfabc, pforce, forcn)


def numpy_stage(u, v, w, uoo, voo, woo, vis, dx, dy, dz, dt, alfapr, pforce, forcn, sl):
    """The reference's expressions, vectorised; arrays [k, j, i]; `sl` the
    interior slices of the component's range."""
    def at(a, di=0, dj=0, dk=0):
        return a[sl[0].start + dk:sl[0].stop + dk, sl[1].start + dj:sl[1].stop + dj, sl[2].start + di:sl[2].stop + di]
    out = []
    for op in range(3):
        c = (u, v, w)[op]
        if op == 0:
            up12 = 0.5 * (at(u) + at(u, 1)); um12 = 0.5 * (at(u) + at(u, -1))
            c1 = (up12 * up12 - um12 * um12) / dx
            c2 = 0.25 * ((at(v) + at(v, 1)) * (at(u) + at(u, 0, 1)) - (at(v, 0, -1) + at(v, 1, -1)) * (at(u) + at(u, 0, -1))) / dy
            c3 = 0.25 * ((at(w) + at(w, 1)) * (at(u) + at(u, 0, 0, 1)) - (at(w, 0, 0, -1) + at(w, 1, 0, -1)) * (at(u) + at(u, 0, 0, -1))) / dz
            oo, visc = at(uoo), at(vis, 1)
        elif op == 1:
            vp12 = 0.5 * (at(v) + at(v, 0, 1)); vm12 = 0.5 * (at(v) + at(v, 0, -1))
            c2 = (vp12 * vp12 - vm12 * vm12) / dy
            c1 = 0.25 * ((at(u) + at(u, 0, 1)) * (at(v) + at(v, 1)) - (at(u, -1) + at(u, -1, 1)) * (at(v) + at(v, -1))) / dx
            c3 = 0.25 * ((at(w) + at(w, 0, 1)) * (at(v) + at(v, 0, 0, 1)) - (at(w, 0, 0, -1) + at(w, 0, 1, -1)) * (at(v) + at(v, 0, 0, -1))) / dz
            oo, visc = at(voo), at(vis, 0, 1)
        else:
            wp12 = 0.5 * (at(w) + at(w, 0, 0, 1)); wm12 = 0.5 * (at(w) + at(w, 0, 0, -1))
            c3 = (wp12 * wp12 - wm12 * wm12) / dz
            c1 = 0.25 * ((at(u) + at(u, 0, 0, 1)) * (at(w) + at(w, 1)) - (at(u, -1) + at(u, -1, 0, 1)) * (at(w) + at(w, -1))) / dx
            c2 = 0.25 * ((at(v) + at(v, 0, 0, 1)) * (at(w) + at(w, 0, 1)) - (at(v, 0, -1) + at(v, 0, -1, 1)) * (at(w) + at(w, 0, -1))) / dy
            oo, visc = at(woo), at(vis, 0, 0, 1)
        st = oo - dt * alfapr * (c1 + c2 + c3)
        dxx, dyy, dzz = dx * dx, dy * dy, dz * dz
        aw = -visc / dxx; ae = -visc / dxx; an = -visc / dyy; as_ = -visc / dyy; at_ = -visc / dzz; ab = -visc / dzz
        ap = -1.0 * (aw + ae + as_ + an + ab + at_)
        diff = -(ap * at(c) + an * at(c, 0, 1) + as_ * at(c, 0, -1) + ae * at(c, 1) + aw * at(c, -1) +
                 at_ * at(c, 0, 0, 1) + ab * at(c, 0, 0, -1))
        st = st + dt * alfapr * diff
        if op == 0 and pforce:
            st = st + dt * alfapr * forcn
        out.append(st)
    return out


def numpy_stage4(u, v, w, uoo, voo, woo, vis, dx, dy, dz, dt, alfapr, pforce, forcn, sl):
    """rungek_conv4th + rungek_diff4th (rungek.for:2-312), vectorised the
    way the reference writes each term; arrays [k, j, i]."""
    def at(a, di=0, dj=0, dk=0):
        return a[sl[0].start + dk:sl[0].stop + dk, sl[1].start + dj:sl[1].stop + dj, sl[2].start + di:sl[2].stop + di]

    def sh(ax, m):  # offset m along axis ax (0 x, 1 y, 2 z) as (di, dj, dk)
        return tuple(m if a == ax else 0 for a in range(3))

    def add(o1, o2):
        return tuple(x + y for x, y in zip(o1, o2))

    def q4(f, ax, base):  # (-f(+1) + 9 f(0) + 9 f(-1) - f(-2)) / 16 along ax, around offset `base`
        return (-at(f, *add(base, sh(ax, 1))) + 9.0 * at(f, *base) + 9.0 * at(f, *add(base, sh(ax, -1)))
                - at(f, *add(base, sh(ax, -2)))) / 16.0

    def d4(p1, p0, m1, m2, h):
        return (-p1 + 27.0 * p0 - 27.0 * m1 + m2) / (24.0 * h)
    vel = (u, v, w)
    oos = (uoo, voo, woo)
    hs = (dx, dy, dz)
    out = []
    for a in range(3):
        c = vel[a]
        terms = []
        for b in range(3):
            if b == a:  # self term: the squared interpolant at faces +2 .. -1
                s = [q4(c, a, sh(a, m)) for m in (2, 1, 0, -1)]
                terms.append(d4(*[x * x for x in s], hs[a]))
            else:  # cross term: c interpolated along b times the b-velocity interpolated along a
                prod = [q4(c, b, sh(b, m + 1)) * q4(vel[b], a, add(sh(b, m), sh(a, 1))) for m in (1, 0, -1, -2)]
                terms.append(d4(*prod, hs[b]))
        st = at(oos[a]) - dt * alfapr * (terms[0] + terms[1] + terms[2])
        visc = at(vis) if a == 0 else at(vis, *sh(a, 1))
        lap = []
        for b in range(3):
            lap.append((-at(c, *sh(b, 2)) + 16.0 * at(c, *sh(b, 1)) - 30.0 * at(c) + 16.0 * at(c, *sh(b, -1))
                        - at(c, *sh(b, -2))) / (12.0 * (hs[b] * hs[b])))
        diff = visc * (lap[0] + lap[1] + lap[2])
        st = st + dt * alfapr * diff
        if a == 0 and pforce:
            st = st + dt * alfapr * forcn
        out.append(st)
    return out


def test_oracle_predictor_4th_order_matches_numpy(oracle):
    """differencing = 2: rungek_conv4th and rungek_diff4th (rungek.for:2-312),
    the oracle against a vectorised evaluation of the same expressions, on a
    periodic block with three ghost layers (the stencils reach i-3 .. i+3);
    pl = 2 is refused."""
    pr = Problem(1, 1, 1, 12, 10, 8, bc=(P,) * 6, ngrid=1, pl=3, dx=0.1, dy=0.125, dz=0.3)
    blocks, rk = rk_inputs(pr, 8)
    given = {k: blocks[0][k].copy() for k in ("u", "v", "w")}
    dt, alfapr, forcn = 0.017, 0.6, 0.2
    assert orc_rk(oracle, pr, blocks, rk, dt, alfapr, pforce=1, forcn=forcn, differencing=2) == 0
    f = blocks[0]
    pl, n = pr.pl, (pr.nz, pr.ny, pr.nx)
    sl = tuple(slice(pl, pl + m) for m in n)
    args = (rk[0]["uoo"], rk[0]["voo"], rk[0]["woo"], rk[0]["vis"], pr.dx, pr.dy, pr.dz, dt, alfapr, 1, forcn, sl)
    us = numpy_stage4(f["u"], given["v"], given["w"], *args)[0]
    vs = numpy_stage4(f["u"], f["v"], given["w"], *args)[1]
    ws = numpy_stage4(f["u"], f["v"], f["w"], *args)[2]
    assert np.array_equal(f["ustar"][sl], us)
    assert np.array_equal(f["vstar"][sl], vs)
    assert np.array_equal(f["wstar"][sl], ws)
    pr2 = Problem(1, 1, 1, 12, 10, 8, bc=(P,) * 6, ngrid=1, pl=2)
    b2, r2 = rk_inputs(pr2, 8)
    assert orc_rk(oracle, pr2, b2, r2, dt, alfapr, differencing=2) == -1


def numpy_weno5(v1, v2, v3, v4, v5):
    """HJ_WENO's fifth-order derivative from five divided differences (weno.for:56-78)."""
    e = 1.0e-6 * np.maximum(np.maximum(np.maximum(np.maximum(v1 * v1, v2 * v2), v3 * v3), v4 * v4), v5 * v5) + 1.0e-99
    t11, t12 = v1 - 2.0 * v2 + v3, v1 - 4.0 * v2 + 3.0 * v3
    t21, t22 = v2 - 2.0 * v3 + v4, v2 - v4
    t31, t32 = v3 - 2.0 * v4 + v5, 3.0 * v3 - 4.0 * v4 + v5
    s1 = (13.0 / 12.0) * (t11 * t11) + 0.25 * (t12 * t12)
    s2 = (13.0 / 12.0) * (t21 * t21) + 0.25 * (t22 * t22)
    s3 = (13.0 / 12.0) * (t31 * t31) + 0.25 * (t32 * t32)
    a1, a2, a3 = 0.1 / ((e + s1) * (e + s1)), 0.6 / ((e + s2) * (e + s2)), 0.3 / ((e + s3) * (e + s3))
    w1, w2, w3 = a1 / (a1 + a2 + a3), a2 / (a1 + a2 + a3), a3 / (a1 + a2 + a3)
    return (w1 * (v1 * (1.0 / 3.0) - v2 * (7.0 / 6.0) + v3 * (11.0 / 6.0)) +
            w2 * (-(v2 * (1.0 / 6.0)) + v3 * (5.0 / 6.0) + v4 * (1.0 / 3.0)) +
            w3 * (v3 * (1.0 / 3.0) + v4 * (5.0 / 6.0) - v5 * (1.0 / 6.0)))


def numpy_weno_derivs(f, ax, ends, h):
    """HJ_WENO along numpy axis ax (2 = x, 1 = y, 0 = z) of field f [k, j, i]:
    (plus, minus), zero outside the computed range; ends = 1-based range
    ends (x, y, z) = component ends + pl_ex + 1."""
    lim = (ends[2], ends[1], ends[0])  # numpy axis order (z, y, x)
    d1 = np.zeros_like(f)
    sl = [slice(0, lim[0]), slice(0, lim[1]), slice(0, lim[2])]
    sl[ax] = slice(0, lim[ax] - 1)
    hi = list(sl)
    hi[ax] = slice(1, lim[ax])
    d1[tuple(sl)] = (f[tuple(hi)] - f[tuple(sl)]) / h
    plus, minus = np.zeros_like(f), np.zeros_like(f)
    n = lim[ax] - 6

    def take(m):
        s2 = [slice(0, lim[0]), slice(0, lim[1]), slice(0, lim[2])]
        s2[ax] = slice(m, m + n)
        return d1[tuple(s2)]
    dst = [slice(0, lim[0]), slice(0, lim[1]), slice(0, lim[2])]
    dst[ax] = slice(3, 3 + n)
    plus[tuple(dst)] = numpy_weno5(take(5), take(4), take(3), take(2), take(1))
    minus[tuple(dst)] = numpy_weno5(take(0), take(1), take(2), take(3), take(4))
    return plus, minus


def test_oracle_predictor_weno_matches_numpy(oracle):
    """differencing = 3: rungek_convWENO (rungek.for:414-582, HJ_WENO of
    weno.for) and rungek_diff2nd, the oracle against a vectorised
    evaluation on a periodic block with pl = 4, pl_ex = 2 (as initial.for
    sets them for WENO)."""
    pr = Problem(1, 1, 1, 12, 10, 8, bc=(P,) * 6, ngrid=1, pl=4, dx=0.1, dy=0.125, dz=0.3)
    blocks, rk = rk_inputs(pr, 9)
    for k in ("u", "v", "w"):  # some exact zeros: the upwinding's third branch
        blocks[0][k][5, 5, 5:9] = 0.0
    given = {k: blocks[0][k].copy() for k in ("u", "v", "w")}
    dt, alfapr, forcn, pl_ex = 0.011, 0.6, 0.15, 2
    assert orc_rk(oracle, pr, blocks, rk, dt, alfapr, pforce=1, forcn=forcn, differencing=3, pl_ex=pl_ex) == 0
    f = blocks[0]
    pl = pr.pl
    sl = tuple(slice(pl, pl + m) for m in (pr.nz, pr.ny, pr.nx))
    ends = (pr.nx + pl + pl_ex + 1, pr.ny + pl + pl_ex + 1, pr.nz + pl + pl_ex + 1)
    hs = {2: pr.dx, 1: pr.dy, 0: pr.dz}

    def at(a, di=0, dj=0, dk=0):
        return a[sl[0].start + dk:sl[0].stop + dk, sl[1].start + dj:sl[1].stop + dj, sl[2].start + di:sl[2].stop + di]

    def upwind(a, ax, fld):
        plus, minus = numpy_weno_derivs(fld, ax, ends, hs[ax])
        return np.where(a > 0.0, at(minus), np.where(a < 0.0, at(plus), 0.0))
    # the u loop sees v, w as given; the v loop w as given (their bounds come later)
    u, v, w = f["u"], given["v"], given["w"]
    uc = at(u)
    vijk = 0.25 * (at(v) + at(v, 1) + at(v, 0, -1) + at(v, 1, -1))
    wijk = 0.25 * (at(w) + at(w, 1) + at(w, 0, 0, -1) + at(w, 1, 0, -1))
    conv_u = uc * upwind(uc, 2, u) + vijk * upwind(vijk, 1, u) + wijk * upwind(wijk, 0, u)
    v = f["v"]
    vc = at(v)
    uijk = 0.25 * (at(u) + at(u, 0, 1) + at(u, -1) + at(u, -1, 1))
    wijk = 0.25 * (at(w) + at(w, 0, 1) + at(w, 0, 0, -1) + at(w, 0, 1, -1))
    conv_v = uijk * upwind(uijk, 2, v) + vc * upwind(vc, 1, v) + wijk * upwind(wijk, 0, v)
    w = f["w"]
    wc = at(w)
    uijk = 0.25 * (at(u) + at(u, 0, 0, 1) + at(u, -1) + at(u, -1, 0, 1))
    vijk = 0.25 * (at(v) + at(v, 0, 0, 1) + at(v, 0, -1) + at(v, 0, -1, 1))
    conv_w = uijk * upwind(uijk, 2, w) + vijk * upwind(vijk, 1, w) + wc * upwind(wc, 0, w)
    # rungek_diff2nd after the three loops, on the final u, v, w
    dxx, dyy, dzz = pr.dx * pr.dx, pr.dy * pr.dy, pr.dz * pr.dz
    for a, (key, oo, conv, vshift) in enumerate((("ustar", "uoo", conv_u, (1, 0, 0)), ("vstar", "voo", conv_v, (0, 1, 0)),
                                                 ("wstar", "woo", conv_w, (0, 0, 1)))):
        c = f["uvw"[a]]
        st = at(rk[0][oo]) - dt * alfapr * conv
        visc = at(rk[0]["vis"], *vshift)
        aw = -visc / dxx; ae = -visc / dxx; an = -visc / dyy; as_ = -visc / dyy; at_ = -visc / dzz; ab = -visc / dzz
        ap = -1.0 * (aw + ae + as_ + an + ab + at_)
        diff = -(ap * at(c) + an * at(c, 0, 1) + as_ * at(c, 0, -1) + ae * at(c, 1) + aw * at(c, -1) +
                 at_ * at(c, 0, 0, 1) + ab * at(c, 0, 0, -1))
        st = st + dt * alfapr * diff
        if a == 0:
            st = st + dt * alfapr * forcn
        assert np.array_equal(f[key][sl], st), key


def test_oracle_predictor_matches_numpy(oracle):
    """One periodic block: boundu/v/w wrap the ghosts; the u predictor reads
    v and w as given, the v predictor w as given (their bounds come after)."""
    pr = Problem(1, 1, 1, 12, 10, 8, bc=(P,) * 6, ngrid=1, pl=2, dx=0.1, dy=0.125, dz=0.3)
    blocks, rk = rk_inputs(pr, 3)
    given = {k: blocks[0][k].copy() for k in ("u", "v", "w")}
    dt, alfapr, forcn = 0.013, 0.7, 0.25
    assert orc_rk(oracle, pr, blocks, rk, dt, alfapr, pforce=1, forcn=forcn) == 0
    f = blocks[0]
    pl, n = pr.pl, (pr.nz, pr.ny, pr.nx)
    sl = tuple(slice(pl, pl + m) for m in n)
    args = (rk[0]["uoo"], rk[0]["voo"], rk[0]["woo"], rk[0]["vis"], pr.dx, pr.dy, pr.dz, dt, alfapr, 1, forcn, sl)
    us = numpy_stage(f["u"], given["v"], given["w"], *args)[0]
    vs = numpy_stage(f["u"], f["v"], given["w"], *args)[1]
    ws = numpy_stage(f["u"], f["v"], f["w"], *args)[2]
    assert np.array_equal(f["ustar"][sl], us)
    assert np.array_equal(f["vstar"][sl], vs)
    assert np.array_equal(f["wstar"][sl], ws)
    # the periodic wrap the bounds applied
    assert np.array_equal(f["u"][:, :, pl - 1], f["u"][:, :, pl + pr.nx - 1])


def test_oracle_predictor_zero_step_is_identity(oracle):
    pr = Problem(2, 1, 1, 8, 8, 8, bc=(1, 2, W, W, P, P), ngrid=2, pl=2)
    blocks, rk = rk_inputs(pr, 4)
    assert orc_rk(oracle, pr, blocks, rk, 0.0, 1.0, alfabc=1, ubulk=0.5) == 0
    pl = pr.pl
    for f, r in zip(blocks, rk):
        I = (slice(pl, pl + pr.nz), slice(pl, pl + pr.ny), slice(pl, pl + pr.nx - 1))
        assert np.array_equal(f["ustar"][I], r["uoo"][I])


def test_oracle_predictor_convective_outflow(oracle):
    """Code 21 on the east face, first stage: every ghost layer of u, v, w
    holds oo(g) - dt*alfapr*(oo(g) - oo(ie))/dx from the start-of-step
    velocity (bounds.for:143-170 and boundv/boundw's branch); ie is one face
    short of the boundary for u.  v's row on the north wall face is checked
    out: the north face comes after the east one and zeroes it there."""
    pr = Problem(1, 1, 1, 12, 8, 8, bc=(1, 21, W, W, P, P), ngrid=1, pl=2, dx=0.1, dy=0.1, dz=0.1)
    blocks, rk = rk_inputs(pr, 6)
    dt, alfapr = 0.02, 0.5
    assert orc_rk(oracle, pr, blocks, rk, dt, alfapr, alfabc=1, pl_ex=1, ubulk=0.3) == 0
    pl, n = pr.pl, pr.nx
    J, K = slice(pl, pl + pr.ny), slice(pl, pl + pr.nz)
    for k, ie in (("u", pl + n - 2), ("v", pl + n - 1), ("w", pl + n - 1)):
        oo = rk[0][k[0] + "oo"]
        Jc = slice(pl, pl + pr.ny - 1) if k == "v" else J
        for ly in range(2):
            g = ie + 1 + ly
            want = oo[K, Jc, g] - dt * alfapr * (oo[K, Jc, g] - oo[K, Jc, ie]) / pr.dx
            assert np.array_equal(blocks[0][k][K, Jc, g], want), (k, ly)


def test_oracle_predictor_refuses_other_branches(oracle):
    pr = Problem(1, 1, 1, 8, 8, 8, ngrid=1, pl=1, stretch_y=2.0)
    blocks, rk = rk_inputs(pr, 5)
    assert orc_rk(oracle, pr, blocks, rk, 0.1, 1.0) == -6
    pr = Problem(1, 1, 1, 8, 8, 8, bc=(7, 2, W, W, W, W), ngrid=1, pl=1)
    blocks, rk = rk_inputs(pr, 5)
    assert orc_rk(oracle, pr, blocks, rk, 0.1, 1.0, alfabc=1) == -1  # code 7 with no inlet values

"""Block layouts and seeded synthetic inputs for the projection path.

A *problem* is a Cartesian box split into ``px x py x pz`` equal blocks of
``nx x ny x nz`` cells, with the six global boundary codes of control.cin
(5 = periodic, anything else = wall, i.e. homogeneous Neumann for p).  Block
ids are numbered x fastest, like infodom.cin.

Inputs follow one parity recipe for every configuration:
``ustar, vstar, wstar`` i.i.d. uniform [-1, 1] (optionally plus smooth
Fourier modes), each component made mean-free over the interior faces, wall
faces zeroed as ``boundu/boundv/boundw`` leave them (bounds.for:2-916).  The
inputs are generated on the *global* grid and sliced into blocks, so every
decomposition of the same box sees the same field.

Arrays use the reference's field layout: Fortran ``(ttc_i, ttc_j, ttc_k)``,
i fastest, ``pl`` ghost layers - here numpy arrays of shape
``(ttc_k, ttc_j, ttc_i)`` in C order, which is the same memory.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from .abi import BlockDesc, Params, Fields, MF3D_PREC_FP64

PERIODIC = 5
WALL = 4


@dataclass
class Problem:
    px: int
    py: int
    pz: int
    nx: int
    ny: int
    nz: int
    bc: tuple = (PERIODIC, PERIODIC, WALL, WALL, PERIODIC, PERIODIC)  # W,E,S,N,B,T
    dx: float = 1.0 / 32
    dy: float = 1.0 / 32
    dz: float = 1.0 / 32
    pl: int = 1
    ngrid: int = 4
    stretch_y: float = 0.0  # tanh stretching factor in y (0 = uniform)
    _hy_global: np.ndarray | None = field(default=None, repr=False)

    @property
    def nblocks(self) -> int:
        return self.px * self.py * self.pz

    @property
    def NX(self) -> int:
        return self.px * self.nx

    @property
    def NY(self) -> int:
        return self.py * self.ny

    @property
    def NZ(self) -> int:
        return self.pz * self.nz

    @property
    def ttc(self) -> tuple:
        return (self.nz + 2 * self.pl, self.ny + 2 * self.pl, self.nx + 2 * self.pl)

    def block_pos(self, b: int) -> tuple:
        return b % self.px, (b // self.px) % self.py, b // (self.px * self.py)

    def extents(self) -> np.ndarray:
        """xsl,xel,ysl,yel,zsl,zel per block (infodom.cin columns 3-8).

        Extents are integer cell counts times the spacing, so adjacent
        blocks share bit-identical face coordinates."""
        e = np.zeros((self.nblocks, 6))
        for b in range(self.nblocks):
            bx, by, bz = self.block_pos(b)
            e[b] = [bx * self.nx * self.dx, (bx + 1) * self.nx * self.dx,
                    by * self.ny * self.dy, (by + 1) * self.ny * self.dy,
                    bz * self.nz * self.dz, (bz + 1) * self.nz * self.dz]
        return e

    # ------------------------------------------------------------------
    # stretching (extension: the reference grid is uniform per block)
    # ------------------------------------------------------------------
    def hy_global(self) -> np.ndarray | None:
        """Global y cell widths with tanh clustering at both walls."""
        if self.stretch_y == 0.0:
            return None
        if self._hy_global is None:
            Ly = self.NY * self.dy
            s = np.arange(self.NY + 1) / self.NY
            beta = self.stretch_y
            yn = 0.5 * Ly * (1.0 + np.tanh(beta * (2.0 * s - 1.0)) / np.tanh(beta))
            self._hy_global = np.diff(yn)
        return self._hy_global

    def block_widths_y(self, b: int) -> np.ndarray | None:
        """Extended widths of block b: ny cells plus W = 2^(ngrid-1) neighbour
        cells each side (wrap on periodic axes, mirror at walls)."""
        h = self.hy_global()
        if h is None:
            return None
        W = 1 << (self.ngrid - 1)
        _, by, _ = self.block_pos(b)
        idx = np.arange(by * self.ny - W, (by + 1) * self.ny + W)
        NY = self.NY
        if self.bc[2] == PERIODIC:
            idx = np.mod(idx, NY)
        else:
            idx = np.where(idx < 0, -1 - idx, idx)
            idx = np.where(idx >= NY, 2 * NY - 1 - idx, idx)
        return np.ascontiguousarray(h[idx])

    # ------------------------------------------------------------------
    def descriptors(self, lib) -> "C.Array":
        """Block descriptors from the neighbour search of ``lib`` (the
        library's ``mf3d_build_topology`` or the oracle's restatement)."""
        ext = np.ascontiguousarray(self.extents().ravel())
        bc6 = (C.c_int * 6)(*self.bc)
        arr = (BlockDesc * self.nblocks)()
        fn = getattr(lib, "mf3d_build_topology", None) or getattr(lib, "orc_build_topology")
        st = fn(self.nblocks, ext.ctypes.data_as(C.POINTER(C.c_double)), bc6,
                C.c_double(self.dx), C.c_double(self.dy), C.c_double(self.dz), arr)
        if st != 0:
            raise RuntimeError(f"topology build failed: {st}")
        # the descriptors point into these arrays: keep every call's alive
        # (descriptors for the library and for the oracle coexist)
        if not hasattr(self, "_keep"):
            self._keep = []
        for b in range(self.nblocks):
            hy = self.block_widths_y(b)
            if hy is not None:
                self._keep.append(hy)
                arr[b].hy = hy.ctypes.data_as(C.POINTER(C.c_double))
        return arr

    def params(self, mg_itrsch=3, irestr=2, iproln=1, maxcy=200, eps=1e-8,
               eps_relative=1, precision=MF3D_PREC_FP64, device=0, pl_ex=0, lsm=0, bounds=0, solver=0,
               nswp=0, differencing=1, alfabc=0, ubulk=0.0) -> Params:
        return Params(ngrid=self.ngrid, mg_itrsch=mg_itrsch, irestr=irestr,
                      iproln=iproln, maxcy=maxcy, eps=eps, eps_relative=eps_relative,
                      pl=self.pl, differencing=differencing, precision=precision, device=device,
                      pl_ex=pl_ex, lsm=lsm, bounds=bounds, solver=solver, nswp=nswp,
                      alfabc=alfabc, ubulk=ubulk)

    def block_density(self, seed: int, lo: float = 0.5, hi: float = 2.0, const: float | None = None):
        """Per-block cell densities (ttc layout) cut from one global field:
        i.i.d. uniform in [lo, hi] (or ``const`` everywhere), ghost layers
        wrapped on periodic axes, so every block sees its neighbours' cells."""
        pl = self.pl
        shp = (self.NZ + 2 * pl, self.NY + 2 * pl, self.NX + 2 * pl)
        if const is not None:
            g = np.full(shp, float(const))
        else:
            g = self.wrap_periodic(np.random.default_rng(seed).uniform(lo, hi, size=shp))
        out = []
        for b in range(self.nblocks):
            bx, by, bz = self.block_pos(b)
            sl = (slice(bz * self.nz, bz * self.nz + self.nz + 2 * pl),
                  slice(by * self.ny, by * self.ny + self.ny + 2 * pl),
                  slice(bx * self.nx, bx * self.nx + self.nx + 2 * pl))
            out.append(np.ascontiguousarray(g[sl]))
        return out

    # ------------------------------------------------------------------
    # seeded inputs
    # ------------------------------------------------------------------
    def global_velocity(self, seed: int, fourier_modes: int = 0, amp: float = 0.1):
        """Global face-velocity arrays with pl ghost layers, shape
        (NZ+2pl, NY+2pl, NX+2pl) each, plus the initial pressure (zeros)."""
        rng = np.random.default_rng(seed)
        pl = self.pl
        shp = (self.NZ + 2 * pl, self.NY + 2 * pl, self.NX + 2 * pl)
        comps = []
        for c in range(3):
            a = rng.uniform(-1.0, 1.0, size=shp)
            if fourier_modes:
                a += self._fourier(rng, fourier_modes, amp, c)
            inner = a[pl:pl + self.NZ, pl:pl + self.NY, pl:pl + self.NX]
            a -= inner.mean()
            comps.append(self.wrap_periodic(a))
        return comps

    def wrap_periodic(self, a: np.ndarray) -> np.ndarray:
        """Ghost layers of a global array made periodic along periodic axes
        (the state exchange_bc leaves them in)."""
        pl = self.pl
        for ax, n, bc in ((2, self.NX, self.bc[0]), (1, self.NY, self.bc[2]), (0, self.NZ, self.bc[4])):
            if bc != PERIODIC:
                continue
            idx = pl + np.mod(np.arange(a.shape[ax]) - pl, n)
            a = np.take(a, idx, axis=ax)
        return np.ascontiguousarray(a)

    def _fourier(self, rng, nmodes, amp, comp):
        pl = self.pl
        z = (np.arange(self.NZ + 2 * pl) - pl + 0.5) / self.NZ
        y = (np.arange(self.NY + 2 * pl) - pl + 0.5) / self.NY
        x = (np.arange(self.NX + 2 * pl) - pl + 0.5) / self.NX
        out = np.zeros((z.size, y.size, x.size))
        for _ in range(nmodes):
            kx, ky, kz = rng.integers(1, 4, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            out += amp * (np.sin(2 * np.pi * kz * z + ph[2])[:, None, None]
                          * np.sin(2 * np.pi * ky * y + ph[1])[None, :, None]
                          * np.sin(2 * np.pi * kx * x + ph[0])[None, None, :])
        return out

    def block_fields(self, seed: int = 1234, fourier_modes: int = 0, p_random: bool = False):
        """Per-block dict of ttc arrays: ustar, vstar, wstar, u, v, w, p, su."""
        us, vs, ws = self.global_velocity(seed, fourier_modes)
        rng = np.random.default_rng(seed + 7)
        pl = self.pl
        pg = (self.wrap_periodic(rng.uniform(-1, 1, size=us.shape)) if p_random else np.zeros_like(us))
        out = []
        for b in range(self.nblocks):
            bx, by, bz = self.block_pos(b)
            sl = (slice(bz * self.nz, bz * self.nz + self.nz + 2 * pl),
                  slice(by * self.ny, by * self.ny + self.ny + 2 * pl),
                  slice(bx * self.nx, bx * self.nx + self.nx + 2 * pl))
            f = {"ustar": us[sl].copy(), "vstar": vs[sl].copy(), "wstar": ws[sl].copy(),
                 "p": pg[sl].copy()}
            # wall faces as boundu/boundv/boundw leave them: zero normal velocity
            isp, iep = pl, pl + self.nx - 1  # 0-based field indices of isp, iep
            jsp, jep = pl, pl + self.ny - 1
            ksp, kep = pl, pl + self.nz - 1
            if bx == 0 and self.bc[0] != PERIODIC:
                f["ustar"][:, :, isp - 1] = 0.0
            if bx == self.px - 1 and self.bc[1] != PERIODIC:
                f["ustar"][:, :, iep] = 0.0
            if by == 0 and self.bc[2] != PERIODIC:
                f["vstar"][:, jsp - 1, :] = 0.0
            if by == self.py - 1 and self.bc[3] != PERIODIC:
                f["vstar"][:, jep, :] = 0.0
            if bz == 0 and self.bc[4] != PERIODIC:
                f["wstar"][ksp - 1, :, :] = 0.0
            if bz == self.pz - 1 and self.bc[5] != PERIODIC:
                f["wstar"][kep, :, :] = 0.0
            f["u"] = f["ustar"].copy()
            f["v"] = f["vstar"].copy()
            f["w"] = f["wstar"].copy()
            f["su"] = np.zeros_like(f["p"])
            out.append(f)
        return out

    def interior(self, a: np.ndarray) -> np.ndarray:
        pl = self.pl
        return a[pl:pl + self.nz, pl:pl + self.ny, pl:pl + self.nx]

    def gather(self, blocks, key: str) -> np.ndarray:
        """Assemble a global interior array (NZ, NY, NX) from block fields."""
        out = np.zeros((self.NZ, self.NY, self.NX))
        for b, f in enumerate(blocks):
            bx, by, bz = self.block_pos(b)
            out[bz * self.nz:(bz + 1) * self.nz, by * self.ny:(by + 1) * self.ny,
                bx * self.nx:(bx + 1) * self.nx] = self.interior(f[key])
        return out


def fields_struct(blocks) -> "C.Array":
    """``mf3d_fields[]`` pointing at numpy arrays (host) of ``blocks``."""
    arr = (Fields * len(blocks))()
    dp = C.POINTER(C.c_double)
    for b, f in enumerate(blocks):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p", "su", "dens"):
            a = f.get(k)
            if a is None and k == "dens":
                continue
            assert a.dtype == np.float64 and a.flags.c_contiguous
            setattr(arr[b], k, a.ctypes.data_as(dp))
    return arr


def domain_problem(nx, ny, nz, bc3, ngrid, h=None, pl=1):
    """A single-block Problem for one batch domain (bc per axis)."""
    h = h if h is not None else 1.0 / max(nx, ny, nz)
    bc = (bc3[0], bc3[0], bc3[1], bc3[1], bc3[2], bc3[2])
    return Problem(1, 1, 1, nx, ny, nz, bc=bc, dx=h, dy=h, dz=h, pl=pl, ngrid=ngrid)


def domain_desc(pr: Problem):
    from .abi import DomainDesc
    d = DomainDesc()
    d.nx, d.ny, d.nz = pr.nx, pr.ny, pr.nz
    d.dx, d.dy, d.dz = pr.dx, pr.dy, pr.dz
    d.bc[0], d.bc[1], d.bc[2] = pr.bc[0], pr.bc[2], pr.bc[4]
    d.ngrid = pr.ngrid
    return d


def random_batch(n, seed, lo=32, hi=192, multiple=8):
    """Domain sizes as the batched configuration draws them: each edge
    log-uniform in [lo, hi] rounded to a multiple of 8; BCs per axis drawn
    from {periodic, wall}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        e = np.exp(rng.uniform(np.log(lo), np.log(hi), size=3))
        nx, ny, nz = (int(max(multiple, round(x / multiple) * multiple)) for x in e)
        bc3 = tuple(int(PERIODIC if b else WALL) for b in rng.integers(0, 2, size=3))
        out.append((nx, ny, nz, bc3))
    return out

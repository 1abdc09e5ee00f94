"""LMR test layouts: unit-cube blocks on a px x py x pz grid, the blocks in
``refine`` at twice the resolution of the others (rdiv 2,
localparameters.for:100-102).  The neighbour search runs over the block
extents, which LMR leaves unchanged (alloc_dom.for:456-1150); the refined
blocks then take twice the cells and half the spacing."""
from __future__ import annotations

import ctypes as C

import numpy as np

from multiflow3d_b200.abi import BlockDesc, Params


class LmrLayout:
    def __init__(self, px, py, pz, n, refine, bc, ngrid_in, pl=2, drop=()):
        self.px, self.py, self.pz, self.n = px, py, pz, n
        self.refine = sorted(refine)
        self.bc = tuple(bc)
        # grid positions (i, j, k) of the blocks, x fastest; `drop` leaves
        # some out (an L-shaped domain has a re-entrant edge)
        self.pos = [(i, j, k) for k in range(pz) for j in range(py) for i in range(px) if (i, j, k) not in drop]
        self.nblocks = len(self.pos)
        self.pl = pl
        # ngrd_gl = ngrid_input + log2(max rdiv) (localparameters.for:33-34)
        self.ngrid = ngrid_in + (1 if self.refine else 0)
        self.h = 1.0 / n

    def extents(self):
        return np.array([[i, i + 1, j, j + 1, k, k + 1] for (i, j, k) in self.pos], dtype=np.float64)

    def descriptors(self, lib):
        ext = np.ascontiguousarray(self.extents().ravel())
        arr = (BlockDesc * self.nblocks)()
        fn = getattr(lib, "mf3d_build_topology", None) or getattr(lib, "orc_build_topology")
        st = fn(self.nblocks, ext.ctypes.data_as(C.POINTER(C.c_double)), (C.c_int * 6)(*self.bc),
                C.c_double(self.h), C.c_double(self.h), C.c_double(self.h), arr)
        if st != 0:
            raise RuntimeError(f"topology build failed: {st}")
        for b in self.refine:
            d = arr[b]
            d.nx, d.ny, d.nz = 2 * d.nx, 2 * d.ny, 2 * d.nz
            d.dx, d.dy, d.dz = d.dx / 2, d.dy / 2, d.dz / 2
        return arr

    def cells(self, b):
        r = 2 if b in self.refine else 1
        return (self.n * r,) * 3

    def ttc(self, b):
        nx, ny, nz = self.cells(b)
        return (nz + 2 * self.pl, ny + 2 * self.pl, nx + 2 * self.pl)

    def params(self, mg_itrsch=3, irestr=2, iproln=1, precision=0):
        return Params(ngrid=self.ngrid, mg_itrsch=mg_itrsch, irestr=irestr, iproln=iproln, maxcy=1, eps=1e-8,
                      eps_relative=1, pl=self.pl, differencing=1, precision=precision)

    def origin(self, b):
        return tuple(float(c) for c in self.pos[b])

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
    """`refine`: block positions of rdiv 2, or a dict position -> rdiv."""

    def __init__(self, px, py, pz, n, refine, bc, ngrid_in, pl=2, drop=()):
        self.px, self.py, self.pz, self.n = px, py, pz, n
        self.rdiv = dict(refine) if isinstance(refine, dict) else {b: 2 for b in refine}
        self.refine = sorted(self.rdiv)
        self.bc = tuple(bc)
        # grid positions (i, j, k) of the blocks, x fastest; `drop` leaves
        # some out (an L-shaped domain has a re-entrant edge)
        self.pos = [(i, j, k) for k in range(pz) for j in range(py) for i in range(px) if (i, j, k) not in drop]
        self.nblocks = len(self.pos)
        self.pl = pl
        # ngrd_gl = ngrid_input + log2(max rdiv) (localparameters.for:33-34)
        self.ngrid_in = ngrid_in
        self.ngrid = ngrid_in + max([0] + [r.bit_length() - 1 for r in self.rdiv.values()])
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
        for b, r in self.rdiv.items():
            d = arr[b]
            d.nx, d.ny, d.nz = r * d.nx, r * d.ny, r * d.nz
            d.dx, d.dy, d.dz = d.dx / r, d.dy / r, d.dz / r
        return arr

    def cells(self, b):
        return (self.n * self.rdiv.get(b, 1),) * 3

    def own_levels(self, b):
        """Levels of the block's own size: ngrid_input + log2(rdiv)."""
        return self.ngrid_in + self.rdiv.get(b, 1).bit_length() - 1

    def ttc(self, b):
        nx, ny, nz = self.cells(b)
        return (nz + 2 * self.pl, ny + 2 * self.pl, nx + 2 * self.pl)

    def params(self, mg_itrsch=3, irestr=2, iproln=1, precision=0):
        return Params(ngrid=self.ngrid, mg_itrsch=mg_itrsch, irestr=irestr, iproln=iproln, maxcy=1, eps=1e-8,
                      eps_relative=1, pl=self.pl, differencing=1, precision=precision)

    def origin(self, b):
        return tuple(float(c) for c in self.pos[b])


def random_layouts(seed, count, n=8, ngrid_in=3):
    """Seeded LMR layouts: grids of up to 3x3x2 blocks, some positions left
    out, a random set of refined blocks, walls or a periodic axis.  Along a
    periodic axis the refinement depends only on the other coordinates, so
    periodic partners share it (alloc_dom.for:210-221)."""
    import numpy as np
    from multiflow3d_b200.problems import PERIODIC, WALL
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        px, py, pz = int(rng.integers(1, 4)), int(rng.integers(1, 4)), int(rng.integers(1, 3))
        if px * py * pz < 2:
            continue
        per = int(rng.integers(0, 4))  # 0: walls; 1..3: that axis periodic
        if per and (px, py, pz)[per - 1] < 2:
            per = 0
        bc = [WALL] * 6
        if per:
            bc[2 * (per - 1)] = bc[2 * (per - 1) + 1] = PERIODIC
        cells = [(i, j, k) for k in range(pz) for j in range(py) for i in range(px)]
        drop = ()
        if not per and len(cells) > 3 and rng.random() < 0.4:
            drop = (cells[int(rng.integers(0, len(cells)))],)
        kept = [c for c in cells if c not in drop]
        # refinement keyed on the coordinates other than the periodic axis
        key = {}
        refine = []
        for b, c in enumerate(kept):
            kk = tuple(v for a, v in enumerate(c) if a != per - 1) if per else c
            if kk not in key:
                key[kk] = bool(rng.random() < 0.4)
            if key[kk]:
                refine.append(b)
        if not refine or len(refine) == len(kept):
            continue
        out.append(LmrLayout(px, py, pz, n, refine, tuple(bc), ngrid_in, drop=drop))
    return out

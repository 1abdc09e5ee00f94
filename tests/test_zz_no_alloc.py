"""mf3d_mgkcyc_device_noalloc: the V-cycle entry point that allocates no
device memory (its pointer tables live in a fixed device array) gives the
result of mf3d_mgkcyc_device on the same inputs, call after call.

The file name sorts last so that the entry point also runs after every
other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.problems import Problem, PERIODIC, WALL
from multiflow3d_b200.solver import Projection

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)
TOL = 1e-12  # relative L2; the two entry points run the same kernels on the same operands


def _ptrs(tensors):
    return (_dp * len(tensors))(*[C.cast(C.c_void_p(t.data_ptr()), _dp) for t in tensors])


def _rel(a, b):
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


@pytest.mark.parametrize("precision", [abi.MF3D_PREC_FP64, abi.MF3D_PREC_FP32])
def test_noalloc_matches_mgkcyc_device(lib, cuda, precision):
    import torch
    pr = Problem(2, 2, 1, 16, 8, 16, bc=(PERIODIC, PERIODIC, WALL, WALL, PERIODIC, PERIODIC), ngrid=3, pl=2)
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, precision=precision)
    proj = Projection(pr.descriptors(lib), prm, lib)
    rng = np.random.default_rng(5)
    rhs = [[torch.from_numpy(rng.uniform(-1, 1, size=pr.ttc)).to(cuda) for _ in range(pr.nblocks)]
           for _ in range(2)]

    def run(fn, su):
        pp = [torch.zeros(pr.ttc, dtype=torch.float64, device=cuda) for _ in range(pr.nblocks)]
        st = fn(proj.ctx, _ptrs(su), _ptrs(pp))
        assert st == abi.MF3D_OK, lib.mf3d_last_error()
        return [t.cpu().numpy() for t in pp]

    ref = [run(lib.mf3d_mgkcyc_device, su) for su in rhs]
    # two no-allocation calls in a row on different right-hand sides, then the
    # existing entry point again: every result equals the reference
    got = [run(lib.mf3d_mgkcyc_device_noalloc, su) for su in rhs]
    again = run(lib.mf3d_mgkcyc_device, rhs[0])
    proj.close()
    for r, g in zip(ref, got):
        for b in range(pr.nblocks):
            assert _rel(g[b], r[b]) <= TOL
            assert np.array_equal(g[b], r[b])
    for b in range(pr.nblocks):
        assert np.array_equal(again[b], ref[0][b])


@pytest.mark.parametrize("precision", [abi.MF3D_PREC_FP64, abi.MF3D_PREC_FP32])
def test_noalloc_first_on_fresh_context_allocates_nothing(lib, cuda, precision):
    """The no-allocation entry point as the first call on a new context: the
    device's free memory is the same before and after two calls (no lazily
    loaded kernel, no pool growth), and the results equal those of
    mf3d_mgkcyc_device on a second context."""
    import torch
    pr = Problem(2, 1, 2, 16, 16, 8, bc=(WALL, WALL, WALL, WALL, PERIODIC, PERIODIC), ngrid=3, pl=1)
    prm = pr.params(mg_itrsch=3, irestr=2, iproln=1, precision=precision)
    rng = np.random.default_rng(9)
    rhs = [[torch.from_numpy(rng.uniform(-1, 1, size=pr.ttc)).to(cuda) for _ in range(pr.nblocks)]
           for _ in range(2)]
    pps = [[torch.zeros(pr.ttc, dtype=torch.float64, device=cuda) for _ in range(pr.nblocks)] for _ in range(2)]
    fresh = Projection(pr.descriptors(lib), prm, lib)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    for su, pp in zip(rhs, pps):
        assert lib.mf3d_mgkcyc_device_noalloc(fresh.ctx, _ptrs(su), _ptrs(pp)) == abi.MF3D_OK, lib.mf3d_last_error()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(cuda)[0]
    fresh.close()
    assert free1 == free0, (free0, free1)
    other = Projection(pr.descriptors(lib), prm, lib)
    for su, pp in zip(rhs, pps):
        ref = [torch.zeros(pr.ttc, dtype=torch.float64, device=cuda) for _ in range(pr.nblocks)]
        assert lib.mf3d_mgkcyc_device(other.ctx, _ptrs(su), _ptrs(ref)) == abi.MF3D_OK
        for b in range(pr.nblocks):
            g, r = pp[b].cpu().numpy(), ref[b].cpu().numpy()
            assert _rel(g, r) <= TOL
            assert np.array_equal(g, r)
    other.close()


def test_noalloc_rejects_too_many_blocks(lib, cuda):
    import torch
    n = abi.MF3D_NOALLOC_MAX_BLOCKS + 1
    pr = Problem(n, 1, 1, 2, 2, 2, bc=(PERIODIC, PERIODIC, WALL, WALL, WALL, WALL), ngrid=1, pl=1)
    prm = pr.params(mg_itrsch=3)
    proj = Projection(pr.descriptors(lib), prm, lib)
    su = [torch.zeros(pr.ttc, dtype=torch.float64, device=cuda) for _ in range(n)]
    pp = [torch.zeros(pr.ttc, dtype=torch.float64, device=cuda) for _ in range(n)]
    st = lib.mf3d_mgkcyc_device_noalloc(proj.ctx, _ptrs(su), _ptrs(pp))
    msg = lib.mf3d_last_error().decode()
    proj.close()
    assert st == abi.MF3D_E_INVALID
    assert "MF3D_NOALLOC_MAX_BLOCKS" in msg

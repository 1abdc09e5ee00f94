"""The failure paths of the projection, each made on the host or through a
bounded device wait - no test faults, traps or hangs the GPU.

The reference prints and stops on these (newsolv_mg.for:59-83); the library
returns a status instead and stays usable:
- a non-finite input -> MF3D_E_NONFINITE (the residual is not finite);
- rmax > 100 after the loop -> MF3D_DIVERGED (newsolv_mg.for:63-64), with the
  same rmax history as the oracle, which reports the same status;
- a device allocation that fails (injected on the host) -> MF3D_E_OOM, then
  a clean mf3d_destroy and a working new context;
- a copy barrier whose phase never completes (one CTA declares more bytes
  than its copies deliver) -> the bounded wait gives up, MF3D_E_TIMEOUT, and
  the same context solves correctly on its next call."""
import ctypes as C

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.abi import SolveInfo
from multiflow3d_b200.problems import Problem, fields_struct
from multiflow3d_b200.solver import Projection

pytestmark = pytest.mark.gpu
_dp = C.POINTER(C.c_double)


def _dev(pr, host, cuda):
    import torch
    return [{k: torch.from_numpy(v.copy()).to(cuda) for k, v in f.items()} for f in host]


def _fields(d):
    arr = (abi.Fields * len(d))()
    for b, f in enumerate(d):
        for k in ("ustar", "vstar", "wstar", "u", "v", "w", "p", "su"):
            setattr(arr[b], k, C.cast(C.c_void_p(f[k].data_ptr()), _dp))
    return arr


def _solve(lib, proj, d, cap):
    info = SolveInfo()
    hist = np.zeros(cap)
    st = lib.mf3d_newsolv_mg_device(proj.ctx, _fields(d), 1.0, 1.0, C.byref(info), hist.ctypes.data_as(_dp), cap)
    return st, info, hist[:max(info.iter, 0)]


def _oracle(oracle, pr, prm, host):
    info = SolveInfo()
    hist = np.zeros(max(prm.maxcy, 1))
    st = oracle.orc_newsolv_mg(pr.descriptors(oracle), pr.nblocks, C.byref(prm), fields_struct(host), 1.0, 1.0,
                               C.byref(info), hist.ctypes.data_as(_dp), prm.maxcy)
    return st, info, hist[:info.iter]


def test_nonfinite_input(lib, oracle, cuda):
    pr = Problem(2, 1, 1, 16, 16, 16, ngrid=3, pl=1)
    host = pr.block_fields(seed=3)
    host[1]["ustar"][5, 6, 7] = np.nan
    prm = pr.params(maxcy=60, eps=1e-9)
    proj = Projection(pr.descriptors(lib), prm, lib)
    st, info, _ = _solve(lib, proj, _dev(pr, host, cuda), prm.maxcy)
    assert st == abi.MF3D_E_NONFINITE, st
    assert "non-finite" in abi.last_error(lib)
    # the context is still usable: the next solve equals the oracle's
    d = _dev(pr, pr.block_fields(seed=3), cuda)
    st2, info2, hist2 = _solve(lib, proj, d, prm.maxcy)
    proj.close()
    ref = pr.block_fields(seed=3)
    st_ref, info_ref, hist_ref = _oracle(oracle, pr, prm, ref)
    assert st2 == st_ref and info2.iter == info_ref.iter
    assert np.array_equal(hist2, hist_ref)
    got = pr.gather([{"p": f["p"].cpu().numpy()} for f in d], "p")
    assert np.array_equal(got, pr.gather(ref, "p"))


def test_diverged_matches_oracle(lib, oracle, cuda):
    """Velocities of order 1e9 and one outer iteration: rmax stays far above
    100, which the reference reports as BIG RMAX (newsolv_mg.for:63-83)."""
    pr = Problem(1, 1, 1, 32, 16, 16, ngrid=3, pl=1)
    host = pr.block_fields(seed=4)
    for f in host:
        for k in ("ustar", "vstar", "wstar", "u", "v", "w"):
            f[k] *= 1e9
    prm = pr.params(maxcy=1, eps=1e-300, eps_relative=0)
    ref = [{k: v.copy() for k, v in f.items()} for f in host]
    st_ref, info_ref, hist_ref = _oracle(oracle, pr, prm, ref)
    proj = Projection(pr.descriptors(lib), prm, lib)
    d = _dev(pr, host, cuda)
    st, info, hist = _solve(lib, proj, d, prm.maxcy)
    proj.close()
    assert st_ref == abi.MF3D_DIVERGED and st == abi.MF3D_DIVERGED, (st_ref, st)
    assert info.rmax > 100.0 and info.iter == info_ref.iter == 1
    assert np.array_equal(hist, hist_ref)
    assert np.array_equal(pr.interior(d[0]["p"].cpu().numpy()), pr.interior(ref[0]["p"]))


def test_injected_allocation_failure(lib, cuda):
    """The host entry point allocates its device mirrors on its first call;
    the first of those allocations fails."""
    pr = Problem(1, 1, 1, 16, 16, 16, ngrid=3, pl=1)
    prm = pr.params(maxcy=30, eps=1e-9)
    proj = Projection(pr.descriptors(lib), prm, lib)
    host = pr.block_fields(seed=5)
    lib.mf3d_test_fail_alloc(0)
    try:
        info = SolveInfo()
        hist = np.zeros(prm.maxcy)
        st = lib.mf3d_newsolv_mg(proj.ctx, fields_struct(host), 1.0, 1.0, C.byref(info), hist.ctypes.data_as(_dp),
                                 prm.maxcy)
    finally:
        lib.mf3d_test_fail_alloc(-1)
    assert st == abi.MF3D_E_OOM, st
    assert "injected" in abi.last_error(lib)
    assert lib.mf3d_destroy(proj.ctx) == abi.MF3D_OK
    proj.ctx = None
    # mf3d_create itself failing part-way (its third allocation) leaves no context behind
    ctx = C.c_void_p()
    lib.mf3d_test_fail_alloc(2)
    try:
        st = lib.mf3d_create(pr.descriptors(lib), 1, C.byref(prm), C.byref(ctx))
    finally:
        lib.mf3d_test_fail_alloc(-1)
    assert st == abi.MF3D_E_OOM and not ctx.value
    # a new context works
    proj = Projection(pr.descriptors(lib), prm, lib)
    res = proj.newsolv_mg(pr.block_fields(seed=5))
    proj.close()
    assert res.status == abi.MF3D_OK


def test_stalled_copy_times_out(lib, oracle, cuda):
    """One half-sweep CTA waits on a barrier whose phase never completes; its
    bounded wait (2 s) gives up, the call returns MF3D_E_TIMEOUT, and the
    next call on the same context equals the oracle."""
    pr = Problem(1, 1, 1, 32, 32, 32, ngrid=3, pl=1)
    prm = pr.params(mg_itrsch=3, maxcy=2, eps=1e-9)
    proj = Projection(pr.descriptors(lib), prm, lib)
    assert lib.mf3d_test_stall_copy(0, 16) == abi.MF3D_OK
    st, _, _ = _solve(lib, proj, _dev(pr, pr.block_fields(seed=6), cuda), prm.maxcy)
    lib.mf3d_test_stall_copy(0, 0)
    assert st == abi.MF3D_E_TIMEOUT, st
    assert "time limit" in abi.last_error(lib)
    d = _dev(pr, pr.block_fields(seed=6), cuda)
    st2, info2, hist2 = _solve(lib, proj, d, prm.maxcy)
    proj.close()
    ref = pr.block_fields(seed=6)
    st_ref, info_ref, hist_ref = _oracle(oracle, pr, prm, ref)
    assert st2 == st_ref and info2.iter == info_ref.iter
    assert np.array_equal(hist2, hist_ref)
    assert np.array_equal(pr.interior(d[0]["p"].cpu().numpy()), pr.interior(ref[0]["p"]))

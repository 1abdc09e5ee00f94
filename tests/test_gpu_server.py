"""The request loop (mf3d_server_*): continuous batching of independent
solves.  Requests join and leave the resident mix at outer-iteration
boundaries; each runs exactly its own solve, so a result is the same alone
and in the mix - bit for bit (tolerance 0), in FP64 and in mixed precision -
and in FP64 equals the oracle's."""
import ctypes as C
import time

import numpy as np
import pytest

from multiflow3d_b200 import abi
from multiflow3d_b200.abi import SolveInfo
from multiflow3d_b200.problems import domain_problem, domain_desc, random_batch, fields_struct
from multiflow3d_b200.solver import Server

pytestmark = pytest.mark.gpu


def domains(n, seed):
    lib = abi.load()
    return [domain_problem(nx, ny, nz, bc, lib.mf3d_max_levels(nx, ny, nz))
            for nx, ny, nz, bc in random_batch(n, seed, lo=16, hi=48)]


def dev_fields(pr, seed, cuda):
    """Device fields, complete on the device (the server's streams do not
    order after the caller's)."""
    import torch
    f = {k: torch.from_numpy(v).to(cuda) for k, v in pr.block_fields(seed=seed)[0].items() if k != "su"}
    torch.cuda.synchronize()
    return f


def wait_all(srv, tickets, timeout=120.0):
    out = {}
    t0 = time.time()
    while len(out) < len(tickets):
        assert time.time() - t0 < timeout, srv.stats()
        for t in tickets:
            if t in out:
                continue
            st, info = srv.poll(t, wait_ms=5)
            if st != abi.MF3D_PENDING:
                out[t] = (st, info)
    return out


@pytest.mark.parametrize("precision", [abi.MF3D_PREC_FP64, abi.MF3D_PREC_FP32])
def test_alone_equals_mix(lib, oracle, cuda, precision):
    doms = domains(6, 17)
    prm = doms[0].params(mg_itrsch=3, maxcy=300, eps=1e-8, precision=precision)
    # alone: one request at a time on its own server
    alone = []
    for d, pr in enumerate(doms):
        srv = Server(prm, lib=lib)
        f = dev_fields(pr, 50 + d, cuda)
        t = srv.submit(domain_desc(pr), f)
        (st, info), = wait_all(srv, [t]).values()
        srv.close()
        alone.append((st, info.info.iter, {k: v.cpu().numpy() for k, v in f.items()}))
    # the mix: requests arrive while others are resident
    srv = Server(prm, lib=lib)
    fields = [dev_fields(pr, 50 + d, cuda) for d, pr in enumerate(doms)]
    tickets = []
    for d, pr in enumerate(doms):
        tickets.append(srv.submit(domain_desc(pr), fields[d]))
        if d % 2 == 1:
            srv.poll(tickets[0], wait_ms=3)  # let a few cycles run before the next arrivals
    res = wait_all(srv, tickets)
    stats = srv.stats()
    srv.close()
    admits = sorted(res[t][1].t_admit for t in tickets)
    assert stats["completed"] == len(doms)
    for d, t in enumerate(tickets):
        st, info = res[t]
        assert st == alone[d][0]
        assert info.info.iter == alone[d][1]
        for k in ("p", "u", "v", "w"):
            assert np.array_equal(fields[d][k].cpu().numpy(), alone[d][2][k]), (d, k)
    if precision == abi.MF3D_PREC_FP64:
        for d, pr in enumerate(doms):
            ref = pr.block_fields(seed=50 + d)
            p = pr.params(mg_itrsch=3, maxcy=300, eps=1e-8)
            info = SolveInfo()
            hist = np.zeros(300)
            st = oracle.orc_newsolv_mg(pr.descriptors(oracle), 1, C.byref(p), fields_struct(ref), 1.0, 1.0,
                                       C.byref(info), hist.ctypes.data_as(C.POINTER(C.c_double)), 300)
            assert res[tickets[d]][1].info.iter == info.iter
            assert np.array_equal(fields[d]["p"].cpu().numpy(), ref[0]["p"])


def test_admission_waits_for_memory(lib, cuda):
    """A cap that holds one request at a time: requests run one after the
    other, in arrival order, and all complete."""
    doms = domains(3, 23)
    prm = doms[0].params(mg_itrsch=3, maxcy=300, eps=1e-8)
    srv = Server(prm, mem_cap_bytes=1.0, lib=lib)  # below any request: admitted only when nothing is resident
    fields = [dev_fields(pr, 70 + d, cuda) for d, pr in enumerate(doms)]
    tickets = [srv.submit(domain_desc(pr), fields[d]) for d, pr in enumerate(doms)]
    res = wait_all(srv, tickets)
    srv.close()
    infos = [res[t][1] for t in tickets]
    for a, b in zip(infos, infos[1:]):
        assert b.t_admit >= a.t_done
    assert all(res[t][0] >= 0 for t in tickets)


def test_unknown_ticket(lib, cuda):
    prm = domains(1, 3)[0].params()
    srv = Server(prm, lib=lib)
    st = lib.mf3d_server_poll(srv.ctx, 12345, None, 0)
    srv.close()
    assert st == abi.MF3D_E_INVALID

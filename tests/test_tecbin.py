"""Restart files `tecbin<id>.bin` (post.for:496-548 writes, initial.for:
689-760 reads).  CPU: the numpy restatement in oracle/tecbin.py against the
committed fixture (written record by record with `struct`, the way
gfortran frames the writer's records), and the library's header parser.
GPU: the device decoder and encoder against the same, byte for byte, on
the fixture and on a full-size block, and a broken record framing."""
import ctypes as C
import hashlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import tecbin as orc_tb  # noqa: E402

from multiflow3d_b200 import abi  # noqa: E402

FIXTURE = os.path.join(ROOT, "tests", "golden", "tecbin0007.bin")
FIXTURE_SHA256 = "f143a7f5ac1505e8289aad88ec6614eb38814433fe7b2fa79d347b988427d60a"


def fixture_bytes():
    with open(FIXTURE, "rb") as fh:
        data = fh.read()
    assert hashlib.sha256(data).hexdigest() == FIXTURE_SHA256
    return data


def test_oracle_reads_fixture():
    head, fields, (x, y, z) = orc_tb.read(fixture_bytes())
    assert head == dict(toti=7, totj=5, totk=4, pl=1, inind=-1, jnind=0, knind=-1)
    assert np.array_equal(x, (np.arange(7) - 1) * 0.125)
    assert np.array_equal(z, (np.arange(4) - 1) * 0.5)
    # the fixture's value rule, field 0 (p) at cell (i, j, k) = (3, 2, 1)
    q = (3 * 7 + 2 * 13 + 1 * 29) % 97
    assert fields["p"][1, 2, 3] == (q - 48) / 8.0
    assert orc_tb.write(7, 5, 4, 1, -1, 0, -1, x, y, z, fields) == fixture_bytes()


def test_library_header_parser(lib):
    data = fixture_bytes()
    info = abi.TecbinInfo()
    assert lib.mf3d_tecbin_info_of(data, len(data), C.byref(info)) == 0
    assert (info.toti, info.totj, info.totk, info.pl) == (7, 5, 4, 1)
    assert (info.inind, info.jnind, info.knind) == (-1, 0, -1)
    assert info.records == 140 and info.data_offset == 52
    assert lib.mf3d_tecbin_size(7, 5, 4) == len(data)
    assert lib.mf3d_tecbin_info_of(data[:-8], len(data) - 8, C.byref(info)) == abi.MF3D_E_INVALID
    bad = bytearray(data)
    bad[0] = 13
    assert lib.mf3d_tecbin_info_of(bytes(bad), len(bad), C.byref(info)) == abi.MF3D_E_INVALID


def _decode(lib, cuda, image: bytes):
    import torch
    info = abi.TecbinInfo()
    st = lib.mf3d_tecbin_info_of(image, len(image), C.byref(info))
    assert st == 0
    dev = torch.from_numpy(np.frombuffer(image, dtype=np.uint8).copy()).to(cuda)
    shape = (info.totk, info.totj, info.toti)
    outs = [torch.empty(shape, dtype=torch.float64, device=cuda) for _ in orc_tb.FIELDS]
    ptrs = (C.c_void_p * 16)(*[o.data_ptr() for o in outs])
    st = lib.mf3d_tecbin_decode_device(C.c_void_p(dev.data_ptr()), C.byref(info), ptrs, 0)
    return st, {f: o.cpu().numpy() for f, o in zip(orc_tb.FIELDS, outs)}


def _encode(lib, cuda, head, xyz, fields):
    import torch
    n = lib.mf3d_tecbin_size(head["toti"], head["totj"], head["totk"])
    img = torch.empty(n, dtype=torch.uint8, device=cuda)
    x, y, z = (torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in xyz)
    fd = [torch.from_numpy(np.ascontiguousarray(fields[f])).to(cuda) for f in orc_tb.FIELDS]
    ptrs = (C.c_void_p * 16)(*[t.data_ptr() for t in fd])
    st = lib.mf3d_tecbin_encode_device(head["toti"], head["totj"], head["totk"], head["pl"], head["inind"],
                                       head["jnind"], head["knind"], C.c_void_p(x.data_ptr()),
                                       C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), ptrs,
                                       C.c_void_p(img.data_ptr()), 0)
    assert st == 0
    return img.cpu().numpy().tobytes()


@pytest.mark.gpu
def test_device_decode_and_encode_fixture(lib, cuda):
    data = fixture_bytes()
    head, ref, xyz = orc_tb.read(data)
    st, got = _decode(lib, cuda, data)
    assert st == 0
    for f in orc_tb.FIELDS:
        assert np.array_equal(got[f].view(np.int64), ref[f].view(np.int64)), f
    assert _encode(lib, cuda, head, xyz, ref) == data


@pytest.mark.gpu
def test_device_round_trip_full_block(lib, cuda):
    """A 128^3 block with two ghost layers (2.4 M records, 0.4 GB): encode on
    the device, compare with the numpy writer byte for byte, decode back."""
    toti = totj = totk = 132
    rng = np.random.default_rng(3)
    fields = {f: rng.standard_normal((totk, totj, toti)) for f in orc_tb.FIELDS}
    xyz = tuple((np.arange(n) - 2) / 128.0 for n in (toti, totj, totk))
    head = dict(toti=toti, totj=totj, totk=totk, pl=2, inind=0, jnind=-1, knind=0)
    img = _encode(lib, cuda, head, xyz, fields)
    assert img == orc_tb.write(toti, totj, totk, 2, 0, -1, 0, *xyz, fields)
    st, got = _decode(lib, cuda, img)
    assert st == 0
    for f in orc_tb.FIELDS:
        assert np.array_equal(got[f], fields[f]), f


@pytest.mark.gpu
def test_device_decode_rejects_broken_framing(lib, cuda):
    data = bytearray(fixture_bytes())
    r = 77
    off = 52 + r * 160 + 156  # the closing length word of cell record 77
    data[off:off + 4] = (151).to_bytes(4, "little")
    st, _ = _decode(lib, cuda, bytes(data))
    assert st == abi.MF3D_E_INVALID
    assert b"record 77" in lib.mf3d_last_error()

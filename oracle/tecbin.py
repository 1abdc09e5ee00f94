"""CPU restatement of the reference's restart-file format `tecbin<id>.bin`
(test infrastructure: the oracle the device decoder and encoder are checked
against; nothing in the library imports it).

The writer is post.for:496-548 (`subroutine tecbin`), the reader
initial.for:689-760.  gfortran writes each unformatted sequential record
framed by its byte length as a 4-byte integer before and after; with
-fdefault-real-8 (makefile:3) reals are 8 bytes, integers stay 4:

    (toti, totj, totk)   int32 x 3          post.for:516
    (pl)                 int32              post.for:517
    (inind, jnind, knind) int32 x 3         post.for:519-524
    then per cell, k outermost, i fastest (post.for:527-539), 19 doubles:
    x(i), y(j), z(k), p, pm, ppm, vis, u, um, uum, v, vm, vvm, w, wm, wwm,
    uvm, uwm, vwm

The reader keeps fields 4..19 (initial.for:718-733) and stops when the
file's pl differs from the run's (initial.for:714-719).
"""
import struct

import numpy as np

FIELDS = ("p", "pm", "ppm", "vis", "u", "um", "uum", "v", "vm", "vvm", "w", "wm", "wwm", "uvm", "uwm", "vwm")
CELL = np.dtype([("n0", "<i4"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8")] + [(f, "<f8") for f in FIELDS] +
                [("n1", "<i4")])
HEADER_BYTES = 52
assert CELL.itemsize == 160


def _framed(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def read(image: bytes):
    """(header dict, {field: array (totk, totj, toti)}, (x, y, z)); raises
    ValueError on a framing or size mismatch."""
    h = struct.unpack_from("<13i", image, 0)
    if (h[0], h[4], h[5], h[7], h[8], h[12]) != (12, 12, 4, 4, 12, 12):
        raise ValueError("header records are not framed as the reference writes them")
    toti, totj, totk, pl, inind, jnind, knind = h[1], h[2], h[3], h[6], h[9], h[10], h[11]
    n = toti * totj * totk
    if len(image) != HEADER_BYTES + n * CELL.itemsize:
        raise ValueError("size does not match the cell records")
    cells = np.frombuffer(image, dtype=CELL, count=n, offset=HEADER_BYTES)
    bad = np.flatnonzero((cells["n0"] != 152) | (cells["n1"] != 152))
    if bad.size:
        raise ValueError(f"cell record {bad[0]} is not framed as 152 bytes")
    shape = (totk, totj, toti)
    fields = {f: cells[f].reshape(shape).copy() for f in FIELDS}
    x = cells["x"].reshape(shape)[0, 0, :].copy()
    y = cells["y"].reshape(shape)[0, :, 0].copy()
    z = cells["z"].reshape(shape)[:, 0, 0].copy()
    head = dict(toti=toti, totj=totj, totk=totk, pl=pl, inind=inind, jnind=jnind, knind=knind)
    return head, fields, (x, y, z)


def write(toti, totj, totk, pl, inind, jnind, knind, x, y, z, fields) -> bytes:
    """The file image the writer produces (missing fields are zeros)."""
    head = (_framed(struct.pack("<3i", toti, totj, totk)) + _framed(struct.pack("<i", pl)) +
            _framed(struct.pack("<3i", inind, jnind, knind)))
    n = toti * totj * totk
    cells = np.zeros(n, dtype=CELL)
    cells["n0"] = 152
    cells["n1"] = 152
    kk, jj, ii = np.meshgrid(np.arange(totk), np.arange(totj), np.arange(toti), indexing="ij")
    cells["x"] = np.asarray(x)[ii.ravel()]
    cells["y"] = np.asarray(y)[jj.ravel()]
    cells["z"] = np.asarray(z)[kk.ravel()]
    for f in FIELDS:
        if f in fields and fields[f] is not None:
            cells[f] = np.asarray(fields[f], dtype=np.float64).ravel()
    return head + cells.tobytes()

"""Writes tests/golden/tecbin0007.bin: a restart file for a block of
ttc extents 7 x 5 x 4 (pl = 1), record by record the way gfortran writes
the `write (88)` statements of post.for:496-548 (each unformatted record
framed by its byte length as a 4-byte integer).  Independent of the numpy
restatement in oracle/tecbin.py and of the device codec: it packs every
record with `struct`.  Values are exact binary fractions plus a few special
bit patterns (signed zero, subnormal, extremes) so that a byte-exact
round trip is meaningful.  Run: python tests/golden/make_tecbin_fixture.py
"""
import os
import struct

TOTI, TOTJ, TOTK, PL = 7, 5, 4, 1
ININD, JNIND, KNIND = -1, 0, -1
SPECIAL = [-0.0, 5e-324, 1.7976931348623157e308, -2.2250738585072014e-308]


def framed(fmt, *vals):
    payload = struct.pack("<" + fmt, *vals)
    n = struct.pack("<i", len(payload))
    return n + payload + n


def value(f, i, j, k):
    q = (i * 7 + j * 13 + k * 29 + f * 3) % 97
    if q < len(SPECIAL):
        return SPECIAL[q]
    return (q - 48) / 8.0 + f / 1024.0


def main():
    out = bytearray()
    out += framed("3i", TOTI, TOTJ, TOTK)
    out += framed("i", PL)
    out += framed("3i", ININD, JNIND, KNIND)
    for k in range(TOTK):
        for j in range(TOTJ):
            for i in range(TOTI):
                x, y, z = (i - PL) * 0.125, (j - PL) * 0.25, (k - PL) * 0.5
                vals = [x, y, z] + [value(f, i, j, k) for f in range(16)]
                out += framed("19d", *vals)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tecbin0007.bin")
    with open(path, "wb") as fh:
        fh.write(bytes(out))
    print(path, len(out))


if __name__ == "__main__":
    main()

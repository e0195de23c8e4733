"""Regenerates seexpr_permutation.inc, the 256-byte permutation of SeExpr's
scalar hash (used by hash(), rand() and the face seeds of XGen scalar
expressions; Disney SeExpr, BSD-3-Clause, Copyright 2011 Disney Enterprises,
Inc.; notice in LICENSES/SeExpr-BSD-3-Clause.txt).

The expression runtime must reproduce the reference's hash bit for bit, so
the table is read off the reference's own xgen_seexpr_hash_finish
(oracle/_ref/libnxg_ref.so, see oracle/Makefile): the finish step tempers
its state and then looks the low byte up in the permutation, returning that
entry in the top byte, so a state whose tempered low byte is i yields
entry i.  It runs only where the reference checkout exists; the generated
file is committed.

    python nanoxgen_b200/csrc/make_permutation_table.py
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
MASK = 0xFFFFFFFF


def temper(s: int) -> int:
    s ^= s >> 11
    s ^= (s << 7) & 0x9D2C5680
    s ^= (s << 15) & 0xEFC60000
    s ^= s >> 18
    return s & MASK


def main() -> None:
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libnxg_ref.so"))
    lib.ref_seexpr_hash_finish.restype = ctypes.c_uint32
    lib.ref_seexpr_hash_finish.argtypes = [ctypes.c_uint32]
    table = [None] * 256
    state = 0
    while any(v is None for v in table):
        low = temper(state) & 0xFF
        if table[low] is None:
            table[low] = lib.ref_seexpr_hash_finish(state) >> 24
        state = (state * 2654435761 + 12345) & MASK
    assert sorted(table) == list(range(256)), "not a permutation"
    lines = [
        "// Generated by make_permutation_table.py -- do not edit.",
        "// SeExpr scalar-hash byte permutation (256 entries).",
        "// Derived from Disney SeExpr under the BSD 3-Clause license.",
        "// Copyright 2011 Disney Enterprises, Inc. All rights reserved.",
        "// SPDX-License-Identifier: BSD-3-Clause (full notice: LICENSES/SeExpr-BSD-3-Clause.txt)",
    ]
    for row in range(0, 256, 16):
        lines.append(" ".join("%3d," % v for v in table[row:row + 16]))
    with open(os.path.join(HERE, "seexpr_permutation.inc"), "w") as handle:
        handle.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()

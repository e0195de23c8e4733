"""Regenerates seexpr_gradients.inc, the 256-entry SeExpr gradient table that
every .nxg v0.2 asset embeds (the reference's include/nanoxgen/seexpr_noise_table.h,
BSD-3-Clause, Copyright 2011 Disney Enterprises, Inc.; notice in
LICENSES/SeExpr-BSD-3-Clause.txt).

The table is part of the asset format, so the builder must write exactly the
reference's bits.  This script takes them from an asset built by the
reference itself (oracle/_ref/libnxg_ref.so, see oracle/Makefile) and prints
each float as a C99 hex literal, so no decimal rounding is involved.  It runs
only where the reference checkout exists; the generated file is committed.

    python nanoxgen_b200/csrc/make_gradient_table.py
"""
import ctypes
import os
import struct
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main() -> None:
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libnxg_ref.so"))
    f3 = ctypes.c_float * 3
    positions = (f3 * 3)(f3(0, 0, 0), f3(1, 0, 0), f3(0, 0, 1))
    tris = (ctypes.c_uint32 * 3)(0, 1, 2)
    counts = (ctypes.c_uint32 * 1)(2)
    cvs = (f3 * 2)(f3(0.25, 0, 0.25), f3(0.25, 1, 0.25))
    normals = (f3 * 1)(f3(0, 1, 0))
    uvs = (ctypes.c_float * 2)(0, 0)
    gtri = (ctypes.c_uint32 * 1)(0xFFFFFFFF)
    bary = (ctypes.c_float * 2)(0, 0)
    radii = (ctypes.c_float * 1)(1.0)
    out = ctypes.c_void_p()
    size = ctypes.c_uint64()
    msg = ctypes.create_string_buffer(256)
    rc = lib.ref_build_asset(positions, 3, None, None, tris, 1, 1, counts, cvs, normals, uvs,
                             gtri, bary, radii, ctypes.byref(out), ctypes.byref(size), msg, 256)
    if rc != 0:
        sys.exit("reference build failed: " + msg.value.decode())
    blob = ctypes.string_at(out, size.value)
    lib.ref_free(out)
    offset = struct.unpack_from("<Q", blob, 120)[0]  # AssetHeader::noise_gradients_offset
    values = struct.unpack_from("<768f", blob, offset)
    lines = [
        "// Generated by make_gradient_table.py -- do not edit.",
        "// SeExpr 3D gradient table (256 x float3), embedded in every .nxg v0.2 asset.",
        "// Derived from Disney SeExpr SeNoiseTables.h under the BSD 3-Clause license.",
        "// Copyright 2011 Disney Enterprises, Inc. All rights reserved.",
        "// SPDX-License-Identifier: BSD-3-Clause (full notice: LICENSES/SeExpr-BSD-3-Clause.txt)",
    ]
    for i in range(256):
        x, y, z = values[3 * i: 3 * i + 3]
        lines.append("{%sf, %sf, %sf}," % (float(x).hex(), float(y).hex(), float(z).hex()))
    with open(os.path.join(HERE, "seexpr_gradients.inc"), "w") as handle:
        handle.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()

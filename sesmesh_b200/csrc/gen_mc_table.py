#!/usr/bin/env python3
"""Transcribes sesmesh's marching-cubes case table into a C include file.

sesmesh meshes with its own 256-case table (generated by the reference under
a uniform face rule, `crates/sesmesh/src/mesh/mc_table.rs:9-285`, read through
`crates/sesmesh/src/mesh/tables.rs:31`).  The triangle order inside each case
and the vertex order inside each triangle decide the OBJ face records, so a
byte-identical mesh needs exactly the same data.  This script parses the two
arrays out of the reference source and writes them as plain C arrays; it runs
only where the reference tree is present and its output is committed
(`mc_table.inc`).  The sha256 of the parsed data is written beside the table
so the tests can check the committed copy without the reference.

Usage: python gen_mc_table.py <path to mc_table.rs> <output .inc>
"""
import hashlib
import re
import sys


def parse(text):
    off_m = re.search(r"TRI_OFFSET:\s*\[u16;\s*257\]\s*=\s*\[(.*?)\];", text, re.S)
    edg_m = re.search(r"TRI_EDGES:\s*\[\[u8;\s*3\];\s*(\d+)\]\s*=\s*\[(.*?)\];", text, re.S)
    if not off_m or not edg_m:
        raise SystemExit("table arrays not found")
    body = re.sub(r"//[^\n]*", "", off_m.group(1))
    offsets = [int(v) for v in re.findall(r"\d+", body)]
    n_tri = int(edg_m.group(1))
    body = re.sub(r"//[^\n]*", "", edg_m.group(2))
    tris = [tuple(int(v) for v in t) for t in re.findall(r"\[(\d+),\s*(\d+),\s*(\d+)\]", body)]
    if len(offsets) != 257 or len(tris) != n_tri or offsets[-1] != n_tri:
        raise SystemExit("unexpected table shape")
    return offsets, tris


def digest(offsets, tris):
    h = hashlib.sha256()
    h.update(",".join(map(str, offsets)).encode())
    h.update(b";")
    h.update(",".join("%d.%d.%d" % t for t in tris).encode())
    return h.hexdigest()


def main():
    src, dst = sys.argv[1], sys.argv[2]
    offsets, tris = parse(open(src).read())
    lines = [
        "// Marching-cubes case table of sesmesh 1.3.2, transcribed by gen_mc_table.py",
        "// from crates/sesmesh/src/mesh/mc_table.rs (data only; identical data is",
        "// required for identical triangle records).",
        "// sha256(data) = " + digest(offsets, tris),
        "#pragma once",
        "#include <stdint.h>",
        "#define SMB_MC_TRIANGLES %d" % len(tris),
        "// Storage qualifier (__constant__ when included by device code).",
        "#ifndef SMB_MC_QUAL",
        "#define SMB_MC_QUAL",
        "#endif",
        "static SMB_MC_QUAL const uint16_t SMB_TRI_OFFSET[257] = {",
    ]
    for i in range(0, 257, 16):
        lines.append("    " + ", ".join(str(v) for v in offsets[i:i + 16]) + ",")
    lines.append("};")
    lines.append("static SMB_MC_QUAL const uint8_t SMB_TRI_EDGES[%d][3] = {" % len(tris))
    for case in range(256):
        row = tris[offsets[case]:offsets[case + 1]]
        if row:
            lines.append("    " + " ".join("{%d, %d, %d}," % t for t in row) + "  // %d" % case)
    lines.append("};")
    open(dst, "w").write("\n".join(lines) + "\n")
    print(digest(offsets, tris))


if __name__ == "__main__":
    main()

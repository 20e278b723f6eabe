"""Extracts the reference's 3D Morton encode tables (x/y/z, 256 entries each) into
morton3d_lut.json, to pin the bit-interleave the oracle and the CUDA z-sort compute.

Source: BananaCore/Banana/NeighborSearch/Morton/Morton3D_LUTs.h (Morton3D_encode_x_256,
Morton3D_encode_y_256, Morton3D_encode_z_256).  Run where the reference tree is available:

    python tests/golden/make_morton_golden.py /path/to/reference
"""
import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(f"usage: python {sys.argv[0]} <reference tree>")
src = Path(sys.argv[1]) / "BananaCore/Banana/NeighborSearch/Morton/Morton3D_LUTs.h"
text = src.read_text()
out = {"source": "BananaCore/Banana/NeighborSearch/Morton/Morton3D_LUTs.h"}
for axis in "xyz":
    m = re.search(r"Morton3D_encode_%s_256\[256\]\s*=\s*\{([^}]*)\}" % axis, text)
    vals = [int(v, 0) for v in re.findall(r"0x[0-9a-fA-F]+|\d+", m.group(1))]
    assert len(vals) == 256, (axis, len(vals))
    out[axis] = vals
dst = Path(__file__).resolve().parent / "morton3d_lut.json"
dst.write_text(json.dumps(out) + "\n")
print(dst)

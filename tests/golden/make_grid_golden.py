"""Extracts the known answers of the reference's Grid unit test into grid_known_answers.json.

Source: BananaCore/Banana/Grid/_Grid.Test.hpp:29-57 (Catch TEST_CASE "Test Grid3D").  The
values are read from the REQUIRE lines of that file; run this script where the reference
tree is available:

    python tests/golden/make_grid_golden.py /path/to/reference
"""
import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(f"usage: python {sys.argv[0]} <reference tree>")
src = Path(sys.argv[1]) / "BananaCore/Banana/Grid/_Grid.Test.hpp"
text = src.read_text()
grid = re.search(r"Grid<3, Real> grid\(Vec3r\((\S+)\), Vec3r\((\S+)\), ([0-9.]+)f\)", text)
ncells = [int(v) for v in re.findall(r"grid\.getNCells\(\)\[\d\] == (\d+)", text)]
valid = re.findall(r"REQUIRE\((!?)grid\.isValidCell\(Vec3i\(([-\d, ]+)\)\)\)", text)
nearest = re.search(r"getNearestValidCellIdx\(Vec3i\(([-\d, ]+)\)\) == Vec3i\(([-\d, ]+)\)", text)
valididx = re.search(r"getValidCellIdx<int>\(Vec3f\(([-\d., ]+)\)\) == Vec3i\(([-\d, ]+)\)", text)
p1 = re.search(r"Vec3f\s+p1 = Vec3f\(([-\d., ]+)\)", text)
p2 = re.search(r"Vec3f\s+p2 = Vec3f\(([-\d., ]+)\)", text)
nl = re.search(r"neighborList\.size\(\) == (\d+)", text)


def vec(s, f=float):
    return [f(x) for x in s.split(",")]


out = {
    "source": "BananaCore/Banana/Grid/_Grid.Test.hpp:29-57",
    "grid": {"bmin": [float(grid.group(1))] * 3, "bmax": [float(grid.group(2))] * 3, "cell_size": float(grid.group(3))},
    "ncells": ncells,
    "is_valid_cell": [{"cell": vec(c, int), "valid": neg != "!"} for neg, c in valid],
    "nearest_valid_cell": {"cell": vec(nearest.group(1), int), "expect": vec(nearest.group(2), int)},
    "valid_cell_idx": {"pos": vec(valididx.group(1)), "expect": vec(valididx.group(2), int)},
    "neighbor_list": {"particles": [vec(p1.group(1)), vec(p2.group(1))], "query": 0, "expect_size": int(nl.group(1))},
}
dst = Path(__file__).resolve().parent / "grid_known_answers.json"
dst.write_text(json.dumps(out, indent=1) + "\n")
print(dst)

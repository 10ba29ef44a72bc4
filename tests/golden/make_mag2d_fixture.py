"""Extract the Magnetostatics2D tensor data file shipped with the reference
(src/modules/cpu/dipole2d/save_test.lua: 16 x 16 x 2 layers, unit cell and
grain size 1e-6 on every axis) into mag2d_save_test.json: the arrays
[dest][src] = [1][1] and [1][2] of the nine components, rows y, columns x, as
printed there (7 significant digits).  The file records no truncation; the
builder reproduces it with truncation 20 on every axis.  Its values carry
the sign of a makeData that added +N; the current makeData
(mag2d_luafuncs.lua:719-729) adds -N.

Reads the reference tree named by REFERENCE=<path> (default: a folder
`reference` beside the repository)."""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("REFERENCE", os.path.join(HERE, "..", "..", "..", "reference"))
SRC = os.path.join(REF, "src", "modules", "cpu", "dipole2d", "save_test.lua")
NAMES = ["XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"]


def main():
    txt = open(SRC).read()
    arrays = {}
    for m in re.finditer(r"(\w\w)\[(\d)\]\[(\d)\] = \[\[\n(.*?)\]\]", txt, re.S):
        ab, d, s, body = m.group(1), int(m.group(2)), int(m.group(3)), m.group(4)
        if d != 1:
            continue
        rows = [[float(v) for v in line.split(",")] for line in body.strip().split("\n")]
        arrays.setdefault(f"{d},{s}", {})[ab] = rows
    out = {"source": "src/modules/cpu/dipole2d/save_test.lua", "nx": 16, "ny": 16, "nz": 2,
           "unit_cell": 1e-6, "grain": 1e-6, "truncation": [20, 20, 20, 20], "sign_of_file": 1,
           "arrays": arrays}
    with open(os.path.join(HERE, "mag2d_save_test.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    main()

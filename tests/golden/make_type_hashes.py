"""Type ids of the reference's encoded objects: hash32(name), the
reference's own MurmurHash3_x86_32 with seed 1000
(src/modules/common/luabaseobject/factory.cpp:123-131), compiled from its
source by oracle/Makefile into oracle/_ref/libmurmur.so and called on the
type names of the SpinSystem stream and on names of every tail length.
Writes type_hashes.json.

Reads the reference tree named by REFERENCE=<path> (default: a folder
`reference` beside the repository)."""
import ctypes
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(HERE, "..", "..", "oracle")
NAMES = ["SpinSystem", "Array.Double", "Array.Float", "Array.Integer", "LLG.Quaternion",
         "LLG.Cartesian", "Exchange", "Dipole", "Anisotropy", "Thermal", "AppliedField",
         "a", "ab", "abc", "abcd", "abcde"]


def main():
    ref = os.environ.get("REFERENCE", os.path.join(HERE, "..", "..", "..", "reference"))
    subprocess.check_call(["make", "-s", "-C", ORACLE, "_ref/libmurmur.so", f"REFERENCE={os.path.abspath(ref)}"])
    lib = ctypes.CDLL(os.path.join(ORACLE, "_ref", "libmurmur.so"))
    fn = lib._Z18MurmurHash3_x86_32PKvijPv
    out = {}
    for name in NAMES:
        b = name.encode()
        res = ctypes.c_int()
        fn(b, len(b), 1000, ctypes.byref(res))
        out[name] = res.value
    doc = {"source": "src/modules/common/luabaseobject/MurmurHash3.cpp, factory.cpp:123-131",
           "seed": 1000, "hash32": out}
    with open(os.path.join(HERE, "type_hashes.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()

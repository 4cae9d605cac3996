"""Extracts the known-answer values that pin the explicit-dynamics path from the reference's
own test files (Peridynamics.jl, test/) into reference_values.json.

The reference is Julia and cannot run in this container, so its tests are read as text: every
number below is copied by a regular expression from the cited test file, and the JSON records
file and line. Run in a container where the reference tree is mounted:

    python tests/golden/make_golden.py /path/to/Peridynamics.jl
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    raise SystemExit("usage: python tests/golden/make_golden.py <path of the Peridynamics.jl tree>")
ROOT = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_values.json")
NUM = r"(-?\d+\.\d+(?:e-?\d+)?)"


def grab(rel, pattern, count=1):
    path = os.path.join(ROOT, rel)
    lines = open(path).read().splitlines()
    for k, line in enumerate(lines, 1):
        m = re.search(pattern, line)
        if m:
            vals = [float(x) for x in m.groups()]
            return {"values": vals[:count] if count > 1 else vals[0], "source": f"{rel}:{k}"}
    raise SystemExit(f"pattern {pattern!r} not found in {rel}")


g = {}
g["osb_two_point_b12"] = grab("test/unit/physics/test_ordinary_state_based.jl", r"b12 = " + NUM)
g["osb_interface_b1"] = grab("test/unit/physics/test_ordinary_state_based.jl", r"b1 = " + NUM)
g["osb_interface_b2"] = grab("test/unit/physics/test_ordinary_state_based.jl", r"b2 = " + NUM)
g["c_nhp_b_int_1"] = grab("test/unit/physics/test_correspondence.jl",
                          r"b_int\[:, 1\] ≈ \[" + NUM + r", " + NUM + r", " + NUM, count=3)
g["c_nhp_b_int_12"] = grab("test/unit/physics/test_correspondence.jl", r"b_int\[1, 2\] ≈ " + NUM)
g["c_nhp_b_int_23"] = grab("test/unit/physics/test_correspondence.jl", r"b_int\[2, 3\] ≈ " + NUM)
g["bb_epsilon_c"] = grab("test/unit/physics/test_bond_based.jl", r"εc ≈ " + NUM)
g["bb_storage_bond_count"] = grab("test/unit/physics/test_bond_based.jl",
                                  r"bond_active == ones\(Bool, (\d+)\)".replace(r"(\d+)", r"(\d+)"))
json.dump(g, open(OUT, "w"), indent=1)
print(json.dumps(g, indent=1))

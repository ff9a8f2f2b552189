"""Generate tests/golden/lattice_tables.json from the reference's lattice tables.

Parses the `#if LATTICE == 27 / 19 / 15` blocks of vars_module.f90 (lines
319-338, 666-684 and 685-703 of the LBFAST sources): the link vectors ex, ey,
ez, the opposite links opp and the weights p(0:nlinks) built from the
parameters p0..p3.  Run with the path of the LBFAST sources' vars_module.f90:
    python tests/golden/make_lattice_golden.py <LBFAST sources>/vars_module.f90
"""
import json
import re
import sys
from fractions import Fraction

src = open(sys.argv[1]).read()
marks = [("27", "#if LATTICE == 27"), ("19", "#elif LATTICE == 19"), ("15", "#elif LATTICE == 15")]
out = {}
for i, (lat, mark) in enumerate(marks):
    a = src.index(mark)
    b = src.index(marks[i + 1][1]) if i + 1 < len(marks) else src.index("#else", a)
    blk = src[a:b]
    if lat == "27":  # the D3Q27 block continues with the high-order tables
        blk = blk[: blk.index("#ifdef HIGHORDER")]

    def ints(name):
        m = re.search(name + r"\s*=\s*\(/([^/]*)/\)", blk)
        return [int(t) for t in m.group(1).replace("&", " ").split(",")]

    params = {}
    for m in re.finditer(r"(p\d)\s*=\s*real\(\s*([0-9.]+)d0\s*/\s*([0-9.]+)d0", blk):
        params[m.group(1)] = Fraction(m.group(2)) / Fraction(m.group(3))
    pm = re.search(r"\bp=\(/([^/]*)/\)", blk)
    w = [float(params[t.strip()]) for t in pm.group(1).replace("&", " ").split(",")]
    out[lat] = {"ex": ints("ex"), "ey": ints("ey"), "ez": ints("ez"), "opp": ints("opp"), "w": w}
    assert all(len(v) == int(lat) for v in out[lat].values()), lat
with open(__file__.replace("make_lattice_golden.py", "lattice_tables.json"), "w") as f:
    json.dump(out, f, indent=1)

"""Generate tests/golden/minv_mrt.npy from the reference's D3Q27 table.

Parses the Fortran array constructor `Minv_mrt(0:nlinks,0:nlinks) = reshape([...])`
in vars_module.f90 (lines 360-521 of the LBFAST sources) and stores it as
minv[r, l] = Minv_mrt(r, l): r the Hermite basis row, l the population.
Run with the path of the LBFAST sources' vars_module.f90:
    python tests/golden/make_minv_golden.py <LBFAST sources>/vars_module.f90
"""
import re
import sys
from fractions import Fraction

import numpy as np

src = open(sys.argv[1]).read()
start = src.index("Minv_mrt(0:nlinks,0:nlinks) = reshape([")
end = src.index("shape=[nlinks+1,nlinks+1])", start)
body = src[start:end]
body = body[body.index("[") + 1:]
# inner arrays [ ... ]
inner = re.findall(r"\[([^\[\]]*)\]", body)
assert len(inner) == 27, len(inner)
cols = []
for arr in inner:
    vals = []
    for tok in arr.replace("&", " ").replace("\n", " ").split(","):
        tok = tok.strip()
        if not tok:
            continue
        tok = tok.replace("_db", "")
        if "/" in tok:
            a, b = tok.split("/")
            vals.append(Fraction(a) / Fraction(b))
        else:
            vals.append(Fraction(tok))
    assert len(vals) == 27, len(vals)
    cols.append([float(v) for v in vals])
# Fortran column-major reshape: inner array l fills Minv_mrt(0:26, l)
minv = np.array(cols).T  # minv[r, l]
np.save(__file__.replace("make_minv_golden.py", "minv_mrt.npy"), minv)
print("saved", minv.shape)

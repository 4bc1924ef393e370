"""Generate ``mc_reference_loops.json`` from the reference's marching-cubes table.

Reads ``src/TurboMC.cu`` of the reference (DWGTech/DWG) AS TEXT and records,
for each of the 256 cube cases:

* ``tri_count`` -- number of triangles the reference emits for the case;
* ``loops``     -- the oriented boundary loops of the case's triangles, as
                   cyclic edge-index sequences rotated to start at their
                   smallest edge (orientation = triangle winding);
* ``tris``      -- the reference's triangles of the case, in its order, as
                   edge-index triples (src/TurboMC.cu:57-314).

The loops pin the polygons that the product derives from the cube geometry;
the triangle lists pin the product's per-case split of those polygons, which
is kept equal to the reference's (the DWG diffusion moves each triangle's
unit normal, so another split of the same polygon changes the result), and
they are the oracle's triangle table.

Usage (needs the reference checkout; the output is committed):
    python tests/golden/make_mc_fixture.py /path/to/reference
"""
import json
import os
import re
import sys
from collections import Counter


def oriented_loops(tris):
    de = Counter()
    for t in tris:
        for k in range(3):
            de[(t[k], t[(k + 1) % 3])] += 1
    bnd = [e for e in de if (e[1], e[0]) not in de]
    nx = {a: b for a, b in bnd}
    loops, seen = [], set()
    for a in sorted(nx):
        if a in seen:
            continue
        loop, c = [a], nx[a]
        seen.add(a)
        while c != a:
            loop.append(c)
            seen.add(c)
            c = nx[c]
        i = loop.index(min(loop))
        loops.append(loop[i:] + loop[:i])
    return sorted(loops)


def main(ref_root):
    src = open(os.path.join(ref_root, "src", "TurboMC.cu")).read()
    start = src.index("triangle_table = {")
    body = src[start:src.index("};", start)]
    rows = re.findall(r"\{([-\d,\s]+)\}", body)
    assert len(rows) == 256, len(rows)
    cases = []
    for ci, r in enumerate(rows):
        v = [int(x) for x in r.split(",")]
        tris = [tuple(v[i:i + 3]) for i in range(0, 16, 3) if v[i] != -1]
        cases.append({"case": ci, "tri_count": len(tris), "loops": oriented_loops(tris),
                      "tris": [list(t) for t in tris]})
    out = {
        "source": "DWGTech/DWG src/TurboMC.cu:57 (triangle_table): triangles per case, their loops and counts",
        "corner_offsets": "corner c at (x + (b0 != b1), y + b1, z + !b2), src/TurboMC.cu:408-413",
        "edges": "edge e joins (e & 7, e<4 ? (e+1)&3 : e<8 ? 4+((e-3)&3) : e-4), src/TurboMC.cu:433-434",
        "cases": cases,
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mc_reference_loops.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("DWG_REFERENCE"):
        sys.exit("usage: make_mc_fixture.py <reference checkout>  (or set DWG_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["DWG_REFERENCE"])

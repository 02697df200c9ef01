"""Generate tests/golden/gs_face_fixtures.json from the reference's own
gather-scatter known-answer tests.

Source: tests/unit/gather_scatter/test_gather_scatter_parallel.pf:38-903 of
the reference (Neko).  Each of the seven tests builds a two-element mesh from
twelve explicitly numbered points, with the second element rotated or
reflected so that a different face pairing occurs, runs gs ADD on
``1 + dof`` (element 1 only) and asserts that the values on the shared face
agree.  This script reads that file as text and records, per test, the point
ids/coordinates, the eight point references of each element (in the order
they are passed to ``mesh%add_element``), the polynomial size and the two
index expressions of the ADD assertion.  It runs only where the reference
checkout exists; the JSON it writes is committed.

Usage: python tests/golden/make_gs_fixtures.py <reference root>
"""
import json
import os
import re
import sys

PF = "tests/unit/gather_scatter/test_gather_scatter_parallel.pf"


def parse(text):
    tests = []
    for m in re.finditer(r"subroutine (test_dofmap_\w+)\(this\)(.*?)end subroutine", text, re.S):
        name, body = m.group(1), m.group(2)
        pts = {}
        for pm in re.finditer(r"call p\((\d+)\)%init\(([-\dd.]+),\s*([-\dd.]+),\s*([-\dd.]+)\)", body):
            pts.setdefault(int(pm.group(1)), {})["xyz"] = [float(v.replace("d", "e")) for v in pm.group(2, 3, 4)]
        for pm in re.finditer(r"call p\((\d+)\)%set_id\((\d+)\)", body):
            pts[int(pm.group(1))]["id"] = int(pm.group(2))
        elems = []
        for em in re.finditer(r"call m%add_element\((\d+),\s*(\d+),(.*?)\)\s*\n", body, re.S):
            refs = [int(v) for v in re.findall(r"p\((\d+)\)", em.group(3))]
            assert len(refs) == 8, (name, em.group(0))
            elems.append(refs)
        lx = int(re.search(r"lx = (\d+)", body).group(1))
        add = body[body.index("Test GS_OP_ADD"):]
        am = re.search(r"@assertEqual\(x%x\(([^)]*)\),\s*x%x\(([^)]*)\)", add)
        tests.append({
            "name": name,
            "lx": lx,
            "points": {str(k): v for k, v in sorted(pts.items())},
            "elements": elems,
            "assert_lhs": am.group(1).replace(" ", ""),
            "assert_rhs": am.group(2).replace(" ", ""),
            "source": f"{PF}:{text[:m.start()].count(chr(10)) + 1}",
        })
    return tests


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_gs_fixtures.py <root of the reference checkout>")
    root = sys.argv[1]
    with open(os.path.join(root, PF)) as f:
        tests = parse(f.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gs_face_fixtures.json")
    with open(out, "w") as f:
        json.dump(tests, f, indent=1)
    print(f"wrote {len(tests)} fixtures to {out}")


if __name__ == "__main__":
    main()

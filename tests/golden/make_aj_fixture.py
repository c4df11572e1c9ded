"""Extract the Abel-Jacobi basis data of set k = 7 (m = 0..8, n = 0..19)
from the reference's EXAMPLES/Basis/aj07.dat (records "k m n", a line of n
roots, a line of k + 1 coefficients of the polynomial in 1 - r^2, as read
by SRC/lib15/ajsetup.f:23-58) into tests/golden/aj07.json.

    python tests/golden/make_aj_fixture.py /path/to/galaxy
"""
import json
import os
import sys


def parse(path, kset=7, maxm=8, maxn=19):
    lines = open(path).read().split("\n")
    out = {"k": kset, "maxm": maxm, "maxn": maxn, "roots": {}, "xcoeff": {},
           "source": "EXAMPLES/Basis/aj07.dat"}
    i = 0
    while i < len(lines):
        head = lines[i].split()
        if len(head) != 3:
            i += 1
            continue
        k, m, n = (int(v) for v in head)
        roots = [float(v) for v in lines[i + 1].split()]
        xc = [float(v) for v in lines[i + 2].split()]
        i += 3
        assert k == kset and len(roots) == n and len(xc) == k + 1, (k, m, n)
        if m <= maxm and n <= maxn:
            out["roots"][f"{m},{n}"] = roots
            out["xcoeff"][f"{m},{n}"] = xc
    for m in range(maxm + 1):
        for n in range(maxn + 1):
            assert f"{m},{n}" in out["roots"], (m, n)
    return out


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python " + os.path.basename(__file__) + " <reference source root>")
    root = sys.argv[1]
    d = parse(os.path.join(root, "EXAMPLES/Basis/aj07.dat"))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "aj07.json"), "w") as f:
        json.dump(d, f)
    print(len(d["roots"]), "functions")

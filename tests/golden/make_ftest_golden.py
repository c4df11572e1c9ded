"""Generate tests/golden/p3d_ftest.json from the reference's p3d force check.

Reads (as text) the reference's input cards EXAMPLES/p3d/ftest/run999.dat
and its printed result EXAMPLES/p3d/ftest/run999.lis, and writes the grid,
the test-mass positions and the four printed (node, FFT value, direct value,
max abs error) rows.  Run in a container that has the reference checkout:

    python tests/golden/make_ftest_golden.py /path/to/galaxy
"""
import json
import os
import re
import sys


def parse(root):
    dat = open(os.path.join(root, "EXAMPLES/p3d/ftest/run999.dat")).read().splitlines()
    lis = open(os.path.join(root, "EXAMPLES/p3d/ftest/run999.lis")).read().splitlines()
    out = {"source": "EXAMPLES/p3d/ftest/run999.dat, EXAMPLES/p3d/ftest/run999.lis:26-30"}
    masses = []
    for line in dat:
        key = line[:10].strip().lower()
        vals = line[10:].split("#")[0].split()
        if key.startswith("grid size"):
            out["nr"], out["na"], out["ngz"] = (int(v) for v in vals[:3])
        elif key.startswith("z spacing"):
            out["dzg"] = float(vals[0])
        elif key.startswith("hash"):
            out["hash"] = int(vals[0])
        elif key.startswith("softl"):
            out["softl"] = float(vals[0])
            out["tsoft"] = int(vals[1]) if len(vals) > 1 else 2
        elif key.startswith("sectors"):
            out["nsect"] = int(vals[0])
        elif key.startswith("posn"):
            masses.append([int(v) for v in vals[:3]])
    out["masses_as_read"] = masses
    # positions after p3ckst's clamping are printed in the .lis
    placed = []
    for line in lis:
        m = re.match(r"\s*Position\s+(\d+)\s+(\d+)\s+(\d+)\s+zone\s+(\d+)", line)
        if m:
            placed.append([int(m.group(i)) for i in (1, 2, 3)])
    out["masses"] = placed
    rows = []
    seen = False
    for line in lis:
        if "Field type" in line:
            seen = True
            continue
        if seen:
            f = line.split()
            if len(f) == 7 and f[0].isdigit():
                rows.append({"type": int(f[0]), "maxerr": float(f[1]), "r": int(f[2]),
                             "z": int(f[3]), "t": int(f[4]), "fft": float(f[5]),
                             "direct": float(f[6])})
    out["rows"] = rows
    return out


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python " + os.path.basename(__file__) + " <reference source root>")
    root = sys.argv[1]
    data = parse(root)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "p3d_ftest.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(data, indent=1))

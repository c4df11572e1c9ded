"""Make tests/golden/run200_head.pcs and run200_golden.json from the
reference's p3d example (EXAMPLES/p3d/run200.pcs0, its data file run200.dat
and its run log run200.lis).  Run in a tree that holds the reference:

    python tests/golden/make_run200_fixture.py /path/to/reference

The fixture keeps every 20th of the 100000 disc particles (the file lists
them from the centre outwards), 5000 in one record (the file layout of
SRC/lib15/loadup.f:36-140)."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from galaxy_b200.pcs import Pcs, read_pcs, write_pcs  # noqa: E402

if len(sys.argv) < 2:
    sys.exit("usage: python " + os.path.basename(__file__) + " <reference source root>")
ref = sys.argv[1]
full = read_pcs(os.path.join(ref, "EXAMPLES", "p3d", "run200.pcs0"))
n = 5000
head = Pcs((n, 0, 0), full.mcoor, n, full.t, full.pm, full.records[::full.n // n][:n])
write_pcs(os.path.join(HERE, "run200_head.pcs"), head)
gold = {
    "source": "EXAMPLES/p3d/run200.pcs0, run200.dat, run200.lis",
    "n_full": full.n, "nsp_full": list(full.nsp), "mcoor": full.mcoor, "pm": full.pm,
    # run200.lis:23-24 "Inner and outer edges of grid are at 0.00 and 60.7652 grid units",
    # "Maximum z distance of grid is 18.50 grid units"
    "grid_outer_edge": 60.7652, "grid_z_max": 18.50,
    # run200.lis:53 "Population 1 mass is 0.50 represented by 100000 particles"
    "disc_mass": 0.5,
    # run200.dat: grid size 85 128 75, z spacing 0.5, hash 8, softl 1.0 with rule 2
    # (cubic spline), sect 1, skip 1; time step 0.025, lscale 10; zones 3 with
    # (step ratio, radius) (2, 1.0) and (4, 2.5); a rigid isothermal halo
    # 'type isot 0.7', scale 1.0 (mass 0.7^2 = 0.49, run200.lis:57)
    "grid": {"nr": 85, "na": 128, "ngz": 75, "dzg": 0.5, "hash": 8, "softl": 1.0,
             "tsoft": 2, "sectors": 1, "skip": [1], "lscale": 10.0, "ts": 0.025},
    "zones": {"nstep": [1, 2, 4], "radius_model": [0.0, 1.0, 2.5]},
    "halo": {"type": "ISOT", "mass": 0.49, "rscale": 1.0},
}
json.dump(gold, open(os.path.join(HERE, "run200_golden.json"), "w"), indent=1)
print("wrote", head.n, "particles")

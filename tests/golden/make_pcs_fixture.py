"""Make tests/golden/run100_head.pcs and run100_golden.json from the
reference's p2d example (EXAMPLES/p2d/run100.pcs0, its run log run100.lis and
data file run100.dat).  Run in a tree that holds the reference:

    python tests/golden/make_pcs_fixture.py /path/to/reference

The fixture keeps the first 3000 particles of the 15000, re-written in
records of 1000 particles (the file layout of SRC/lib15/loadup.f:36-140)."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from galaxy_b200.pcs import Pcs, read_pcs, write_pcs  # noqa: E402

if len(sys.argv) < 2:
    sys.exit("usage: python " + os.path.basename(__file__) + " <reference source root>")
ref = sys.argv[1]
full = read_pcs(os.path.join(ref, "EXAMPLES", "p2d", "run100.pcs0"))
head = Pcs((3000, 0, 0), full.mcoor, 1000, full.t, full.pm, full.records[:3000])
write_pcs(os.path.join(HERE, "run100_head.pcs"), head)
gold = {
    "source": "EXAMPLES/p2d/run100.pcs0, run100.lis, run100.dat",
    "n_full": full.n, "mcoor": full.mcoor, "per_record_full": full.per_record, "t": full.t,
    "pm": full.pm,
    "records_sum_full": float(full.records.astype(np.float64).sum()),
    # run100.lis:57 "Mass represented by particles = 0.857301"
    "mass_represented": 0.857301,
    # run100.lis:15 "Inner and outer edges of grid are at 0.00 and 90.4726 grid units"
    "grid_outer_edge": 90.4726,
    # run100.dat: grid size 93 128, HASH 2, softl 3.67879, sectors 2, lscale 10, time step 0.02
    "grid": {"nr": 93, "na": 128, "hash": 2, "softl": 3.67879, "sectors": 2, "lscale": 10.0,
             "ts": 0.02},
}
json.dump(gold, open(os.path.join(HERE, "run100_golden.json"), "w"), indent=1)
print("wrote", head.n, "particles")

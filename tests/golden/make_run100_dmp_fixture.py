"""Make tests/golden/run100_dmp.npz from the reference's p2d example run
(EXAMPLES/p2d/run100.dmp0 .. run100.dmp80: restart dumps of run100 every
500 steps, two time-step zones, the m = 0 harmonic skipped in favour of
the analytic disc force).  Run in a tree that holds the reference:

    python tests/golden/make_run100_dmp_fixture.py /path/to/reference

Kept: the whole state at step 0 (15000 particle records in grid units with
zone-step velocities, their zones from the dump's lists, the solve's mass
array and zone 2's newest array); every 5th particle at steps 500 and 1000
with its zone; and the m = 2 amplitude A2 = mean exp(2 i phi) of all the
particles at every dump (steps 0 .. 4000)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from galaxy_b200.dmp import read_dmp  # noqa: E402

if len(sys.argv) < 2:
    sys.exit("usage: python " + os.path.basename(__file__) + " <reference source root>")
ref = sys.argv[1]
ex = os.path.join(ref, "EXAMPLES", "p2d")
d0 = read_dmp(os.path.join(ex, "run100.dmp0"))
sub = np.arange(0, d0.records.shape[0], 5)
out = dict(
    records0=d0.records, zone0=d0.zone.astype(np.int8), mass0=d0.mass,
    zone2_new0=d0.zone_mass[2][3], lstep0=np.array([d0.zone_mass[2][0], d0.zone_mass[2][2]]),
    istep0=d0.istep, lscale=d0.lscale, ts=d0.ts, pmass=d0.pmass, softl=d0.softl,
    nsect=d0.nsect, tsoft=d0.tsoft, nr=d0.grid["nr"], na=d0.grid["na"], ng=d0.grid["ng"],
    skipped=np.array(d0.grid["skipped"]), rgrid=d0.grid["rgrid"], sub=sub,
    # run100.dat: 'type soft 0.367879' (epsilon; rstar = 1 + epsilon, inimod.f:74),
    # 'mass 1.', 'scale 1.0 8.0', 'zones 2' with 'step ratio 2, radius 3.0'
    epsilon=0.367879, disc_mass=1.0, rscale=1.0, nstep=np.array([1, 2]),
    zone_radius_model=np.array([0.0, 3.0]))
steps, a2 = [], []
for k in range(9):
    dk = read_dmp(os.path.join(ex, f"run100.dmp{10 * k}" if k else "run100.dmp0"))
    ph = np.arctan2(dk.records[:, 1].astype(np.float64), dk.records[:, 0].astype(np.float64))
    steps.append(dk.istep)
    a2.append(np.mean(np.exp(2j * ph)))
    if dk.istep in (500, 1000):
        out[f"records{dk.istep}_sub"] = dk.records[sub]
        out[f"zone{dk.istep}_sub"] = dk.zone[sub].astype(np.int8)
out["a2_steps"] = np.array(steps)
out["a2"] = np.array(a2)
np.savez_compressed(os.path.join(HERE, "run100_dmp.npz"), **out)
print("steps", steps, "|A2|", np.abs(a2))

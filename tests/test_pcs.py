"""The reference's particle files (.pcs) and the pcs2dmp-style start of a run,
on the reference's own p2d example (EXAMPLES/p2d/run100.pcs0: the first 3000
of its 15000 particles, tests/golden/make_pcs_fixture.py), pinned on its run
log (run100.lis) and stepped on the GPU against the FP64 oracle."""
import json
import os

import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_RMAP_STDPOL
from galaxy_b200.pcs import Pcs, read_pcs, write_pcs, start_run
from oracle import oracle as ox

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold():
    return json.load(open(os.path.join(GOLD, "run100_golden.json")))


def cfg_run100(g):
    # run100.dat: grid size 93 128, HASH 2, softl 3.67879 (Plummer), sectors 2,
    # 'skip 0': no m = 0 on the grid, the analytic force of the softened disc
    # (mass 1, rstar = 1 + epsilon, epsilon = softl / lscale) instead
    gr = g["grid"]
    L, ts = gr["lscale"], gr["ts"]
    return make_config(2, gr["nr"], gr["na"], ng=gr["hash"] + 1, nsect=gr["sectors"],
                       skip=(0,), rmap=GX_RMAP_STDPOL, softl=gr["softl"], tsoft=1, halo=2,
                       halo_v2=L ** 3 * ts ** 2, halo_rc=(1.0 + gr["softl"] / L) * L)


def test_pcs_reads_the_reference_layout(gold, tmp_path):
    p = read_pcs(os.path.join(GOLD, "run100_head.pcs"))
    assert p.nsp == (3000, 0, 0) and p.mcoor == gold["mcoor"] and p.per_record == 1000
    assert p.t == gold["t"] and p.pm == np.float32(gold["pm"])
    # the mass the reference reports for its 15000 particles (run100.lis)
    assert abs(gold["pm"] * gold["n_full"] - gold["mass_represented"]) < 1e-6
    # round trip: the same bytes
    q = tmp_path / "again.pcs"
    write_pcs(str(q), p)
    assert q.read_bytes() == open(os.path.join(GOLD, "run100_head.pcs"), "rb").read()
    # grid units as loadup stores them (x lscale, v lscale ts, pm lscale^3 ts^2)
    gr = gold["grid"]
    rec, pmass = p.grid_units(gr["lscale"], gr["ts"])
    assert rec.shape == (3000, 4)
    assert np.allclose(rec[:, :2], p.records[:, :2] * gr["lscale"], rtol=1e-6)
    assert np.allclose(rec[:, 2:], p.records[:, 2:] * gr["lscale"] * gr["ts"], rtol=1e-6)
    assert abs(pmass - gold["pm"] * gr["lscale"] ** 3 * gr["ts"] ** 2) < 1e-12


def test_particles_at_the_origin_are_discarded():
    r = np.array([[0, 0, 1, 1], [1, 0, 0, 0]], np.float32)
    rec, _ = Pcs((2, 0, 0), 4, 2, 0.0, 1.0, r).grid_units(10.0, 0.1)
    assert rec.shape == (1, 4)


def test_grid_edge_matches_the_reference_run_log(gold):
    g = ox.geometry(cfg_run100(gold))
    assert abs(g.rgrid - gold["grid_outer_edge"]) < 5e-4


@pytest.mark.gpu
def test_reference_example_steps_track_the_oracle(gold):
    gr = gold["grid"]
    p = read_pcs(os.path.join(GOLD, "run100_head.pcs"))
    cfg = cfg_run100(gold)
    gal = start_run(cfg, p, gr["lscale"], gr["ts"], tcent=False)
    with gal:
        geo = gal.geo
        assert abs(geo.rgrid - gold["grid_outer_edge"]) < 5e-4
        nsteps = 5
        gal.step(nsteps)
        pos = gal.unload().astype(np.float64)
    rec, pmass = p.grid_units(gr["lscale"], gr["ts"])
    c64 = cfg_run100(gold)
    c64.pmass = pmass
    ref, _, _ = ox.step(c64, ox.green(c64, 64), rec.astype(np.float64), nsteps, prec=64)
    scale = np.abs(ref[:, :2]).max()
    d = np.abs(pos[:, :2] - ref[:, :2]).max(axis=1)
    assert d.max() / scale < 1e-3 and np.mean(d > 2e-5 * scale) < 1e-3

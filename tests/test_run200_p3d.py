"""The reference's p3d example (EXAMPLES/p3d/run200): its particle file
(every 20th of its 100000 disc particles, tests/golden/make_run200_fixture.py)
on its 85 x 128 x 75 grid with cubic-spline softening, the m = 1 harmonic
skipped, a rigid isothermal halo and three time-step zones.  The grid is
pinned on the run log (run200.lis: outer edge, vertical extent); the GPU
steps follow the FP64 oracle's zone steps."""
import json
import os

import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_RMAP_STDPOL
from galaxy_b200.pcs import read_pcs
from oracle import oracle as ox

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold():
    return json.load(open(os.path.join(GOLD, "run200_golden.json")))


def run200(gold, pm):
    gr, h = gold["grid"], gold["halo"]
    L, ts = gr["lscale"], gr["ts"]
    cfg = make_config(3, gr["nr"], gr["na"], ngz=gr["ngz"], dzg=gr["dzg"], ng=gr["hash"] + 1,
                      nsect=gr["sectors"], skip=tuple(gr["skip"]), rmap=GX_RMAP_STDPOL,
                      softl=gr["softl"], tsoft=gr["tsoft"], pmass=pm,
                      # ISOT (frhalo.f:55-56): F = -(M/a) x / (x^2 + a^2) in model
                      # units, x = r / a; in grid units v^2 = (M/a) L^2 ts^2, rc = a L
                      halo=1, halo_v2=h["mass"] / h["rscale"] * L ** 2 * ts ** 2,
                      halo_rc=h["rscale"] * L)
    nstep = gold["zones"]["nstep"]
    zbr = [r * L for r in gold["zones"]["radius_model"]]
    return cfg, nstep, zbr


def load(gold):
    p = read_pcs(os.path.join(GOLD, "run200_head.pcs"))
    gr = gold["grid"]
    rec, pm = p.grid_units(gr["lscale"], gr["ts"])
    return p, rec, pm


def test_run200_file_and_grid_match_the_reference_log(gold):
    p, rec, pm = load(gold)
    assert p.nsp == (5000, 0, 0) and p.mcoor == gold["mcoor"] == 6
    assert p.pm == np.float32(gold["pm"])
    # the particles carry the disc mass of the log (100000 of them)
    assert abs(gold["pm"] * gold["n_full"] - 0.476880) < 1e-5
    cfg, _, _ = run200(gold, pm)
    g = ox.geometry(cfg)
    assert abs(g.rgrid - gold["grid_outer_edge"]) < 5e-4
    assert abs(g.zm - gold["grid_z_max"]) < 1e-5
    assert list(g.lg[:9]) == [0, 1, 0, 0, 0, 0, 0, 0, 0]  # m = 1 skipped


@pytest.mark.gpu
def test_run200_zoned_steps_track_the_oracle(gold):
    p, rec, pm = load(gold)
    cfg, nstep, zbr = run200(gold, pm)
    G = ox.green(cfg, 64)
    zr = ox.ZoneRun(cfg, G, rec.astype(np.float64), nstep, zbr)
    nsteps = 8
    zr.step(nsteps)
    ref = zr.records()
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.set_zones(nstep, zbr)
        gal.loadup(rec)
        gal.masset()
        zone0, _ = gal.zone_info()
        gal.step(nsteps)
        pos = gal.unload().astype(np.float64)
        zone, istep = gal.zone_info()
    assert istep == nsteps
    assert np.bincount(zone0, minlength=5)[1:4].min() > 100  # all three zones populated
    assert np.mean(zone == zr.zone) > 0.999
    scale = np.abs(ref[:, :3]).max()
    d = np.abs(pos[:, :3] - ref[:, :3]).max(axis=1)
    assert np.mean(d > 2e-5 * scale) < 2e-3 and d.max() / scale < 1e-3, (d.max() / scale)
    dv = np.abs(pos[:, 3:] - ref[:, 3:]).max(axis=1)
    assert np.median(dv) < 1e-5 * np.abs(ref[:, 3:]).max()


@pytest.mark.gpu
def test_run200_partial_grid_solves_give_the_whole_grid_trajectories(gold):
    """3D: zones 1..m < 3 move on most steps and the field is synthesised over
    their rings only (p3fndf.f:66-80); the run is the whole-grid run bit for bit"""
    from galaxy_b200 import GX_FLAG_WHOLE_GRID
    p, rec, pm = load(gold)
    cfg, nstep, zbr = run200(gold, pm)
    out = []
    for flags in (0, GX_FLAG_WHOLE_GRID):
        cfg.flags = flags
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.set_zones(nstep, zbr)
            gal.loadup(rec)
            gal.masset()
            gal.step(2 * max(nstep) + 1)
            out.append((gal.unload(), gal.zone_info()[0]))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])

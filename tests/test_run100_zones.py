"""The reference's own p2d example run, restarted from its dump.

run100 (EXAMPLES/p2d/run100.dat): 15000 particles of a softened Kuz'min-
Toomre disc on a 93 x 128 grid, sectors 2, HASH 2, two time-step zones
(zone 2 beyond 3 length units steps every 2 steps), and 'skip 0': the m = 0
harmonic is left out of the grid and the analytic disc force is applied
instead (filset.f:3-5, axifrc.f, frdisc.f:27-29, inimod.f:74).  The
reference dumped the run every 500 steps; tests/golden/run100_dmp.npz holds
its state at step 0, every 5th particle at steps 500 and 1000, and the m = 2
amplitude at every dump (tests/golden/make_run100_dmp_fixture.py).

The FP64 oracle and the GPU path start from the step-0 dump and must follow
the reference's later dumps: particle positions after 500 and 1000 steps,
the zone lists, and the growth of the m = 2 mode (run100.dat quotes the
predicted eigenfrequency 0.540 + 0.158i)."""
import os

import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_RMAP_STDPOL, GX_GRID_MASS
from oracle import oracle as ox

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run100_dmp.npz")


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(GOLD))


def run100(fx):
    """config, zone step factors and boundaries (grid units) of run100"""
    L, ts = float(fx["lscale"]), float(fx["ts"])
    cfg = make_config(2, int(fx["nr"]), int(fx["na"]), ng=int(fx["ng"]), nsect=int(fx["nsect"]),
                      skip=(0,), rmap=GX_RMAP_STDPOL, softl=float(fx["softl"]),
                      tsoft=int(fx["tsoft"]), pmass=float(fx["pmass"]), halo=2,
                      halo_v2=float(fx["disc_mass"]) * L ** 3 * ts ** 2,
                      halo_rc=(1.0 + float(fx["epsilon"])) * float(fx["rscale"]) * L)
    nstep = [int(v) for v in fx["nstep"]]
    zbr = [float(v) * L for v in fx["zone_radius_model"]]
    return cfg, nstep, zbr


def base_records(rec, zone, nstep, nz=2):
    """velocities from zone-step to base-step units (adjvls.f)"""
    r = rec.astype(np.float32).copy()
    on = zone <= nz
    t = np.asarray(nstep, np.float32)[np.minimum(zone, nz) - 1]
    r[on, 2:] = r[on, 2:] * (np.float32(1) / t[on])[:, None]
    return r


def pos_err(a, b):
    d = np.abs(a[:, :2].astype(np.float64) - b[:, :2].astype(np.float64)).max(axis=1)
    return np.median(d), d.max()


def a2(rec):
    ph = np.arctan2(rec[:, 1].astype(np.float64), rec[:, 0].astype(np.float64))
    return np.abs(np.mean(np.exp(2j * ph)))


@pytest.fixture(scope="module")
def oracle_run(fx):
    cfg, nstep, zbr = run100(fx)
    G = ox.green(cfg, 64)
    rec = base_records(fx["records0"], fx["zone0"].astype(np.int32), nstep)
    return ox.ZoneRun(cfg, G, rec.astype(np.float64), nstep, zbr)


def test_zones_and_zone_masses_match_the_reference_dump(fx, oracle_run):
    zr = oracle_run
    assert zr.z.istep == 0
    assert (zr.zone == fx["zone0"]).all()
    assert np.bincount(zr.zone).tolist() == [0, 11964, 3036]
    # the velocities back in zone-step units are the dump's
    assert np.array_equal(zr.pos.astype(np.float32), fx["records0"])
    m = fx["mass0"].astype(np.float64)
    assert np.abs(zr.mass - m).max() / np.abs(m).max() < 1e-5
    n2 = fx["zone2_new0"].astype(np.float64)
    assert np.abs(zr.zm[1] - n2).max() / np.abs(n2).max() < 1e-5


def test_oracle_follows_the_reference_dumps(fx, oracle_run):
    zr = oracle_run
    sub = fx["sub"]
    tol = {500: (3e-5, 3e-4), 1000: (1e-4, 1e-3)}
    done = 0
    for s in (500, 1000):
        zr.step(s - done)
        done = s
        assert (zr.zone[sub] == fx[f"zone{s}_sub"]).all(), s
        med, mx = pos_err(zr.pos[sub], fx[f"records{s}_sub"])
        assert med < tol[s][0] and mx < tol[s][1], (s, med, mx)


def test_oracle_m2_mode_grows_as_the_reference(fx):
    cfg, nstep, zbr = run100(fx)
    G = ox.green(cfg, 64)
    rec = base_records(fx["records0"], fx["zone0"].astype(np.int32), nstep)
    zr = ox.ZoneRun(cfg, G, rec.astype(np.float64), nstep, zbr)
    ref = np.abs(fx["a2"])
    got = [a2(zr.pos)]
    for _ in fx["a2_steps"][1:]:
        zr.step(500)
        got.append(a2(zr.pos))
    got = np.array(got)
    assert np.all(np.abs(got[1:] / ref[1:] - 1) < 0.02), got / ref
    # growth rate between steps 1000 and 3000 (ts = 0.02 per step)
    rate = np.log(got[6] / got[2]) / (2000 * float(fx["ts"]))
    assert abs(rate - 0.158) < 0.005, rate


# -- GPU -------------------------------------------------------------------
def gpu_run(fx):
    cfg, nstep, zbr = run100(fx)
    gal = Galaxy(cfg)
    gal.greenm()
    gal.set_zones(nstep, zbr)
    gal.loadup(base_records(fx["records0"], fx["zone0"].astype(np.int32), nstep))
    gal.masset()
    return gal, nstep


@pytest.mark.gpu
def test_gpu_zone_masset_matches_the_reference_dump(fx):
    gal, nstep = gpu_run(fx)
    with gal:
        zone, istep = gal.zone_info()
        assert istep == 0 and (zone == fx["zone0"]).all()
        m = fx["mass0"].astype(np.float64)
        assert np.abs(gal.grid(GX_GRID_MASS) - m).max() / np.abs(m).max() < 1e-5
        # loadup scaled the velocities, unload undoes it exactly
        back = gal.unload()
        assert np.array_equal(back, base_records(fx["records0"], fx["zone0"].astype(np.int32),
                                                 nstep))


@pytest.mark.gpu
def test_gpu_follows_the_reference_dumps(fx):
    gal, nstep = gpu_run(fx)
    sub = fx["sub"]
    tol = {500: (3e-5, 5e-4), 1000: (1e-4, 2e-3)}
    with gal:
        done = 0
        for s in (500, 1000):
            gal.step(s - done)
            done = s
            zone, istep = gal.zone_info()
            assert istep == s
            assert np.mean(zone[sub] == fx[f"zone{s}_sub"]) > 0.999, s
            got = gal.unload()
            ref = base_records(fx[f"records{s}_sub"], fx[f"zone{s}_sub"].astype(np.int32), nstep)
            med, mx = pos_err(got[sub], ref)
            assert med < tol[s][0] and mx < tol[s][1], (s, med, mx)
            dv = np.abs(got[sub, 2:] - ref[:, 2:]).max(axis=1)
            assert np.median(dv) < 1e-6, (s, np.median(dv))


@pytest.mark.gpu
def test_gpu_m2_mode_grows_as_the_reference(fx):
    gal, _ = gpu_run(fx)
    ref = np.abs(fx["a2"])
    with gal:
        got = [a2(gal.unload())]
        for _ in fx["a2_steps"][1:]:
            gal.step(500)
            got.append(a2(gal.unload()))
    got = np.array(got)
    assert np.all(np.abs(got[1:] / ref[1:] - 1) < 0.03), got / ref
    rate = np.log(got[6] / got[2]) / (2000 * float(fx["ts"]))
    assert abs(rate - 0.158) < 0.005, rate


@pytest.mark.gpu
def test_gpu_tmcent_uses_each_zones_step(fx):
    """tmcent moves a zone-z velocity by -a t^2 / 2 in zone-step units,
    i.e. -a t / 2 in base-step units (getacc.f:141-150, tmcgrp.f)"""
    gal, nstep = gpu_run(fx)
    with gal:
        gal.findf(False)
        acc = gal.getacc(want_pot=False)
        v0 = gal.unload()[:, 2:].astype(np.float64)
        gal.tmcent(True)
        v1 = gal.unload()[:, 2:].astype(np.float64)
    zone = fx["zone0"].astype(np.int32)
    t = np.asarray(nstep, np.float64)[np.minimum(zone, 2) - 1]
    want = -0.5 * acc.astype(np.float64) * t[:, None]
    assert np.abs((v1 - v0) - want).max() < 1e-6 * np.abs(v0).max()


@pytest.mark.gpu
def test_gpu_zone_api_checks_and_empty_runs(fx):
    from galaxy_b200 import GxError, GX_PREC_FP64
    cfg, nstep, zbr = run100(fx)
    with Galaxy(cfg) as gal:
        for bad_nstep, bad_zbr in (([2, 2], zbr),             # nstep[0] must be 1
                                   ([1, 2, 4], [0.0, 40.0, 20.0]),  # boundaries descending
                                   ([1, 2], [0.0, 1e4])):       # boundary outside the grid
            with pytest.raises(GxError):
                gal.set_zones(bad_nstep, bad_zbr)
        gal.set_zones(nstep, zbr)
        # no particles: masset, steps and the zone report still work
        gal.greenm()
        gal.loadup(np.zeros((0, 4), np.float32))
        gal.masset()
        gal.step(3)
        zone, istep = gal.zone_info()
        assert zone.size == 0 and istep == 3
        assert not np.any(gal.grid(GX_GRID_MASS))
        # zones are set before the particles
        gal.loadup(base_records(fx["records0"][:100], fx["zone0"][:100].astype(np.int32), nstep))
        with pytest.raises(GxError):
            gal.set_zones(nstep, zbr)
    # not on the plain FP64 path
    cfg64, _, _ = run100(fx)
    cfg64.precision = GX_PREC_FP64
    with Galaxy(cfg64) as gal:
        with pytest.raises(GxError):
            gal.set_zones(nstep, zbr)


@pytest.mark.gpu
def test_gpu_partial_grid_solves_give_the_whole_grid_trajectories(fx):
    """on the steps where only zone 1 moves the field is synthesised over
    zone 1's rings only (findf.f:41-54); every moving particle reads the
    same field values as in the whole-grid solve, so the run is the same
    bit for bit"""
    from galaxy_b200 import GX_FLAG_WHOLE_GRID
    cfg, nstep, zbr = run100(fx)
    rec = base_records(fx["records0"], fx["zone0"].astype(np.int32), nstep)
    out = []
    for flags in (0, GX_FLAG_WHOLE_GRID):
        cfg.flags = flags
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.set_zones(nstep, zbr)
            gal.loadup(rec)
            gal.masset()
            gal.step(301)
            out.append((gal.unload(), gal.zone_info()[0], gal.grid(GX_GRID_MASS)))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.gpu
def test_gpu_partial_grid_range_covers_the_moving_zone(fx):
    """the field rings of a partial solve run from jrad(1) to krad(1): the
    rings of zone 1's cells and their outer neighbours (massgn.f:75-76)"""
    gal, nstep = gpu_run(fx)
    nr = int(fx["nr"])
    with gal:
        src, fld = gal.zone_rings()
        assert fld == (1, nr)  # step 0: both zones move
        gal.step(1)
        src, fld = gal.zone_rings()
        rec = gal.unload()
        zone, istep = gal.zone_info()
    assert istep == 1
    key, _, on = ox.weight(gal.cfg, rec, old=False, prec=32)
    na = int(fx["na"])
    ring = key // na
    z1 = (zone == 1) & on.astype(bool)
    assert fld == (int(ring[z1].min()) + 1, int(ring[z1].max()) + 2)
    assert fld[1] < nr - 10  # narrower than the grid
    # the sources span every zone's mass
    assert 1 <= src[0] <= fld[0] and fld[1] < src[1] <= nr

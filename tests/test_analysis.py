"""On-device analysis: the 'danl' density harmonics of the grid rings
(SRC/lib15/densty.f:82-118, 190-250) and the global integrals of icheck.

The oracle's danl is checked on masses whose harmonics are known, the GPU's
against the oracle on the same mass grid, and on the reference's run100
restart dump (tests/golden/run100_dmp.npz)."""
import os

import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_GRID_MASS, GX_RMAP_LOG, GX_RMAP_STDPOL
from oracle import oracle as ox

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run100_dmp.npz")


def cfg2():
    return make_config(2, 40, 64, ng=9, rmap=GX_RMAP_STDPOL, softl=1.0, tsoft=1, pmass=1.0)


def test_oracle_danl_of_known_harmonics():
    cfg = cfg2()
    g = ox.geometry(cfg)
    th = 2 * np.pi * np.arange(g.na) / g.na
    # ring i carries 1 + 0.3 cos(2 th) + 0.1 sin(3 th)
    ring = 1 + 0.3 * np.cos(2 * th) + 0.1 * np.sin(3 * th)
    mass = np.tile(ring, g.nr)
    d = ox.danl(cfg, mass, 10.0, 0.02)
    assert d.shape == (g.nr, g.ng)
    assert np.allclose(d[:, 2], 0.15, atol=1e-12)     # (0.3 na / 2) / na
    assert np.allclose(d[:, 3], 0.05j, atol=1e-12)    # sine sum over m = 0 term
    others = np.delete(d[:, 1:], [1, 2], axis=1)
    assert np.abs(others).max() < 1e-12
    # m = 0: the ring's surface density summed over spokes
    r = [np.float32(0.0)] + [np.expm1(np.float32(g.ua) * np.float32(i + 0.5)) for i in range(g.nr)]
    area = 0.5 * np.float32(g.alpha) * (np.float32(r[1]) ** 2 - np.float32(r[0]) ** 2)
    assert abs(d[0, 0].real - g.na / (10.0 * 0.02 ** 2) / area) < 1e-5 * d[0, 0].real
    # an empty ring reports no harmonics
    mass[:g.na] = 0
    assert np.all(ox.danl(cfg, mass, 10.0, 0.02)[0] == 0)


@pytest.mark.gpu
def test_gpu_danl_matches_oracle_on_the_reference_run():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_run100_zones import gpu_run
    fx = dict(np.load(GOLD))
    L, ts = float(fx["lscale"]), float(fx["ts"])
    gal, _ = gpu_run(fx)
    got = {}
    with gal:
        for steps in (0, 3000):
            if steps:
                gal.step(steps)  # leaves the mass of the new positions in place
            m = gal.grid(GX_GRID_MASS).astype(np.float64)
            d = gal.danl(L, ts)
            ref = ox.danl(gal.cfg, m, L, ts)
            assert np.abs(d[:, 0] - ref[:, 0]).max() < 1e-5 * np.abs(ref[:, 0]).max()
            assert np.abs(d[:, 1:] - ref[:, 1:]).max() < 1e-5, steps
            got[steps] = d
    # at step 0 the harmonics are those of the dump's own mass array
    ref0 = ox.danl(gal.cfg, fx["mass0"].astype(np.float64), L, ts)
    assert np.abs(got[0][:, 1:] - ref0[:, 1:]).max() < 1e-5
    # by step 3000 the bar mode dominates the inner rings' m = 2 harmonic
    assert np.abs(got[3000][:20, 2]).max() > 30 * np.abs(got[0][:20, 2]).max()


def _icheck_ref(cfg, rec, acc, pot, tz, pm, halo_pot=None):
    """the oracle's icheck of the on-grid particles with time-centred base-step
    velocities v + a t / 2 (cencds.f:26-48); pe = pm (pot_grid / 2 + pot_halo)"""
    nd = cfg.ndim
    key, _, on = ox.weight(cfg, rec, old=False, prec=32)
    on = on.astype(bool)
    r = rec.astype(np.float64).copy()
    r[:, nd:] += 0.5 * acc.astype(np.float64) * tz[:, None]
    pg = pot.astype(np.float64) - (0 if halo_pot is None else halo_pot)
    d = ox.icheck(cfg, r[on], acc[on], pg[on], pm)
    if halo_pot is not None:
        d.pe += pm * halo_pot[on].sum()
    return d, int(on.sum())


def _close(a, b, tol):
    for f in ("ke", "pe", "lz", "virial", "a2_re", "a2_im"):
        x, y = getattr(a, f), getattr(b, f)
        assert abs(x - y) <= tol * max(abs(y), 1e-300), (f, x, y)


@pytest.mark.gpu
def test_gpu_icheck_matches_oracle_integrals():
    """icheck.f:61-92 on a 3D disc with a rigid halo: energies, Lz, virial,
    A2 and the on-grid count against the oracle on the same accelerations"""
    from galaxy_b200.disk import kt_disk
    nr = 32
    cfg = make_config(3, nr, 64, ngz=15, dzg=0.1, ng=9, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / (nr - 1)),
                      rmap_r0=0.05, softl=0.2, tsoft=1, pmass=1.0)
    rec, pm = kt_disk(100000, seed=4, rmax=6.0, ndim=3, z0=0.1, dt=0.025)  # some off the grid
    cfg.pmass = pm
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.findf(True)
        acc, pot = gal.getacc(want_pot=True)
        d = gal.icheck()
    ref, non = _icheck_ref(cfg, rec, acc, pot, np.ones(len(rec)), np.float32(pm))
    assert d.n_on_grid == non and 0 < non < len(rec)
    _close(d, ref, 1e-6)


@pytest.mark.gpu
def test_gpu_icheck_with_zones_on_the_reference_run():
    """run100 at step 0: each zone's velocities time-centred with its own
    step, the analytic disc's potential added in full"""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_run100_zones import gpu_run
    fx = dict(np.load(GOLD))
    gal, nstep = gpu_run(fx)
    with gal:
        gal.findf(True)
        acc, pot = gal.getacc(want_pot=True)
        d = gal.icheck()
        rec = gal.unload()
        zone, _ = gal.zone_info()
        cfg = gal.cfg
    # the softened Kuz'min-Toomre disc's potential, -K / sqrt(r^2 + Rs^2)
    r2 = rec[:, 0].astype(np.float64) ** 2 + rec[:, 1].astype(np.float64) ** 2
    hp = -np.float64(np.float32(cfg.halo_v2)) / np.sqrt(r2 + np.float64(np.float32(cfg.halo_rc)) ** 2)
    tz = np.asarray(nstep, np.float64)[np.minimum(zone, 2) - 1]
    ref, non = _icheck_ref(cfg, rec, acc, pot, tz, np.float32(cfg.pmass), halo_pot=hp)
    assert d.n_on_grid == non
    _close(d, ref, 2e-6)

"""Batched ensemble of 2D discs (gx_ensemble_*): each disc against its own
single-disc run and the FP64 oracle, the A2 series against the particles,
determinism across the graph and direct launch paths and across the
autotuner's launch shapes."""
import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_RMAP_LOG
from galaxy_b200.disk import kt_disk
from galaxy_b200.ensemble import Ensemble
from oracle import oracle as ox

pytestmark = pytest.mark.gpu


def cfg_c1():
    # 64 log-spaced rings 0.05 .. 5 x 128 spokes, m = 0..8, Plummer 0.1
    return make_config(2, 64, 128, ng=9, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / 63),
                       rmap_r0=0.05, softl=0.1, tsoft=1, pmass=1.0)


def discs(counts, seed0=100):
    recs, pms = [], []
    for i, n in enumerate(counts):
        rec, pm = kt_disk(n, seed=seed0 + i, rmax=4.8, ndim=2, dt=0.025)
        recs.append(rec.astype(np.float32))
        pms.append(pm)
    return recs, np.array(pms, np.float32)


def close_positions(pos, ref, tol=2e-5):
    scale = np.abs(ref[:, :2]).max()
    d = np.abs(pos[:, :2].astype(np.float64) - ref[:, :2]).max(axis=1)
    return d.max() / scale, np.mean(d > tol * scale)


def a2_of(cfg, rec):
    """mean e^{2 i phi} over the particles whose cell (massgn's) is on the grid"""
    with Galaxy(cfg) as gal:
        key, _ = gal.weight(rec, old=False)
    on = key >= 0
    x = rec[on, 0].astype(np.float64)
    y = rec[on, 1].astype(np.float64)
    r2 = x * x + y * y
    return np.mean(((x * x - y * y) + 2j * x * y) / r2)


def test_ensemble_discs_match_single_runs_and_oracle():
    cfg = cfg_c1()
    recs, pms = discs([4000, 15000, 9000])
    nsteps = 6
    ens = Ensemble(cfg, recs, pms, max_steps=nsteps)
    ens.step(nsteps)
    out = ens.unload()
    ens.close()
    for d, rec in enumerate(recs):
        c = cfg_c1()
        c.pmass = float(pms[d])
        with Galaxy(c) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.step(nsteps)
            single = gal.unload().astype(np.float64)
        dx, frac = close_positions(out[d], single)
        assert dx < 1e-4 and frac < 1e-3, (d, dx, frac)
    # disc 0 against the FP64 oracle's trajectory
    c = cfg_c1()
    c.pmass = float(pms[0])
    G = ox.green(c, 64)
    ref_pos, _, _ = ox.step(c, G, recs[0].astype(np.float64), nsteps, prec=64)
    dx, frac = close_positions(out[0], ref_pos)
    assert dx < 1e-3 and frac < 1e-3, (dx, frac)


def test_ensemble_a2_series_matches_particles():
    cfg = cfg_c1()
    recs, pms = discs([3000, 12000])
    ens = Ensemble(cfg, recs, pms, max_steps=8)
    a0 = ens.a2()
    assert a0.shape == (1, 2)
    for d in range(2):
        assert abs(a0[0, d] - a2_of(cfg, recs[d])) < 1e-10
    ens.step(5)
    a = ens.a2()
    assert a.shape == (6, 2)
    out = ens.unload()
    ens.close()
    for d in range(2):
        assert abs(a[5, d] - a2_of(cfg, out[d])) < 1e-10, (d, a[5, d], a2_of(cfg, out[d]))


def test_ensemble_graph_and_direct_launches_agree_bitwise():
    cfg = cfg_c1()
    recs, pms = discs([5000, 20000, 700, 11000], seed0=300)
    e1 = Ensemble(cfg, recs, pms, max_steps=20)
    e1.step(20)  # one replay of the 16-step graph + 4 direct launches
    e2 = Ensemble(cfg, recs, pms, max_steps=20)
    for _ in range(20):
        e2.step(1)
    p1, p2 = e1.unload(), e2.unload()
    a1, a2 = e1.a2(), e2.a2()
    e1.close()
    e2.close()
    for x, y in zip(p1, p2):
        assert np.array_equal(x, y)
    assert np.array_equal(a1, a2)


def test_ensemble_tuner_restores_state_and_keeps_results():
    cfg = cfg_c1()
    recs, pms = discs([6000, 30000, 2500], seed0=500)
    e1 = Ensemble(cfg, recs, pms, max_steps=40)
    threads, chunk = e1.tune()
    assert threads in (256, 512, 1024) and chunk in (4096, 8192, 16384, 32768)
    assert e1.steps_done() == 0
    conf = e1.config()
    assert conf["threads"] == threads and conf["chunk"] == chunk
    e1.step(5)
    e2 = Ensemble(cfg, recs, pms, max_steps=40)
    e2.step(5)
    p1, p2 = e1.unload(), e2.unload()
    a1, a2 = e1.a2(), e2.a2()
    e1.close()
    e2.close()
    # the integer deposit makes the fields, hence the trajectories, independent
    # of the launch shape; the A2 sums only change their rounding
    for x, y in zip(p1, p2):
        assert np.array_equal(x, y)
    assert np.abs(a1 - a2).max() < 1e-12

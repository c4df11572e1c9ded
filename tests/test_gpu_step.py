"""GPU parity of the particle side: cell keys (bit-exact against the
oracle's FP32 mirror of SRC/lib15/weight.f), mass assignment (massgn),
interpolated accelerations (grdacc), multi-step trajectories, determinism,
and the plain FP64 path."""
import numpy as np
import pytest

from galaxy_b200 import (Galaxy, make_config, GX_PREC_FP64, GX_PREC_MIXED, GX_RMAP_LOG,
                         GX_RMAP_STDPOL, GX_GRID_MASS)
from galaxy_b200.disk import kt_disk
from oracle import oracle as ox

pytestmark = pytest.mark.gpu


def cfg3(precision=GX_PREC_MIXED, halo=0):
    # log-spaced rings 0.05 .. 5 (the benchmark's ring table), 3D
    nr = 32
    return make_config(3, nr, 64, ngz=15, dzg=0.1, ng=9, rmap=GX_RMAP_LOG,
                       rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.2,
                       tsoft=1, pmass=1.0, halo=halo, halo_v2=0.49 * 0.025 ** 2,
                       halo_rc=1.0, precision=precision)


def cfg2(precision=GX_PREC_MIXED, nsect=1):
    # the reference's standard map u = ln(1 + r)/alpha, 2D
    return make_config(2, 40, 64, ng=9, nsect=nsect, rmap=GX_RMAP_STDPOL, softl=1.0,
                       tsoft=1, pmass=1.0, precision=precision)


def disk3(n, seed=1):
    rec, pm = kt_disk(n, seed=seed, rmax=4.5, ndim=3, z0=0.1, dt=0.025)
    return rec, pm


def disk2(n, seed=2):
    rec, pm = kt_disk(n, seed=seed, rmax=5.0, ndim=2, dt=0.025, lscale=5.0)
    return rec, pm


def boundary_points(cfg, n=4000, seed=7):
    """Particles placed on ring radii, spoke angles and plane heights, where
    truncation is most sensitive."""
    g = ox.geometry(cfg)
    rng = np.random.default_rng(seed)
    ju = rng.integers(0, g.nr - 1, n)
    jt = rng.integers(0, g.na, n)
    if cfg.rmap == GX_RMAP_STDPOL:
        r = np.expm1(np.float32(g.ua) * ju.astype(np.float32))
    else:
        r = np.exp(np.float32(g.ua) * (ju.astype(np.float32) - np.float32(g.uoffs)))
    r = r.astype(np.float32) * (1 + rng.integers(-2, 3, n) * np.float32(6e-8))
    th = 2 * np.pi * jt / g.na + rng.integers(-2, 3, n) * 1e-7
    x = (r * np.cos(th)).astype(np.float32)
    y = (r * np.sin(th)).astype(np.float32)
    if cfg.ndim == 2:
        return np.stack([x, y, 0 * x, 0 * x], axis=1).astype(np.float32)
    jz = rng.integers(0, g.ngz, n)
    z = (jz * np.float32(cfg.dzg) - np.float32(g.zm)).astype(np.float32)
    return np.stack([x, y, z, 0 * x, 0 * x, 0 * x], axis=1).astype(np.float32)


@pytest.mark.parametrize("which", ["3d", "2d", "2d-sectors"])
@pytest.mark.parametrize("old", [False, True])
def test_keys_bit_exact_against_reference_arithmetic(which, old):
    cfg = cfg3() if which == "3d" else cfg2(nsect=2 if which == "2d-sectors" else 1)
    rec = disk3(50000)[0] if which == "3d" else disk2(50000)[0]
    rec = np.concatenate([rec, boundary_points(cfg)])
    okey, owt, oon = ox.weight(cfg, rec, old=old, prec=32)
    with Galaxy(cfg) as gal:
        key, wt = gal.weight(rec, old=old)
    mism = np.nonzero(key != np.where(oon, okey, -1))[0]
    assert mism.size == 0, (mism.size, rec[mism[:5]], key[mism[:5]], okey[mism[:5]])
    on = oon.astype(bool)
    assert np.abs(wt[on] - owt[on]).max() < 2e-5


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_masset_matches_oracle(which):
    cfg = cfg3() if which == "3d" else cfg2()
    rec = disk3(200000)[0] if which == "3d" else disk2(200000)[0]
    ref, jrk = ox.masset(cfg, rec.astype(np.float64), prec=64)
    with Galaxy(cfg) as gal:
        gal.loadup(rec)
        gal.masset()
        m = gal.grid(GX_GRID_MASS).astype(np.float64)
    assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6
    assert np.abs(m - ref).max() / ref.max() < 2e-6


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_getacc_matches_oracle(which):
    cfg = cfg3(halo=1) if which == "3d" else cfg2()
    rec = disk3(50000)[0] if which == "3d" else disk2(50000)[0]
    G = ox.green(cfg, 64)
    mass, jrk = ox.masset(cfg, rec.astype(np.float64), prec=64)
    f = ox.findf(cfg, G, mass, lpot=True, jrk=jrk, prec=64, polar=False)
    acc_ref, pot_ref = ox.grdacc(cfg, rec.astype(np.float64), f, phys=True, prec=64)
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.findf(True)
        acc, pot = gal.getacc()
    num = np.linalg.norm(acc - acc_ref)
    den = np.linalg.norm(acc_ref)
    assert num / den < 1e-5, num / den
    assert np.linalg.norm(pot - pot_ref) / np.linalg.norm(pot_ref) < 1e-5


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_steps_track_oracle_fp64(which):
    cfg = cfg3() if which == "3d" else cfg2()
    rec, pm = disk3(20000) if which == "3d" else disk2(20000)
    cfg.pmass = pm
    G = ox.green(cfg, 64)
    nsteps = 4
    ref_pos, ref_mass, _ = ox.step(cfg, G, rec.astype(np.float64), nsteps, prec=64)
    # the FP64 path's positions are read back as float32 records
    for prec, tol in ((GX_PREC_MIXED, 2e-5), (GX_PREC_FP64, 2e-7)):
        cfg.precision = prec
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.step(nsteps)
            pos = gal.unload().astype(np.float64)
            m = gal.grid(GX_GRID_MASS)
        nd = cfg.ndim
        scale = np.abs(ref_pos[:, :nd]).max()
        dx = np.abs(pos[:, :nd] - ref_pos[:, :nd]).max() / scale
        # a particle whose cell differs by round-off after a few steps moves
        # by a force difference of the interpolation slope; compare the bulk
        frac = np.mean(np.abs(pos[:, :nd] - ref_pos[:, :nd]).max(axis=1) > tol * scale)
        assert frac < 1e-3 and dx < 1e-3, (prec, dx, frac)
        assert np.abs(m - ref_mass).max() / ref_mass.max() < (1e-4 if prec == GX_PREC_MIXED else 1e-6)


def test_mixed_step_is_bitwise_deterministic():
    cfg = cfg3()
    rec, pm = disk3(100000, seed=5)
    cfg.pmass = pm
    outs = []
    for _ in range(2):
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.step(3)
            outs.append((gal.unload(), gal.grid(GX_GRID_MASS)))
    assert np.array_equal(outs[0][0].view(np.uint32), outs[1][0].view(np.uint32))
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))


def test_mixed_force_error_vs_fp64_path():
    """Force relative error <= 1e-5 (global L2) of the mixed path against
    the FP64 path at the same particles, 3D, 400k particles."""
    cfg = make_config(3, 64, 128, ngz=45, dzg=0.04, ng=17, rmap=GX_RMAP_LOG,
                      rmap_a=float(np.log(100.0) / 63), rmap_r0=0.05, softl=0.1, tsoft=1)
    rec, pm = kt_disk(400000, seed=9, rmax=4.8, ndim=3, z0=0.1, dt=0.02)
    cfg.pmass = pm
    res = {}
    for prec in (GX_PREC_MIXED, GX_PREC_FP64):
        cfg.precision = prec
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.findf(True)
            res[prec] = gal.getacc()
    a32, p32 = res[GX_PREC_MIXED]
    a64, p64 = res[GX_PREC_FP64]
    err = np.linalg.norm(a32 - a64) / np.linalg.norm(a64)
    perr = np.linalg.norm(p32 - p64) / np.linalg.norm(p64)
    assert err < 1e-5, err
    assert perr < 1e-5, perr


def test_compensated_drift_tracks_the_exact_sum():
    """GX_FLAG_COMPENSATED: the drift x += v carries its rounding error in a
    low part.  With no mass the step is a pure drift, so after T steps the
    stored (FP32) position must be the FP32 rounding of x0 + T v (summed
    exactly), while the plain FP32 drift accumulates one rounding per step."""
    from galaxy_b200 import GX_FLAG_COMPENSATED
    rng = np.random.default_rng(5)
    n, T = 4000, 3000
    r = rng.uniform(0.5, 3.0, n)
    th = rng.uniform(0, 2 * np.pi, n)
    rec = np.zeros((n, 4), np.float32)
    rec[:, 0] = r * np.cos(th)
    rec[:, 1] = r * np.sin(th)
    rec[:, 2:] = rng.uniform(-1e-3, 1e-3, (n, 2))
    exact = rec[:, :2].astype(np.float64) + T * rec[:, 2:].astype(np.float64)
    err = {}
    for flags in (0, GX_FLAG_COMPENSATED):
        cfg = cfg2()
        cfg.pmass = 0.0
        cfg.flags = flags
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.step(T)
            out = gal.unload()
        assert np.array_equal(out[:, 2:], rec[:, 2:])  # no force: velocities unchanged
        ulp = np.spacing(np.abs(exact).astype(np.float32)).astype(np.float64)
        err[flags] = np.max(np.abs(out[:, :2] - exact) / ulp)
    assert err[GX_FLAG_COMPENSATED] <= 1.0, err
    assert err[0] > 8 * err[GX_FLAG_COMPENSATED], err

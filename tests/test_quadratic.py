"""p3d quadratic (27-point) interpolation, the 'inte 3' card (jmass = 3):
weights (SRC/lib15/weight.f:251-314), mass assignment (massgn.f:173-202) and
force interpolation (grdacc.f:267-299).

No shipped example of the reference uses this scheme, so there is no
reference output to pin it on: the oracle's restatement is checked by the
scheme's own properties (the weights sum to one and reproduce linear
functions of the node coordinates, the deposit conserves mass), and the GPU
path against the oracle (keys bit for bit against its FP32 mirror, masses,
accelerations and trajectories against FP64)."""
import numpy as np
import pytest

from galaxy_b200 import (Galaxy, make_config, GX_FLAG_QUADRATIC, GX_PREC_FP64, GX_RMAP_LOG,
                         GX_GRID_MASS, GxError)
from galaxy_b200.disk import kt_disk
from oracle import oracle as ox


def cfgq(halo=0):
    nr = 32
    return make_config(3, nr, 64, ngz=15, dzg=0.1, ng=9, rmap=GX_RMAP_LOG,
                       rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.2,
                       tsoft=1, pmass=1.0, halo=halo, halo_v2=0.49 * 0.025 ** 2, halo_rc=1.0,
                       flags=GX_FLAG_QUADRATIC)


def disk(n, seed=1):
    return kt_disk(n, seed=seed, rmax=4.5, ndim=3, z0=0.1, dt=0.025)


def node_coords(cfg, key):
    """(t, z, u) index of the central node of each key"""
    g = ox.geometry(cfg)
    jt = key % g.na
    row = key // g.na
    return jt, row % g.ngz, row // g.ngz


def test_oracle_weights_sum_to_one_and_reproduce_linear_functions():
    cfg = cfgq()
    rec = disk(20000)[0].astype(np.float64)
    key, wt, on = ox.weight(cfg, rec, old=True, prec=64)
    on = on.astype(bool)
    assert wt.shape[1] == 27
    assert np.abs(wt[on].sum(axis=1) - 1).max() < 1e-12
    g = ox.geometry(cfg)
    # continuous coordinates of each particle in index units
    r = np.hypot(rec[:, 0], rec[:, 1])
    ua = float(np.float32(cfg.rmap_a))
    u = np.log(r) / ua - np.log(float(np.float32(cfg.rmap_r0))) / ua
    t = np.mod(np.arctan2(rec[:, 1], rec[:, 0]) * g.na / (2 * np.pi), g.na)
    dzg = float(np.float32(cfg.dzg))
    z = (rec[:, 2] + 0.5 * dzg * (g.ngz - 1)) / dzg
    jt, jz, ju = node_coords(cfg, key)
    # sum_l w_l * offset_l along each axis = coordinate - central node,
    # where no index was clamped (interior particles)
    l = np.arange(27)
    oi, oj, ok = l % 3 - 1, (l // 3) % 3 - 1, l // 9 - 1
    inner = on & (ju >= 1) & (u + 0.5 < g.nr - 1) & (z + 0.5 < g.ngz - 1) & (u >= 0.5)
    dt = np.mod(t - jt + g.na / 2, g.na) - g.na / 2
    for off, want in ((oi, dt), (oj, z - jz), (ok, u - ju)):
        got = (wt * off[None, :]).sum(axis=1)
        assert np.abs(got[inner] - want[inner]).max() < 1e-9


def test_oracle_quadratic_deposit_conserves_mass():
    cfg = cfgq()
    rec, pm = disk(30000)
    cfg.pmass = pm
    mass, jrk = ox.masset(cfg, rec.astype(np.float64), prec=64)
    key, wt, on = ox.weight(cfg, rec.astype(np.float64), prec=64)
    _, jz, ju = node_coords(cfg, key)
    g = ox.geometry(cfg)
    on = on.astype(bool)
    # nodes fall outside the mesh only below the first ring's bottom plane
    # (ju = 1, jz = 0); none of these particles is there
    assert not np.any(on & (ju == 1) & (jz == 0))
    pmf = float(np.float32(pm))  # the config holds the particle mass in FP32
    assert abs(mass.sum() - pmf * on.sum()) < 1e-12 * on.sum() * pmf
    # ring range as massgn.f:180-181 tracks it: jrad = ju, krad = ju + 2
    assert jrk[0] == ju[on].min() and jrk[1] == min(ju[on].max() + 2, g.nr)


def test_quadratic_is_rejected_where_it_is_not_built():
    c2 = make_config(2, 32, 64, ng=5, softl=1.0, flags=GX_FLAG_QUADRATIC)
    with pytest.raises(GxError):
        Galaxy(c2)
    c64 = cfgq()
    c64.precision = GX_PREC_FP64
    with pytest.raises(GxError):
        Galaxy(c64)


# -- GPU --------------------------------------------------------------------
def boundary_points(cfg, n=4000, seed=7):
    """particles on the half-integer boundaries the quadratic scheme truncates at"""
    g = ox.geometry(cfg)
    rng = np.random.default_rng(seed)
    u = rng.integers(0, g.nr - 1, n) + np.float32(0.5)
    t = rng.integers(0, g.na, n) + 0.5
    r = np.exp(np.float32(g.ua) * (u.astype(np.float32) - np.float32(g.uoffs))).astype(np.float32)
    r = r * (1 + rng.integers(-2, 3, n) * np.float32(6e-8))
    th = 2 * np.pi * t / g.na + rng.integers(-2, 3, n) * 1e-7
    jz = rng.integers(0, g.ngz - 1, n) + 0.5
    z = (jz * np.float32(cfg.dzg) - np.float32(g.zm)).astype(np.float32)
    x = (r * np.cos(th)).astype(np.float32)
    y = (r * np.sin(th)).astype(np.float32)
    return np.stack([x, y, z, 0 * x, 0 * x, 0 * x], axis=1).astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("old", [False, True])
def test_gpu_quadratic_keys_bit_exact(old):
    cfg = cfgq()
    rec = np.concatenate([disk(50000)[0], boundary_points(cfg)])
    okey, owt, oon = ox.weight(cfg, rec, old=old, prec=32)
    with Galaxy(cfg) as gal:
        key, wt = gal.weight(rec, old=old)
    mism = np.nonzero(key != np.where(oon, okey, -1))[0]
    assert mism.size == 0, (mism.size, rec[mism[:5]], key[mism[:5]], okey[mism[:5]])
    on = oon.astype(bool)
    assert np.abs(wt[on] - owt[on]).max() < 2e-5


@pytest.mark.gpu
def test_gpu_quadratic_masset_matches_oracle_and_is_deterministic():
    cfg = cfgq()
    rec, pm = disk(200000)
    cfg.pmass = pm
    ref, jrk = ox.masset(cfg, rec.astype(np.float64), prec=64)
    ms = []
    for _ in range(2):
        with Galaxy(cfg) as gal:
            gal.loadup(rec)
            gal.masset()
            ms.append(gal.grid(GX_GRID_MASS))
    assert np.array_equal(ms[0], ms[1])
    m = ms[0].astype(np.float64)
    assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6
    assert np.abs(m - ref).max() / ref.max() < 2e-6


@pytest.mark.gpu
def test_gpu_quadratic_getacc_matches_oracle():
    cfg = cfgq(halo=1)
    rec, pm = disk(50000)
    cfg.pmass = pm
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
    assert np.linalg.norm(acc - acc_ref) / np.linalg.norm(acc_ref) < 1e-5
    assert np.linalg.norm(pot - pot_ref) / np.linalg.norm(pot_ref) < 1e-5


@pytest.mark.gpu
def test_gpu_quadratic_steps_track_oracle_fp64():
    cfg = cfgq()
    rec, pm = disk(20000)
    cfg.pmass = pm
    G = ox.green(cfg, 64)
    nsteps = 4
    ref_pos, ref_mass, _ = ox.step(cfg, G, rec.astype(np.float64), nsteps, prec=64)
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.step(nsteps)
        pos = gal.unload().astype(np.float64)
        m = gal.grid(GX_GRID_MASS)
    scale = np.abs(ref_pos[:, :3]).max()
    d = np.abs(pos[:, :3] - ref_pos[:, :3]).max(axis=1)
    assert np.mean(d > 2e-5 * scale) < 1e-3 and d.max() / scale < 1e-3
    assert np.abs(m - ref_mass).max() / ref_mass.max() < 1e-4


@pytest.mark.gpu
def test_gpu_quadratic_with_time_step_zones_tracks_oracle():
    """the two extensions together: p3d, quadratic, three zones (the radii
    and step factors of the reference's p3d example, EXAMPLES/p3d/run200.dat)"""
    cfg = cfgq()
    rec, pm = disk(20000)
    cfg.pmass = pm
    G = ox.green(cfg, 64)
    nstep, zbr = [1, 2, 4], [0.0, 1.0, 2.5]
    zr = ox.ZoneRun(cfg, G, rec.astype(np.float64), nstep, zbr)
    zr.step(8)
    ref = zr.records()
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.set_zones(nstep, zbr)
        gal.loadup(rec)
        gal.masset()
        gal.step(8)
        pos = gal.unload().astype(np.float64)
        zone, istep = gal.zone_info()
    assert istep == 8
    assert np.mean(zone == zr.zone) > 0.999
    scale = np.abs(ref[:, :3]).max()
    d = np.abs(pos[:, :3] - ref[:, :3]).max(axis=1)
    assert np.mean(d > 2e-5 * scale) < 2e-3 and d.max() / scale < 1e-3


@pytest.mark.gpu
def test_gpu_quadratic_keys_with_sectors_and_an_empty_deposit():
    """sector folding (nsect = 2) ahead of the nearest-node rule; no particles"""
    cfg = cfgq()
    cfg.nsect = 2
    cfg.ng = 9
    rec = np.concatenate([disk(20000)[0], boundary_points(cfg, 2000)])
    for old in (False, True):
        okey, owt, oon = ox.weight(cfg, rec, old=old, prec=32)
        with Galaxy(cfg) as gal:
            key, wt = gal.weight(rec, old=old)
        assert np.array_equal(key, np.where(oon, okey, -1)), old
    with Galaxy(cfgq()) as gal:
        gal.loadup(np.zeros((0, 6), np.float32))
        gal.masset()
        assert not np.any(gal.grid(GX_GRID_MASS))


@pytest.mark.gpu
def test_gpu_quadratic_at_the_largest_spoke_count():
    """na = 512, the largest spoke count: 27 rows of 512 fixed-point bins
    (55 KB of shared memory per deposit CTA) and the 27-point gather.  The
    FP32 spoke coordinate resolves 6e-5 spokes near 512 (its ulp), so the
    masses are compared per cell in units of one particle's mass."""
    nr = 24
    cfg = make_config(3, nr, 512, ngz=15, dzg=0.1, ng=5, rmap=GX_RMAP_LOG,
                      rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.2,
                      tsoft=1, pmass=1.0, flags=GX_FLAG_QUADRATIC)
    rec, pm = disk(60000, seed=5)
    cfg.pmass = pm
    ref, _ = ox.masset(cfg, rec.astype(np.float64), prec=64)
    okey, _, oon = ox.weight(cfg, rec, old=False, prec=32)
    with Galaxy(cfg) as gal:
        key, _ = gal.weight(rec, old=False)
        gal.loadup(rec)
        gal.masset()
        m = gal.grid(GX_GRID_MASS).astype(np.float64)
    assert np.array_equal(key, np.where(oon, okey, -1))
    assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6
    assert np.abs(m - ref).max() < 5e-4 * pm

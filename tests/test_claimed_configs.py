"""GPU parity at the configurations the benchmark numbers are quoted on.

* 3D bench grid: 128 log-spaced rings (0.05 .. 5) x 256 spokes x 125 planes
  (dz = 0.04), m = 0..16, Plummer 0.1, on 1M particles of the seeded
  Kuzmin-Toomre disc with a sech^2 layer (z0 = 0.1), dt = 0.02: cell keys bit
  for bit against the FP32 mirror of SRC/lib15/weight.f:196-250 (a 200k
  sample plus particles placed on cell boundaries at 256 spokes and 125
  planes), masset against the FP64 oracle (massgn.f:140-172), the polar
  fields of findf(lpot) (p3manl.f:62-109, p3conv.f:137-230,
  p3fsyn.f:59-129) and the interpolated force and potential (grdacc.f:189-266)
  against the FP64 oracle, each at a relative L2 error <= 1e-5, and a few
  steps against the oracle's FP64 trajectory.
* 2D bench grid: 64 log rings x 128 spokes, m = 0..8, Plummer 0.1, 100k
  particles, 200 steps at dt = 0.025 against the oracle's FP64 trajectory
  (step.f:135-290, stpgrp.f:26-32), for the mixed and the plain FP64 path.
* The field solve's transforms on five more grids, each with the per-ring
  kernels and with the general ones (GX_FLAG_ROWBLOCK_TRANSFORMS): grids
  beyond the tensor-core vertical synthesis (more than 64 even or odd
  vertical wavenumbers; more than 72 spectral columns), a grid it takes, and
  m = 0 alone and m = 0..1, against the oracle.
"""
import numpy as np
import pytest

from galaxy_b200 import (Galaxy, make_config, GX_PREC_FP64, GX_PREC_MIXED, GX_RMAP_LOG,
                         GX_GRID_MASS, GX_GRID_FR, GX_GRID_FT, GX_GRID_FZ, GX_GRID_POT,
                         GX_FLAG_ROWBLOCK_TRANSFORMS)
from galaxy_b200.disk import kt_disk
from oracle import oracle as ox

pytestmark = pytest.mark.gpu

# force and potential relative L2 error bound of the mixed path against FP64
TOL_FIELD = 1e-5


def cfg_bench3(precision=GX_PREC_MIXED):
    """The 3D benchmark grid."""
    nr = 128
    return make_config(3, nr, 256, ngz=125, dzg=0.04, ng=17, rmap=GX_RMAP_LOG,
                       rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.1,
                       tsoft=1, precision=precision)


def cfg_bench2(precision=GX_PREC_MIXED):
    """The 2D benchmark grid."""
    nr = 64
    return make_config(2, nr, 128, ng=9, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / (nr - 1)),
                       rmap_r0=0.05, softl=0.1, tsoft=1, precision=precision)


def on_boundaries(cfg, n, seed=7):
    """Particles within a few ulp of ring radii, spoke angles and plane
    heights, where the truncation to a cell is most sensitive."""
    g = ox.geometry(cfg)
    rng = np.random.default_rng(seed)
    ju = rng.integers(0, g.nr - 1, n)
    jt = rng.integers(0, g.na, n)
    r = np.exp(np.float32(g.ua) * (ju.astype(np.float32) - np.float32(g.uoffs))).astype(np.float32)
    r = r * (1 + rng.integers(-3, 4, n) * np.float32(6e-8))
    th = 2 * np.pi * jt / g.na + rng.integers(-3, 4, n) * 1e-7
    x = (r * np.cos(th)).astype(np.float32)
    y = (r * np.sin(th)).astype(np.float32)
    if cfg.ndim == 2:
        return np.stack([x, y, 0 * x, 0 * x], axis=1).astype(np.float32)
    jz = rng.integers(0, g.ngz, n)
    z = (jz * np.float32(cfg.dzg) - np.float32(g.zm)).astype(np.float32)
    z = z + rng.integers(-2, 3, n).astype(np.float32) * np.float32(1e-8)
    return np.stack([x, y, z, 0 * x, 0 * x, 0 * x], axis=1).astype(np.float32)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def bench3():
    """1M particles on the 3D bench grid with the FP64 oracle's mass, polar
    and Cartesian fields, and Green table."""
    import os
    ox.set_threads(os.cpu_count() or 1)
    rec, pm = kt_disk(1_000_000, seed=12345, rmax=4.8, ndim=3, z0=0.1, dt=0.02)
    cfg = cfg_bench3()
    cfg.pmass = pm
    G = ox.green(cfg, 64)
    pos64 = rec.astype(np.float64)
    mass, jrk = ox.masset(cfg, pos64, prec=64)
    fpol = ox.findf(cfg, G, mass, lpot=True, jrk=jrk, prec=64, polar=True)
    fcart = ox.findf(cfg, G, mass, lpot=True, jrk=jrk, prec=64, polar=False)
    yield dict(cfg=cfg, rec=rec, pm=pm, G=G, mass=mass, jrk=jrk, fpol=fpol, fcart=fcart)
    ox.set_threads(1)


@pytest.mark.parametrize("old", [False, True])
def test_bench3_keys_bit_exact(bench3, old):
    cfg = bench3["cfg"]
    rec = np.concatenate([bench3["rec"][:200_000], on_boundaries(cfg, 50_000)])
    okey, owt, oon = ox.weight(cfg, rec, old=old, prec=32)
    with Galaxy(cfg) as gal:
        key, wt = gal.weight(rec, old=old)
    mism = np.nonzero(key != np.where(oon, okey, -1))[0]
    assert mism.size == 0, (mism.size, rec[mism[:5]], key[mism[:5]], okey[mism[:5]])
    on = oon.astype(bool)
    # the weights are products of the cell fractions, which the fast path
    # forms from its own log and atan2: within 4 ulp of the largest cell
    # coordinate (na = 256 spokes) of the reference's FP32 fractions
    assert np.abs(wt[on] - owt[on]).max() < 4 * np.spacing(np.float32(256.0))


def test_bench3_masset_fields_force_potential_vs_fp64_oracle(bench3):
    cfg = bench3["cfg"]
    rec = bench3["rec"]
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        m = gal.grid(GX_GRID_MASS).astype(np.float64)
        gal.findf_polar(True)
        f = np.stack([gal.grid(GX_GRID_FR), gal.grid(GX_GRID_FT), gal.grid(GX_GRID_FZ),
                      gal.grid(GX_GRID_POT)]).astype(np.float64)
        gal.findf(True)
        acc, pot = gal.getacc()
    # against the FP32 mirror (the same FP32 cells as the reference; the cell
    # fractions come from the fast FP32 log and atan2, within ~2e-5 of the
    # mirror's at 128 rings and 256 spokes, the keys bit for bit)
    ref32, _ = ox.masset(cfg, rec, prec=32)
    ref32 = ref32.astype(np.float64)
    assert np.abs(m - ref32).max() / ref32.max() < 2e-5
    # against FP64 cells: the FP32 cell coordinates (u = log r / alpha up to
    # 128 rings carries ~1e-5 absolute) move weight between cells by that
    # much per particle; the L2 error is what reaches the field
    ref = bench3["mass"]
    assert abs(m.sum() - ref.sum()) / ref.sum() < 1e-6
    assert rel(m, ref) < 1e-5, rel(m, ref)
    for t in range(4):
        assert rel(f[t], bench3["fpol"][t]) < TOL_FIELD, (t, rel(f[t], bench3["fpol"][t]))
    idx = np.arange(0, rec.shape[0], 5)
    acc_ref, pot_ref = ox.grdacc(cfg, rec[idx].astype(np.float64), bench3["fcart"], phys=True,
                                 prec=64)
    ea, ep = rel(acc[idx], acc_ref), rel(pot[idx], pot_ref)
    assert ea < TOL_FIELD and ep < TOL_FIELD, (ea, ep)


def test_bench3_steps_track_oracle_fp64(bench3):
    cfg = bench3["cfg"]
    rec = bench3["rec"][:300_000]
    c = cfg_bench3()
    c.pmass = bench3["pm"]
    nsteps = 5
    ref_pos, ref_mass, _ = ox.step(c, bench3["G"], rec.astype(np.float64), nsteps, prec=64)
    with Galaxy(c) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.step(nsteps)
        pos = gal.unload().astype(np.float64)
        m = gal.grid(GX_GRID_MASS).astype(np.float64)
    scale = np.abs(ref_pos[:, :3]).max()
    d = np.abs(pos[:, :3] - ref_pos[:, :3]).max(axis=1) / scale
    assert np.mean(d > 2e-5) < 1e-3 and d.max() < 1e-3, (np.mean(d > 2e-5), d.max())
    assert np.abs(m - ref_mass).max() / ref_mass.max() < 1e-4


def _a2(p):
    ph = np.arctan2(p[:, 1], p[:, 0])
    return np.mean(np.exp(2j * ph))


@pytest.mark.parametrize("precision,tol", [(GX_PREC_MIXED, 2e-5), (GX_PREC_FP64, 2e-7)])
def test_bench2_200_steps_track_oracle_fp64(precision, tol):
    """The 2D bench configuration over its 200 steps (100k particles,
    dt = 0.025).  The mixed path's positions stay within 2e-5 of the
    position scale for all but 0.1 % of the particles (the FP32 mirror of
    the reference drifts from the FP64 trajectory by 1.1e-6 at the 99.9th
    percentile over the same run); the FP64 path is read back as float32."""
    import os
    ox.set_threads(os.cpu_count() or 1)
    rec, pm = kt_disk(100_000, seed=12345, rmax=4.8, ndim=2, dt=0.025)
    cfg = cfg_bench2(GX_PREC_FP64)
    cfg.pmass = pm
    nsteps = 200
    ref_pos, ref_mass, _ = ox.step(cfg, ox.green(cfg, 64), rec.astype(np.float64), nsteps, prec=64)
    ox.set_threads(1)
    cfg.precision = precision
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.step(nsteps)
        pos = gal.unload().astype(np.float64)
        m = gal.grid(GX_GRID_MASS).astype(np.float64)
    scale = np.abs(ref_pos[:, :2]).max()
    d = np.abs(pos[:, :2] - ref_pos[:, :2]).max(axis=1) / scale
    assert np.mean(d > tol) < 1e-3 and d.max() < 1e-3, (np.mean(d > tol), d.max())
    mtol = 1e-4 if precision == GX_PREC_MIXED else 1e-6
    assert np.abs(m - ref_mass).max() / ref_mass.max() < mtol
    a, b = _a2(pos), _a2(ref_pos)
    assert abs(a - b) < 1e-4 * abs(b), (a, b)


# Transform kernels by grid.  By default the per-ring kernels take every
# grid below; with GX_FLAG_ROWBLOCK_TRANSFORMS the general kernels run:
# the forward k_fwd_az + k_fwd_z, and for the vertical synthesis the
# tensor-core k_synz_tc ("std") or, where it does not take the grid, the FP32
# k_synz (68 even wavenumbers at ngz = 135, 81 spectral columns at
# m = 0..40), then k_synaz.
FALLBACK = {
    "ngz135": dict(nr=32, na=32, ngz=135, dzg=0.02, ng=5),
    "m0..40": dict(nr=32, na=128, ngz=15, dzg=0.1, ng=41),
    "std": dict(nr=32, na=64, ngz=45, dzg=0.05, ng=9),
    # m = 0 alone (the ring synthesis's m = 0 units only; the forward takes
    # the general kernels, its ring kernel having no m >= 1 column) and m = 0..1
    "ng1": dict(nr=32, na=64, ngz=15, dzg=0.1, ng=1),
    "ng2": dict(nr=32, na=64, ngz=15, dzg=0.1, ng=2),
}


@pytest.mark.parametrize("rowblock", [False, True], ids=["ring", "rowblock"])
@pytest.mark.parametrize("case", sorted(FALLBACK))
def test_fp32_vertical_synthesis_grids_vs_oracle(case, rowblock):
    p = FALLBACK[case]
    nr = p["nr"]
    cfg = make_config(3, nr, p["na"], ngz=p["ngz"], dzg=p["dzg"], ng=p["ng"], rmap=GX_RMAP_LOG,
                      rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=0.2, tsoft=1,
                      flags=GX_FLAG_ROWBLOCK_TRANSFORMS if rowblock else 0)
    rec, pm = kt_disk(100_000, seed=31, rmax=4.5, ndim=3, z0=0.3, dt=0.02)
    cfg.pmass = pm
    G = ox.green(cfg, 64)
    mass, jrk = ox.masset(cfg, rec.astype(np.float64), prec=64)
    fpol = ox.findf(cfg, G, mass, lpot=True, jrk=jrk, prec=64, polar=True)
    ref_pos, _, _ = ox.step(cfg, G, rec.astype(np.float64), 3, prec=64)
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.findf_polar(True)
        f = np.stack([gal.grid(GX_GRID_FR), gal.grid(GX_GRID_FT), gal.grid(GX_GRID_FZ),
                      gal.grid(GX_GRID_POT)]).astype(np.float64)
        gal.step(3)
        pos = gal.unload().astype(np.float64)
    for t in range(4):
        if not np.any(fpol[t]):
            # no such force (the azimuthal one with m = 0 alone): zero as well
            assert not np.any(f[t]), t
            continue
        assert rel(f[t], fpol[t]) < TOL_FIELD, (t, rel(f[t], fpol[t]))
    scale = np.abs(ref_pos[:, :3]).max()
    d = np.abs(pos[:, :3] - ref_pos[:, :3]).max(axis=1) / scale
    assert np.mean(d > 2e-5) < 1e-3 and d.max() < 1e-3, (np.mean(d > 2e-5), d.max())

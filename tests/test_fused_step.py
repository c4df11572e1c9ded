"""The fused particle pass on the bucketed store (gx_bucket.cu) against the
row-sorted deposit (gx_deposit.cu, GX_FLAG_SORTED_DEPOSIT).

Both compute the same positions (the same push arithmetic) and the same
integer fixed-point mass sums, so every case must agree bit for bit: the
particles (read back in load order) and the mass array, after steps that
cross the entry points which compact the bucketed store (getacc, tmcent,
icheck, unload) and re-bucket it.  Cases: 3D and 2D discs; the compensated
position update; particles moving several cells per step (segments
overflow, corners fall outside the deposit window, particles leave the
grid); the 3D benchmark grid; a context with no particles."""
import numpy as np
import pytest

from galaxy_b200 import (Galaxy, make_config, GX_FLAG_COMPENSATED, GX_FLAG_SORTED_DEPOSIT,
                         GX_RMAP_LOG, GX_RMAP_STDPOL, GX_GRID_MASS)
from galaxy_b200.disk import kt_disk

pytestmark = pytest.mark.gpu


def cfg3(nr=32, na=64, ngz=15, dzg=0.1, ng=9, softl=0.2):
    return make_config(3, nr, na, ngz=ngz, dzg=dzg, ng=ng, rmap=GX_RMAP_LOG,
                       rmap_a=float(np.log(100.0) / (nr - 1)), rmap_r0=0.05, softl=softl, tsoft=1)


def cfg2():
    return make_config(2, 40, 64, ng=9, rmap=GX_RMAP_STDPOL, softl=1.0, tsoft=1)


def case(name):
    if name == "3d":
        rec, pm = kt_disk(200_000, seed=1, rmax=4.5, ndim=3, z0=0.1, dt=0.025)
        return cfg3(), rec, pm, 0
    if name == "2d":
        rec, pm = kt_disk(200_000, seed=2, rmax=5.0, ndim=2, dt=0.025, lscale=5.0)
        return cfg2(), rec, pm, 0
    if name == "3d-compensated":
        rec, pm = kt_disk(100_000, seed=3, rmax=4.5, ndim=3, z0=0.1, dt=0.025)
        return cfg3(), rec, pm, GX_FLAG_COMPENSATED
    if name == "3d-fast-movers":
        rec, pm = kt_disk(100_000, seed=4, rmax=4.5, ndim=3, z0=0.1, dt=0.025)
        rec = rec.copy()
        rec[:, 3:] *= 25.0   # several cells per step: overflow, out-of-window corners, off-grid
        return cfg3(), rec, pm, 0
    if name == "2d-fast-movers":
        rec, pm = kt_disk(100_000, seed=5, rmax=5.0, ndim=2, dt=0.025, lscale=5.0)
        rec = rec.copy()
        rec[:, 2:] *= 25.0
        return cfg2(), rec, pm, 0
    if name == "bench3":
        rec, pm = kt_disk(1_000_000, seed=12345, rmax=4.8, ndim=3, z0=0.1, dt=0.02)
        return cfg3(nr=128, na=256, ngz=125, dzg=0.04, ng=17, softl=0.1), rec, pm, 0
    raise KeyError(name)


def run(cfg, rec, pm, flags):
    cfg.pmass = pm
    cfg.flags = flags
    out = []
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        gal.findf(True)
        gal.tmcent(True)
        gal.step(3)
        out.append(gal.grid(GX_GRID_MASS))
        gal.findf(True)
        acc, pot = gal.getacc()        # compacts the bucketed store
        out += [acc, pot]
        gal.step(2)
        gal.findf(True)
        gal.icheck()                   # compacts it again (its sums are not compared)
        gal.step(1, phys=True)
        out.append(gal.unload())
        out.append(gal.grid(GX_GRID_MASS))
        gal.step(2)                    # re-bucketed from the compacted store
        out.append(gal.unload())
        out.append(gal.grid(GX_GRID_MASS))
    return out


@pytest.mark.parametrize("name", ["3d", "2d", "3d-compensated", "3d-fast-movers",
                                  "2d-fast-movers", "bench3"])
def test_fused_step_is_bitwise_the_sorted_deposit(name):
    cfg, rec, pm, flags = case(name)
    a = run(cfg, rec, pm, flags)
    b = run(cfg, rec, pm, flags | GX_FLAG_SORTED_DEPOSIT)
    for k, (x, y) in enumerate(zip(a, b)):
        assert x.shape == y.shape
        same = x.view(np.uint32) == y.view(np.uint32)
        assert same.all(), (name, k, int((~same).sum()))
    if "fast" in name:
        # the run did move particles across several rows and off the grid
        pos = a[-2]
        assert np.isfinite(pos).all()


def test_fused_step_empty_context():
    cfg = cfg3()
    cfg.pmass = 1.0
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(np.zeros((0, 6), np.float32))
        gal.masset()
        gal.step(2)
        assert gal.unload().shape == (0, 6)
        assert not gal.grid(GX_GRID_MASS).any()


def test_fused_2d_graph_replay_is_bitwise_the_sorted_deposit():
    """A 2D run long enough that the fused path replays pairs of steps from
    a CUDA graph (captured once the mass is a fused pass's): the same
    particles and mass, bit for bit, as the sorted deposit's plain
    launches, over two calls."""
    cfg, rec, pm, _ = case("2d")
    out = []
    for flags in (0, GX_FLAG_SORTED_DEPOSIT):
        cfg.pmass = pm
        cfg.flags = flags
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            gal.step(21)
            gal.step(14, phys=True)
            out.append((gal.unload(), gal.grid(GX_GRID_MASS)))
    for x, y in zip(out[0], out[1]):
        assert (x.view(np.uint32) == y.view(np.uint32)).all()

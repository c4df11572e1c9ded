"""Adjoint of the 2D step (gx_adjoint): the FP64 oracle adjoint against
central finite differences of the oracle's own FP64 trajectory (CPU), and
the GPU adjoint against the FP64 oracle gradient (GPU)."""
import numpy as np
import pytest

from galaxy_b200 import Galaxy, make_config, GX_RMAP_LOG
from galaxy_b200.disk import kt_disk
from oracle import oracle as ox

DT = 0.025


def cfg_adj(nr=32, na=64, ng=5, pmass=1.0):
    # log rings 0.05 .. 5, Plummer 0.2, cored isothermal halo r_c = 1, v0 = 0.7
    return make_config(2, nr, na, ng=ng, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / (nr - 1)),
                       rmap_r0=0.05, softl=0.2, tsoft=1, pmass=pmass, halo=1,
                       halo_v2=0.49 * DT * DT, halo_rc=1.0)


def disc(n, seed):
    rec, pm = kt_disk(n, seed=seed, rmax=4.5, ndim=2, dt=DT, halo_v2=0.49, halo_rc=1.0)
    return rec.astype(np.float32), pm


def test_oracle_adjoint_matches_central_differences():
    rec, pm = disc(400, 3)
    cfg = cfg_adj(pmass=pm)
    G = ox.green(cfg, 64)
    T = 6
    pos = rec.astype(np.float64)
    J, grad, dth = ox.adj_gradient(cfg, G, pos, T)
    assert J > 0
    h = 1e-5
    rng = np.random.default_rng(0)
    for _ in range(8):
        p, k = int(rng.integers(len(pos))), int(rng.integers(4))
        a, b = pos.copy(), pos.copy()
        a[p, k] += h
        b[p, k] -= h
        fd = (ox.adj_forward(cfg, G, a, T)[0] - ox.adj_forward(cfg, G, b, T)[0]) / (2 * h)
        assert abs(grad[p, k] - fd) <= 1e-6 * abs(fd) + 1e-12, (p, k, grad[p, k], fd)
    for k in range(2):
        c1, c2 = cfg_adj(pmass=pm), cfg_adj(pmass=pm)
        if k == 0:
            c1.halo_rc += 1e-4
            c2.halo_rc -= 1e-4
            d = c1.halo_rc - c2.halo_rc
        else:
            c1.halo_v2 += 1e-4 * c1.halo_v2
            c2.halo_v2 -= 1e-4 * c2.halo_v2
            d = c1.halo_v2 - c2.halo_v2
        fd = (ox.adj_forward(c1, G, pos, T)[0] - ox.adj_forward(c2, G, pos, T)[0]) / d
        assert abs(dth[k] - fd) <= 1e-5 * abs(fd), (k, dth[k], fd)


@pytest.mark.gpu
@pytest.mark.parametrize("ckpt", [1, 4, 12])
def test_gpu_adjoint_matches_fp64_oracle(ckpt):
    rec, pm = disc(3000, 11)
    cfg = cfg_adj(pmass=pm)
    T = 12
    J_ref, g_ref, th_ref = ox.adj_gradient(cfg, ox.green(cfg, 64), rec.astype(np.float64), T)
    with Galaxy(cfg) as gal:
        gal.greenm()
        gal.loadup(rec)
        gal.masset()
        J, grad, dth, drift = gal.adjoint(T, ckpt)
        # the context holds the initial particles again
        back = gal.unload()
    assert np.array_equal(back, rec)
    # measured on a B200: J 1.7e-8, gradient 2.9e-6 (each component <= 3.0e-6),
    # halo-parameter derivatives <= 8.2e-6, relative to the FP64 oracle
    assert abs(J - J_ref) < 1e-6 * J_ref, (J, J_ref)
    err = np.linalg.norm(grad - g_ref) / np.linalg.norm(g_ref)
    assert err < 3e-5, err
    for k in range(4):
        ek = np.linalg.norm(grad[:, k] - g_ref[:, k]) / np.linalg.norm(g_ref[:, k])
        assert ek < 3e-5, (k, ek)
    assert np.all(np.abs(dth - th_ref) < 1e-4 * np.abs(th_ref)), (dth, th_ref)
    # time reversal in FP32 over at most ckpt steps stays close to the checkpoints
    assert drift < 1e-3, drift


@pytest.mark.gpu
def test_gpu_adjoint_is_deterministic_up_to_fp64_atomics():
    rec, pm = disc(5000, 21)
    cfg = cfg_adj(pmass=pm)
    outs = []
    for _ in range(2):
        with Galaxy(cfg) as gal:
            gal.greenm()
            gal.loadup(rec)
            gal.masset()
            outs.append(gal.adjoint(10, 5))
    (J1, g1, t1, _), (J2, g2, t2, _) = outs
    assert J1 == J2
    assert np.linalg.norm(g1 - g2) <= 1e-6 * np.linalg.norm(g1)
    assert np.all(np.abs(t1 - t2) <= 1e-9 * np.abs(t1))

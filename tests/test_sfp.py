"""SFP (Abel-Jacobi, k = 7, m = 0..8, n = 0..19) coefficient sum and forces.

CPU: the oracle's restatement of ajfun/ajder/sfptab/sfpval (table of nrtab
radii + 5-point Lagrange interpolation, the reference's algorithm) agrees
with direct evaluation of the basis functions, and its coefficient sum
agrees with the direct-evaluation sum.
GPU: gx_sfp_sum (tensor-core moments: mma.sync and tcgen05, FP16 hi/lo
operands) and its FP64 path against the oracle's FP64 sum; gx_sfp_acc
against the oracle's sfpacc; the SFP-driven time loop gx_sfp_step against
the oracle's FP64 loop (sfpadd + sfpacc + stpgrp).
Basis data: tests/golden/aj07.json (tests/golden/make_aj_fixture.py).
"""
import os

import numpy as np
import pytest

from galaxy_b200.disk import exp_disk
from galaxy_b200.sfp import Basis
from oracle import oracle as ox


@pytest.fixture(scope="module")
def basis(golden_dir):
    return Basis.from_json(os.path.join(golden_dir, "aj07.json"), maxm=8, maxn=19)


def test_table_interpolation_matches_direct_basis(basis):
    """sfpval's 5-point Lagrange interpolation (sfpval.f:33-52) on the
    1001-radius table reproduces ajfun; the coefficient sum built on it
    equals the sum of directly evaluated functions."""
    pos = exp_disk(3000, seed=4).astype(np.float64)
    maxr = 6.0
    C = ox.sfp_coeffs(basis, pos, maxr)
    r = np.hypot(pos[:, 0], pos[:, 1])
    ph = np.arctan2(pos[:, 1], pos[:, 0])
    D = np.zeros_like(C)
    for m, n in basis.functions():
        U = np.array([ox.ajfun(basis, m, n, ri / maxr) for ri in r])
        if m == 0:
            D[n, 8] = U.sum()
        else:
            D[n, 8 + m] = (U * np.cos(m * ph)).sum()
            D[n, 8 - m] = (U * np.sin(m * ph)).sum()
    D /= maxr ** 2
    assert np.linalg.norm(C - D) / np.linalg.norm(D) < 1e-9


def test_ajder_is_the_derivative_of_ajfun(basis):
    h = 1e-6
    for m, n in [(0, 0), (2, 5), (8, 19), (5, 11)]:
        for p in (0.2, 0.5, 0.9):
            fd = (ox.ajfun(basis, m, n, p + h) - ox.ajfun(basis, m, n, p - h)) / (2 * h)
            assert abs(ox.ajder(basis, m, n, p) - fd) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [400000, 1000, 129])
def test_sfp_sum_matches_fp64_oracle(basis, n):
    """precision 0: warp-level mma.sync tensor cores; 2: tcgen05 tensor cores
    (TMEM accumulator); 1: FP64 CUDA cores.  n = 129 and 1000 leave partial
    rounds and idle CTAs."""
    from galaxy_b200.sfp import Sfp
    pos = exp_disk(n, seed=11)
    ref = ox.sfp_coeffs(basis, pos.astype(np.float64), 6.0, pmass=2.5e-6)
    with Sfp(basis, 6.0) as s:
        s.load(pos)
        c32 = s.sum(pmass=2.5e-6, precision=0)
        ctc5 = s.sum(pmass=2.5e-6, precision=2)
        c64 = s.sum(pmass=2.5e-6, precision=1)
        again = s.sum(pmass=2.5e-6, precision=0)
    e32 = np.linalg.norm(c32 - ref) / np.linalg.norm(ref)
    etc5 = np.linalg.norm(ctc5 - ref) / np.linalg.norm(ref)
    e64 = np.linalg.norm(c64 - ref) / np.linalg.norm(ref)
    # positions are float32 on the device; the oracle uses the same floats
    assert e64 < 1e-9, e64
    assert e32 < 1e-6, e32
    assert etc5 < 1e-6, etc5
    assert np.array_equal(c32, again)


@pytest.mark.gpu
def test_sfp_forces_match_oracle(basis):
    from galaxy_b200.sfp import Sfp
    pos = exp_disk(50000, seed=12)
    coeff = ox.sfp_coeffs(basis, pos.astype(np.float64), 6.0, pmass=1e-5)
    acc_ref, pot_ref = ox.sfp_acc(basis, coeff, pos.astype(np.float64), 6.0)
    with Sfp(basis, 6.0) as s:
        s.load(pos)
        acc, pot = s.acc(coeff)
    assert np.linalg.norm(acc - acc_ref) / np.linalg.norm(acc_ref) < 1e-5
    assert np.linalg.norm(pot - pot_ref) / np.linalg.norm(pot_ref) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 2])
def test_sfp_step_tracks_oracle(basis, precision):
    """gx_sfp_step against the same loop on the oracle in FP64 (step.f:
    sfpadd over the current positions, sfpacc, then v += a dt, x += v dt),
    10 steps of 20k particles of the exponential disc set rotating in their
    own initial field.  The loop on the device keeps FP32 positions and
    velocities and evaluates the basis exactly (Chebyshev series) where the
    oracle interpolates the reference's table."""
    from galaxy_b200.sfp import Sfp
    n, nsteps, dt, maxr = 20000, 10, 0.05, 6.0
    pm = 1.0 / n
    pos = exp_disk(n, seed=21).astype(np.float64)
    c0 = ox.sfp_coeffs(basis, pos, maxr, pmass=pm)
    a0, _ = ox.sfp_acc(basis, c0, pos, maxr)
    r = np.hypot(pos[:, 0], pos[:, 1])
    ar = -(a0[:, 0] * pos[:, 0] + a0[:, 1] * pos[:, 1]) / np.maximum(r, 1e-12)
    vc = np.sqrt(np.maximum(r * ar, 0.0))
    vel = np.stack([-vc * pos[:, 1], vc * pos[:, 0]], axis=1) / np.maximum(r, 1e-12)[:, None]
    rec = np.concatenate([pos, vel], axis=1).astype(np.float32)
    x = rec[:, :2].astype(np.float64)
    v = rec[:, 2:].astype(np.float64)
    for _ in range(nsteps):
        c = ox.sfp_coeffs(basis, x, maxr, pmass=pm)
        a, _ = ox.sfp_acc(basis, c, x, maxr)
        v = v + a * dt
        x = x + v * dt
    c_ref = ox.sfp_coeffs(basis, x, maxr, pmass=pm)
    with Sfp(basis, maxr) as s:
        s.load(rec)
        c_gpu = s.step(nsteps, dt, pmass=pm, precision=precision)
        out = s.unload()
    assert out.shape == (n, 4)
    dx = np.abs(out[:, :2] - x).max() / np.abs(x).max()
    dv = np.abs(out[:, 2:] - v).max() / np.abs(v).max()
    ec = np.linalg.norm(c_gpu - c_ref) / np.linalg.norm(c_ref)
    assert dx < 1e-5 and dv < 1e-4, (dx, dv)
    assert ec < 1e-5, ec
    # the particles did move: 10 steps of a rotating disc
    assert np.abs(out[:, :2] - rec[:, :2]).max() > 0.1


@pytest.mark.gpu
def test_sfp_sum_64_chebyshev_terms(basis):
    """A basis whose functions need 64 Chebyshev terms: the aj07 roots with
    the polynomial in 1 - r^2 extended to k = 16 (degree up to maxn + k +
    maxm / 2 = 39 in x), so the sum runs the 4-tile mma.sync kernels.  Both
    device paths against the oracle's table sum; the tcgen05 path, which
    takes 32 terms at most, refuses the basis."""
    from galaxy_b200 import GxError
    from galaxy_b200.sfp import Basis, Sfp
    rng = np.random.default_rng(5)
    k = 16
    roots, xc = {}, {}
    for m in range(basis.maxm + 1):
        for n in range(basis.maxn + 1):
            roots[(m, n)] = list(basis.roots[m, n, :n])
            base = list(basis.xcoeff[m, n, :])
            xc[(m, n)] = base + list(0.05 * abs(base[0]) * rng.standard_normal(k + 1 - len(base)))
    b16 = Basis(k, roots, xc, maxm=basis.maxm, maxn=basis.maxn)
    pos = exp_disk(300_000, seed=13)
    ref = ox.sfp_coeffs(b16, pos.astype(np.float64), 6.0, pmass=2.5e-6)
    with Sfp(b16, 6.0) as s:
        s.load(pos)
        c32 = s.sum(pmass=2.5e-6, precision=0)
        c64 = s.sum(pmass=2.5e-6, precision=1)
        with pytest.raises(GxError):
            s.sum(pmass=2.5e-6, precision=2)
    e32 = np.linalg.norm(c32 - ref) / np.linalg.norm(ref)
    e64 = np.linalg.norm(c64 - ref) / np.linalg.norm(ref)
    assert e64 < 1e-7, e64
    assert e32 < 1e-6, e32

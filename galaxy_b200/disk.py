"""Seeded synthetic disks of the benchmark shapes (host side, numpy).

The reference draws its initial conditions with its own DF machinery
(SRC/lib15/df*.f, SRC/progs/smooth.f); those programs are outside the PM
step.  These generators stand in for them with seeded inputs of the same
shapes: a Kuzmin-Toomre disc Sigma ~ (1 + r^2)^-3/2 truncated at rmax
(inverse CDF M(<r) ~ 1 - (1 + r^2)^-1/2), circular speed of the
(untruncated) Kuzmin-Toomre potential v_c^2 = M r^2 / (1 + r^2)^(3/2),
Gaussian radial dispersion from Toomre Q (sigma_R = 3.36 Q Sigma / kappa),
azimuthal dispersion from the epicyclic ratio kappa / (2 Omega), and in 3D
a sech^2(z/z0) layer with sigma_z^2 = pi Sigma z0 (isothermal sheet).
G = 1, total disc mass M.  Output is in the internal units of the step:
positions in grid units (x lscale), velocities as displacement per step
(v lscale dt), and pmass = (M / N) lscale^3 dt^2 (SRC/lib15/loadup.f:99).
"""
import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def kt_disk(n, seed=12345, rmax=5.0, q=1.2, mass=1.0, ndim=2, z0=0.1, halo_v2=0.0,
            halo_rc=1.0, dt=0.025, lscale=1.0, dtype=np.float32):
    """Return (records [n, 2*ndim], pmass) for a Kuzmin-Toomre disc."""
    g = _rng(seed)
    f = 1.0 - (1.0 + rmax * rmax) ** -0.5
    u = g.random(n)
    r = np.sqrt(1.0 / (1.0 - u * f) ** 2 - 1.0)
    phi = 2.0 * np.pi * g.random(n)
    # rotation curve: disc (+ optional cored isothermal halo, frhalo.f:55-56)
    vc2_disk = mass * r * r / (1.0 + r * r) ** 1.5
    vc2 = vc2_disk + halo_v2 * r * r / (r * r + halo_rc * halo_rc)
    vc = np.sqrt(vc2)
    # Omega^2 = vc^2 / r^2; kappa^2 = R dOmega^2/dR + 4 Omega^2
    om2 = vc2 / np.maximum(r * r, 1e-12)
    dom2 = (mass * (-3.0 * r) / (1.0 + r * r) ** 2.5
            + halo_v2 * (-2.0 * r) / (r * r + halo_rc * halo_rc) ** 2)
    kap2 = np.maximum(r * dom2 + 4.0 * om2, 1e-12)
    kap = np.sqrt(kap2)
    sigma = mass / (2.0 * np.pi) * (1.0 + r * r) ** -1.5
    sr = 3.36 * q * sigma / kap
    sp = sr * kap / (2.0 * np.sqrt(om2))
    vr = g.normal(0.0, 1.0, n) * sr
    vp = vc + g.normal(0.0, 1.0, n) * sp
    c, s = np.cos(phi), np.sin(phi)
    x, y = r * c, r * s
    vx, vy = vr * c - vp * s, vr * s + vp * c
    if ndim == 2:
        rec = np.stack([x, y, vx, vy], axis=1)
        pos_scale = np.array([lscale, lscale, lscale * dt, lscale * dt])
    else:
        uz = g.random(n)
        z = z0 * np.arctanh(np.clip(2.0 * uz - 1.0, -1 + 1e-12, 1 - 1e-12))
        sz = np.sqrt(np.pi * sigma * z0)
        vz = g.normal(0.0, 1.0, n) * sz
        rec = np.stack([x, y, z, vx, vy, vz], axis=1)
        pos_scale = np.array([lscale] * 3 + [lscale * dt] * 3)
    rec = rec * pos_scale
    pmass = mass / n * lscale ** 3 * dt * dt
    return rec.astype(dtype), pmass


def exp_disk(n, seed=12345, rmax=6.0, dtype=np.float32):
    """Exponential disc Sigma ~ e^-r truncated at rmax (positions only)."""
    g = _rng(seed)
    # inverse CDF of M(<r) ~ 1 - (1 + r) e^-r by bisection on a table
    rr = np.linspace(0.0, rmax, 200001)
    cdf = 1.0 - (1.0 + rr) * np.exp(-rr)
    cdf /= cdf[-1]
    r = np.interp(g.random(n), cdf, rr)
    phi = 2.0 * np.pi * g.random(n)
    return np.stack([r * np.cos(phi), r * np.sin(phi)], axis=1).astype(dtype)

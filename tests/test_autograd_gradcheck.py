"""Gradient-check harness of the hand-written adjoint through its
torch.autograd binding (galaxy_b200.autograd): the gradient of J = |A2| after
T steps of the 2D mixed path (cored isothermal halo r_c = 1, v0 = 0.7) with
respect to the initial records and the halo parameters, taken by backward()
through the adjoint, against central finite differences of the GPU's own
forward step (gx_step) and against the FP64 oracle gradient."""
import numpy as np
import pytest

from galaxy_b200 import make_config, GX_RMAP_LOG
from galaxy_b200.disk import kt_disk
from oracle import oracle as ox

pytestmark = pytest.mark.gpu
DT = 0.025


def cfg_adj(pmass):
    nr = 32
    return make_config(2, nr, 64, ng=5, rmap=GX_RMAP_LOG, rmap_a=float(np.log(100.0) / (nr - 1)),
                       rmap_r0=0.05, softl=0.2, tsoft=1, pmass=pmass, halo=1,
                       halo_v2=0.49 * DT * DT, halo_rc=1.0)


def test_autograd_adjoint_matches_central_differences_of_the_gpu_forward():
    import torch
    from galaxy_b200.autograd import forward_objective, pm_objective
    rec, pm = kt_disk(3000, seed=11, rmax=4.5, ndim=2, dt=DT, halo_v2=0.49, halo_rc=1.0)
    rec = rec.astype(np.float32)
    cfg = cfg_adj(pm)
    T = 12
    coords = torch.tensor(rec, requires_grad=True)
    theta = torch.tensor([cfg.halo_rc, cfg.halo_v2], dtype=torch.float64, requires_grad=True)
    J = pm_objective(coords, theta, cfg, T, 4)
    J.backward()
    g = coords.grad.numpy().astype(np.float64)
    gth = theta.grad.numpy()
    # the same objective as the plain forward step
    J0 = forward_objective(cfg, rec, T)
    assert abs(J.item() - J0) < 1e-5 * J0, (J.item(), J0)
    # and as the FP64 oracle's gradient
    J_ref, g_ref, th_ref = ox.adj_gradient(cfg, ox.green(cfg, 64), rec.astype(np.float64), T)
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 3e-5
    # central differences of the GPU forward on seeded records outside the
    # inner rings (there cells are smaller than the step's reach, and the
    # piecewise-linear weights make J kinked at that scale), step 1e-5
    r = np.hypot(rec[:, 0], rec[:, 1])
    rng = np.random.default_rng(0)
    parts = rng.choice(np.nonzero(r > 1.0)[0], size=3, replace=False)
    scale = np.abs(g).max()
    for p in parts:
        for k in range(4):
            a, b = rec.copy(), rec.copy()
            a[p, k] += np.float32(1e-5)
            b[p, k] -= np.float32(1e-5)
            fd = (forward_objective(cfg, a, T) - forward_objective(cfg, b, T)) / \
                (float(a[p, k]) - float(b[p, k]))
            assert abs(g[p, k] - fd) <= 2e-2 * abs(fd) + 1e-3 * scale, (p, k, g[p, k], fd)
    for k in range(2):
        th = np.array([cfg.halo_rc, cfg.halo_v2], np.float64)
        d = 1e-3 * th[k]
        tp, tm = th.copy(), th.copy()
        tp[k] += d
        tm[k] -= d
        fd = (forward_objective(cfg, rec, T, tp) - forward_objective(cfg, rec, T, tm)) / (2 * d)
        assert abs(gth[k] - fd) <= 2e-2 * abs(fd), (k, gth[k], fd)

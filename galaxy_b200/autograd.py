"""torch.autograd binding of the hand-written adjoint (gx_adjoint), for
gradient checks.

``pm_objective(coords, theta, cfg, nsteps, ckpt_every)`` (a
torch.autograd.Function) returns the
objective J = |A2(t_final)| of a 2D run started from the particle records
``coords`` (n x 4 float32: x, y, vx, vy in grid units) with the cored
isothermal halo ``theta`` = (halo_rc, halo_v2) (frhalo.f:55-56), after
``nsteps`` leapfrog steps of the mixed path; A2 = (1/n) sum_p e^{2 i phi_p}
over all particles.  The forward pass runs the adjoint once (it recomputes
the forward trajectory by time reversal from checkpoints every
``ckpt_every`` steps) and keeps its gradient; ``backward`` scales it by the
incoming gradient.  ``forward_objective`` is the same J from the plain
forward step (gx_step), the function whose central differences the adjoint
is checked against.

The product path does not use torch: this module is the thin wrapper of a
gradient-check harness, importing torch only when it is used.
"""
import numpy as np

from . import Galaxy


def _context(cfg, theta):
    c = type(cfg).from_buffer_copy(cfg)
    c.halo_rc = float(theta[0])
    c.halo_v2 = float(theta[1])
    return c


def forward_objective(cfg, coords, nsteps, theta=None):
    """J = |A2| after nsteps steps of the plain forward path (gx_step) from
    the records coords, with the halo parameters theta = (halo_rc, halo_v2)
    (default: those of cfg)."""
    c = _context(cfg, theta if theta is not None else (cfg.halo_rc, cfg.halo_v2))
    with Galaxy(c) as gal:
        gal.greenm()
        gal.loadup(np.ascontiguousarray(coords, np.float32))
        gal.masset()
        gal.step(nsteps)
        p = gal.unload().astype(np.float64)
    phi = np.arctan2(p[:, 1], p[:, 0])
    return float(abs(np.mean(np.exp(2j * phi))))


def _function():
    import torch

    class PMObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, coords, theta, cfg, nsteps, ckpt_every):
            c = _context(cfg, theta.detach().cpu().numpy())
            rec = np.ascontiguousarray(coords.detach().cpu().numpy(), np.float32)
            with Galaxy(c) as gal:
                gal.greenm()
                gal.loadup(rec)
                gal.masset()
                J, grad, dth, _ = gal.adjoint(int(nsteps), int(ckpt_every))
            ctx.save_for_backward(torch.from_numpy(grad).to(coords.dtype),
                                  torch.from_numpy(dth).to(theta.dtype))
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            grad, dth = ctx.saved_tensors
            return gJ * grad, gJ * dth, None, None, None

    return PMObjective


_PM = None


def pm_objective(coords, theta, cfg, nsteps, ckpt_every=50):
    """J(coords, theta) as a differentiable torch scalar (see the module)."""
    global _PM
    if _PM is None:
        _PM = _function()
    return _PM.apply(coords, theta, cfg, nsteps, ckpt_every)

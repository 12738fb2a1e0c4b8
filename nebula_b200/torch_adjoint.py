"""torch.autograd binding of the seed-replay adjoint (separate from the C ABI).

``ScanProblem`` holds one scan (geometry, materials, primaries, seed, pixel
grid) and two simulations on the device: a forward one and an adjoint one.
``se_yield(theta, problem)`` returns the per-pixel SE yield as a tensor that
is differentiable with respect to ``theta`` (6 values: inelastic IMFP scale,
elastic IMFP scale and work function, for materials 0 and 1):

* forward: sets theta and runs the plain transport; yield = SE count /
  primaries of the pixel;
* backward: sets theta and replays the same primaries with the same seed in
  the adjoint simulation (identical trajectories), which returns per-pixel
  sums of the score functions of every detected SE; the vector-Jacobian
  product is contracted on the host in float64.

The gradients are those of the C ABI (``nbl_sim_gradients``): score-function
estimates for the mean-free-path scales; for the work functions, with
``w_step > 0`` (the default, 0.05 eV), the signed-tally difference of a
replay whose primaries run with the work functions shifted by
``w_step * (+-1)``, which carries the deterministic effects of a crossing
(energy shift, refraction) as well as the transmission probability; with
``w_step = 0`` the transmission probability's score alone.  With
``w_step > 0`` the backward pass uses the forward pass's signed tallies, so
it must follow a forward pass at the same theta (as autograd does).
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Simulation


class ScanProblem:
    def __init__(self, geometry, materials, primaries, tally, seed=1, capacity=1 << 21, device=0, w_step=0.05,
                 physics=None):
        self.primaries = primaries
        self.tally = tuple(tally)
        nx, ny = self.tally
        counts = np.zeros((ny, nx), np.float64)
        ok = (primaries["px"] >= 0) & (primaries["px"] < nx) & (primaries["py"] >= 0) & (primaries["py"] < ny)
        np.add.at(counts, (primaries["py"][ok], primaries["px"][ok]), 1.0)
        self.per_pixel = counts
        self.w_step = float(w_step)
        self._forward_theta = None
        self.forward_sim = Simulation(geometry, materials, capacity=capacity, seed=seed, tally=tally, device=device,
                                      physics=physics)
        self.adjoint_sim = Simulation(geometry, materials, capacity=capacity, seed=seed, tally=tally, device=device,
                                      adjoint=True, adjoint_w_step=self.w_step, physics=physics)

    def set_seed(self, seed):
        """Run both simulations with another random-number key (a new,
        independent sample of the same scan)."""
        self.forward_sim.set_seed(seed)
        self.adjoint_sim.set_seed(seed)
        self._forward_theta = None

    def theta0(self):
        return torch.tensor(self.forward_sim.get_theta(), dtype=torch.float64)

    def _run(self, sim, theta):
        sim.set_theta(np.asarray(theta, np.float32))
        sim.reset()
        sim.push(self.primaries)
        sim.run()
        sim.flush_detected()

    def forward(self, theta):
        self._run(self.forward_sim, theta)
        self._forward_theta = np.asarray(theta, np.float32).copy()
        se, bse, _ = self.forward_sim.tallies()
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(self.per_pixel > 0, se / self.per_pixel, 0.0)

    def jacobian(self, theta):
        """d(SE yield of each pixel)/d theta, shape (ny, nx, 6).  With a
        work-function step, the forward run at the same theta is reused (run
        here if the last forward pass was at another theta)."""
        th = np.asarray(theta, np.float32)
        if self.w_step > 0 and (self._forward_theta is None or not np.array_equal(self._forward_theta, th)):
            self.forward(th)
        self._run(self.adjoint_sim, theta)
        gs, _ = self.adjoint_sim.gradients(self.forward_sim if self.w_step > 0 else None)
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(self.per_pixel[..., None] > 0, gs / self.per_pixel[..., None], 0.0)

    def close(self):
        self.forward_sim.close()
        self.adjoint_sim.close()


class _SEYield(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, problem):
        th = theta.detach().cpu().numpy().astype(np.float64)
        ctx.problem = problem
        ctx.theta = th
        return torch.from_numpy(problem.forward(th)).to(theta.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        J = ctx.problem.jacobian(ctx.theta)
        g = np.einsum("yx,yxk->k", grad_out.detach().cpu().numpy().astype(np.float64), J)
        return torch.from_numpy(g).to(grad_out.dtype), None


def se_yield(theta: torch.Tensor, problem: ScanProblem) -> torch.Tensor:
    """Per-pixel SE yield, differentiable in ``theta`` through the adjoint."""
    return _SEYield.apply(theta, problem)

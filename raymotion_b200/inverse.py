"""Material fitting with the path-replay adjoint (rmcuda_backward).

Parameters are optimised normalised to their ranges (u = (p - lo) / (hi - lo),
clamped to [0, 1]) with Adam.  Across ranks the fit is data parallel: each
rank renders and differentiates its own frames (its own seeds), and ``step``
averages the ranks' gradients with one all-reduce of n_materials x 8 floats
(8 KB for 256 materials; NCCL over NVLink on GPUs, gloo on CPU) before the
identical Adam update, so every rank holds the same parameters.  This is the
only data exchange of the workload; rendering itself runs as replicas.
"""
from __future__ import annotations

import torch


def _world() -> int:
    import torch.distributed as dist
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


class MaterialFit:
    """Adam on normalised material parameters (rows: materials, columns:
    albedo rgb, roughness, emission rgb, IOR); ``mask`` selects the fitted
    entries, the others stay at ``true``."""

    def __init__(self, start: torch.Tensor, true: torch.Tensor, mask: torch.Tensor, lo: torch.Tensor,
                 hi: torch.Tensor, lr: float = 1e-2):
        self.true, self.mask, self.lo, self.hi = true, mask, lo, hi
        self.u = ((start - lo) / (hi - lo)).clone().requires_grad_(True)
        self.opt = torch.optim.Adam([self.u], lr=lr)

    def params(self) -> torch.Tensor:
        return torch.where(self.mask, self.lo + (self.hi - self.lo) * self.u.detach().clamp(0, 1), self.true)

    def step(self, grad: torch.Tensor) -> torch.Tensor:
        """One update from this rank's dL/dparams (n_materials x 8, any shape of that size);
        returns the gradient used (the mean over ranks)."""
        g = grad.reshape(self.u.shape).to(self.u.dtype).clone()
        world = _world()
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(g)
            g /= world
        self.opt.zero_grad()
        self.u.grad = torch.where(self.mask, g * (self.hi - self.lo), torch.zeros_like(self.u))
        self.opt.step()
        with torch.no_grad():
            self.u.clamp_(0, 1)
        return g

"""Differentiable Siddon projector for PyTorch.

FIR has no gradient path; its reconstruction is OSEM only.  This module
exposes the same system matrix A (FIR's Siddon traversal, projections.cc) as
a ``torch.autograd.Function``: the forward pass is the multi-frame forward
projector (``fir_forward_frames``) and the backward pass is the matched
backprojector (``fir_backward_frames``), which retraces the paths instead of
storing them.  Both run on the GPU through the C ABI; there is no CPU path.

Shapes: images ``[F, nz, ny, nx]`` (or ``[nz, ny, nx]``), sinograms
``[F, n_bins]`` (or ``[n_bins]``), FIR's file order of bins.  float32 uses
FIR's arithmetic (each frame's projection equals ``fir_forward``); float64
runs double sums and double atomics, for gradient checks finer than float.

Also here: the attenuated Poisson negative log-likelihood, a quadratic
26-neighbour smoothness penalty and an L-BFGS reconstruction built on them.
"""
from __future__ import annotations

import math
import time
from typing import Optional

import torch

from .capi import Context, proj_geometry
from .geometry import ProjSpec, ScannerSpec, VolSpec


class SiddonProjector:
    """The system matrix of one scanner, sinogram geometry and volume."""

    def __init__(self, scanner: ScannerSpec, proj: ProjSpec, vol: VolSpec, device: int = 0,
                 geometry: Optional[int] = None):
        self.ctx = Context(scanner, device=device)
        if geometry is not None:
            from .capi import FIR_OPT_GEOMETRY

            self.ctx.set_option(FIR_OPT_GEOMETRY, geometry)
        self.scanner, self.proj, self.vol = scanner, proj, vol
        self.n_bins = proj_geometry(proj)["n_bins"]
        self.device = torch.device("cuda", device)

    def close(self):
        self.ctx.close()

    def _frames(self, x: torch.Tensor, n: int):
        return x.reshape(-1, n).shape[0]

    def project(self, x: torch.Tensor) -> torch.Tensor:
        """A x without autograd (frames kept)."""
        single = x.dim() == 3
        xf = x.reshape(-1, *self.vol.shape_zyx).contiguous()
        y = torch.empty(xf.shape[0], self.n_bins, dtype=x.dtype, device=x.device)
        self.ctx.forward_frames(self.vol.with_frames(xf.shape[0]), xf, self.proj, y)
        return y[0] if single else y

    def backproject(self, y: torch.Tensor) -> torch.Tensor:
        """A^T y without autograd (frames kept)."""
        single = y.dim() == 1
        yf = y.reshape(-1, self.n_bins).contiguous()
        x = torch.empty(yf.shape[0], *self.vol.shape_zyx, dtype=y.dtype, device=y.device)
        self.ctx.backward_frames(self.proj, yf, self.vol.with_frames(yf.shape[0]), x)
        return x[0] if single else x

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        """Differentiable A x."""
        return _Project.apply(x, self)


class _Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, op: SiddonProjector):
        ctx.op = op
        return op.project(x)

    @staticmethod
    def backward(ctx, gy):
        return ctx.op.backproject(gy), None


class _BackProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, op: SiddonProjector):
        ctx.op = op
        return op.backproject(y)

    @staticmethod
    def backward(ctx, gx):
        return ctx.op.project(gx), None


def backproject(y: torch.Tensor, op: SiddonProjector) -> torch.Tensor:
    """Differentiable A^T y (its backward is the forward projector)."""
    return _BackProject.apply(y, op)


def expected_counts(x, op: SiddonProjector, atten=None, bias=None):
    """Model mean of the measurement: (A x) * atten + bias, where atten holds
    the attenuation factors exp(-A mu) = 1 / ACF (ProjData::exponential gives
    the ACF)."""
    yb = op(x)
    if atten is not None:
        yb = yb * atten
    if bias is not None:
        yb = yb + bias
    return yb


def poisson_nll(ybar: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """sum(ybar - y log ybar), with 0 log 0 = 0 (bins no LOR of the model
    reaches and no count fell in)."""
    return (ybar - torch.xlogy(y, ybar)).sum()


# the 13 offsets of half the 26-neighbourhood (each neighbour pair once),
# with weight 1 / distance in voxels
_HALF26 = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
           if (dz, dy, dx) > (0, 0, 0)]


def quadratic_penalty(x: torch.Tensor, beta: float) -> torch.Tensor:
    """beta/2 * sum over 26-neighbour pairs (j, k) of (x_j - x_k)^2 / |j - k|,
    |j - k| the centre distance in voxels (1, sqrt 2, sqrt 3); per frame,
    summed over frames."""
    xs = x.reshape(-1, *x.shape[-3:])
    total = xs.new_zeros(())
    nz, ny, nx = xs.shape[-3:]
    for dz, dy, dx in _HALF26:
        a = xs[:, max(dz, 0):nz + min(dz, 0), max(dy, 0):ny + min(dy, 0), max(dx, 0):nx + min(dx, 0)]
        b = xs[:, max(-dz, 0):nz + min(-dz, 0), max(-dy, 0):ny + min(-dy, 0), max(-dx, 0):nx + min(-dx, 0)]
        w = 1.0 / math.sqrt(dz * dz + dy * dy + dx * dx)
        total = total + w * ((a - b) ** 2).sum()
    return 0.5 * beta * total


def penalized_nll(x, y, op: SiddonProjector, beta: float, atten=None, bias=None):
    """Poisson NLL of the attenuated model plus the quadratic penalty."""
    return poisson_nll(expected_counts(x, op, atten, bias), y) + quadratic_penalty(x, beta)


def reconstruct_lbfgs(op: SiddonProjector, y, beta: float, atten=None, bias=None, x0=None, steps: int = 50,
                      history: int = 10):
    """Penalized-likelihood reconstruction by L-BFGS (torch.optim.LBFGS, strong
    Wolfe line search, ``steps`` iterations).  Non-negativity through the
    parametrisation x = softplus(theta).  Returns (x, stats) with the loss
    history and the device time per gradient evaluation (forward projection,
    loss, backward projection)."""
    shape = (y.shape[0],) + tuple(op.vol.shape_zyx) if y.dim() == 2 else tuple(op.vol.shape_zyx)
    if x0 is None:
        x0 = torch.ones(shape, dtype=y.dtype, device=y.device)
    theta = (x0.clamp_min(1e-6).expm1().clamp_min(1e-12).log()).detach().requires_grad_(True)
    opt = torch.optim.LBFGS([theta], lr=1.0, max_iter=steps, history_size=history, line_search_fn="strong_wolfe",
                            tolerance_grad=0.0, tolerance_change=0.0)
    losses, times = [], []
    stream = torch.cuda.current_stream(y.device)

    def closure():
        opt.zero_grad()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        x = torch.nn.functional.softplus(theta)
        loss = penalized_nll(x, y, op, beta, atten, bias)
        loss.backward()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
        losses.append(float(loss.detach()))
        return loss

    t0 = time.perf_counter()
    opt.step(closure)
    wall = time.perf_counter() - t0
    x = torch.nn.functional.softplus(theta).detach()
    return x, {"losses": losses, "gradient_ms": times, "evaluations": len(times), "wall_s": wall}

"""Reconstruction loops over the device operators (tensors stay on the GPU).

* ``fdk`` -- cosine/Parker weighting, ramp filter and weighted voxel-driven
  backprojection (mat_codes/filtering.m + backprojection.m as one call);
* ``sirt`` -- x <- x + lam * C A^T R (b - A x) with R, C the inverse row and
  column sums (the normalised form of nefct/functions/sart.py:29-39);
* ``cg`` -- conjugate gradients on A^T A x = A^T b (the normal equations that
  nefct/functions/conj_grad.py:76-101 iterates on), with its scalars kept on
  the device;
  both loops can run as one captured CUDA graph per iteration (``graph=True``):
  the first iteration runs eagerly, the second is recorded and the rest are
  replays, with no host synchronisation inside an iteration;
* ``motion_project`` -- the 4D forward of project_t.py:153-160 with the
  cpp/deform warp: per phase, warp the reference volume by that phase's
  displacement field and project the phase's views; differentiable in the
  reference volume and every field (the warped volumes are not stored: the
  backward of the warp needs only its inputs).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, ops

__all__ = ["fdk", "sirt", "cg", "motion_project", "sinusoid_field"]


def fdk(sino: torch.Tensor, geom: ops.ConeBeam, window: str = "ram-lak", parker: int = 0) -> torch.Tensor:
    return ops.fdk_backproject(ops.fdk_filter(sino, geom, window, parker), geom)


def _iterate(step, n_iter: int, graph: bool, callback, state) -> None:
    """Runs step() n_iter times; with graph=True the first call runs eagerly on
    a side stream (its allocations warm the caching allocator), the second is
    recorded into a CUDA graph and the remaining ones are replays of it."""
    if n_iter <= 0:
        return
    if not graph:
        for it in range(n_iter):
            step()
            if callback is not None:
                callback(it, state)
        return
    side = torch.cuda.Stream(device=state.device)
    side.wait_stream(torch.cuda.current_stream(state.device))
    with torch.cuda.stream(side):
        step()
    torch.cuda.current_stream(state.device).wait_stream(side)
    if callback is not None:
        callback(0, state)
    if n_iter == 1:
        return
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    for it in range(1, n_iter):
        g.replay()
        if callback is not None:
            callback(it, state)
    del g


def sirt(b: torch.Tensor, geom: ops.ConeBeam, n_iter: int, flags: int = _lib.LINE_INTEGRAL, x0=None,
         lam: float = 1.0, callback=None, graph: bool = False) -> torch.Tensor:
    ones_v = torch.ones(geom.vol_shape, device=b.device, dtype=b.dtype)
    ones_s = torch.ones(geom.sino_shape, device=b.device, dtype=b.dtype)
    rs = ops.cb_forward(ones_v, geom, flags)
    cs = ops.cb_backward(ones_s, geom, flags)
    R = torch.where(rs > 0, 1.0 / rs.clamp_min(1e-30), torch.zeros_like(rs))
    C = torch.where(cs > 0, 1.0 / cs.clamp_min(1e-30), torch.zeros_like(cs))
    del rs, cs, ones_v, ones_s
    x = torch.zeros(geom.vol_shape, device=b.device, dtype=b.dtype) if x0 is None else x0.clone()
    ax = torch.empty_like(b)
    atr = torch.empty_like(x)

    def step():
        ops.cb_forward(x, geom, flags, out=ax)
        ax.sub_(b).neg_().mul_(R)                 # R (b - A x)
        ops.cb_backward(ax, geom, flags, out=atr)
        x.addcmul_(atr, C, value=lam)

    _iterate(step, n_iter, graph, callback, x)
    return x


def cg(b: torch.Tensor, geom: ops.ConeBeam, n_iter: int, flags: int = _lib.LINE_INTEGRAL, x0=None,
       callback=None, graph: bool = False) -> torch.Tensor:
    """Conjugate gradients on A^T A x = A^T b; alpha and beta stay 0-dim
    device tensors, so an iteration never waits for the host.  Once the
    residual is exactly zero (a zero right-hand side, or exact
    convergence) both step sizes are 0 and the iterate stays put."""
    ax = torch.empty_like(b)
    aty = ops.cb_backward(b, geom, flags)
    x = torch.zeros(geom.vol_shape, device=b.device, dtype=b.dtype) if x0 is None else x0.clone()
    ata = torch.empty_like(x)

    def normal(v):                                # A^T A v into ata
        ops.cb_forward(v, geom, flags, out=ax)
        ops.cb_backward(ax, geom, flags, out=ata)
        return ata

    r = aty - normal(x)
    p = r.clone()

    def dot(u, v):                                # float32 products, float64 sum
        return (u * v).sum(dtype=torch.float64)

    rsold = dot(r, r)

    zero = torch.zeros((), dtype=torch.float64, device=b.device)

    def safe_div(num, den):                       # 0 where den is 0 (converged: r = 0 or p = 0)
        return torch.where(den > 0, num / torch.where(den > 0, den, torch.ones_like(den)), zero)

    def step():
        ap = normal(p)
        alpha = safe_div(rsold, dot(p, ap))
        x.add_(p * alpha.float())
        r.sub_(ap * alpha.float())
        rsnew = dot(r, r)
        p.mul_(safe_div(rsnew, rsold).float()).add_(r)
        rsold.copy_(rsnew)

    _iterate(step, n_iter, graph, callback, x)
    return x


def sinusoid_field(shape, amplitude: float, rng: np.random.Generator, terms: int = 4, device=None) -> list:
    """Three displacement components [nz, ny, nx] (voxels), each a sum of
    `terms` seeded low-frequency sinusoids scaled to max |m| = amplitude."""
    nz, ny, nx = shape
    z = torch.linspace(0, 1, nz, device=device, dtype=torch.float64).view(-1, 1, 1)
    y = torch.linspace(0, 1, ny, device=device, dtype=torch.float64).view(1, -1, 1)
    x = torch.linspace(0, 1, nx, device=device, dtype=torch.float64).view(1, 1, -1)
    out = []
    for _ in range(3):
        f = torch.zeros(shape, device=device, dtype=torch.float64)
        for _ in range(terms):
            kx, ky, kz = rng.integers(0, 3, 3)
            ph = rng.uniform(0, 2 * np.pi)
            a = rng.uniform(0.3, 1.0)
            f += a * torch.sin(2 * np.pi * (kx * x + ky * y + kz * z) + ph)
        f *= amplitude / float(f.abs().max().clamp_min(1e-12))
        out.append(f.float().contiguous())
    return out


def motion_project(ref: torch.Tensor, fields: list, geoms: list, flags: int = 0) -> list:
    """Per phase p: project(warp(ref, fields[p]), geoms[p]); differentiable."""
    return [ops.project(ops.warp(ref, *m), g, flags) for m, g in zip(fields, geoms)]

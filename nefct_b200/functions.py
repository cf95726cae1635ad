"""Drop-in operators with the reference's call signatures.

Mirrors nefct/functions/project.py:63-98 (Project3D),
back_project.py:244-277 (BackProject3D), project_t.py:112-163 (Project3DT),
back_project_t.py:332-374 (BackProject3DT), sart.py:21-39 (SART) and
conj_grad.py:67-101 (ConjGrad), and adds FDK (the MATLAB pipeline of
mat_codes/filtering.m + backprojection.m as one operator).

The TensorFlow ops are replaced by the sm_100a kernels of libnefct_b200.so.
``data`` may be numpy (copied to the current CUDA device and back, like the
reference's per-call numpy round trip) or a CUDA torch tensor (stays on the
device).  Geometry is passed in physical units; the kernels normalise to
voxel units themselves, so no ``unit_size`` rescaling of the result is
needed (the reference rescales because it hands voxel units to its ops).

Extra keyword ``mode`` (default keeps the reference's behaviour):
  Project3D:     'ref'  weights carry 1/L^2 as siddon_3d's forward does;
                 'line' plain line integrals.
  BackProject3D: 'ref'  siddon_3d's backproject_device semantics;
                 'transpose' the exact transpose of Project3D('ref');
                 'line' the exact transpose of Project3D('line').
"""
from __future__ import annotations

from typing import Callable

import numpy as np
import torch

from . import _lib, ops
from .base import nef_class
from .data import Image, Image3D, Image3DT, ProjectionSequence3D
from .geometry import ScannerConfig3D

__all__ = ["cone_beam", "Project3D", "BackProject3D", "Project3DT", "BackProject3DT", "FDK", "SART",
           "ConjGrad", "WarpDeformer"]

_FWD_FLAGS = {"ref": _lib.REF_FORWARD, "line": _lib.LINE_INTEGRAL}
_BP_FLAGS = {"ref": _lib.REF_BACKPROJECT, "transpose": _lib.REF_FORWARD, "line": _lib.LINE_INTEGRAL}


def cone_beam(config: ScannerConfig3D, shape, center, size, angles, offsets=None) -> ops.ConeBeam:
    """Kernel-convention geometry from the reference's python geometry.

    Python SID (source -> detector) is the kernel's SAD and python SAD
    (source -> axis) the kernel's SID (quirk Q12).  Detector offsets are
    physical (mm, or radians for a cylindrical detector's a axis), as in
    DetectorDirectAConfig.meshgrid."""
    da, db = config.detector_a.unit_size, config.detector_b.unit_size
    a_shift = 0.5 + float(config.detector_a.offset or 0.0) / da
    b_shift = 0.5 + float(config.detector_b.offset or 0.0) / db
    angles = np.asarray(angles, dtype=np.float32).reshape(-1)
    offs = None
    if offsets is not None:
        o = np.asarray(offsets, dtype=np.float32).reshape(-1)
        if o.size == 1 and angles.size > 1:
            o = np.full(angles.size, o[0], np.float32)
        if np.any(o != 0):
            offs = o
    return ops.ConeBeam(tuple(shape), angles, float(config.SAD), float(config.SID),
                        config.detector_a.number, da, config.detector_b.number, db, a_shift, b_shift,
                        tuple(float(c) for c in center), tuple(float(s) for s in size),
                        "flat" if config.is_flat else "cyl", offs)


def _device():
    if not torch.cuda.is_available():
        raise _lib.NefctError(_lib.ERR_INVALID, "no CUDA device: the projector runs on the GPU only")
    return torch.device("cuda", torch.cuda.current_device())


def _vol_in(data) -> tuple[torch.Tensor, bool]:
    """[nx, ny, nz] numpy/tensor -> contiguous [nz, ny, nx] float32 CUDA tensor."""
    if isinstance(data, torch.Tensor):
        t = data if data.is_cuda else data.to(_device())
        return t.permute(2, 1, 0).contiguous().float(), False
    a = np.ascontiguousarray(np.asarray(data, dtype=np.float32).transpose())
    return torch.from_numpy(a).to(_device(), non_blocking=False), True


def _sino_in(data) -> tuple[torch.Tensor, bool]:
    """[na, nb, nv] -> contiguous [nv, nb, na] float32 CUDA tensor."""
    return _vol_in(data)


def _out(t: torch.Tensor, as_numpy: bool):
    """[k, j, i] device tensor -> [i, j, k] numpy (or device tensor view)."""
    t = t.permute(2, 1, 0)
    if as_numpy:
        return np.ascontiguousarray(t.cpu().numpy())
    return t


@nef_class
class Project3D:
    config: ScannerConfig3D
    angles: list
    offsets: list
    mode: str = "ref"

    def __call__(self, image: Image) -> ProjectionSequence3D:
        offsets = self.offsets
        if offsets is None:
            offsets = np.zeros(len(self.angles), np.float32)
        geom = cone_beam(self.config, image.shape, image.center, image.size, self.angles, offsets)
        vol, as_np = _vol_in(image.data)
        sino = ops.cb_forward(vol, geom, _FWD_FLAGS[self.mode])
        return ProjectionSequence3D(_out(sino, as_np), self.config, self.angles, offsets)


@nef_class
class BackProject3D:
    config: ScannerConfig3D
    shape: list
    unit_size: float
    mode: str = "ref"

    def __call__(self, proj: ProjectionSequence3D) -> Image3D:
        size = [s * self.unit_size for s in self.shape]
        geom = cone_beam(self.config, self.shape, [0, 0, 0], size, proj.angles, proj.offsets)
        sino, as_np = _sino_in(proj.data)
        vol = ops.cb_backward(sino, geom, _BP_FLAGS[self.mode])
        return Image3D(_out(vol, as_np), [0, 0, 0], size)


@nef_class
class FDK:
    """Cone-beam FDK (flat detector): cosine (+ Parker) weighting and ramp
    filtering (mat_codes/filtering.m, ParkerWeight.m) then voxel-driven
    weighted backprojection (backprojection.m with pixel_3d's geometry)."""
    config: ScannerConfig3D
    shape: list
    unit_size: float
    filter: str = "ram-lak"
    parker: int = 0

    def __call__(self, proj: ProjectionSequence3D) -> Image3D:
        size = [s * self.unit_size for s in self.shape]
        geom = cone_beam(self.config, self.shape, [0, 0, 0], size, proj.angles, None)
        sino, as_np = _sino_in(proj.data)
        filt = ops.fdk_filter(sino, geom, self.filter, self.parker)
        vol = ops.fdk_backproject(filt, geom)
        return Image3D(_out(vol, as_np), [0, 0, 0], size)


def _groups(timestamps, n):
    ts = np.zeros(n) if timestamps is None else np.asarray(timestamps).reshape(-1)
    order = []
    for t in dict.fromkeys(ts.tolist()):
        order.append((t, np.nonzero(ts == t)[0]))
    return ts, order


@nef_class
class Project3DT:
    """Per-view deformed projection (project_t.py:112-163).  The reference
    deforms and projects one view at a time; views that share a timestamp
    see the same deformed image, so they are projected in one launch."""
    config: ScannerConfig3D
    angles: list
    offsets: list
    timestamps: list
    deformer: Callable
    mode: str = "ref"

    def __call__(self, image: Image3D) -> ProjectionSequence3D:
        angles = np.asarray(self.angles, np.float32).reshape(-1)
        nv = angles.size
        offsets = np.zeros(nv, np.float32) if self.offsets is None else np.asarray(self.offsets, np.float32)
        ts, groups = _groups(self.timestamps, nv)
        as_np = not isinstance(image.data, torch.Tensor)
        out = torch.empty((nv, self.config.detector_b.number, self.config.detector_a.number),
                          dtype=torch.float32, device=_device())
        for t, idx in groups:
            image_ = self.deformer(image, t)
            geom = cone_beam(self.config, image.shape, image.center, image.size, angles[idx], offsets[idx])
            vol, _ = _vol_in(image_.data)
            out[torch.as_tensor(idx, device=out.device)] = ops.cb_forward(vol, geom, _FWD_FLAGS[self.mode])
        return ProjectionSequence3D(_out(out, as_np), self.config, self.angles, offsets, ts)


@nef_class
class BackProject3DT:
    """Per-view backprojection followed by the deformer (back_project_t.py:
    332-374).  The deformer is linear in its image argument (a warp), so the
    views of one timestamp are backprojected together and deformed once."""
    config: ScannerConfig3D
    shape: list
    unit_size: float
    timestamps: list
    deformer: Callable
    mode: str = "ref"

    def __call__(self, proj: ProjectionSequence3D) -> Image3DT:
        size = [s * self.unit_size for s in self.shape]
        angles = np.asarray(proj.angles, np.float32).reshape(-1)
        nv = angles.size
        offsets = np.asarray(proj.offsets, np.float32).reshape(-1)
        if offsets.size != nv:
            offsets = np.full(nv, offsets[0] if offsets.size else 0.0, np.float32)
        _, groups = _groups(proj.timestamps, nv)
        sino, as_np = _sino_in(proj.data)
        acc = None
        for t, idx in groups:
            geom = cone_beam(self.config, self.shape, [0, 0, 0], size, angles[idx], offsets[idx])
            sub = sino[torch.as_tensor(idx, device=sino.device)].contiguous()
            b = ops.cb_backward(sub, geom, _BP_FLAGS[self.mode])
            d = self.deformer(b.permute(2, 1, 0), t, self.timestamps)
            d = d.data if hasattr(d, "data") else d
            acc = d if acc is None else acc + d
        if as_np:
            acc = acc.cpu().numpy()
        return Image3DT(acc, [0, 0, 0], size, self.timestamps)


@nef_class
class WarpDeformer:
    """Deformer built on the cpp/deform warp: ``fields`` maps a timestamp to
    (mx, my, mz) displacement volumes [nx, ny, nz] in voxels."""
    fields: dict

    def __call__(self, image, time, timestamps=None):
        data = image.data if hasattr(image, "data") else image
        f = self.fields.get(float(time))
        if f is None:
            return image
        vol, as_np = _vol_in(data)
        m = [_vol_in(c)[0] for c in f]
        out = _out(ops.warp_forward(vol, *m), as_np)
        return image.update(data=out) if hasattr(image, "data") else out


@nef_class
class SART:
    """x <- x + lambda * BP(p - A x) / emap (sart.py:29-39)."""
    n_iter: int
    lambda_: float
    emap: Image
    project: Callable
    back_project: Callable

    def __call__(self, projection: ProjectionSequence3D, x: Image = None) -> Image:
        if x is None:
            x = self.emap * 0
        em = self.emap.data
        for _ in range(self.n_iter):
            bp = self.back_project(projection - self.project(x))
            ratio = _div_no_nan(bp.data, em)
            x = x.update(data=x.data + ratio * self.lambda_)
        return x


def _div_no_nan(a, b):
    if isinstance(a, torch.Tensor):
        b = b if isinstance(b, torch.Tensor) else torch.as_tensor(b, device=a.device)
        return torch.where(b != 0, a / torch.where(b != 0, b, torch.ones_like(b)), torch.zeros_like(a))
    b = np.asarray(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(b != 0, a / np.where(b != 0, b, 1), 0).astype(np.float32)


@nef_class
class ConjGrad:
    """Conjugate gradients on BP(A x) = BP(p) (conj_grad.py:76-101).  The
    total-variation branch of the reference is not on the projector path."""
    n_iter: int
    project: Callable
    back_project: Callable
    total_vari: object = None
    invert_total_vari: object = None
    mu: float = 0.0

    def __call__(self, projection: ProjectionSequence3D, x: Image = None, d=None) -> Image:
        if self.total_vari is not None:
            raise NotImplementedError("the total-variation term is outside the projector path")
        b = self.back_project(projection)
        if x is None:
            x = b * 0
        A = lambda v: self.back_project(self.project(v))
        r = b - A(x)
        p = r
        dot = (lambda u, v: float((u * v).sum()))
        rsold = dot(r.data, r.data)
        for _ in range(self.n_iter):
            Ap = A(p)
            alpha = rsold / dot(p.data, Ap.data)
            x = x + p * alpha
            r = r - Ap * alpha
            rsnew = dot(r.data, r.data)
            p = r + p * (rsnew / rsold)
            rsold = rsnew
        return x

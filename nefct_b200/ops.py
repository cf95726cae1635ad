"""Torch-level operators over the C ABI (device tensors in, device tensors out).

Every op runs the sm_100a kernels of libnefct_b200.so on the tensors' CUDA
device and the current torch stream.  There is no CPU path: a CPU tensor is
an error.  Layouts are the reference's device layouts: volumes
[nz, ny, nx] (x fastest), sinograms [nv, nb, na].

Differentiable wrappers (torch.autograd.Function):

* ``project`` -- forward projector; its backward is the hand-written exact
  transpose (``cb_backward`` with the same flags);
* ``backproject`` -- the transpose; its backward is the forward;
* ``warp`` -- cpp/deform trilinear warp; backward gives the image adjoint
  and the displacement-field gradient.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import NefctError

__all__ = ["ConeBeam", "cb_forward", "cb_backward", "cb_count_intersections", "lor_forward",
           "lor_backward", "fdk_filter", "fdk_backproject", "warp_forward", "warp_adjoint",
           "warp_grad_dvf", "warp_invert", "project", "backproject", "warp", "DDGeometry", "dd_forward",
           "dd_backward", "dd_backproject", "dd_project", "parker_direction", "NefctError"]


@dataclass(eq=False)
class ConeBeam:
    """Circular cone-beam geometry in the kernel convention of the C ABI.

    shape is (nx, ny, nz); center/size give the volume box (size defaults to
    one unit per voxel).  src_iso is the source-to-axis distance (the
    reference kernel's ``SID``), src_det the source-to-detector distance (its
    ``SAD``).  Detector cell ia sits at a = (ia + a_shift)*da - na*da/2
    (radians for a cylindrical detector), row ib at b = (ib + b_shift)*db -
    nb*db/2.
    """
    shape: tuple
    angles: np.ndarray
    src_iso: float
    src_det: float
    na: int
    da: float
    nb: int
    db: float
    a_shift: float = 0.5
    b_shift: float = 0.5
    center: tuple = (0.0, 0.0, 0.0)
    size: tuple | None = None
    det_kind: str = "flat"
    z_offsets: np.ndarray | None = None

    def __post_init__(self):
        self.shape = tuple(int(s) for s in self.shape)
        self.angles = np.ascontiguousarray(np.asarray(self.angles, dtype=np.float32).reshape(-1))
        if self.z_offsets is not None:
            self.z_offsets = np.ascontiguousarray(np.asarray(self.z_offsets, dtype=np.float32).reshape(-1))
            if self.z_offsets.size != self.angles.size:
                raise ValueError("z_offsets must have one entry per view")
        if self.size is None:
            self.size = tuple(float(s) for s in self.shape)
        if self.det_kind not in ("flat", "cyl"):
            raise ValueError("det_kind must be 'flat' or 'cyl'")

    @property
    def nv(self) -> int:
        return int(self.angles.size)

    @property
    def vol_shape(self) -> tuple:
        nx, ny, nz = self.shape
        return (nz, ny, nx)

    @property
    def sino_shape(self) -> tuple:
        return (self.nv, self.nb, self.na)

    def grid(self) -> _lib.Grid:
        nx, ny, nz = self.shape
        return _lib.Grid(nx, ny, nz, *[float(c) for c in self.center], *[float(s) for s in self.size])

    def struct(self) -> _lib.CBGeom:
        g = _lib.CBGeom()
        g.grid = self.grid()
        g.nv = self.nv
        g.angles = self.angles.ctypes.data_as(C.POINTER(C.c_float))
        g.z_offsets = (self.z_offsets.ctypes.data_as(C.POINTER(C.c_float))
                       if self.z_offsets is not None else None)
        g.src_iso, g.src_det = float(self.src_iso), float(self.src_det)
        g.na, g.da, g.a_shift = int(self.na), float(self.da), float(self.a_shift)
        g.nb, g.db, g.b_shift = int(self.nb), float(self.db), float(self.b_shift)
        g.det_kind = _lib.DET_CYL if self.det_kind == "cyl" else _lib.DET_FLAT
        return g

    def subset(self, views) -> "ConeBeam":
        """The same scanner restricted to the given view indices."""
        idx = np.asarray(views)
        return ConeBeam(self.shape, self.angles[idx], self.src_iso, self.src_det, self.na, self.da,
                        self.nb, self.db, self.a_shift, self.b_shift, self.center, self.size,
                        self.det_kind, None if self.z_offsets is None else self.z_offsets[idx])


def _check_tensor(t: torch.Tensor, shape: tuple, name: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise NefctError(_lib.ERR_INVALID, f"{name} must be a CUDA tensor (there is no CPU path)")
    if t.dtype not in (torch.float32, torch.float64):
        raise NefctError(_lib.ERR_INVALID, f"{name} must be float32 or float64, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise NefctError(_lib.ERR_INVALID, f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise NefctError(_lib.ERR_INVALID, f"{name} must be contiguous")


def _stream(t: torch.Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _suffix(t: torch.Tensor) -> str:
    return "_f64" if t.dtype == torch.float64 else ""


def _workspace(geom: ConeBeam, flags: int, like: torch.Tensor):
    """Workspace from torch's caching allocator.  Its memory is reused only by
    work ordered after the current stream's, so dropping it right after the
    enqueue is safe."""
    g = geom.struct()
    n = _lib.load().nefct_cb_workspace_bytes(C.byref(g), flags) * (2 if like.dtype == torch.float64 else 1)
    if n == 0:
        return None, 0
    return torch.empty(n, dtype=torch.uint8, device=like.device), n


def cb_forward(vol: torch.Tensor, geom: ConeBeam, flags: int = _lib.REF_FORWARD,
               out: torch.Tensor | None = None) -> torch.Tensor:
    """Cone-beam forward projection [nz,ny,nx] -> [nv,nb,na]."""
    _check_tensor(vol, geom.vol_shape, "vol")
    if out is None:
        out = torch.empty(geom.sino_shape, dtype=vol.dtype, device=vol.device)
    else:
        _check_tensor(out, geom.sino_shape, "out")
    with torch.cuda.device(vol.device):
        g = geom.struct()
        ws, wn = _workspace(geom, flags, vol)
        _lib.call("nefct_cb_forward" + _suffix(vol), C.byref(g), vol.data_ptr(), out.data_ptr(), flags,
                  ws.data_ptr() if ws is not None else None, wn, _stream(vol))
    return out


def cb_backward(sino: torch.Tensor, geom: ConeBeam, flags: int = _lib.REF_FORWARD,
                out: torch.Tensor | None = None) -> torch.Tensor:
    """Backprojection [nv,nb,na] -> [nz,ny,nx].  With the forward's flags it
    is that forward's exact transpose; with REF_BACKPROJECT the reference's
    own backprojection."""
    _check_tensor(sino, geom.sino_shape, "sino")
    if out is None:
        out = torch.empty(geom.vol_shape, dtype=sino.dtype, device=sino.device)
    else:
        _check_tensor(out, geom.vol_shape, "out")
    with torch.cuda.device(sino.device):
        g = geom.struct()
        ws, wn = _workspace(geom, flags, sino)
        _lib.call("nefct_cb_backward" + _suffix(sino), C.byref(g), sino.data_ptr(), out.data_ptr(), flags,
                  ws.data_ptr() if ws is not None else None, wn, _stream(sino))
    return out


def cb_count_intersections(geom: ConeBeam, flags: int = _lib.REF_FORWARD, device="cuda") -> int:
    """Ray-voxel contributions of the forward walk (the throughput unit)."""
    cnt = torch.zeros(1, dtype=torch.int64, device=device)
    with torch.cuda.device(cnt.device):
        g = geom.struct()
        _lib.call("nefct_cb_count_intersections", C.byref(g), flags, cnt.data_ptr(), _stream(cnt))
    return int(cnt.item())


def _lor_grid(shape, center, size):
    nx, ny, nz = shape
    size = size if size is not None else (nx, ny, nz)
    return _lib.Grid(nx, ny, nz, *[float(c) for c in center], *[float(s) for s in size])


def _check_order(order, n, device):
    if order is None:
        return None
    if order.dtype != torch.int32 or order.dim() != 1 or order.shape[0] != n or order.device != device:
        raise NefctError(_lib.ERR_INVALID, "order must be an int32 permutation of the lines on their device")
    return order.contiguous()


def lor_order(lors: torch.Tensor, shape, center=(0.0, 0.0, 0.0), size=None) -> torch.Tensor:
    """Walk order for a large unsorted line list: an int32 permutation that
    groups nearly parallel neighbouring lines (pass it as ``order`` to
    lor_forward / lor_backward; compute it once per list)."""
    if lors.dim() != 2 or lors.shape[0] != 6:
        raise NefctError(_lib.ERR_INVALID, "lors must be [6, n]")
    _check_tensor(lors, tuple(lors.shape), "lors")
    n = lors.shape[1]
    keys = torch.empty(n, dtype=torch.int32, device=lors.device)
    g = _lor_grid(shape, center, size)
    with torch.cuda.device(lors.device):
        _lib.call("nefct_lor_order_keys", C.byref(g), lors.data_ptr(), n, keys.data_ptr(), _stream(lors))
    return torch.argsort(keys).to(torch.int32)


def lor_forward(lors: torch.Tensor, vol: torch.Tensor, shape, center=(0.0, 0.0, 0.0), size=None,
                flags: int = _lib.LOR_REF_FORWARD, order: torch.Tensor | None = None) -> torch.Tensor:
    """cpp/siddon Projection: lors [6, n] -> line integrals [n] (optionally
    walked in ``order`` from lor_order; results keep the lines' order)."""
    nx, ny, nz = shape
    _check_tensor(vol, (nz, ny, nx), "vol")
    if lors.dim() != 2 or lors.shape[0] != 6:
        raise NefctError(_lib.ERR_INVALID, "lors must be [6, n]")
    _check_tensor(lors, tuple(lors.shape), "lors")
    n = lors.shape[1]
    order = _check_order(order, n, lors.device)
    out = torch.empty(n, dtype=torch.float32, device=vol.device)
    g = _lor_grid(shape, center, size)
    with torch.cuda.device(vol.device):
        if order is None:
            _lib.call("nefct_lor_forward", C.byref(g), lors.data_ptr(), n, vol.data_ptr(), out.data_ptr(), flags,
                      _stream(vol))
        else:
            _lib.call("nefct_lor_forward_ordered", C.byref(g), lors.data_ptr(), n, order.data_ptr(),
                      vol.data_ptr(), out.data_ptr(), flags, _stream(vol))
    return out


def lor_backward(lors: torch.Tensor, vals: torch.Tensor, shape, center=(0.0, 0.0, 0.0), size=None,
                 flags: int = _lib.LOR_REF_BACKPROJECT, order: torch.Tensor | None = None) -> torch.Tensor:
    """cpp/siddon Backprojection: values [n] along lors [6, n] -> volume."""
    nx, ny, nz = shape
    if lors.dim() != 2 or lors.shape[0] != 6:
        raise NefctError(_lib.ERR_INVALID, "lors must be [6, n]")
    _check_tensor(lors, tuple(lors.shape), "lors")
    _check_tensor(vals, (lors.shape[1],), "vals")
    n = lors.shape[1]
    order = _check_order(order, n, lors.device)
    out = torch.empty((nz, ny, nx), dtype=torch.float32, device=vals.device)
    g = _lor_grid(shape, center, size)
    with torch.cuda.device(vals.device):
        if order is None:
            _lib.call("nefct_lor_backward", C.byref(g), lors.data_ptr(), n, vals.data_ptr(), out.data_ptr(),
                      flags, _stream(vals))
        else:
            _lib.call("nefct_lor_backward_ordered", C.byref(g), lors.data_ptr(), n, order.data_ptr(),
                      vals.data_ptr(), out.data_ptr(), flags, _stream(vals))
    return out


def fdk_filter(sino: torch.Tensor, geom: ConeBeam, window: str | int = "ram-lak", parker: int = 0) -> torch.Tensor:
    """Cosine (+ Parker) weighting and ramp filtering (mat_codes/filtering.m)."""
    _check_tensor(sino, geom.sino_shape, "sino")
    if sino.dtype != torch.float32:
        raise NefctError(_lib.ERR_INVALID, "fdk_filter is float32")
    w = _lib.WINDOWS[window.lower()] if isinstance(window, str) else int(window)
    out = torch.empty_like(sino)
    with torch.cuda.device(sino.device):
        g = geom.struct()
        _lib.call("nefct_fdk_filter", C.byref(g), sino.data_ptr(), out.data_ptr(), w, int(parker), _stream(sino))
    return out


def parker_direction(geom: ConeBeam) -> int:
    """ParkerWeight.m's ``dir`` for this scan: +1 when the view angles
    increase, -1 when they decrease.

    The ray through detector coordinate a at view angle phi points along
    phi + g, g = atan(a / src_det) (a grows counter-clockwise: the detector
    offset is along (-sin phi, cos phi)), so its conjugate ray is measured at
    view phi + pi + 2 g with fan angle -g.  ParkerWeight.m's
    pweight = beta - fanang + dir * g (degrees, beta = view index * dang)
    moves by exactly 180 between a ray and its conjugate -- so that its sin^2
    and cos^2 ramps add to one over every redundant pair -- only for
    dir = +1 when beta grows with the angle; a scan that turns the other way
    walks beta backwards and needs dir = -1."""
    a = np.asarray(geom.angles, np.float64)
    if a.size < 2 or a[1] == a[0]:
        raise NefctError(_lib.ERR_INVALID, "Parker weighting needs at least two distinct view angles")
    return 1 if a[1] > a[0] else -1


def fdk_backproject(filtered: torch.Tensor, geom: ConeBeam, weight: bool = True) -> torch.Tensor:
    """Voxel-driven bilinear backprojection (pixel_3d semantics) with the FDK
    distance weight (backprojection.m) unless weight=False."""
    _check_tensor(filtered, geom.sino_shape, "filtered")
    if filtered.dtype != torch.float32:
        raise NefctError(_lib.ERR_INVALID, "fdk_backproject is float32")
    out = torch.empty(geom.vol_shape, dtype=torch.float32, device=filtered.device)
    with torch.cuda.device(filtered.device):
        g = geom.struct()
        # tap-quad workspace (one chunk of views) from the caching allocator
        wn = _lib.load().nefct_fdk_workspace_bytes(C.byref(g))
        ws = torch.empty(wn, dtype=torch.uint8, device=filtered.device)
        _lib.call("nefct_fdk_backproject_ws", C.byref(g), filtered.data_ptr(), out.data_ptr(),
                  0 if weight else _lib.FDK_NO_WEIGHT, ws.data_ptr(), wn, _stream(filtered))
    return out


def _check_warp(img, *others):
    _check_tensor(img, tuple(img.shape), "img")
    if img.dim() != 3:
        raise NefctError(_lib.ERR_INVALID, "warp volumes are [nz, ny, nx]")
    for t in others:
        _check_tensor(t, tuple(img.shape), "displacement/gradient")
        if t.dtype != img.dtype:
            raise NefctError(_lib.ERR_INVALID, "warp inputs must share one dtype")


def warp_forward(img, mx, my, mz) -> torch.Tensor:
    """cpp/deform Deform: out[i] = trilinear(img, i + m[i])."""
    _check_warp(img, mx, my, mz)
    nz, ny, nx = img.shape
    out = torch.empty_like(img)
    with torch.cuda.device(img.device):
        _lib.call("nefct_warp_forward" + _suffix(img), img.data_ptr(), mx.data_ptr(), my.data_ptr(),
                  mz.data_ptr(), nx, ny, nz, out.data_ptr(), _stream(img))
    return out


def warp_adjoint(gout, mx, my, mz) -> torch.Tensor:
    _check_warp(gout, mx, my, mz)
    nz, ny, nx = gout.shape
    out = torch.empty_like(gout)
    with torch.cuda.device(gout.device):
        _lib.call("nefct_warp_adjoint" + _suffix(gout), gout.data_ptr(), mx.data_ptr(), my.data_ptr(),
                  mz.data_ptr(), nx, ny, nz, out.data_ptr(), _stream(gout))
    return out


def warp_grad_dvf(img, mx, my, mz, gout):
    _check_warp(img, mx, my, mz, gout)
    nz, ny, nx = img.shape
    gx, gy, gz = torch.empty_like(img), torch.empty_like(img), torch.empty_like(img)
    with torch.cuda.device(img.device):
        _lib.call("nefct_warp_grad_dvf" + _suffix(img), img.data_ptr(), mx.data_ptr(), my.data_ptr(),
                  mz.data_ptr(), gout.data_ptr(), nx, ny, nz, gx.data_ptr(), gy.data_ptr(), gz.data_ptr(),
                  _stream(img))
    return gx, gy, gz


def warp_invert(mx, my, mz, iters: int = 30):
    """Inverse displacement field (DeformInvert, deform_tex.cu.cc:78-99)."""
    _check_warp(mx, my, mz)
    if mx.dtype != torch.float32:
        raise NefctError(_lib.ERR_INVALID, "warp_invert is float32")
    nz, ny, nx = mx.shape
    ix, iy, iz = torch.empty_like(mx), torch.empty_like(mx), torch.empty_like(mx)
    with torch.cuda.device(mx.device):
        _lib.call("nefct_warp_invert", mx.data_ptr(), my.data_ptr(), mz.data_ptr(), nx, ny, nz, int(iters),
                  ix.data_ptr(), iy.data_ptr(), iz.data_ptr(), _stream(mx))
    return ix, iy, iz


class DDGeometry:
    """Geometry of the distance-driven pair (dist_3d_back_fdk.cu.cc's
    conventions): voxel units with the grid centred on the rotation axis;
    shape (nx, ny, nz); src_iso = source-axis (the reference's SAD), src_det
    = source-detector (its SID); bin ia at (ia + 0.5) * da + a_offset -
    na * da / 2 (radians for a cylindrical detector), rows likewise; per-view
    z offsets (None = 0)."""

    def __init__(self, shape, angles, src_iso, src_det, na, da, nb, db, a_offset=0.0, b_offset=0.0,
                 det_kind="flat", z_offsets=None):
        self.shape = tuple(int(v) for v in shape)
        self.angles = np.ascontiguousarray(np.asarray(angles, np.float32).reshape(-1))
        self.z_offsets = None if z_offsets is None else np.ascontiguousarray(
            np.asarray(z_offsets, np.float32).reshape(-1))
        if self.z_offsets is not None and self.z_offsets.size != self.angles.size:
            raise NefctError(_lib.ERR_INVALID, f"{self.z_offsets.size} z offsets for {self.angles.size} views")
        self.src_iso, self.src_det = float(src_iso), float(src_det)
        self.na, self.da, self.nb, self.db = int(na), float(da), int(nb), float(db)
        self.a_offset, self.b_offset = float(a_offset), float(b_offset)
        self.det_kind = det_kind

    @property
    def nv(self) -> int:
        return int(self.angles.size)

    @property
    def vol_shape(self) -> tuple:
        nx, ny, nz = self.shape
        return (nz, ny, nx)

    @property
    def proj_shape(self) -> tuple:
        return (self.nv, self.nb, self.na)

    def struct(self) -> _lib.DDGeom:
        nx, ny, nz = self.shape
        return _lib.DDGeom(nx, ny, nz, self.nv, self.angles.ctypes.data_as(C.POINTER(C.c_float)),
                           self.z_offsets.ctypes.data_as(C.POINTER(C.c_float)) if self.z_offsets is not None
                           else None, self.src_iso, self.src_det, self.na, self.da, self.a_offset, self.nb, self.db,
                           self.b_offset, _lib.DET_CYL if self.det_kind == "cyl" else _lib.DET_FLAT)


def _dd_call(name: str, src: torch.Tensor, geom: DDGeometry, flags: int, out_shape: tuple) -> torch.Tensor:
    if not isinstance(src, torch.Tensor) or not src.is_cuda:
        raise NefctError(_lib.ERR_INVALID, f"{name} needs a CUDA tensor (there is no CPU path)")
    if src.dtype not in (torch.float32, torch.float64):
        raise NefctError(_lib.ERR_INVALID, f"{name} takes float32 or float64, got {src.dtype}")
    src = src.contiguous()
    out = torch.empty(out_shape, dtype=src.dtype, device=src.device)
    g = geom.struct()
    with torch.cuda.device(src.device):
        if src.dtype == torch.float64:
            _lib.call(f"nefct_dd_{name}_f64", C.byref(g), src.data_ptr(), out.data_ptr(), flags, _stream(src))
        else:
            wn = _lib.load().nefct_dd_workspace_bytes(C.byref(g))
            ws = torch.empty(wn, dtype=torch.uint8, device=src.device)
            _lib.call(f"nefct_dd_{name}", C.byref(g), src.data_ptr(), out.data_ptr(), flags, ws.data_ptr(), wn,
                      _stream(src))
    return out


def dd_forward(vol: torch.Tensor, geom: DDGeometry, flags: int = 0) -> torch.Tensor:
    """Distance-driven forward projection [nz][ny][nx] -> [nv][nb][na]: the
    exact transpose of dd_backward with the same flags (flags 0: with the FDK
    weight, the transpose of the reference's FDK backprojection;
    FDK_NO_WEIGHT: footprint-weighted line integrals)."""
    _check_tensor(vol, geom.vol_shape, "vol")
    return _dd_call("forward", vol, geom, flags, geom.proj_shape)


def dd_backward(proj: torch.Tensor, geom: DDGeometry, flags: int = 0) -> torch.Tensor:
    """Distance-driven backprojection [nv][nb][na] -> [nz][ny][nx] (flags 0:
    dist_3d_back_fdk's FDK-weighted backprojection)."""
    _check_tensor(proj, geom.proj_shape, "proj")
    return _dd_call("backward", proj, geom, flags, geom.vol_shape)


def dd_backproject(proj, shape, angles, src_iso: float, src_det: float, da: float, db: float,
                   a_offset: float = 0.0, b_offset: float = 0.0, det_kind: str = "flat", z_offsets=None):
    """Distance-driven FDK-weighted backprojection (back_project_{flat,cyli}_fdk_gpu,
    nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:257-298).

    proj: float32 CUDA tensor [nv][nb][na]; shape (nx, ny, nz); geometry in
    voxel units with the grid centred on the axis; src_iso = source-axis
    (the reference's SAD), src_det = source-detector (its SID); bin ia sits at
    (ia + 0.5) * da + a_offset - na * da / 2.  Returns [nz][ny][nx]."""
    if not isinstance(proj, torch.Tensor) or not proj.is_cuda:
        raise NefctError(_lib.ERR_INVALID, "dd_backproject needs a CUDA tensor (there is no CPU path)")
    if proj.dtype != torch.float32 or proj.dim() != 3:
        raise NefctError(_lib.ERR_INVALID, "proj must be float32 [nv][nb][na]")
    proj = proj.contiguous()
    nv, nb, na = proj.shape
    geom = DDGeometry(shape, angles, src_iso, src_det, na, da, nb, db, a_offset, b_offset, det_kind, z_offsets)
    if geom.nv != nv:
        raise NefctError(_lib.ERR_INVALID, f"{geom.nv} angles for {nv} views")
    out = torch.empty(geom.vol_shape, dtype=torch.float32, device=proj.device)
    g = geom.struct()
    wn = _lib.load().nefct_dd_workspace_bytes(C.byref(g))
    ws = torch.empty(wn, dtype=torch.uint8, device=proj.device)
    with torch.cuda.device(proj.device):
        _lib.call("nefct_dd_backproject", C.byref(g), proj.data_ptr(), out.data_ptr(), ws.data_ptr(), wn,
                  _stream(proj))
    return out


# ---------------- autograd ----------------

class _Project(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol, geom, flags):
        ctx.geom, ctx.flags = geom, flags
        return cb_forward(vol.contiguous(), geom, flags)

    @staticmethod
    def backward(ctx, g):
        return cb_backward(g.contiguous(), ctx.geom, ctx.flags), None, None


class _Backproject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sino, geom, flags):
        ctx.geom, ctx.flags = geom, flags
        return cb_backward(sino.contiguous(), geom, flags)

    @staticmethod
    def backward(ctx, g):
        return cb_forward(g.contiguous(), ctx.geom, ctx.flags), None, None


class _Warp(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img, mx, my, mz):
        img, mx, my, mz = (t.contiguous() for t in (img, mx, my, mz))
        # only the inputs are saved; the warped volume is recomputed by nobody:
        # neither derivative needs it
        ctx.save_for_backward(img, mx, my, mz)
        return warp_forward(img, mx, my, mz)

    @staticmethod
    def backward(ctx, g):
        img, mx, my, mz = ctx.saved_tensors
        g = g.contiguous()
        gi = warp_adjoint(g, mx, my, mz) if ctx.needs_input_grad[0] else None
        gx = gy = gz = None
        if any(ctx.needs_input_grad[1:]):
            gx, gy, gz = warp_grad_dvf(img, mx, my, mz, g)
        return gi, gx, gy, gz


class _DDProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol, geom, flags):
        ctx.geom, ctx.flags = geom, flags
        return dd_forward(vol.contiguous(), geom, flags)

    @staticmethod
    def backward(ctx, g):
        return dd_backward(g.contiguous(), ctx.geom, ctx.flags), None, None


def dd_project(vol: torch.Tensor, geom: DDGeometry, flags: int = 0) -> torch.Tensor:
    """Differentiable distance-driven forward projection (backward = the
    hand-written exact transpose, dd_backward with the same flags)."""
    return _DDProject.apply(vol, geom, flags)


def project(vol: torch.Tensor, geom: ConeBeam, flags: int = _lib.REF_FORWARD) -> torch.Tensor:
    """Differentiable forward projection; backward = exact transpose."""
    return _Project.apply(vol, geom, flags)


def backproject(sino: torch.Tensor, geom: ConeBeam, flags: int = _lib.REF_FORWARD) -> torch.Tensor:
    """Differentiable exact transpose of ``project`` with the same flags."""
    return _Backproject.apply(sino, geom, flags)


def warp(img, mx, my, mz) -> torch.Tensor:
    """Differentiable cpp/deform warp (gradients w.r.t. image and field)."""
    return _Warp.apply(img, mx, my, mz)

"""TEST INFRASTRUCTURE: CPU oracles of the projector hot path.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It is the checker, never the product
path: ``nefct_b200`` does not import it and has no CPU fallback.

Two layers:

* ``liboracle.so`` -- a plain-C restatement of the reference's slab-split
  Siddon walk, its cone-beam and LOR drivers, the pixel_3d voxel-driven
  backprojection, the cpp/deform warp, and an exact FP64 Siddon
  (``nefct_oracle.c``, file:line citations inside).
* ``_ref/libnefct_ref.so`` -- the reference's own device routines compiled as
  host C++ from the reference sources (``ref_shim.cc``, ``Makefile``).  Used to
  pin the restatement and as the "reference" CPU baseline.  Present only when
  it was built (it needs the reference checkout at build time).
* ``_ref/libnefct_ref_gpu.so`` -- the reference's siddon_3d flat-detector
  pair, pixel_3d backprojection, cpp/siddon LOR pair, distance-driven FDK
  backprojection and cpp/deform warp with their host launchers, compiled by nvcc for the GPU (``ref_gpu_shim.cu``): the
  reference's own CUDA path, run on device buffers for parity and for timing
  beside the library.
* ``_ref/libnefct_ref_tex.so`` -- the reference's texture-based DVF inversion
  (``deform_tex.cu.cc``) compiled by nvcc for the GPU (``ref_tex_shim.cu``):
  hardware texture filtering has no host form, so this one checker runs on
  the GPU, on device buffers.

The FDK filter restatement of the MATLAB code lives in ``oracle.fdk``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libnefct_ref.so")
_REF_TEX = os.path.join(HERE, "_ref", "libnefct_ref_tex.so")
_REF_GPU = os.path.join(HERE, "_ref", "libnefct_ref_gpu.so")

TIE_GE, SKIP_SHORT, INV_L2, Q5_TRIPLE_L = 1, 2, 4, 8
CB_FWD = TIE_GE | INV_L2
CB_BP = SKIP_SHORT
LOR_FWD = SKIP_SHORT | INV_L2 | Q5_TRIPLE_L
LOR_BP = SKIP_SHORT


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float),
                ("sx", C.c_float), ("sy", C.c_float), ("sz", C.c_float)]


def build(ref: str | None = None) -> None:
    """Run oracle/Makefile: the C restatement, plus oracle/_ref when a
    reference checkout is named (``ref``, else the NEFCT_REF environment
    variable)."""
    env = dict(os.environ)
    if ref:
        env["NEFCT_REF"] = ref
    subprocess.run(["make", "-s", "-C", HERE], check=True, env=env)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
    return _lib


def have_ref() -> bool:
    return os.path.exists(_REF)


def have_ref_tex() -> bool:
    return os.path.exists(_REF_TEX)


def have_ref_gpu() -> bool:
    return os.path.exists(_REF_GPU)


_ref_gpu = None


def _ref_gpu_lib():
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(_REF_GPU):
            raise FileNotFoundError("oracle/_ref/libnefct_ref_gpu.so was not built")
        _ref_gpu = C.CDLL(_REF_GPU)
        args = ([C.c_void_p] + [C.c_int] * 3 + [C.c_float] * 6 + [C.c_void_p] + [C.c_int] * 3 + [C.c_float] * 6
                + [C.c_void_p])
        for name in ("ref_gpu_project_flat", "ref_gpu_backproject_flat", "ref_gpu_pixel_backproject_flat"):
            fn = getattr(_ref_gpu, name)
            fn.restype = C.c_int
            fn.argtypes = args
        _ref_gpu.ref_gpu_dd_backproject_flat.restype = C.c_int
        _ref_gpu.ref_gpu_dd_backproject_flat.argtypes = ([C.c_void_p] + [C.c_int] * 3 + [C.c_void_p] * 2
                                                         + [C.c_int] + [C.c_float] * 4 + [C.c_int]
                                                         + [C.c_float] * 2 + [C.c_int] + [C.c_void_p])
        _ref_gpu.ref_gpu_deform.restype = C.c_int
        _ref_gpu.ref_gpu_deform.argtypes = [C.c_void_p] * 4 + [C.c_int] * 3 + [C.c_void_p]
        lor_args = [C.c_void_p] + [C.c_int] * 4 + [C.c_float] * 6 + [C.c_void_p] * 2
        for name in ("ref_gpu_lor_forward", "ref_gpu_lor_backward"):
            fn = getattr(_ref_gpu, name)
            fn.restype = C.c_int
            fn.argtypes = lor_args
    return _ref_gpu


def _check_gpu(err, what):
    if err:
        raise RuntimeError(f"reference CUDA {what} failed: CUDA error {err}")


def ref_gpu_pixel_backproject(sino, shape, corner, size, angles, SID, SAD, na, da, ai, nb, db, bi):
    """The reference's pixel_3d BackProjectFlatKernel through backproject_flat
    (pixel.cu.cc:98-175) on the GPU.  sino: float32 CUDA tensor
    [nv][nb][na]; shape (nx, ny, nz), corner = the grid's low corner (Q10),
    size in mm; returns the volume [nz][ny][nx].  Synchronises."""
    import torch
    lib_ = _ref_gpu_lib()
    assert sino.is_cuda and sino.dtype == torch.float32 and sino.is_contiguous()
    nx, ny, nz = shape
    out = torch.zeros((nz, ny, nx), dtype=torch.float32, device=sino.device)
    _check_gpu(lib_.ref_gpu_pixel_backproject_flat(sino.data_ptr(), nx, ny, nz, *corner, *size,
                                                  angles.contiguous().data_ptr(), na, nb, int(angles.numel()),
                                                  SID, SAD, da, ai, db, bi, out.data_ptr()),
               "pixel_3d backprojection")
    return out


def ref_gpu_dd_backproject(proj, shape, angles, offsets, SID, SAD, na, da, ai, nb, db, bi):
    """The reference's distance-driven back_project_fdk_kernel through
    back_project_flat_fdk_gpu (dist_3d_back_fdk.cu.cc:17-276) on the GPU, in
    its naming (SID source-detector, SAD source-axis, voxel units).  proj:
    float32 CUDA tensor [nv][nb][na]; angles, offsets: float32 CUDA tensors
    [nv]; returns the volume [nz][ny][nx] (zeroed, then added into).
    Synchronises."""
    import torch
    lib_ = _ref_gpu_lib()
    assert proj.is_cuda and proj.dtype == torch.float32 and proj.is_contiguous()
    nx, ny, nz = shape
    out = torch.zeros((nz, ny, nx), dtype=torch.float32, device=proj.device)
    _check_gpu(lib_.ref_gpu_dd_backproject_flat(proj.data_ptr(), nx, ny, nz, offsets.contiguous().data_ptr(),
                                                angles.contiguous().data_ptr(), int(angles.numel()), SID, SAD,
                                                da, ai, na, db, bi, nb, out.data_ptr()),
               "distance-driven backprojection")
    return out


def ref_gpu_deform(img, mx, my, mz):
    """The reference's cpp/deform DeformKernel through deform()
    (deform.cu.cc:14-46, 112-126) on the GPU: float32 CUDA tensors
    [nz][ny][nx]; returns the warped image (zero where the reference writes
    nothing, Q13).  Synchronises."""
    import torch
    lib_ = _ref_gpu_lib()
    ts = [t.contiguous() for t in (img, mx, my, mz)]
    for t in ts:
        assert t.is_cuda and t.dtype == torch.float32 and t.shape == ts[0].shape
    nz, ny, nx = ts[0].shape
    out = torch.zeros_like(ts[0])
    _check_gpu(lib_.ref_gpu_deform(*[t.data_ptr() for t in ts], nx, ny, nz, out.data_ptr()), "deform")
    return out


def ref_gpu_lor(forward: bool, lors, shape, center, size, x):
    """The reference's cpp/siddon ProjectKernel / BackProjectKernel through
    projection / backprojection (siddon_gpu.cu.cc:652-747), launched as the
    reference launches them (32 CTAs of 1024 threads).  lors: float32 CUDA
    tensor [6][n]; x: the volume [nz][ny][nx] (forward) or the line values [n]
    (backprojection).  Outputs are zeroed first (the reference leaves skipped
    lines unwritten, Q4, and accumulates into an unzeroed volume, Q6).
    Synchronises."""
    import torch
    lib_ = _ref_gpu_lib()
    assert lors.is_cuda and lors.dtype == torch.float32 and lors.is_contiguous() and lors.shape[0] == 6
    n = int(lors.shape[1])
    nx, ny, nz = shape
    if forward:
        out = torch.zeros(n, dtype=torch.float32, device=lors.device)
        err = lib_.ref_gpu_lor_forward(lors.data_ptr(), n, nx, ny, nz, *center, *size, x.contiguous().data_ptr(),
                                       out.data_ptr())
    else:
        out = torch.zeros((nz, ny, nx), dtype=torch.float32, device=lors.device)
        err = lib_.ref_gpu_lor_backward(lors.data_ptr(), n, nx, ny, nz, *center, *size, x.contiguous().data_ptr(),
                                        out.data_ptr())
    _check_gpu(err, "LOR " + ("forward" if forward else "backprojection"))
    return out


def ref_gpu_cb(forward: bool, g: Grid, x, angles, SID, SAD, na, da, ai, nb, db, bi, out=None):
    """The reference's own CUDA cone-beam pair (flat detector) on the GPU:
    ProjectFlatKernel through project_flat (siddon.cu.cc:323-356, 392-420),
    or BackProjectFlatKernel through backproject_flat (:766-832, 834-862),
    launched as the reference launches them (16 x 16 x 4 threads, legacy
    default stream).  x: contiguous float32 CUDA tensor, the volume [nz][ny][nx]
    (forward) or the sinogram [nv][nb][na] (backprojection); angles: float32
    CUDA tensor [nv].  The backprojection accumulates into ``out`` (zeroed
    here when not given), as the reference's atomics do.  Synchronises."""
    import torch
    lib_ = _ref_gpu_lib()
    assert x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
    nv = int(angles.numel())
    if out is None:
        shape = (nv, nb, na) if forward else (g.nz, g.ny, g.nx)
        out = torch.zeros(shape, dtype=torch.float32, device=x.device)
    fn = lib_.ref_gpu_project_flat if forward else lib_.ref_gpu_backproject_flat
    err = fn(x.data_ptr(), g.nx, g.ny, g.nz, g.cx, g.cy, g.cz, g.sx, g.sy, g.sz,
             angles.contiguous().data_ptr(), na, nb, nv, SID, SAD, da, ai, db, bi, out.data_ptr())
    _check_gpu(err, "forward" if forward else "backprojection")
    return out


_ref_tex = None


def ref_tex_invert(mx, my, mz):
    """The reference's DeformInvertKernel (deform_tex.cu.cc:78-99, 30
    Gauss-Seidel passes over linear-filtered, clamp-addressed textures) run
    through its host function invert() (:102-168) on the GPU.  mx, my, mz:
    contiguous float32 CUDA tensors [nz][ny][nx]; returns the inverse field's
    three components as new CUDA tensors.  Synchronises the device."""
    import torch
    global _ref_tex
    if _ref_tex is None:
        if not os.path.exists(_REF_TEX):
            raise FileNotFoundError("oracle/_ref/libnefct_ref_tex.so was not built")
        _ref_tex = C.CDLL(_REF_TEX)
        _ref_tex.ref_tex_invert.restype = C.c_int
        _ref_tex.ref_tex_invert.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [C.c_void_p] * 3
    ms = [m.contiguous() for m in (mx, my, mz)]
    for m in ms:
        assert m.is_cuda and m.dtype == torch.float32 and m.dim() == 3
    nz, ny, nx = ms[0].shape
    out = [torch.empty_like(ms[0]) for _ in range(3)]
    torch.cuda.synchronize()
    err = _ref_tex.ref_tex_invert(*[m.data_ptr() for m in ms], nx, ny, nz, *[o.data_ptr() for o in out])
    if err:
        raise RuntimeError(f"reference texture inversion failed: CUDA error {err}")
    return out


def ref_threads() -> int:
    """OpenMP threads the reference build runs on (OMP_NUM_THREADS, else
    every host core)."""
    return int(ref().ref_max_threads())


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise FileNotFoundError("oracle/_ref/libnefct_ref.so was not built")
        _ref = C.CDLL(_REF)
    return _ref


def _p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def grid(shape, center=(0.0, 0.0, 0.0), size=None) -> Grid:
    """shape is (nx, ny, nz); the volume array is [nz][ny][nx] (x fastest)."""
    nx, ny, nz = shape
    if size is None:
        size = (float(nx), float(ny), float(nz))
    return Grid(nx, ny, nz, *[float(c) for c in center], *[float(s) for s in size])


def trig(angles, use_cosf: bool) -> tuple[np.ndarray, np.ndarray]:
    a = _f32(angles)
    cs = np.empty_like(a)
    sn = np.empty_like(a)
    L = lib()
    L.or_trig_f32(_p(a), C.c_int(a.size), C.c_int(int(use_cosf)), _p(cs), _p(sn))
    return cs, sn


def cb_forward(g: Grid, vol, angles, src_iso, src_det, na, da, ai, nb, db, bi, *, cyl=False,
               flags=CB_FWD, off=None, use_cosf=False, f64=False):
    """Sinogram [nv][nb][na] of vol [nz][ny][nx]; returns (sino, intersections)."""
    L = lib()
    nv = len(angles)
    if f64:
        a = _f64(angles)
        cs, sn = np.cos(a), np.sin(a)
        v = _f64(vol)
        out = np.zeros((nv, nb, na), np.float64)
        fn, cv, conv = L.or_cb_forward_f64, C.c_double, _f64
    else:
        cs, sn = trig(angles, use_cosf)
        v = _f32(vol)
        out = np.zeros((nv, nb, na), np.float32)
        fn, cv, conv = L.or_cb_forward_f32, C.c_float, _f32
    fn.restype = C.c_longlong
    o = None if off is None else conv(off)
    cnt = fn(C.byref(g), _p(v), _p(conv(cs)), _p(conv(sn)), _p(o), C.c_int(nv), cv(src_iso),
             cv(src_det), C.c_int(na), cv(da), cv(ai), C.c_int(nb), cv(db), cv(bi),
             C.c_int(int(cyl)), C.c_uint(flags), _p(out))
    return out, int(cnt)


def cb_backward(g: Grid, sino, angles, src_iso, src_det, na, da, ai, nb, db, bi, *, cyl=False,
                flags=CB_BP, q8=False, off=None, use_cosf=False, f64=False):
    """Scatter a [nv][nb][na] sinogram into a new [nz][ny][nx] volume."""
    L = lib()
    nv = len(angles)
    shape = (g.nz, g.ny, g.nx)
    if f64:
        a = _f64(angles)
        cs, sn = np.cos(a), np.sin(a)
        s = _f64(sino)
        out = np.zeros(shape, np.float64)
        fn, cv, conv = L.or_cb_backward_f64, C.c_double, _f64
    else:
        cs, sn = trig(angles, use_cosf)
        s = _f32(sino)
        out = np.zeros(shape, np.float32)
        fn, cv, conv = L.or_cb_backward_f32, C.c_float, _f32
    o = None if off is None else conv(off)
    fn(C.byref(g), _p(s), _p(conv(cs)), _p(conv(sn)), _p(o), C.c_int(nv), cv(src_iso), cv(src_det),
       C.c_int(na), cv(da), cv(ai), C.c_int(nb), cv(db), cv(bi), C.c_int(int(cyl)),
       C.c_uint(flags), C.c_int(int(q8)), _p(out))
    return out


def cb_exact(g: Grid, vol, angles, src_iso, src_det, na, da, ai, nb, db, bi, *, cyl=False,
             inv_l2=True, off=None):
    """Exact FP64 line integrals (classical Siddon) of every cone-beam ray."""
    L = lib()
    nv = len(angles)
    out = np.zeros((nv, nb, na), np.float64)
    o = None if off is None else _f64(off)
    L.or_cb_exact_f64(C.byref(g), _p(_f64(vol)), _p(_f64(angles)), _p(o), C.c_int(nv),
                      C.c_double(src_iso), C.c_double(src_det), C.c_int(na), C.c_double(da),
                      C.c_double(ai), C.c_int(nb), C.c_double(db), C.c_double(bi),
                      C.c_int(int(cyl)), C.c_int(int(inv_l2)), _p(out))
    return out


def lor_forward(g: Grid, vol, lors, flags=LOR_FWD):
    L = lib()
    lr = _f32(lors)
    n = lr.shape[1]
    out = np.zeros(n, np.float32)
    L.or_lor_forward_f32.restype = C.c_longlong
    cnt = L.or_lor_forward_f32(C.byref(g), _p(_f32(vol)), _p(lr), C.c_longlong(n), C.c_uint(flags), _p(out))
    return out, int(cnt)


def lor_backward(g: Grid, vals, lors, flags=LOR_BP):
    L = lib()
    lr = _f32(lors)
    out = np.zeros((g.nz, g.ny, g.nx), np.float32)
    L.or_lor_backward_f32(C.byref(g), _p(_f32(vals)), _p(lr), C.c_longlong(lr.shape[1]),
                          C.c_uint(flags), _p(out))
    return out


def pixel_backproject(sino, angles, shape, corner, size, src_iso, src_det, na, da, ai, nb, db, bi,
                      *, cyl=False, fdk=False, f64=False):
    """Voxel-driven bilinear backprojection (pixel_3d), optional FDK weight."""
    L = lib()
    nx, ny, nz = shape
    nv = len(angles)
    if f64:
        conv, cv, fn, dt = _f64, C.c_double, L.or_pixel_backproject_f64, np.float64
    else:
        conv, cv, fn, dt = _f32, C.c_float, L.or_pixel_backproject_f32, np.float32
    out = np.zeros((nz, ny, nx), dt)
    fn(_p(conv(sino)), _p(conv(angles)), C.c_int(nv), C.c_int(nx), C.c_int(ny), C.c_int(nz),
       _p(conv(corner)), _p(conv(size)), cv(src_iso), cv(src_det), C.c_int(na), cv(da), cv(ai),
       C.c_int(nb), cv(db), cv(bi), C.c_int(int(cyl)), C.c_int(int(fdk)), _p(out))
    return out


def deform(img, mx, my, mz, f64=False):
    L = lib()
    conv = _f64 if f64 else _f32
    img = conv(img)
    nz, ny, nx = img.shape
    out = np.zeros_like(img)
    fn = L.or_deform_f64 if f64 else L.or_deform_f32
    fn(_p(img), _p(conv(mx)), _p(conv(my)), _p(conv(mz)), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(out))
    return out


def warp_invert(mx, my, mz, iters=30):
    L = lib()
    mx, my, mz = _f32(mx), _f32(my), _f32(mz)
    nz, ny, nx = mx.shape
    out = [np.zeros_like(mx) for _ in range(3)]
    L.or_warp_invert_f32(_p(mx), _p(my), _p(mz), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(iters),
                         *[_p(o) for o in out])
    return out


def dd_backproject(proj, angles, shape, SID, SAD, na, da, ai, nb, db, bi, *, cyl=False, off=None,
                   use_cosf=True):
    """Distance-driven FDK-weighted backprojection (dist_3d_back_fdk): voxel
    units, grid centred on the axis, SID = source-detector, SAD =
    source-axis; proj is [nv][nb][na]."""
    L = lib()
    nx, ny, nz = shape
    nv = len(angles)
    cs, sn = trig(angles, use_cosf)
    o = np.zeros(nv, np.float32) if off is None else _f32(off)
    out = np.zeros((nz, ny, nx), np.float32)
    L.or_dd_backproject_f32(_p(_f32(proj)), _p(_f32(cs)), _p(_f32(sn)), _p(o), C.c_int(nv), C.c_float(SID),
                            C.c_float(SAD), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(na), C.c_float(da),
                            C.c_float(ai), C.c_int(nb), C.c_float(db), C.c_float(bi), C.c_int(int(cyl)),
                            C.c_int(int(use_cosf)), _p(out))
    return out


# ---------------- the reference itself, compiled for the host ----------------

def ref_cb_forward(g: Grid, vol, angles, SID, SAD, na, da, ai, nb, db, bi, *, cyl=False, f64=False):
    """siddon_3d project_flat/project_cyli (kernel naming: SID = source to
    axis, SAD = source to detector)."""
    R = ref()
    nv = len(angles)
    if f64:
        conv, cv, fn, dt = _f64, C.c_double, R.ref_s3d_project_f64, np.float64
    else:
        conv, cv, fn, dt = _f32, C.c_float, R.ref_s3d_project, np.float32
    out = np.zeros((nv, nb, na), dt)
    fn(C.c_int(int(cyl)), _p(conv(vol)), C.c_int(g.nx), C.c_int(g.ny), C.c_int(g.nz),
       cv(g.cx), cv(g.cy), cv(g.cz), cv(g.sx), cv(g.sy), cv(g.sz), _p(conv(angles)), C.c_int(na),
       C.c_int(nb), C.c_int(nv), cv(SID), cv(SAD), cv(da), cv(ai), cv(db), cv(bi), _p(out))
    return out


def ref_cb_backward(g: Grid, sino, angles, SID, SAD, na, da, ai, nb, db, bi, *, cyl=False, f64=False,
                    atomic=False):
    """The reference's backprojection.  Default: deterministic (fixed chunks
    of rows, chunk volumes summed in order; 16 volume-sized buffers).
    atomic=True: atomic adds into one volume (the host form of the device
    atomics: no extra volumes, summation order set by scheduling) -- for
    timing and for volumes too large for 16 copies."""
    R = ref()
    nv = len(angles)
    if f64:
        conv, cv, fn, dt = _f64, C.c_double, R.ref_s3d_backproject_f64, np.float64
    else:
        conv, cv, dt = _f32, C.c_float, np.float32
        fn = R.ref_s3d_backproject_atomic if atomic else R.ref_s3d_backproject
    s = conv(sino).reshape(-1)
    if cyl:
        # Q8 indexing reaches ia + iv*na + ib*na*nb; pad with zeros past the end
        need = (na - 1) + (nv - 1) * na + (nb - 1) * na * nb + 1
        if need > s.size:
            s = np.concatenate([s, np.zeros(need - s.size, s.dtype)])
    out = np.zeros((g.nz, g.ny, g.nx), dt)
    fn(C.c_int(int(cyl)), _p(s), C.c_int(g.nx), C.c_int(g.ny), C.c_int(g.nz), cv(g.cx), cv(g.cy),
       cv(g.cz), cv(g.sx), cv(g.sy), cv(g.sz), _p(conv(angles)), C.c_int(na), C.c_int(nb), C.c_int(nv),
       cv(SID), cv(SAD), cv(da), cv(ai), cv(db), cv(bi), _p(out))
    return out


def ref_lor_forward(g: Grid, vol, lors):
    R = ref()
    lr = _f32(lors)
    n = lr.shape[1]
    out = np.zeros(n, np.float32)
    R.ref_lor_project(_p(lr), C.c_longlong(n), _p(_f32(vol)), C.c_int(g.nx), C.c_int(g.ny),
                      C.c_int(g.nz), C.c_float(g.cx), C.c_float(g.cy), C.c_float(g.cz),
                      C.c_float(g.sx), C.c_float(g.sy), C.c_float(g.sz), _p(out))
    return out


def ref_lor_backward(g: Grid, vals, lors):
    R = ref()
    lr = _f32(lors)
    out = np.zeros((g.nz, g.ny, g.nx), np.float32)
    R.ref_lor_backproject(_p(lr), C.c_longlong(lr.shape[1]), _p(_f32(vals)), C.c_int(g.nx),
                          C.c_int(g.ny), C.c_int(g.nz), C.c_float(g.cx), C.c_float(g.cy),
                          C.c_float(g.cz), C.c_float(g.sx), C.c_float(g.sy), C.c_float(g.sz), _p(out))
    return out


def ref_pixel_backproject(sino, angles, shape, corner, size, SID, SAD, na, da, ai, nb, db, bi, *, cyl=False):
    R = ref()
    nx, ny, nz = shape
    out = np.zeros((nz, ny, nx), np.float32)
    R.ref_pixel_backproject(C.c_int(int(cyl)), _p(_f32(sino)), C.c_int(nx), C.c_int(ny), C.c_int(nz),
                            _p(_f32(corner)), _p(_f32(size)), _p(_f32(angles)), C.c_int(na),
                            C.c_int(nb), C.c_int(len(angles)), C.c_float(SID), C.c_float(SAD),
                            C.c_float(da), C.c_float(ai), C.c_float(db), C.c_float(bi), _p(out))
    return out


def ref_deform(img, mx, my, mz):
    R = ref()
    img = _f32(img)
    nz, ny, nx = img.shape
    out = np.zeros_like(img)
    R.ref_deform(_p(img), _p(_f32(mx)), _p(_f32(my)), _p(_f32(mz)), C.c_int(nx), C.c_int(ny),
                 C.c_int(nz), _p(out))
    return out


def ref_dd_backproject(proj, angles, shape, SID, SAD, na, da, ai, nb, db, bi, *, cyl=False, off=None):
    """back_project_{flat,cyli}_fdk_gpu of dist_3d_back_fdk.cu.cc:257-298
    (into a zeroed volume)."""
    R = ref()
    nx, ny, nz = shape
    nv = len(angles)
    o = np.zeros(nv, np.float32) if off is None else _f32(off)
    out = np.zeros((nz, ny, nx), np.float32)
    R.ref_dd_backproject(C.c_int(int(cyl)), _p(_f32(proj)), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(o),
                         _p(_f32(angles)), C.c_int(nv), C.c_float(SID), C.c_float(SAD), C.c_float(da),
                         C.c_float(ai), C.c_int(na), C.c_float(db), C.c_float(bi), C.c_int(nb), _p(out))
    return out

"""Op-level mirrors of the reference's TensorFlow custom ops on this path.

Same op names (TensorFlow's snake_case python wrappers), same inputs, attrs
and output shapes as the registered ops, including their quirks:

* ``siddon_3d``  nefct/cc/siddon_3d/siddon.cc:11-80 -- ProjectFlat,
  ProjectCyli (the op passes ``da`` as the row pitch, Q7), BackProjectFlat,
  BackProjectCyli (sinogram read transposed, Q8);
* ``pixel_3d``   nefct/cc/pixel_3d/pixel.cc:11-47 -- voxel-driven
  BackProjectFlat / BackProjectCyli (``center`` is the grid's low corner,
  Q10; ``ai`` counts from the pixel centre, Q9);
* ``siddon``     cpp/siddon/siddon_gpu.cc:11-35 -- Projection,
  Backprojection (LOR pair);
* ``deform``     cpp/deform/deform.cc:12-22 -- Deform;
* ``distance_3d`` nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:257-298 --
  back_project_flat_fdk_gpu / back_project_cyli_fdk_gpu (host entry points
  of the distance-driven FDK backprojection; the reference registers no op
  for them).  They add into the caller's ``image``, as there.  Also
  project_flat_three / project_cyli_three, the forward ops of dist_3d_mod
  that nefct/functions/project.py:11-16, :88-97 calls with keyword attrs
  (shape, offsets, angles, SID, SAD, na, da, ai, nb, db, bi; voxel units,
  SID = source-detector, SAD = source-axis, ai/bi physical offsets in
  voxels): the reference ships no source for them, so they are this
  library's distance-driven line integrals (nefct_dd_forward without the
  FDK weight: footprint overlap fractions times |p2 - p1| / |driving
  component|, summed per bin), whose exact transpose is
  nefct_dd_backward.

Tensors are CUDA torch tensors.  ``grid``/``center``/``size`` may be
sequences or tensors; the reference reads them back from the device with
blocking copies, here they are plain host values.  Backprojection outputs
have the op's declared shape (nx, ny, nz) over the kernel's x-fastest memory,
exactly like the TensorFlow tensors (reshape to (nz, ny, nx) for a
[z][y][x] view).
"""
from __future__ import annotations

import types

import numpy as np
import torch

from . import _lib, ops

__all__ = ["siddon_3d", "pixel_3d", "siddon", "deform", "distance_3d"]


def _host3(v, cast):
    if isinstance(v, torch.Tensor):
        v = v.detach().cpu().numpy()
    v = np.asarray(v).reshape(-1)
    if v.size != 3:
        raise _lib.NefctError(_lib.ERR_INVALID, "grid/center/size need 3 entries")
    return tuple(cast(x) for x in v)


def _angles(angle):
    if isinstance(angle, torch.Tensor):
        angle = angle.detach().cpu().numpy()
    return np.asarray(angle, np.float32).reshape(-1)


def _geom(grid, center, size, angle, SID, SAD, na, da, ai, nb, db, bi, cyl):
    g = _host3(grid, int)
    return ops.ConeBeam(g, _angles(angle), float(SID), float(SAD), int(na), float(da), int(nb), float(db),
                        float(ai), float(bi), _host3(center, float), _host3(size, float),
                        "cyl" if cyl else "flat")


def _flat_volume(image, g):
    nx, ny, nz = g
    if image.numel() != nx * ny * nz:
        raise _lib.NefctError(_lib.ERR_INVALID, f"image has {image.numel()} elements, grid needs {nx * ny * nz}")
    return image.contiguous().view(nz, ny, nx)


def _project(cyl):
    def op(image, grid, center, size, angle, SID, SAD, na, da, ai, nb, db, bi):
        # Q7: the op hands da to the kernel where db belongs (siddon.cc:155, 211)
        geom = _geom(grid, center, size, angle, SID, SAD, na, da, ai, nb, da, bi, cyl)
        return ops.cb_forward(_flat_volume(image, geom.shape), geom, _lib.REF_FORWARD)
    op.__name__ = "project_cyli" if cyl else "project_flat"
    return op


def _backproject(cyl):
    def op(projection_value, grid, center, size, angle, SID, SAD, na, da, ai, nb, db, bi, nx, ny, nz):
        geom = _geom(grid, center, size, angle, SID, SAD, na, da, ai, nb, db, bi, cyl)
        flags = _lib.REF_BACKPROJECT | (_lib.Q8_INDEX if cyl else 0)
        sino = projection_value.contiguous().view(geom.sino_shape)
        vol = ops.cb_backward(sino, geom, flags)
        return vol.view(int(nx), int(ny), int(nz))
    op.__name__ = "back_project_cyli" if cyl else "back_project_flat"
    return op


def _pixel_backproject(cyl):
    def op(projection_value, grid, center, size, angle, SID, SAD, na, da, ai, nb, db, bi, nx, ny, nz):
        corner = _host3(center, float)
        sz = _host3(size, float)
        mid = tuple(c + s / 2.0 for c, s in zip(corner, sz))
        # pixel_3d's ai/bi count from the pixel centre: siddon_3d's shift minus 1/2 (Q9)
        geom = _geom(grid, mid, sz, angle, SID, SAD, na, da, float(ai) + 0.5, nb, db, float(bi) + 0.5, cyl)
        sino = projection_value.contiguous().view(geom.sino_shape)
        vol = ops.fdk_backproject(sino, geom, weight=False)
        return vol.view(int(nx), int(ny), int(nz))
    op.__name__ = "back_project_cyli" if cyl else "back_project_flat"
    return op


# Line lists at least this long are walked in lor_order (a key pass and a
# sort, ~1 ms for 16 Mi lines, against a 6-8x slower walk in list order); the
# results keep the lines' order, so the ops behave exactly as in list order
# (the backprojection up to the summation order of its float reductions).
_LOR_AUTO_ORDER = 1 << 20


def _lor_walk_order(lors, g, center, size):
    if lors.shape[1] < _LOR_AUTO_ORDER:
        return None
    return ops.lor_order(lors, g, center, size)


def _projection(lors, image, grid, center, size):
    g = _host3(grid, int)
    lors = lors.contiguous()
    c, s = _host3(center, float), _host3(size, float)
    return ops.lor_forward(lors, _flat_volume(image, g), g, c, s, _lib.LOR_REF_FORWARD,
                           order=_lor_walk_order(lors, g, c, s))


def _backprojection(image, lors, lors_value, grid, center, size):
    g = _host3(grid, int)
    lors = lors.contiguous()
    c, s = _host3(center, float), _host3(size, float)
    vol = ops.lor_backward(lors, lors_value.contiguous(), g, c, s, _lib.LOR_REF_BACKPROJECT,
                           order=_lor_walk_order(lors, g, c, s))
    return vol.view(image.shape)


def _deform(image, mx, my, mz, grid):
    g = _host3(grid, int)
    vol = _flat_volume(image, g)
    out = ops.warp_forward(vol, *[_flat_volume(m, g) for m in (mx, my, mz)])
    return out.view(image.shape)


siddon_3d = types.SimpleNamespace(project_flat=_project(False), project_cyli=_project(True),
                                  back_project_flat=_backproject(False), back_project_cyli=_backproject(True))
pixel_3d = types.SimpleNamespace(back_project_flat=_pixel_backproject(False),
                                 back_project_cyli=_pixel_backproject(True))
siddon = types.SimpleNamespace(projection=_projection, backprojection=_backprojection)
deform = types.SimpleNamespace(deform=_deform)


def _dd_backproject(cyl):
    def op(pv_values, shape, offsets, angles, nv, SID, SAD, da, ai, na, db, bi, nb, image):
        """pv_values [nv][nb][na]; shape (nx, ny, nz); SID = source-detector,
        SAD = source-axis (this file's naming); image (nx, ny, nz) over
        x-fastest memory is added to and returned."""
        nx, ny, nz = _host3(shape, int)
        ang = _angles(angles)[:int(nv)]
        off = None if offsets is None else np.asarray(
            offsets.detach().cpu().numpy() if isinstance(offsets, torch.Tensor) else offsets, np.float32)
        pv = pv_values.reshape(int(nv), int(nb), int(na))
        vol = ops.dd_backproject(pv, (nx, ny, nz), ang, float(SAD), float(SID), float(da), float(db), float(ai),
                                 float(bi), "cyl" if cyl else "flat", off)
        image += vol.reshape(image.shape)
        return image
    return op


def _dd_project(cyl):
    def op(image, shape, offsets, angles, SID, SAD, na, da, ai, nb, db, bi):
        """image: the volume over x-fastest memory (the transposed numpy /
        [nz, ny, nx] tensor the reference hands over); returns [nv, nb, na].
        The bin centre is (i + 0.5) * d + ai - n * d / 2, as in the
        backprojection of dist_3d_back_fdk.cu.cc:45-60."""
        nx, ny, nz = (int(v) for v in shape)
        ang = _angles(angles)
        off = None if offsets is None else _angles(offsets)
        if off is not None and off.size == 1 and ang.size > 1:
            off = np.full(ang.size, off[0], np.float32)
        g = ops.DDGeometry((nx, ny, nz), ang, float(SAD), float(SID), int(na), float(da), int(nb), float(db),
                           float(ai), float(bi), "cyl" if cyl else "flat", off)
        vol = image if isinstance(image, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(image, np.float32))
        if not vol.is_cuda:
            vol = vol.cuda()
        return ops.dd_forward(vol.reshape(nz, ny, nx).contiguous().float(), g, _lib.FDK_NO_WEIGHT)
    return op


distance_3d = types.SimpleNamespace(back_project_flat_fdk_gpu=_dd_backproject(False),
                                    back_project_cyli_fdk_gpu=_dd_backproject(True),
                                    project_flat_three=_dd_project(False), project_cyli_three=_dd_project(True))

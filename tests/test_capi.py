"""CPU: the C-ABI library loads, exports every symbol the header declares, and
rejects bad arguments with a status (no GPU work is started by these calls:
validation happens before any CUDA call)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "nefct_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(nefct_[a-z0-9_]+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported(nefct_lib):
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(nefct_lib, s), s


def test_python_binding_covers_header(nefct_lib):
    from nefct_b200 import _lib
    assert sorted(_lib.symbols()) == declared_symbols()


def test_version_and_status_strings(nefct_lib):
    assert b"sm_100a" in nefct_lib.nefct_version()
    assert nefct_lib.nefct_status_string(0) == b"ok"
    assert nefct_lib.nefct_status_string(3).startswith(b"workspace")


def _geom(**kw):
    import nefct_b200 as nb
    base = dict(shape=(16, 16, 16), angles=np.linspace(0, 6.28, 8, dtype=np.float32), src_iso=100.0,
                src_det=200.0, na=32, da=1.0, nb=24, db=1.0)
    base.update(kw)
    return nb.ConeBeam(**base)


@pytest.mark.parametrize("kw,needle", [
    (dict(na=0), b"detector"),
    (dict(shape=(0, 16, 16)), b"grid dimensions"),
    (dict(da=0.0), b"pitch"),
    (dict(angles=np.array([0.0, np.nan], np.float32)), b"angle 1"),
    (dict(size=(16.0, -1.0, 16.0)), b"size"),
])
def test_invalid_geometry_is_rejected(nefct_lib, kw, needle):
    g = _geom(**kw).struct()
    st = nefct_lib.nefct_cb_forward(C.byref(g), None, None, 0, None, 0, None)
    assert st == 1
    assert needle in nefct_lib.nefct_last_error()


def test_forward_needs_workspace(nefct_lib):
    g = _geom().struct()
    # non-NULL fake pointers: validation fails on the workspace before any CUDA call
    st = nefct_lib.nefct_cb_forward(C.byref(g), C.c_void_p(16), C.c_void_p(16), 0, None, 0, None)
    assert st == 3
    assert nefct_lib.nefct_cb_workspace_bytes(C.byref(g), 0) == 16 ** 3 * 4
    assert nefct_lib.nefct_cb_workspace_bytes(C.byref(g), 0x20) == 0


def test_unknown_flags_rejected(nefct_lib):
    g = _geom().struct()
    st = nefct_lib.nefct_cb_forward(C.byref(g), C.c_void_p(16), C.c_void_p(16), 0x4000, None, 0, None)
    assert st == 1 and b"flag" in nefct_lib.nefct_last_error()


def test_fdk_rejects_cylindrical_and_bad_window(nefct_lib):
    g = _geom(det_kind="cyl").struct()
    assert nefct_lib.nefct_fdk_filter(C.byref(g), C.c_void_p(16), C.c_void_p(32), 0, 0, None) == 5
    g = _geom().struct()
    assert nefct_lib.nefct_fdk_filter(C.byref(g), C.c_void_p(16), C.c_void_p(32), 9, 0, None) == 1
    assert nefct_lib.nefct_fdk_filter(C.byref(g), C.c_void_p(16), C.c_void_p(16), 0, 0, None) == 1


def test_warp_rejects_bad_grid(nefct_lib):
    assert nefct_lib.nefct_warp_forward(None, None, None, None, 0, 4, 4, None, None) == 1


def test_ops_refuse_cpu_tensors(nefct_lib):
    import torch
    import nefct_b200 as nb
    g = _geom()
    with pytest.raises(nb.NefctError, match="CUDA tensor"):
        nb.ops.cb_forward(torch.zeros(g.vol_shape), g)


def test_deterministic_workspace_size(nefct_lib):
    g = _geom().struct()
    n = 16 ** 3
    assert nefct_lib.nefct_cb_workspace_bytes(C.byref(g), 0x40) == 256 + 16 * n
    assert nefct_lib.nefct_cb_workspace_bytes(C.byref(g), 0x40 | 0x20) == 256 + 8 * n


def test_fdk_filter_rejects_wide_detectors(nefct_lib):
    """The filter's transforms go up to 4096 points: more than 2048 columns is
    refused before any device work."""
    g = _geom(na=2049).struct()
    assert nefct_lib.nefct_fdk_filter(C.byref(g), C.c_void_p(16), C.c_void_p(32), 0, 0, None) == 5
    assert b"2048" in nefct_lib.nefct_last_error()


def test_batch_plan_validates_problems(nefct_lib):
    from nefct_b200 import _lib
    probs = (_lib.CBProblem * 97)()
    plan, ws = C.c_void_p(), C.c_size_t()
    assert nefct_lib.nefct_cb_batch_plan(probs, 97, 0, C.byref(plan), C.byref(ws)) == 1   # > 96 problems
    assert b"96" in nefct_lib.nefct_last_error()
    probs = (_lib.CBProblem * 1)()
    probs[0].geom = _geom().struct()
    assert nefct_lib.nefct_cb_batch_plan(probs, 1, 0, C.byref(plan), C.byref(ws)) == 1     # NULL buffers
    assert b"NULL" in nefct_lib.nefct_last_error()
    probs[0].vol = probs[0].sino = probs[0].grad = probs[0].back = 16
    assert nefct_lib.nefct_cb_batch_plan(probs, 1, 0x4000, C.byref(plan), C.byref(ws)) == 1  # unknown flags


def test_batch_set_buffers_is_host_only(nefct_lib):
    """Planning and re-pointing a plan's buffers make no CUDA call (fake
    device pointers are only stored); a NULL plan is refused."""
    from nefct_b200 import _lib
    probs = (_lib.CBProblem * 2)()
    for i in range(2):
        probs[i].geom = _geom().struct()
        probs[i].vol = probs[i].sino = probs[i].grad = probs[i].back = 256 * (i + 1)
    plan, ws = C.c_void_p(), C.c_size_t()
    assert nefct_lib.nefct_cb_batch_plan(probs, 2, 0, C.byref(plan), C.byref(ws)) == 0
    try:
        vols = (C.c_void_p * 2)(4096, None)
        assert nefct_lib.nefct_cb_batch_set_buffers(plan, vols, None, None, None) == 0
        assert nefct_lib.nefct_cb_batch_set_buffers(plan, None, None, vols, None) == 0
    finally:
        nefct_lib.nefct_cb_batch_destroy(plan)
    assert nefct_lib.nefct_cb_batch_set_buffers(None, None, None, None, None) == 1


def test_dd_rejects_bad_geometry(nefct_lib):
    from nefct_b200 import _lib
    ang = (C.c_float * 2)(0.0, float("nan"))
    g = _lib.DDGeom(nx=8, ny=8, nz=8, nv=2, angles=ang, z_offsets=None, src_iso=100.0, src_det=200.0, na=16,
                    da=1.0, a_offset=0.0, nb=8, db=1.0, b_offset=0.0, det_kind=0)
    ws = nefct_lib.nefct_dd_workspace_bytes(C.byref(g))
    assert ws == 8 * 8 * 8 * 4
    assert nefct_lib.nefct_dd_backproject(C.byref(g), C.c_void_p(16), C.c_void_p(32), C.c_void_p(64), ws, None) == 1
    assert b"view 1" in nefct_lib.nefct_last_error()
    ang[1] = 0.5
    g.det_kind = 7
    assert nefct_lib.nefct_dd_backproject(C.byref(g), C.c_void_p(16), C.c_void_p(32), C.c_void_p(64), ws, None) == 1
    g.det_kind = 0
    assert nefct_lib.nefct_dd_backproject(C.byref(g), C.c_void_p(16), C.c_void_p(32), C.c_void_p(64), 4, None) == 3


def test_noalloc_refuses_grids_beyond_its_scratch(nefct_lib):
    """The allocation-free forward checks the grid against its fixed 32 MiB
    scratch before any CUDA call."""
    import nefct_b200 as nb
    from nefct_b200 import _lib
    g = nb.ConeBeam((256, 256, 256), [0.0], 600.0, 1200.0, 64, 1.0, 64, 1.0)
    s = g.struct()
    st = nefct_lib.nefct_cb_forward_noalloc(C.byref(s), C.c_void_p(256), C.c_void_p(256), 0, None)
    assert st == _lib.ERR_INVALID
    assert b"at most 8388608 voxels" in nefct_lib.nefct_last_error()


def test_dd_pair_rejects_bad_arguments(nefct_lib):
    """The distance-driven pair validates geometry, flags, buffers and the
    workspace before any CUDA call."""
    from nefct_b200 import _lib, ops
    g = ops.DDGeometry((8, 8, 8), np.linspace(0, 3, 4), 50.0, 100.0, 16, 1.0, 8, 1.0)
    s = g.struct()
    ws = C.c_void_p(256)
    assert nefct_lib.nefct_dd_forward(C.byref(s), C.c_void_p(256), C.c_void_p(256), 0x1, ws, 1 << 20, None) == \
        _lib.ERR_INVALID
    assert b"unknown flag" in nefct_lib.nefct_last_error()
    assert nefct_lib.nefct_dd_forward(C.byref(s), None, C.c_void_p(256), 0, ws, 1 << 20, None) == _lib.ERR_INVALID
    st = nefct_lib.nefct_dd_backward(C.byref(s), C.c_void_p(256), C.c_void_p(256), 0, ws, 16, None)
    assert st == _lib.ERR_WORKSPACE and b"workspace" in nefct_lib.nefct_last_error()
    bad = ops.DDGeometry((0, 8, 8), np.linspace(0, 3, 4), 50.0, 100.0, 16, 1.0, 8, 1.0).struct()
    assert nefct_lib.nefct_dd_forward_f64(C.byref(bad), C.c_void_p(256), C.c_void_p(256), 0, None) == \
        _lib.ERR_INVALID


def test_probes_reject_bad_arguments(nefct_lib):
    from nefct_b200 import _lib
    assert nefct_lib.nefct_probe_l2_read(C.c_void_p(256), 6, 1, 8, C.c_void_p(256), None) == _lib.ERR_INVALID
    assert nefct_lib.nefct_probe_l2_read(C.c_void_p(260), 8, 1, 8, C.c_void_p(256), None) == _lib.ERR_INVALID
    assert nefct_lib.nefct_probe_l2_red(C.c_void_p(256), 8, 0, 8, None) == _lib.ERR_INVALID
    assert nefct_lib.nefct_probe_l2_red(None, 8, 1, 8, None) == _lib.ERR_INVALID


@pytest.mark.parametrize("kw,needle", [
    (dict(shape=((1 << 20) + 1, 1, 1)), b"<= 2^20"),
    (dict(shape=(2048, 2048, 1024)), b"2^31"),
    (dict(nb=65536), b"65535"),
])
def test_size_limits_are_rejected(nefct_lib, kw, needle):
    """Grid dimensions above 2^20, grids of 2^31 voxels or more and more than
    65535 detector rows are refused with a status before any CUDA call."""
    g = _geom(**kw).struct()
    st = nefct_lib.nefct_cb_forward(C.byref(g), C.c_void_p(256), C.c_void_p(256), 0, C.c_void_p(256), 1 << 40,
                                    None)
    assert st == 1
    assert needle in nefct_lib.nefct_last_error()


def test_lor_negative_count_is_rejected(nefct_lib):
    from nefct_b200 import _lib
    grid = _lib.Grid(8, 8, 8, 0, 0, 0, 8, 8, 8)
    assert nefct_lib.nefct_lor_forward(C.byref(grid), C.c_void_p(256), -1, C.c_void_p(256), C.c_void_p(256), 0,
                                       None) == _lib.ERR_INVALID


def test_fdk_quad_workspace_is_checked(nefct_lib):
    from nefct_b200 import _lib
    g = _geom().struct()
    need = nefct_lib.nefct_fdk_workspace_bytes(C.byref(g))
    assert need == 8 * 32 * 24 * 16          # all 8 views fit one chunk of tap quads
    st = nefct_lib.nefct_fdk_backproject_ws(C.byref(g), C.c_void_p(256), C.c_void_p(256), 0, C.c_void_p(256),
                                            need - 16, None)
    assert st == _lib.ERR_WORKSPACE
    st = nefct_lib.nefct_fdk_backproject_ws(C.byref(g), C.c_void_p(256), C.c_void_p(256), 0, C.c_void_p(264),
                                            need, None)
    assert st == _lib.ERR_INVALID and b"aligned" in nefct_lib.nefct_last_error()


def test_cone_beam_refuses_lor_only_flag(nefct_lib):
    """NEFCT_Q5 is a quirk of the LOR projector: the cone-beam calls refuse it
    before any CUDA call instead of ignoring it."""
    from nefct_b200 import _lib
    g = _geom().struct()
    ws = C.c_void_p(256)
    for fn in ("nefct_cb_forward", "nefct_cb_backward"):
        st = getattr(nefct_lib, fn)(C.byref(g), C.c_void_p(256), C.c_void_p(256), _lib.Q5, ws, 1 << 20, None)
        assert st == _lib.ERR_UNSUPPORTED, fn
        assert b"LOR" in nefct_lib.nefct_last_error()
    st = nefct_lib.nefct_cb_forward_noalloc(C.byref(g), C.c_void_p(256), C.c_void_p(256), _lib.Q5, None)
    assert st == _lib.ERR_UNSUPPORTED

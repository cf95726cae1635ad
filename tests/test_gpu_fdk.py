"""GPU parity of FDK: the filter against the numpy restatement of
filtering.m / ParkerWeight.m, the voxel-driven backprojection against the
reference's pixel_3d (fixtures) and the oracle, and an end-to-end
reconstruction of a phantom."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import ops
from oracle import fdk as ofdk
from tests.golden.make_golden import DB, NA, NB, SRC_DET, SRC_ISO
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("window", ["ram-lak", "shepp-logan", "cosine", "hamming", "hann"])
@pytest.mark.parametrize("parker", [0, 1, -1])
def test_filter_vs_restatement(cuda, window, parker):
    nv, nb_, na = 40, 12, 100
    if parker:
        ang = np.deg2rad(np.arange(nv) * (220.0 / nv)).astype(np.float32)
    else:
        ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((8, 8, 8), ang, 300.0, 600.0, na, 1.3, nb_, 1.1)
    sino = np.random.default_rng(4).random((nv, nb_, na), dtype=np.float32)
    out = ops.fdk_filter(torch.from_numpy(sino).to(cuda), g, window, parker).cpu().numpy()
    ref = ofdk.fdk_filter(sino, 600.0, 300.0, 1.3, 1.1, window=window, parker=parker, angles=ang)
    assert_parity(out, ref)


@pytest.mark.parametrize("na,nb_", [(1, 1), (33, 5), (2048, 3)])
def test_filter_sizes_vs_restatement(cuda, na, nb_):
    """Transform lengths from 64 (one column) to 4096 (the widest supported
    detector, whose transform buffers need more than 48 KB of shared memory),
    an odd row count (the last row pair holds one row), odd log2 L (33 columns:
    L = 128)."""
    nv = 3
    ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((8, 8, 8), ang, 300.0, 600.0, na, 0.4, nb_, 1.1)
    sino = np.random.default_rng(na).random((nv, nb_, na), dtype=np.float32)
    for window in ("ram-lak", "shepp-logan"):
        out = ops.fdk_filter(torch.from_numpy(sino).to(cuda), g, window).cpu().numpy()
        ref = ofdk.fdk_filter(sino, 600.0, 300.0, 0.4, 1.1, window=window, angles=ang)
        assert_parity(out, ref)


def test_pixel_backprojection_vs_reference_fixtures(cuda, golden):
    corner = golden["pixel/corner"]
    sino = torch.from_numpy(golden["pixel/sino"]).to(cuda)
    for cyl, key, da in ((False, "pixel/flat", 2.5), (True, "pixel/cyl", 0.012)):
        op = nb.cc.pixel_3d.back_project_cyli if cyl else nb.cc.pixel_3d.back_project_flat
        out = op(sino, [24, 20, 16], corner, [48.0, 40.0, 32.0], golden["angles"], SRC_ISO, SRC_DET, NA, da, 0.0,
                 NB, DB, 0.0, 24, 20, 16)
        out = out.reshape(16, 20, 24).cpu().numpy()
        assert_parity(out, golden[key])


@pytest.mark.skipif("not __import__('oracle').have_ref()")
@pytest.mark.parametrize("phi", [0.0, 0.7, 2.9])
def test_fdk_distance_weight_pinned_by_reference_kernel(cuda, oracle_lib, phi):
    """The FDK distance weight src_iso^2 / (src_iso + x cos + y sin)^2
    (backprojection.m:11-12) is pinned against the reference's own kernel
    that applies it, dist_3d_back_fdk.cu.cc:153-154 (built for the host):
    for one view of an all-ones projection, that kernel's output divided by
    this library's weight-free distance-driven backprojection (same
    footprints and fractions) is the reference's weight per voxel; the
    voxel-driven FDK backprojection's weighted / unweighted ratio must
    equal it (1 mm voxels, grid centred on the axis, even sizes so both
    place voxel centres at (i + 0.5 - n / 2))."""
    n, na, nbr, sid, sdd = 32, 96, 80, 60.0, 120.0
    ang = np.array([phi], np.float32)
    ones = np.ones((1, nbr, na), np.float32)
    dg = ops.DDGeometry((n, n, n), ang, sid, sdd, na, 1.0, nbr, 1.0)
    ref_w = oracle_lib.ref_dd_backproject(ones, ang, (n, n, n), sdd, sid, na, 1.0, 0.0, nbr, 1.0, 0.0)
    ours_nw = ops.dd_backward(torch.from_numpy(ones).to(cuda), dg, nb._lib.FDK_NO_WEIGHT).cpu().numpy()
    g = nb.ConeBeam((n, n, n), ang, sid, sdd, na, 1.0, nbr, 1.0, size=(float(n),) * 3)
    t = torch.from_numpy(ones).to(cuda)
    fw = ops.fdk_backproject(t, g, weight=True).cpu().numpy()
    fnw = ops.fdk_backproject(t, g, weight=False).cpu().numpy()
    inside = (ours_nw > 1e-3 * ours_nw.max()) & (fnw > 0.5)
    assert inside.sum() > 0.3 * n ** 3
    w_ref = ref_w[inside] / ours_nw[inside]
    w_ours = fw[inside] / fnw[inside]
    # float32: each side is a ratio of two sums of ~20 rounded footprint
    # terms (atomic order differs between the host build and the GPU), so
    # agreement is to a few 1e-6; a wrong weight formula is off by ~1e-1
    np.testing.assert_allclose(w_ours, w_ref, rtol=2e-5)


def test_weighted_backprojection_vs_oracle(cuda, oracle_lib):
    ang = np.linspace(0, 2 * np.pi, 50, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((30, 26, 22), ang, 250.0, 500.0, 64, 1.7, 48, 1.4, center=(1.0, -2.0, 0.5),
                    size=(30.0, 26.0, 22.0))
    sino = np.random.default_rng(9).random(g.sino_shape, dtype=np.float32)
    out = ops.fdk_backproject(torch.from_numpy(sino).to(cuda), g).cpu().numpy()
    corner = [c - s / 2 for c, s in zip(g.center, g.size)]
    ref = oracle_lib.pixel_backproject(sino, ang, g.shape, np.array(corner, np.float32), g.size, 250.0, 500.0,
                                       64, 1.7, 0.0, 48, 1.4, 0.0, fdk=True)
    assert_parity(out, ref)


def test_weighted_backprojection_long_axis_vs_oracle(cuda, oracle_lib):
    """A grid whose three axes hold more voxels together than the kernel
    parameters' table of voxel centres (6144): the kernels compute the
    centres themselves, with the same result."""
    ang = np.linspace(0, 2 * np.pi, 24, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((6, 5, 6200), ang, 250.0, 500.0, 40, 1.7, 48, 1.4, center=(0.5, -0.5, 0.3),
                    size=(6.0, 5.0, 62.0))
    sino = np.random.default_rng(10).random(g.sino_shape, dtype=np.float32)
    out = ops.fdk_backproject(torch.from_numpy(sino).to(cuda), g).cpu().numpy()
    corner = [c - s / 2 for c, s in zip(g.center, g.size)]
    ref = oracle_lib.pixel_backproject(sino, ang, g.shape, np.array(corner, np.float32), g.size, 250.0, 500.0,
                                       40, 1.7, 0.0, 48, 1.4, 0.0, fdk=True)
    assert np.abs(ref).max() > 0
    assert_parity(out, ref)


def test_fdk_reconstructs_phantom(cuda):
    """Line-integral projections of a 64^3 ellipsoid phantom, Ram-Lak FDK:
    the interior is recovered (relative error of the central region)."""
    rows = np.array([[1.0, 0.6, 0.5, 0.4, 0, 0, 0, 0, 0, 0], [0.5, 0.2, 0.25, 0.2, 0.2, 0.1, 0, 30, 0, 0]])
    ph = nb.ellipsoid_phantom(64, rows, device=cuda)              # [x, y, z]
    vol = ph.permute(2, 1, 0).contiguous()
    ang = np.linspace(0, 2 * np.pi, 180, endpoint=False)
    g = nb.ConeBeam((64, 64, 64), ang, 400.0, 800.0, 160, 2.0, 128, 2.0, size=(64.0,) * 3)
    sino = ops.cb_forward(vol, g, nb._lib.LINE_INTEGRAL)
    rec = ops.fdk_backproject(ops.fdk_filter(sino, g), g)
    c = slice(20, 44)
    err = (rec[c, c, c] - vol[c, c, c]).norm() / vol[c, c, c].norm()
    assert float(err) < 0.15, float(err)


def test_short_scan_parker_close_to_full_scan(cuda):
    """A 180 deg + fan short scan with Parker weights in the direction
    derived from the geometry (ops.parker_direction: +1 for increasing
    angles) reconstructs close to the full scan, and clearly better than with
    the flipped direction (which weights the redundant rays wrongly)."""
    rows = np.array([[1.0, 0.5, 0.5, 0.45, 0, 0, 0, 0, 0, 0]])
    vol = nb.ellipsoid_phantom(48, rows, device=cuda).permute(2, 1, 0).contiguous()
    full = np.linspace(0, 2 * np.pi, 240, endpoint=False)
    gf = nb.ConeBeam((48, 48, 48), full, 300.0, 600.0, 128, 2.0, 64, 2.0, size=(48.0,) * 3)
    rf = ops.fdk_backproject(ops.fdk_filter(ops.cb_forward(vol, gf, nb._lib.LINE_INTEGRAL), gf), gf)
    fan = 2 * np.degrees(np.arctan(128 * 2.0 / 2 / 600.0))
    step = 1.5
    n = int(np.ceil((180 + fan) / step)) + 1
    c = slice(12, 36)
    errs = {}
    for sign in (1, -1):
        short = sign * np.deg2rad(np.arange(n) * step - fan / 2)
        gs = nb.ConeBeam((48, 48, 48), short, 300.0, 600.0, 128, 2.0, 64, 2.0, size=(48.0,) * 3)
        d = ops.parker_direction(gs)
        assert d == sign
        lines = ops.cb_forward(vol, gs, nb._lib.LINE_INTEGRAL)
        for flip in (1, -1):
            rs = ops.fdk_backproject(ops.fdk_filter(lines, gs, parker=d * flip), gs)
            errs[(sign, flip)] = float((rs[c, c, c] - rf[c, c, c]).norm() / rf[c, c, c].norm())
    for sign in (1, -1):
        assert errs[(sign, 1)] < 0.1, errs
        assert errs[(sign, -1)] > 1.5 * errs[(sign, 1)], errs


@pytest.mark.parametrize("weight", [True, False])
@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_tap_quad_backprojection_is_bitwise_equal(cuda, weight, cyl):
    """nefct_fdk_backproject_ws (taps read as quads from a repacked chunk)
    gives the bits of nefct_fdk_backproject (four loads per tap set), over
    several view chunks, with taps at the detector's last row and column."""
    import ctypes as C
    from nefct_b200 import _lib
    lib = _lib.load()
    nv = 300                                    # three view chunks (up to 128 views each)
    g = nb.ConeBeam((40, 36, 30), np.linspace(0, 2 * np.pi, nv, endpoint=False), 90.0, 180.0, 61,
                    0.02 if cyl else 1.3, 47, 1.2, size=(40.0, 36.0, 30.0), det_kind="cyl" if cyl else "flat")
    sino = torch.rand(g.sino_shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(2))
    s = g.struct()
    flags = 0 if weight else _lib.FDK_NO_WEIGHT
    stream = torch.cuda.current_stream(cuda).cuda_stream
    plain = torch.empty(g.vol_shape, device=cuda)
    _lib.check(lib.nefct_fdk_backproject(C.byref(s), sino.data_ptr(), plain.data_ptr(), flags, stream))
    wn = lib.nefct_fdk_workspace_bytes(C.byref(s))
    ws = torch.empty(wn, dtype=torch.uint8, device=cuda)
    quad = torch.full(g.vol_shape, float("nan"), device=cuda)
    _lib.check(lib.nefct_fdk_backproject_ws(C.byref(s), sino.data_ptr(), quad.data_ptr(), flags, ws.data_ptr(), wn,
                                            stream))
    torch.cuda.synchronize()
    assert torch.equal(quad, plain)
    assert float(plain.abs().max()) > 0

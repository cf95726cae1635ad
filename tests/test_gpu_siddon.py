"""GPU parity of the Siddon kernels (called through the C ABI via ctypes).

Tolerances (float32): rel-L2 <= 1e-5 and max-abs <= 1e-4 * max|ref| against
the reference (golden fixtures / reference build / oracle restatement);
FP64 identities to 1e-12.
"""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib, ops
from tests.golden.make_golden import AI, BI, CASES, DB, NA, NB, SRC_DET, SRC_ISO

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4


def assert_parity(out, ref, rel=REL_L2, mabs=MAX_ABS):
    out = np.asarray(out, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = np.abs(ref).max()
    assert scale > 0
    r = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    m = np.abs(out - ref).max() / scale
    assert r <= rel and m <= mabs, f"rel-L2 {r:.3e} max-abs/max {m:.3e}"
    return r


def _geom(case, angles):
    name, grid, centre, size, cyl, da = case
    return nb.ConeBeam(grid, angles, SRC_ISO, SRC_DET, NA, da, NB, DB, AI, BI, centre, size,
                       "cyl" if cyl else "flat")


@pytest.mark.parametrize("flags", [0, _lib.NO_TRANSPOSE], ids=["transposed", "direct"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_forward_vs_reference_fixtures(cuda, golden, case, flags):
    g = _geom(case, golden["angles"])
    vol = torch.from_numpy(golden[f"{case[0]}/vol"]).to(cuda)
    out = ops.cb_forward(vol, g, flags).cpu().numpy()
    assert_parity(out, golden[f"{case[0]}/fwd"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_forward_vs_restatement_tight(cuda, golden, oracle_lib, case):
    """Same per-view trig as the GPU (double rounded): only weight rounding differs."""
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    vol = golden[f"{name}/vol"]
    out = ops.cb_forward(torch.from_numpy(vol).to(cuda), g).cpu().numpy()
    port, _ = oracle_lib.cb_forward(oracle_lib.grid(grid, centre, size), vol, golden["angles"], SRC_ISO,
                                    SRC_DET, NA, da, AI, NB, DB, BI, cyl=cyl, use_cosf=False)
    assert_parity(out, port, rel=1e-6, mabs=1e-5)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_backprojection_vs_fixtures(cuda, golden, case):
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    sino = torch.from_numpy(golden[f"{name}/sino_in"]).to(cuda)
    flags = _lib.REF_BACKPROJECT | (_lib.Q8_INDEX if cyl else 0)
    out = ops.cb_backward(sino, g, flags).cpu().numpy()
    assert_parity(out, golden[f"{name}/bp"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_intersection_count_matches_reference(cuda, golden, case):
    g = _geom(case, golden["angles"])
    assert ops.cb_count_intersections(g) == int(golden[f"{case[0]}/count"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_exact_transpose_vs_oracle(cuda, golden, oracle_lib, case):
    """cb_backward with the forward's flags equals the oracle's scatter with
    the forward's weights (tie >=, 1/L^2, no skip)."""
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    sino = golden[f"{name}/sino_in"]
    out = ops.cb_backward(torch.from_numpy(sino).to(cuda), g, 0).cpu().numpy()
    ref = oracle_lib.cb_backward(oracle_lib.grid(grid, centre, size), sino, golden["angles"], SRC_ISO,
                                 SRC_DET, NA, da, AI, NB, DB, BI, cyl=cyl, flags=oracle_lib.CB_FWD)
    assert_parity(out, ref)


@pytest.mark.parametrize("flags", [0, _lib.LINE_INTEGRAL, _lib.REF_BACKPROJECT])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_adjoint_identity_f64(cuda, case, flags):
    """<A x, y> == <x, A^T y> to rounding in FP64 for every flag set."""
    g = _geom(case, np.linspace(0, 2 * np.pi, 17, endpoint=False) + 0.05)
    gen = torch.Generator(device=cuda).manual_seed(34)
    x = torch.randn(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen)
    y = torch.randn(g.sino_shape, dtype=torch.float64, device=cuda, generator=gen)
    ax = ops.cb_forward(x, g, flags)
    aty = ops.cb_backward(y, g, flags)
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0) * 1e2


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_f32_error_vs_fp64_oracle(cuda, golden, oracle_lib, case):
    """The error of the float32 forward and exact transpose against the FP64
    build of the same discretisation (the oracle's walk in double), stated:
    on these fixtures the float32 walk itself (the oracle's, on the CPU) is
    ~7e-7 (forward) and ~1.2e-6 (transpose) rel-L2 from the FP64 walk, and
    the GPU stays within 1e-5."""
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    og = oracle_lib.grid(grid, centre, size)
    args = (golden["angles"], SRC_ISO, SRC_DET, NA, da, AI, NB, DB, BI)
    vol, sino = golden[f"{name}/vol"], golden[f"{name}/sino_in"]
    ref_f, _ = oracle_lib.cb_forward(og, vol, *args, cyl=cyl, f64=True)
    ref_b = oracle_lib.cb_backward(og, sino, *args, cyl=cyl, flags=oracle_lib.CB_FWD, f64=True)
    out_f = ops.cb_forward(torch.from_numpy(vol).to(cuda), g).cpu().numpy()
    out_b = ops.cb_backward(torch.from_numpy(sino).to(cuda), g, 0).cpu().numpy()
    assert_parity(out_f, ref_f)
    assert_parity(out_b, ref_b)


def test_f64_forward_vs_reference_f64(cuda, golden):
    for case in CASES:
        g = _geom(case, golden["angles"])
        vol = torch.from_numpy(golden[f"{case[0]}/vol"].astype(np.float64)).to(cuda)
        out = ops.cb_forward(vol, g).cpu().numpy()
        assert_parity(out, golden[f"{case[0]}/fwd64"], rel=1e-6, mabs=1e-6)


def test_finite_difference_fp64_autograd(cuda):
    """loss = ||A x - b||^2 on 32^3 / 60 views in FP64: autograd (hand-written
    transpose) against central differences along a random direction."""
    g = nb.ConeBeam((32, 32, 32), np.linspace(0, 2 * np.pi, 60, endpoint=False), 120.0, 240.0, 48, 1.5, 40, 1.5)
    gen = torch.Generator(device=cuda).manual_seed(5)
    x = torch.rand(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen).requires_grad_()
    b = torch.rand(g.sino_shape, dtype=torch.float64, device=cuda, generator=gen)
    d = torch.randn(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen)
    loss = ((nb.project(x, g) - b) ** 2).sum()
    loss.backward()
    # the loss is exactly quadratic in x, so a large step has no truncation
    # error; the rounding error of the difference is ~eps * loss / h
    h = 0.5
    with torch.no_grad():
        fp = ((ops.cb_forward(x + h * d, g) - b) ** 2).sum()
        fm = ((ops.cb_forward(x - h * d, g) - b) ** 2).sum()
    fd = float((fp - fm) / (2 * h))
    an = float((x.grad * d).sum())
    assert abs(fd - an) <= 1e-9 * abs(an) + 1e-14 * float(loss) / h


def test_many_views_chunked_and_offsets(cuda, oracle_lib):
    """> 1024 views (several launches) and per-view z offsets."""
    nv = 1100
    ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    off = np.linspace(-3, 3, nv).astype(np.float32)
    g = nb.ConeBeam((12, 12, 10), ang, 60.0, 120.0, 20, 1.5, 9, 1.5, z_offsets=off)
    vol = np.random.default_rng(3).random((10, 12, 12), dtype=np.float32)
    out = ops.cb_forward(torch.from_numpy(vol).to(cuda), g).cpu().numpy()
    ref, _ = oracle_lib.cb_forward(oracle_lib.grid((12, 12, 10)), vol, ang, 60.0, 120.0, 20, 1.5, 0.5, 9, 1.5,
                                   0.5, off=off)
    assert_parity(out, ref)


def test_64cube_90views_full_size_vs_reference(cuda, oracle_lib):
    """The 64^3 workload (64^3 at 2 mm, 10 seeded ellipsoids, 90 views, 128x96
    at 2 mm, source-axis 500 mm, source-detector 1000 mm): forward and
    reference backprojection element-wise against the reference build (or
    the restatement when the build is absent)."""
    vol = nb.ellipsoid_phantom(64, nb.random_ellipsoids(10, 1)).numpy().transpose(2, 1, 0).copy()
    ang = np.linspace(0, 2 * np.pi, 90, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((64, 64, 64), ang, 500.0, 1000.0, 128, 2.0, 96, 2.0, size=(128.0, 128.0, 128.0))
    og = oracle_lib.grid((64, 64, 64), (0, 0, 0), (128.0, 128.0, 128.0))
    out = ops.cb_forward(torch.from_numpy(vol).to(cuda), g).cpu().numpy()
    if oracle_lib.have_ref():
        ref = oracle_lib.ref_cb_forward(og, vol, ang, 500.0, 1000.0, 128, 2.0, 0.5, 96, 2.0, 0.5)
    else:
        ref, _ = oracle_lib.cb_forward(og, vol, ang, 500.0, 1000.0, 128, 2.0, 0.5, 96, 2.0, 0.5, use_cosf=True)
    assert_parity(out, ref)
    sino = np.ascontiguousarray(ref)
    bp = ops.cb_backward(torch.from_numpy(sino).to(cuda), g, _lib.REF_BACKPROJECT).cpu().numpy()
    if oracle_lib.have_ref():
        rb = oracle_lib.ref_cb_backward(og, sino, ang, 500.0, 1000.0, 128, 2.0, 0.5, 96, 2.0, 0.5)
    else:
        rb = oracle_lib.cb_backward(og, sino, ang, 500.0, 1000.0, 128, 2.0, 0.5, 96, 2.0, 0.5, use_cosf=True)
    assert_parity(bp, rb)


def test_lor_pair_vs_fixtures(cuda, golden):
    lors = torch.from_numpy(golden["lor/lors"]).to(cuda)
    vol = torch.from_numpy(golden["lor/vol"]).to(cuda)
    out = ops.lor_forward(lors, vol, (24, 20, 16), size=(48.0, 40.0, 32.0)).cpu().numpy()
    assert_parity(out, golden["lor/fwd"])
    assert np.all(out[:5] == 0)
    vals = torch.from_numpy(golden["lor/vals"]).to(cuda)
    bp = ops.lor_backward(lors, vals, (24, 20, 16), size=(48.0, 40.0, 32.0)).cpu().numpy()
    assert_parity(bp, golden["lor/bp"])


@pytest.mark.parametrize("flags", [_lib.REF_FORWARD, _lib.TIE_GT])
def test_driving_axis_tie(cuda, oracle_lib, flags):
    """Rays with |xd| == |yd| exactly: >= (forward) drives x, > drives y (Q3)."""
    n = 64
    t = np.linspace(-9, 9, n).astype(np.float32)
    lors = np.stack([t - 20, t - 20, np.full(n, 0.7, np.float32), t + 20, t + 20, np.full(n, 3.1, np.float32)])
    lors = np.ascontiguousarray(lors.astype(np.float32))
    vol = np.random.default_rng(1).random((16, 16, 16), dtype=np.float32)
    og = oracle_lib.grid((16, 16, 16), (0, 0, 0), (16.0, 16.0, 16.0))
    oflags = oracle_lib.INV_L2 | (0 if flags & _lib.TIE_GT else oracle_lib.TIE_GE)
    ref, _ = oracle_lib.lor_forward(og, vol, lors, flags=oflags)
    out = ops.lor_forward(torch.from_numpy(lors).to(cuda), torch.from_numpy(vol).to(cuda), (16, 16, 16),
                          flags=flags).cpu().numpy()
    assert_parity(out, ref)


def test_rays_missing_volume_are_zero(cuda):
    g = nb.ConeBeam((16, 16, 16), [0.0, 1.0], 100.0, 200.0, 64, 4.0, 8, 1.0, a_shift=40.0)
    out = ops.cb_forward(torch.ones(g.vol_shape, device=cuda), g)
    assert float(out.abs().max()) == 0.0


def test_linearity_and_adjoint_256cube_360views(cuda):
    """Size-independent properties at the 256^3 / 360-view workload's full size (256^3,
    360 views, 512x384): linearity, and <Ax,y> = <x,A^T y> in float32."""
    ang = np.linspace(0, 2 * np.pi, 360, endpoint=False)
    g = nb.ConeBeam((256, 256, 256), ang, 600.0, 1200.0, 512, 1.2, 384, 1.2, size=(256.0,) * 3)
    gen = torch.Generator(device=cuda).manual_seed(1)
    x = torch.rand(g.vol_shape, device=cuda, generator=gen)
    y = torch.rand(g.sino_shape, device=cuda, generator=gen)
    ax = ops.cb_forward(x, g, _lib.LINE_INTEGRAL)
    a2x = ops.cb_forward(2.0 * x, g, _lib.LINE_INTEGRAL)
    assert float((a2x - 2 * ax).abs().max()) <= 1e-6 * float(ax.abs().max())
    aty = ops.cb_backward(y, g, _lib.LINE_INTEGRAL)
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_adjoint_512cube_720views_normal(cuda):
    """Adjoint dot-product test of the differentiable-projector scan at full size
    (512^3 at 1 mm, 720 views, 1024x768 at 1 mm, SID 700 / SDD 1400 mm) with
    x, y ~ N(0, 1) (seeds 34, 35).  Signed values make both inner products
    sums with cancellation, so float32 rounding shows at ~1e-6 of them."""
    ang = np.linspace(0, 2 * np.pi, 720, endpoint=False)
    g = nb.ConeBeam((512, 512, 512), ang, 700.0, 1400.0, 1024, 1.0, 768, 1.0, size=(512.0,) * 3)
    x = torch.randn(g.vol_shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(34))
    y = torch.randn(g.sino_shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(35))
    lhs = float((ops.cb_forward(x, g).double() * y.double()).sum())
    rhs = float((x.double() * ops.cb_backward(y, g).double()).sum())
    rel = abs(lhs - rhs) / abs(lhs)
    assert rel < 1e-5, (lhs, rhs, rel)
    del x, y
    torch.cuda.empty_cache()


@pytest.mark.parametrize("size", [(40.0, 36.0, 30.0), (40.0, 46.8, 24.0)], ids=["cubic", "anisotropic"])
def test_launch_shapes_give_identical_forward(cuda, size):
    """Launch shapes do not change the per-ray arithmetic: the forward is
    bitwise identical across rows (columns) per CTA, grid orders and the two
    walks (thread per ray, column warps), for cubic voxels and for voxels
    of 1 x 1.3 x 0.8 mm (the walks' division path).  The geometry has a
    partial last row tile (45 rows) and row tiles that straddle the central
    row (z slopes of both signs in one warp); the transpose gets zero rays
    inside a warp.  The transpose agrees to float rounding (atomic summation
    order)."""
    from nefct_b200 import autotune
    g = nb.ConeBeam((40, 36, 30), np.linspace(0, 2 * np.pi, 33, endpoint=False), 150.0, 300.0, 70, 1.3, 45, 1.1,
                    size=size)
    gen = torch.Generator(device=cuda).manual_seed(8)
    vol = torch.rand(g.vol_shape, device=cuda, generator=gen)
    y = torch.rand(g.sino_shape, device=cuda, generator=gen)
    y[3, 10:14] = 0
    y[5, :, 7] = 0
    saved = autotune.current()
    try:
        outs, backs = {}, []
        for rows in (1, 2, 4, 8):
            for order in (0, 1):
                for walk in (0, 3):
                    autotune.apply(rows, order, walk)
                    outs.setdefault(walk, []).append(ops.cb_forward(vol, g).cpu())
                    backs.append(ops.cb_backward(y, g).cpu().double())
        for walk, group in outs.items():
            for i, o in enumerate(group[1:]):
                assert torch.equal(o, group[0]), f"walk {walk} variant {i + 1}"
        assert torch.equal(outs[3][0], outs[0][0])
        for b in backs[1:]:
            assert float((b - backs[0]).norm() / backs[0].norm()) < 1e-6
        rec = autotune.tune_cone_beam(g, 0, cuda, reps=1, use_cache=False)
        assert rec["rows"] in (2, 4, 8) and rec["order"] in (0, 1) and rec["walk"] in (0, 1, 2, 3)
        assert len([k for k in rec["ms"] if k.count("/") == 2]) == 12      # rows x order x walk, both directions
        assert all(f"{k}/fwd" in rec["ms"] and f"{k}/bwd" in rec["ms"] for k in rec["ms"] if k.count("/") == 2)
    finally:
        autotune.apply(saved["rows"], saved["order"], saved["walk"])


@pytest.mark.parametrize("walk", [0, 3])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_walks_vs_reference(cuda, golden, case, walk):
    """Forward and reference backprojection (incl. Q8 for the cylindrical
    case) with both walks against the reference fixtures."""
    from nefct_b200 import autotune
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    saved = autotune.current()
    try:
        autotune.apply(saved["rows"], saved["order"], walk)
        out = ops.cb_forward(torch.from_numpy(golden[f"{name}/vol"]).to(cuda), g).cpu().numpy()
        assert_parity(out, golden[f"{name}/fwd"])
        bp = ops.cb_backward(torch.from_numpy(golden[f"{name}/sino_in"]).to(cuda), g,
                             _lib.REF_BACKPROJECT | (_lib.Q8_INDEX if cyl else 0)).cpu().numpy()
        assert_parity(bp, golden[f"{name}/bp"])
    finally:
        autotune.apply(saved["rows"], saved["order"], saved["walk"])


@pytest.mark.parametrize("flags", [0, _lib.LINE_INTEGRAL, _lib.REF_BACKPROJECT, _lib.NO_TRANSPOSE])
def test_deterministic_transpose_is_bitwise_reproducible(cuda, flags):
    """NEFCT_DETERMINISTIC: 64-bit fixed-point sums give the same bits on
    every run, and agree with the float-atomic transpose to float rounding."""
    g = nb.ConeBeam((48, 40, 36), np.linspace(0, 2 * np.pi, 40, endpoint=False), 140.0, 280.0, 80, 1.2, 60, 1.1,
                    size=(48.0, 40.0, 36.0))
    gen = torch.Generator(device=cuda).manual_seed(21)
    y = torch.randn(g.sino_shape, device=cuda, generator=gen)
    runs = [ops.cb_backward(y, g, flags | _lib.DETERMINISTIC) for _ in range(3)]
    for r in runs[1:]:
        assert torch.equal(r, runs[0])
    # same float contributions as the atomic path; only the summation differs
    assert_parity(runs[0].cpu().numpy(), ops.cb_backward(y, g, flags).cpu().numpy())
    # positive values (no cancellation): within float rounding of FP64 sums
    yp = torch.rand(g.sino_shape, device=cuda, generator=gen)
    det = ops.cb_backward(yp, g, flags | _lib.DETERMINISTIC)
    ref = ops.cb_backward(yp.double(), g, flags).float()
    assert_parity(det.cpu().numpy(), ref.cpu().numpy())


def test_deterministic_autograd_matches_float_path(cuda):
    g = nb.ConeBeam((32, 32, 32), np.linspace(0, 2 * np.pi, 30, endpoint=False), 100.0, 200.0, 48, 1.4, 40, 1.4)
    x = torch.rand(g.vol_shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(3))
    grads = []
    for flags in (0, _lib.DETERMINISTIC):
        xi = x.clone().requires_grad_()
        (nb.project(xi, g, flags) ** 2).sum().backward()
        grads.append(xi.grad)
    assert_parity(grads[1].cpu().numpy(), grads[0].cpu().numpy(), rel=1e-6, mabs=1e-5)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_exact_mode_vs_fp64_exact_oracle(cuda, golden, oracle_lib, case):
    """NEFCT_EXACT (FP64 set-up, FP32 stepping) against the FP64 exact
    Siddon oracle: the FP32 stepping error stays below 1e-5 rel-L2."""
    name, grid, centre, size, cyl, da = case
    g = _geom(case, golden["angles"])
    vol = golden[f"{name}/vol"]
    da32 = float(np.float32(da))        # the geometry travels as float32
    ex = oracle_lib.cb_exact(oracle_lib.grid(grid, centre, size), vol, golden["angles"], SRC_ISO, SRC_DET, NA, da32,
                             AI, NB, DB, BI, cyl=cyl)
    for flags in (_lib.EXACT, _lib.EXACT | _lib.NO_TRANSPOSE):
        out = ops.cb_forward(torch.from_numpy(vol).to(cuda), g, flags).cpu().numpy()
        assert_parity(out, ex)
    out64 = ops.cb_forward(torch.from_numpy(vol.astype(np.float64)).to(cuda), g, _lib.EXACT).cpu().numpy()
    assert_parity(out64, ex, rel=1e-10, mabs=1e-9)


def test_exact_mode_chord_lengths(cuda):
    """Known answer: with plain line integrals of a volume of ones, each ray
    sums the length of its chord through the box."""
    n, s = 10, 20.0
    ang = np.array([0.3, 1.1, 2.0], np.float32)
    g = nb.ConeBeam((n, n, n), ang, 50.0, 100.0, 24, 2.0, 18, 2.0, size=(s, s, s))
    out = ops.cb_forward(torch.ones(g.vol_shape, device=cuda), g, _lib.EXACT | _lib.NO_INV_L2).cpu().numpy()
    # chord of each ray through the box, analytically (slab method in FP64)
    cs, sn = np.cos(ang.astype(np.float64)), np.sin(ang.astype(np.float64))
    for v in range(3):
        for ib in range(18):
            for ia in range(24):
                a = (ia + 0.5) * 2.0 - 24.0
                b = (ib + 0.5) * 2.0 - 18.0
                p1 = np.array([-50 * cs[v], -50 * sn[v], 0.0])
                p2 = np.array([50 * cs[v] - a * sn[v], 50 * sn[v] + a * cs[v], b])
                d = p2 - p1
                t0, t1 = 0.0, 1.0
                for k in range(3):
                    lo, hi = (-s / 2 - p1[k]) / d[k], (s / 2 - p1[k]) / d[k]
                    t0, t1 = max(t0, min(lo, hi)), min(t1, max(lo, hi))
                chord = max(0.0, t1 - t0) * np.linalg.norm(d)
                assert abs(out[v, ib, ia] - chord) <= 2e-5 * s


@pytest.mark.parametrize("flags", [_lib.EXACT, _lib.EXACT | _lib.NO_INV_L2])
def test_exact_mode_adjoint_identity_f64(cuda, flags):
    g = nb.ConeBeam((22, 26, 18), np.linspace(0, 2 * np.pi, 19, endpoint=False) + 0.07, 90.0, 180.0, 40, 1.3, 30,
                    1.2, size=(22.0, 26.0, 18.0), center=(0.4, -0.3, 0.2))
    gen = torch.Generator(device=cuda).manual_seed(9)
    x = torch.randn(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen)
    y = torch.randn(g.sino_shape, dtype=torch.float64, device=cuda, generator=gen)
    lhs = float((ops.cb_forward(x, g, flags) * y).sum())
    rhs = float((x * ops.cb_backward(y, g, flags)).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


# Odd geometries for both walks against the restatement (same per-view trig):
# steep cone (z slope > 1 per slab, z floors jump by 2), odd grid counts,
# a single detector row / column, views on the axes and on the diagonal,
# z offsets that push whole views out of the grid, a 1-voxel-thick grid.
_EDGE = {
    "steep_cone": dict(shape=(20, 20, 20), src_iso=25.0, src_det=50.0, na=24, da=2.0, nb=64, db=3.0),
    "odd_counts": dict(shape=(33, 17, 9), src_iso=90.0, src_det=180.0, na=41, da=1.7, nb=23, db=1.3),
    "one_row": dict(shape=(24, 24, 12), src_iso=80.0, src_det=160.0, na=50, da=1.0, nb=1, db=1.0),
    "one_column": dict(shape=(24, 24, 12), src_iso=80.0, src_det=160.0, na=1, da=1.0, nb=40, db=0.8),
    "thin_grid": dict(shape=(30, 28, 1), src_iso=70.0, src_det=140.0, na=36, da=1.5, nb=9, db=0.4),
}
_EDGE_ANGLES = np.array([0.0, np.pi / 4, np.pi / 2, 0.7, np.pi, 3 * np.pi / 4, 5.5], np.float32)


@pytest.mark.parametrize("walk", [0, 3], ids=["thread-walk", "column-warps"])
@pytest.mark.parametrize("name", sorted(_EDGE))
def test_edge_geometries_vs_restatement(cuda, oracle_lib, name, walk):
    from nefct_b200 import autotune
    e = _EDGE[name]
    off = np.array([0.0, 0.5, -0.5, 40.0, 0.0, -1.0, 0.25], np.float32)      # view 3 mostly misses the grid
    g = nb.ConeBeam(e["shape"], _EDGE_ANGLES, e["src_iso"], e["src_det"], e["na"], e["da"], e["nb"], e["db"],
                    size=tuple(float(v) for v in e["shape"]), z_offsets=off)
    rng = np.random.default_rng(5)
    vol = rng.random(g.vol_shape, dtype=np.float32)
    y = rng.random(g.sino_shape, dtype=np.float32)
    og = oracle_lib.grid(e["shape"], (0, 0, 0), tuple(float(v) for v in e["shape"]))
    args = (_EDGE_ANGLES, e["src_iso"], e["src_det"], e["na"], e["da"], 0.5, e["nb"], e["db"], 0.5)
    ref_f, _ = oracle_lib.cb_forward(og, vol, *args, off=off)
    ref_b = oracle_lib.cb_backward(og, y, *args, off=off, flags=oracle_lib.CB_FWD)
    saved = autotune.current()
    try:
        autotune.apply(saved["rows"], saved["order"], walk)
        out_f = ops.cb_forward(torch.from_numpy(vol).to(cuda), g).cpu().numpy()
        out_b = ops.cb_backward(torch.from_numpy(y).to(cuda), g).cpu().numpy()
    finally:
        autotune.apply(saved["rows"], saved["order"], saved["walk"])
    assert np.abs(ref_f).max() > 0
    assert_parity(out_f, ref_f, rel=1e-6, mabs=1e-5)
    assert_parity(out_b, ref_b, rel=1e-6, mabs=1e-5)
    miss = ref_f == 0                      # rays that miss the grid (the volume has no zero voxel)
    assert miss.any() and float(np.abs(out_f[miss]).max()) == 0.0


def test_lor_ordered_walk_same_results(cuda):
    """The ordered walk of a large unsorted line list returns the unordered
    walk's forward bitwise (same per-line code, results at each line's
    index) and its backward to float rounding; the order is a permutation."""
    rng = np.random.default_rng(31)
    n = 200_000
    p1, p2 = rng.uniform(0, 2 * np.pi, n), rng.uniform(0, 2 * np.pi, n)
    lors = np.stack([40 * np.cos(p1), 40 * np.sin(p1), rng.uniform(-15, 15, n),
                     40 * np.cos(p2), 40 * np.sin(p2), rng.uniform(-15, 15, n)]).astype(np.float32)
    lors[:, :7] = np.array([[0, 0, 0, 3, 0, 0]], np.float32).T          # short lines (Q4)
    d_lors = torch.from_numpy(lors).to(cuda)
    vol = torch.rand((20, 24, 28), device=cuda, generator=torch.Generator(device=cuda).manual_seed(3))
    vals = torch.rand(n, device=cuda, generator=torch.Generator(device=cuda).manual_seed(4))
    shape, size = (28, 24, 20), (56.0, 48.0, 40.0)
    order = ops.lor_order(d_lors, shape, size=size)
    assert order.dtype == torch.int32 and torch.equal(torch.sort(order.long()).values, torch.arange(n, device=cuda))
    f0 = ops.lor_forward(d_lors, vol, shape, size=size)
    f1 = ops.lor_forward(d_lors, vol, shape, size=size, order=order)
    assert torch.equal(f0, f1)
    b0 = ops.lor_backward(d_lors, vals, shape, size=size).double()
    b1 = ops.lor_backward(d_lors, vals, shape, size=size, order=order).double()
    assert float((b1 - b0).norm() / b0.norm()) < 1e-6


@pytest.mark.parametrize("flags", [0, _lib.REF_BACKPROJECT])
def test_deterministic_transpose_same_bits_in_both_walks(cuda, flags):
    """The column warps reduce the same per-contribution fixed-point integers
    as the thread walk: the deterministic transposes agree bit for bit."""
    from nefct_b200 import autotune
    g = nb.ConeBeam((36, 30, 26), np.linspace(0, 2 * np.pi, 21, endpoint=False) + 0.1, 110.0, 230.0, 66, 1.2, 41,
                    1.1, size=(36.0, 30.0, 26.0), z_offsets=np.linspace(-1, 1, 21))
    y = torch.randn(g.sino_shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(12))
    saved = autotune.current()
    outs = []
    try:
        for walk in (0, 3):
            autotune.apply(saved["rows"], saved["order"], walk)
            outs.append(ops.cb_backward(y, g, flags | _lib.DETERMINISTIC).cpu())
    finally:
        autotune.apply(saved["rows"], saved["order"], saved["walk"])
    assert torch.equal(outs[0], outs[1])
    assert float(outs[0].abs().max()) > 0


def test_forward_transpose_capture_in_cuda_graph(cuda):
    """The single-problem forward and transpose (column warps: copies,
    memsets, kernels, folds; per-view tables in kernel parameters) record
    into a CUDA graph and replay to the eager results."""
    g = nb.ConeBeam((48, 40, 32), np.linspace(0, 2 * np.pi, 30, endpoint=False), 120.0, 240.0, 64, 1.2, 40, 1.1,
                    size=(48.0, 40.0, 32.0))
    gen = torch.Generator(device=cuda).manual_seed(77)
    vol = torch.rand(g.vol_shape, device=cuda, generator=gen)
    y = torch.rand(g.sino_shape, device=cuda, generator=gen)
    sino = torch.empty(g.sino_shape, device=cuda)
    back = torch.empty(g.vol_shape, device=cuda)
    ref_s, ref_b = ops.cb_forward(vol, g), ops.cb_backward(y, g)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):                       # warm-up outside the capture
        ops.cb_forward(vol, g, out=sino)
        ops.cb_backward(y, g, out=back)
    torch.cuda.current_stream().wait_stream(s)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        ops.cb_forward(vol, g, out=sino)
        ops.cb_backward(y, g, out=back)
    sino.zero_()
    back.fill_(float("nan"))
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(sino, ref_s)
    assert_parity(back.cpu().numpy(), ref_b.cpu().numpy(), rel=1e-6, mabs=1e-5)


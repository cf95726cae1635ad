"""GPU parity of the distance-driven FDK backprojection (dist_3d_back_fdk)."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import ops
from tests.golden.make_golden import (DD_AI, DD_BI, DD_DA, DD_DA_CYL, DD_DB, DD_GRID, DD_NA, DD_NB, DD_SAD,
                                      DD_SID)
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_dd_vs_reference_fixtures(cuda, golden, cyl):
    """Against the reference's own kernel (host build), which evaluates the
    view and detector-angle trigonometry with cosf/sinf (here: the
    double-precision functions, rounded)."""
    key, da = ("dd/cyl", DD_DA_CYL) if cyl else ("dd/flat", DD_DA)
    proj = torch.from_numpy(golden["dd/proj"]).to(cuda)
    out = ops.dd_backproject(proj, DD_GRID, golden["angles"], DD_SAD, DD_SID, da, DD_DB, DD_AI, DD_BI,
                             "cyl" if cyl else "flat", golden["dd/off"])
    assert_parity(out.cpu().numpy(), golden[key])


@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_dd_vs_restatement_tight(cuda, oracle_lib, cyl):
    """Same trigonometry as the restatement: only the summation order of the
    reductions differs.  Views on both sides of the 45-degree switch of the
    driving axis, z offsets, a partial row tile (45 rows) and zero bins."""
    rng = np.random.default_rng(23)
    shape, na, nbins = (30, 26, 20), 37, 45
    ang = np.array([0.2, np.pi / 4 - 2e-3, np.pi / 4 + 2e-3, 1.9, 3.3, 5.0], np.float32)
    proj = rng.random((ang.size, nbins, na), dtype=np.float32)
    proj[2, 5:9] = 0
    off = rng.uniform(-2, 2, ang.size).astype(np.float32)
    sad, sid, da = 70.0, 150.0, (0.009 if cyl else 1.1)
    ref = oracle_lib.dd_backproject(proj, ang, shape, sid, sad, na, da, 0.2, nbins, 1.05, -0.3, cyl=cyl, off=off,
                                    use_cosf=False)
    out = ops.dd_backproject(torch.from_numpy(proj).to(cuda), shape, ang, sad, sid, da, 1.05, 0.2, -0.3,
                             "cyl" if cyl else "flat", off).cpu().numpy()
    assert_parity(out, ref, rel=1e-6, mabs=1e-5)


def test_dd_op_mirror_accumulates(cuda, golden):
    """back_project_flat_fdk_gpu adds into the caller's image, as the
    reference's host function does."""
    proj = torch.from_numpy(golden["dd/proj"]).to(cuda)
    nx, ny, nz = DD_GRID
    image = torch.ones((nx, ny, nz), device=cuda)
    out = nb.cc.distance_3d.back_project_flat_fdk_gpu(proj, DD_GRID, golden["dd/off"], golden["angles"],
                                                      proj.shape[0], DD_SID, DD_SAD, DD_DA, DD_AI, DD_NA, DD_DB,
                                                      DD_BI, DD_NB, image)
    assert out is image
    assert_parity(out.cpu().numpy().reshape(nz, ny, nx) - 1.0, golden["dd/flat"], rel=1e-5, mabs=1e-4)


def _dd_geom(cyl, nv=7, seed=0):
    rng = np.random.default_rng(seed)
    ang = np.array([0.2, np.pi / 4 - 2e-3, np.pi / 4 + 2e-3, 1.9, 3.3, 4.1, 5.0], np.float32)[:nv]
    return ops.DDGeometry((26, 22, 18), ang, 70.0, 150.0, 33, 0.009 if cyl else 1.1, 41, 1.05, 0.2, -0.3,
                          "cyl" if cyl else "flat", rng.uniform(-2, 2, ang.size).astype(np.float32))


@pytest.mark.parametrize("flags", [0, nb._lib.FDK_NO_WEIGHT], ids=["fdk-weight", "line-integral"])
@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_dd_pair_adjoint_identity_f64(cuda, cyl, flags):
    """<A x, y> = <x, A^T y> to rounding in FP64: the distance-driven forward
    is the exact transpose of the backprojection with the same flags (views
    on both sides of the 45-degree switch of the driving axis, z offsets,
    a partial row tile)."""
    g = _dd_geom(cyl)
    gen = torch.Generator(device=cuda).manual_seed(3)
    x = torch.randn(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen)
    y = torch.randn(g.proj_shape, dtype=torch.float64, device=cuda, generator=gen)
    lhs = float((ops.dd_forward(x, g, flags) * y).sum())
    rhs = float((x * ops.dd_backward(y, g, flags)).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0), (lhs, rhs)


@pytest.mark.parametrize("flags", [0, nb._lib.FDK_NO_WEIGHT], ids=["fdk-weight", "line-integral"])
def test_dd_float_pair_vs_f64(cuda, flags):
    """The float32 pair against its FP64 build (same footprints; weights
    rounded in float32, reciprocals approximate), and the float32 adjoint
    identity; dd_backward with flags 0 is the reference's FDK
    backprojection (nefct_dd_backproject)."""
    g = _dd_geom(False)
    gen = torch.Generator(device=cuda).manual_seed(4)
    x = torch.rand(g.vol_shape, device=cuda, generator=gen)
    y = torch.rand(g.proj_shape, device=cuda, generator=gen)
    fx = ops.dd_forward(x, g, flags)
    by = ops.dd_backward(y, g, flags)
    assert_parity(fx.cpu().numpy(), ops.dd_forward(x.double(), g, flags).cpu().numpy(), rel=1e-6, mabs=1e-5)
    assert_parity(by.cpu().numpy(), ops.dd_backward(y.double(), g, flags).cpu().numpy(), rel=1e-6, mabs=1e-5)
    lhs, rhs = float((fx.double() * y.double()).sum()), float((x.double() * by.double()).sum())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)
    if flags == 0:
        ref = ops.dd_backproject(y, g.shape, g.angles, g.src_iso, g.src_det, g.da, g.db, g.a_offset, g.b_offset,
                                 g.det_kind, g.z_offsets)
        assert_parity(by.cpu().numpy(), ref.cpu().numpy(), rel=1e-6, mabs=1e-5)


def test_dd_line_integrals_of_ones_are_chords(cuda):
    """Known answer: without the FDK weight, a bin whose footprints lie
    inside the grid sums (overlap fractions, which add to one per slab) x
    |p2 - p1| / |driving component| over the slabs, i.e. the length of its
    central ray's chord through the box."""
    n = 40
    ang = np.array([0.3, 1.0, 2.6], np.float32)
    g = ops.DDGeometry((n, n, n), ang, 200.0, 400.0, 16, 1.0, 12, 1.0)
    out = ops.dd_forward(torch.ones(g.vol_shape, dtype=torch.float64, device=cuda), g,
                         nb._lib.FDK_NO_WEIGHT).cpu().numpy()
    for v, a in enumerate(ang.astype(np.float64)):
        cs, sn = np.cos(a), np.sin(a)
        for ib in range(12):
            for ia in range(16):
                u = (ia + 0.5) * 1.0 - 8.0
                w = (ib + 0.5) * 1.0 - 6.0
                p1 = np.array([-200.0 * cs, -200.0 * sn, 0.0])
                p2 = np.array([200.0 * cs - u * sn, 200.0 * sn + u * cs, w])
                d = p2 - p1
                t0, t1 = 0.0, 1.0
                for k in range(3):
                    lo, hi = (-n / 2 - p1[k]) / d[k], (n / 2 - p1[k]) / d[k]
                    t0, t1 = max(t0, min(lo, hi)), min(t1, max(lo, hi))
                chord = max(0.0, t1 - t0) * np.linalg.norm(d)
                assert abs(out[v, ib, ia] - chord) <= 0.03 * chord, (v, ib, ia, out[v, ib, ia], chord)


def test_dd_autograd_finite_difference_f64(cuda):
    """loss = ||A x - b||^2 through ops.dd_project (backward = dd_backward):
    autograd against a central difference in FP64 (exact for a quadratic)."""
    g = _dd_geom(False, seed=5)
    gen = torch.Generator(device=cuda).manual_seed(6)
    x = torch.rand(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen).requires_grad_()
    b = torch.rand(g.proj_shape, dtype=torch.float64, device=cuda, generator=gen)
    d = torch.randn(g.vol_shape, dtype=torch.float64, device=cuda, generator=gen)
    loss = ((ops.dd_project(x, g) - b) ** 2).sum()
    loss.backward()
    h = 0.5
    with torch.no_grad():
        fp = ((ops.dd_forward(x + h * d, g) - b) ** 2).sum()
        fm = ((ops.dd_forward(x - h * d, g) - b) ** 2).sum()
    fd = float((fp - fm) / (2 * h))
    an = float((x.grad * d).sum())
    assert abs(fd - an) <= 1e-9 * abs(an) + 1e-13 * float(loss) / h


def test_dd_project_op_mirror(cuda):
    """cc.distance_3d.project_flat_three with the keyword attrs of
    nefct/functions/project.py:79-97 returns [nv, nb, na] line integrals of
    the distance-driven forward (no FDK weight)."""
    shape, na, nbins = (24, 20, 16), 30, 18
    ang = np.linspace(0, 2 * np.pi, 9, endpoint=False).astype(np.float32)
    vol = torch.rand((16, 20, 24), device=cuda, generator=torch.Generator(device=cuda).manual_seed(2))
    out = nb.cc.distance_3d.project_flat_three(vol, shape=shape, offsets=[0.0] * 9, angles=list(ang), SID=160.0,
                                               SAD=80.0, na=na, da=1.2, ai=0.1, nb=nbins, db=1.1, bi=-0.2)
    g = ops.DDGeometry(shape, ang, 80.0, 160.0, na, 1.2, nbins, 1.1, 0.1, -0.2)
    assert out.shape == (9, nbins, na)
    assert torch.equal(out, ops.dd_forward(vol, g, nb._lib.FDK_NO_WEIGHT))

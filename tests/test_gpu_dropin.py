"""GPU: the drop-in operators with the reference's call signatures."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib, ops
from tests.golden.make_golden import AI, BI, DB, NA, NB, SRC_DET, SRC_ISO
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


def _scanner(mode="flat"):
    return nb.ScannerConfig3D(mode, 800.0, 400.0, nb.DetectorDirectAConfig(96, 192.0),
                              nb.DetectorDirectBConfig(64, 128.0))


def test_project3d_numpy_roundtrip_vs_oracle(cuda, oracle_lib):
    sc = _scanner()
    data = nb.phantom(32) * 1.0                     # [x, y, z]
    img = nb.Image3D(data, [0, 0, 0], [64.0, 64.0, 64.0])
    ang = np.linspace(0, 2 * np.pi, 30, endpoint=False).astype(np.float32)
    proj = nb.Project3D(sc, ang, None)(img)
    assert isinstance(proj.data, np.ndarray) and proj.data.shape == (96, 64, 30)
    og = oracle_lib.grid((32, 32, 32), (0, 0, 0), (64.0, 64.0, 64.0))
    ref, _ = oracle_lib.cb_forward(og, np.ascontiguousarray(data.transpose()), ang, 400.0, 800.0, 96, 2.0, 0.5,
                                   64, 2.0, 0.5)
    assert_parity(proj.data, ref.transpose())


def test_backproject3d_modes(cuda):
    sc = _scanner()
    ang = np.linspace(0, 2 * np.pi, 20, endpoint=False).astype(np.float32)
    p = nb.ProjectionSequence3D(np.random.default_rng(1).random((96, 64, 20), dtype=np.float32), sc, ang)
    b_ref = nb.BackProject3D(sc, [32, 32, 32], 2.0)(p)
    b_tr = nb.BackProject3D(sc, [32, 32, 32], 2.0, "transpose")(p)
    assert b_ref.data.shape == (32, 32, 32) and b_ref.size == [64.0, 64.0, 64.0]
    # the reference backprojection lacks the 1/L^2 of the transpose (Q2)
    assert float(b_ref.data.sum()) > 1e3 * float(b_tr.data.sum())


def test_project3d_device_tensors_stay_on_device(cuda):
    sc = _scanner()
    img = nb.Image3D(torch.rand(32, 32, 32, device=cuda), [0, 0, 0], [64.0] * 3)
    proj = nb.Project3D(sc, np.linspace(0, 3, 10), None, "line")(img)
    assert proj.data.is_cuda and tuple(proj.data.shape) == (96, 64, 10)


def test_sart_reduces_residual(cuda):
    sc = _scanner()
    ang = np.linspace(0, 2 * np.pi, 40, endpoint=False).astype(np.float32)
    x_true = nb.Image3D(torch.from_numpy(nb.phantom(32)).to(cuda), [0, 0, 0], [64.0] * 3)
    fwd = nb.Project3D(sc, ang, None, "line")
    bwd = nb.BackProject3D(sc, [32, 32, 32], 2.0, "line")
    p = fwd(x_true)
    ones = p.update(data=torch.ones_like(p.data))
    emap = bwd(ones)
    # the reference's SART (sart.py:29-39) normalises by the column sums only,
    # so the step must absorb the row sums (ray lengths)
    lam = 1.0 / float(fwd(x_true.update(data=torch.ones_like(x_true.data))).data.max())
    r = [float(p.data.norm())]
    x = None
    for _ in range(4):
        x = nb.SART(5, lam, emap, fwd, bwd)(p, x)
        r.append(float((p - fwd(x)).data.norm()))
    assert all(b < a for a, b in zip(r, r[1:])), r
    assert r[-1] < 0.5 * r[0], r


def test_project3dt_with_warp_deformer_matches_manual(cuda):
    sc = _scanner()
    ang = np.linspace(0, 2 * np.pi, 12, endpoint=False).astype(np.float32)
    ts = np.repeat([0.0, 1.0, 2.0], 4)
    shape = (24, 24, 24)
    rng = np.random.default_rng(2)
    fields = {t: [rng.uniform(-2, 2, shape).astype(np.float32) for _ in range(3)] for t in (1.0, 2.0)}
    deformer = nb.WarpDeformer(fields)
    img = nb.Image3D(rng.random(shape, dtype=np.float32), [0, 0, 0], [48.0] * 3)
    out = nb.Project3DT(sc, ang, None, ts, deformer)(img)
    for t in (0.0, 1.0, 2.0):
        idx = np.nonzero(ts == t)[0]
        warped = deformer(img, t)
        ref = nb.Project3D(sc, ang[idx], None)(warped)
        np.testing.assert_allclose(out.data[:, :, idx], ref.data, rtol=1e-6, atol=1e-9)


def test_op_mirrors_reproduce_quirks(cuda, golden):
    """ProjectFlat passes da as the row pitch (Q7); BackProjectCyli reads the
    sinogram transposed (Q8) -- both as the TensorFlow ops do."""
    name, grid, centre, size = "cyl_iso", (24, 20, 16), (0.5, 0.5, -1.0), (48.0, 40.0, 32.0)
    sino = torch.from_numpy(golden[f"{name}/sino_in"]).to(cuda)
    out = nb.cc.siddon_3d.back_project_cyli(sino, grid, centre, size, golden["angles"], SRC_ISO, SRC_DET, NA,
                                            0.012, AI, NB, DB, BI, *grid)
    assert_parity(out.reshape(16, 20, 24).cpu().numpy(), golden[f"{name}/bp"])
    vol = torch.from_numpy(golden["flat_iso/vol"]).to(cuda)
    a = nb.cc.siddon_3d.project_flat(vol, (24, 20, 16), (1.0, -0.5, 0.25), (48.0, 40.0, 32.0), golden["angles"],
                                     SRC_ISO, SRC_DET, NA, 2.5, AI, NB, 9.0, BI)
    g = nb.ConeBeam((24, 20, 16), golden["angles"], SRC_ISO, SRC_DET, NA, 2.5, NB, 2.5, AI, BI,
                    (1.0, -0.5, 0.25), (48.0, 40.0, 32.0))
    np.testing.assert_array_equal(a.cpu().numpy(), ops.cb_forward(vol, g).cpu().numpy())


def test_lor_op_mirrors_order_long_lists(cuda):
    """The Projection / Backprojection mirrors walk lists of >= 2^20 lines in
    lor_order: the forward equals the list-order walk bit for bit, the
    backprojection to float rounding (summation order of the reductions)."""
    n, shape, size = (1 << 20) + 4097, (32, 28, 24), (64.0, 56.0, 48.0)
    gen = torch.Generator(device=cuda).manual_seed(12)
    ang = torch.rand(2, n, device=cuda, generator=gen) * (2 * np.pi)
    zz = (torch.rand(2, n, device=cuda, generator=gen) - 0.5) * 60.0
    lors = torch.stack([50.0 * torch.cos(ang[0]), 50.0 * torch.sin(ang[0]), zz[0],
                        50.0 * torch.cos(ang[1]), 50.0 * torch.sin(ang[1]), zz[1]]).contiguous()
    image = torch.rand(shape, device=cuda, generator=gen)          # [nx, ny, nz] of the TF op
    vals = torch.rand(n, device=cuda, generator=gen)
    center = (0.0, 0.0, 0.0)
    a = nb.cc.siddon.projection(lors, image, shape, center, size)
    a0 = ops.lor_forward(lors, image.contiguous().view(24, 28, 32), shape, center, size, _lib.LOR_REF_FORWARD)
    assert torch.equal(a, a0)
    b = nb.cc.siddon.backprojection(image, lors, vals, shape, center, size).double()
    b0 = ops.lor_backward(lors, vals, shape, center, size, _lib.LOR_REF_BACKPROJECT).view(image.shape).double()
    assert float((b - b0).norm() / b0.norm()) < 1e-6


def test_empty_and_degenerate_inputs(cuda):
    """An empty LOR list gives an empty forward and a zero backprojection; a
    zero sinogram transposes to an exactly zero volume; a one-voxel grid seen
    by a 1 x 1 detector in one view projects and transposes consistently."""
    from nefct_b200 import ops
    vol = torch.rand((8, 8, 8), device=cuda)
    lors = torch.empty((6, 0), device=cuda)
    assert ops.lor_forward(lors, vol, (8, 8, 8)).numel() == 0
    bp = ops.lor_backward(lors, torch.empty(0, device=cuda), (8, 8, 8))
    assert bp.shape == (8, 8, 8) and float(bp.abs().max()) == 0.0
    g = nb.ConeBeam((8, 8, 8), np.linspace(0, 2 * np.pi, 7, endpoint=False), 40.0, 80.0, 12, 1.0, 10, 1.0)
    back = ops.cb_backward(torch.zeros(g.sino_shape, device=cuda), g)
    assert float(back.abs().max()) == 0.0
    g1 = nb.ConeBeam((1, 1, 1), [0.3], 40.0, 80.0, 1, 2.0, 1, 2.0, size=(1.0, 1.0, 1.0))
    x = torch.full((1, 1, 1), 3.0, device=cuda)
    y = torch.full((1, 1, 1), 2.0, device=cuda)
    ax = ops.cb_forward(x, g1)
    aty = ops.cb_backward(y, g1)
    assert float(ax) > 0
    assert abs(float((ax * y).sum()) - float((x * aty).sum())) <= 1e-6 * float((ax * y).sum())

"""GPU parity at the benchmarked scans' full sizes, element-wise on view
subsets, against the reference's own projector code built for the host
(oracle/_ref; the oracle restatement when that build is absent).

* the FDK scanner (256^3 at 1 mm, 30 ellipsoids, 360 views, 512 x 384 at
  1.2 mm, 600 / 1200 mm) and the differentiable-projector scan (512^3 at
  1 mm, 50 ellipsoids, 720 views, 1024 x 768 at 1 mm, 700 / 1400 mm): the
  forward of sampled views and the reference backprojection of the
  reference's own sinogram, rel-L2 <= 1e-5 and max-abs <= 1e-4 x max; the
  forward's error against the oracle's FP64 walk is stated;
* the autograd gradient (the hand-written exact transpose) against the
  reference's own backprojector: the reference's forward weights carry
  1 / L^2 and its backprojection does not (siddon.cu.cc:86 vs :526), so
  A^T y = BP_ref(y / L^2), with L the ray length in voxels, for rays that
  are neither exactly diagonal nor short;
* the distance-driven FDK backprojection and the trilinear warp at the FDK
  scanner's and the motion workload's sizes.
"""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib, ops

pytestmark = pytest.mark.gpu

SCANS = {
    "fdk_scanner": dict(n=256, ell=30, seed=2, nv=360, na=512, nb=384, px=1.2, si=600.0, sd=1200.0,
                        views=[0, 37, 95, 180, 241, 333]),
    "diff_projector": dict(n=512, ell=50, seed=3, nv=720, na=1024, nb=768, px=1.0, si=700.0, sd=1400.0,
                           views=[13, 250, 431, 690]),
}


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.abs(a - b).max() / np.abs(b).max())


def ref_forward(oracle_lib, og, vol, ang, args):
    if oracle_lib.have_ref():
        return oracle_lib.ref_cb_forward(og, vol, ang, *args)
    return oracle_lib.cb_forward(og, vol, ang, *args, use_cosf=True)[0]


def ref_backproject(oracle_lib, og, sino, ang, args, atomic):
    if oracle_lib.have_ref():
        return oracle_lib.ref_cb_backward(og, sino, ang, *args, atomic=atomic)
    return oracle_lib.cb_backward(og, sino, ang, *args, use_cosf=True)


@pytest.mark.parametrize("name", sorted(SCANS))
def test_scan_view_subset_vs_reference(cuda, oracle_lib, name):
    s = SCANS[name]
    n = s["n"]
    ang_all = np.linspace(0, 2 * np.pi, s["nv"], endpoint=False).astype(np.float32)
    ang = ang_all[s["views"]]
    g = nb.ConeBeam((n, n, n), ang_all, s["si"], s["sd"], s["na"], s["px"], s["nb"], s["px"],
                    size=(float(n),) * 3).subset(s["views"])
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(s["ell"], s["seed"]), device=cuda).permute(2, 1, 0)
    vol = vol.contiguous()
    og = oracle_lib.grid((n, n, n), (0, 0, 0), (float(n),) * 3)
    args = (s["si"], s["sd"], s["na"], s["px"], 0.5, s["nb"], s["px"], 0.5)
    vol_np = vol.cpu().numpy()
    ref_s = ref_forward(oracle_lib, og, vol_np, ang, args)
    out_s = ops.cb_forward(vol, g, 0).cpu().numpy()
    r, m = rel(out_s, ref_s)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    # stated: the float32 forward against the oracle's FP64 walk of the same views
    f64, _ = oracle_lib.cb_forward(og, vol_np, ang, *args, f64=True)
    r64, _ = rel(out_s, f64)
    rr64, _ = rel(ref_s, f64)
    assert r64 <= 1e-5 and r64 <= 10 * rr64 + 1e-6, (r64, rr64)
    del vol
    ref_b = ref_backproject(oracle_lib, og, ref_s, ang, args, atomic=n > 256)
    out_b = ops.cb_backward(torch.from_numpy(ref_s).to(cuda), g, _lib.REF_BACKPROJECT).cpu().numpy()
    r, m = rel(out_b, ref_b)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    torch.cuda.empty_cache()


def test_autograd_gradient_vs_reference_backprojector(cuda, oracle_lib):
    """The 64^3 workload (64^3 at 2 mm, 90 views, 128 x 96 at 2 mm, 500 /
    1000 mm) with the views offset by 0.01 rad (no exactly diagonal rays):
    d/dx sum(A(x) * y) from autograd against BP_ref(y / L^2)."""
    n, nv, na, nbr, px, si, sd, vox = 64, 90, 128, 96, 2.0, 500.0, 1000.0, 2.0
    ang = (np.linspace(0, 2 * np.pi, nv, endpoint=False) + 0.01).astype(np.float32)
    g = nb.ConeBeam((n, n, n), ang, si, sd, na, px, nbr, px, size=(n * vox,) * 3)
    gen = torch.Generator(device=cuda).manual_seed(41)
    x = torch.rand(g.vol_shape, device=cuda, generator=gen).requires_grad_()
    y = torch.rand(g.sino_shape, device=cuda, generator=gen) + 0.5
    (nb.project(x, g) * y).sum().backward()
    grad = x.grad.cpu().numpy()
    # L^2 of each ray in voxel units: |p2 - p1|^2 = SDD^2 + a^2 + b^2 (flat detector)
    a = (np.arange(na) + 0.5) * px - na * px / 2
    b = (np.arange(nbr) + 0.5) * px - nbr * px / 2
    L2 = (sd ** 2 + a[None, :] ** 2 + b[:, None] ** 2) / vox ** 2
    yl = (y.cpu().numpy().astype(np.float64) / L2[None]).astype(np.float32)
    og = oracle_lib.grid((n, n, n), (0, 0, 0), (n * vox,) * 3)
    ref = ref_backproject(oracle_lib, og, yl, ang, (si, sd, na, px, 0.5, nbr, px, 0.5), atomic=False)
    r, m = rel(grad, ref)
    assert r <= 1e-5 and m <= 1e-4, (r, m)


def test_distance_driven_full_size_vs_reference(cuda, oracle_lib):
    """The distance-driven FDK backprojection at the FDK scanner's size
    (256^3, 512 x 384 bins of 1.2 voxels, 600 / 1200 voxels), 8 views,
    against the reference's dist_3d_back_fdk kernel built for the host."""
    if not oracle_lib.have_ref():
        pytest.skip("the reference's host build is absent")
    n, na, nbr, px, sad, sid = 256, 512, 384, 1.2, 600.0, 1200.0
    ang = (np.linspace(0, 2 * np.pi, 8, endpoint=False) + 0.3).astype(np.float32)
    proj = torch.rand((8, nbr, na), device=cuda, generator=torch.Generator(device=cuda).manual_seed(5))
    ours = ops.dd_backproject(proj, (n, n, n), ang, sad, sid, px, px).cpu().numpy()
    ref = oracle_lib.ref_dd_backproject(proj.cpu().numpy(), ang, (n, n, n), sid, sad, na, px, 0.0, nbr, px, 0.0)
    r, m = rel(ours, ref)
    assert r <= 1e-5 and m <= 1e-4, (r, m)


def test_warp_full_size_vs_reference(cuda, oracle_lib):
    """The trilinear warp at the motion workload's size (256^3, a field of
    four sinusoids per component up to 5 voxels) against the reference's
    DeformKernel built for the host."""
    if not oracle_lib.have_ref():
        pytest.skip("the reference's host build is absent")
    n = 256
    gen = torch.Generator(device=cuda).manual_seed(5)
    img = torch.rand((n, n, n), device=cuda, generator=gen)
    z, y, x = torch.meshgrid(*[torch.arange(n, device=cuda, dtype=torch.float32)] * 3, indexing="ij")
    rng = np.random.default_rng(5)
    m = []
    for _ in range(3):
        f = torch.zeros_like(img)
        for _ in range(4):
            k, ph = rng.uniform(0.5, 3, 3) * 2 * np.pi / n, rng.uniform(0, 2 * np.pi)
            f += 1.25 * torch.sin(float(k[0]) * x + float(k[1]) * y + float(k[2]) * z + float(ph))
        m.append(f.contiguous())
    ours = ops.warp_forward(img, *m).cpu().numpy()
    ref = oracle_lib.ref_deform(img.cpu().numpy(), *[a.cpu().numpy() for a in m])
    r, mx = rel(ours, ref)
    assert r <= 1e-5 and mx <= 1e-4, (r, mx)

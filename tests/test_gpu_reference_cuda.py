"""GPU: the library against the reference's own CUDA kernels, built
unchanged by nvcc from the reference sources (oracle/_ref/libnefct_ref_gpu.so:
siddon_3d's ProjectFlatKernel / BackProjectFlatKernel, pixel_3d's
BackProjectFlatKernel, cpp/siddon's ProjectKernel / BackProjectKernel and
dist_3d_back_fdk's back_project_fdk_kernel and cpp/deform's DeformKernel
with their host launchers) and run on the same GPU.

* parity: the library's outputs against the reference's CUDA kernels,
  element-wise (rel-L2 <= 1e-5, max-abs <= 1e-4 x max): the cone-beam pair on
  the 64^3 workload at full size and on views of the 512^3 scan, the
  voxel-driven and the distance-driven backprojections on the FDK scanner,
  the LOR pair on 1 Mi ring lines, the warp at 256^3;
* speed: each reference launch beside the library's call for the same work,
  both timed with CUDA events after a warm-up call, the fastest of three
  (printed with -s).
"""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib, ops

pytestmark = [pytest.mark.gpu, pytest.mark.skipif("not __import__('oracle').have_ref_gpu()")]


def rel(a, b):
    a, b = a.double(), b.double()
    return float((a - b).norm() / b.norm()), float((a - b).abs().max() / b.abs().max())


def _events(fn, reps=3):
    """fn's output and its fastest of `reps` timed calls (after a warm-up)."""
    fn()                                      # warm-up (allocations, first launch)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return out, best


def test_reference_cuda_kernels_64cube(cuda, oracle_lib):
    """The 64^3 workload (64^3 at 2 mm, 10 ellipsoids, 90 views, 128 x 96 at
    2 mm, 500 / 1000 mm), every view."""
    n, nv, na, nbr, px, si, sd, vox = 64, 90, 128, 96, 2.0, 500.0, 1000.0, 2.0
    ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    g = nb.ConeBeam((n, n, n), ang, si, sd, na, px, nbr, px, size=(n * vox,) * 3)
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(10, 1), device=cuda).permute(2, 1, 0).contiguous()
    og = oracle_lib.grid((n, n, n), (0, 0, 0), (n * vox,) * 3)
    d_ang = torch.from_numpy(ang).to(cuda)
    args = (si, sd, na, px, 0.5, nbr, px, 0.5)
    ref_s = oracle_lib.ref_gpu_cb(True, og, vol, d_ang, *args)
    r, m = rel(ops.cb_forward(vol, g, 0), ref_s)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    ref_b = oracle_lib.ref_gpu_cb(False, og, ref_s, d_ang, *args)
    r, m = rel(ops.cb_backward(ref_s, g, _lib.REF_BACKPROJECT), ref_b)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    if oracle_lib.have_ref():
        # the same reference code built for the host: device vs host math only
        host = torch.from_numpy(oracle_lib.ref_cb_forward(og, vol.cpu().numpy(), ang, *args)).to(cuda)
        r, _ = rel(ref_s, host)
        assert r <= 1e-5, r


def test_reference_cuda_kernels_512cube_speed(cuda, oracle_lib):
    """72 of the 720 views (every 10th) of the 512^3 scan (512^3 at 1 mm, 50
    ellipsoids, 1024 x 768 at 1 mm, 700 / 1400 mm): parity, and the time of
    the reference's CUDA forward + backprojection against the library's
    forward + exact transpose on the same views."""
    n, na, nbr, px, si, sd = 512, 1024, 768, 1.0, 700.0, 1400.0
    ang_all = np.linspace(0, 2 * np.pi, 720, endpoint=False).astype(np.float32)
    views = list(range(0, 720, 10))
    ang = ang_all[views]
    g = nb.ConeBeam((n, n, n), ang_all, si, sd, na, px, nbr, px, size=(float(n),) * 3).subset(views)
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(50, 3), device=cuda).permute(2, 1, 0).contiguous()
    og = oracle_lib.grid((n, n, n), (0, 0, 0), (float(n),) * 3)
    d_ang = torch.from_numpy(ang).to(cuda)
    args = (si, sd, na, px, 0.5, nbr, px, 0.5)
    ref_s, t_ref_f = _events(lambda: oracle_lib.ref_gpu_cb(True, og, vol, d_ang, *args))
    out_s, t_f = _events(lambda: ops.cb_forward(vol, g, 0))
    r, m = rel(out_s, ref_s)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    del out_s
    ref_b, t_ref_b = _events(lambda: oracle_lib.ref_gpu_cb(False, og, ref_s, d_ang, *args))
    out_b = ops.cb_backward(ref_s, g, _lib.REF_BACKPROJECT)
    r, m = rel(out_b, ref_b)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    del out_b, ref_b
    _, t_b = _events(lambda: ops.cb_backward(ref_s, g, 0))          # the exact transpose
    print(f"\n512^3, 72 views: reference CUDA forward {t_ref_f:.1f} ms, backprojection {t_ref_b:.1f} ms; "
          f"library forward {t_f:.1f} ms, transpose {t_b:.1f} ms; "
          f"speed-up {(t_ref_f + t_ref_b) / (t_f + t_b):.2f}x (forward {t_ref_f / t_f:.2f}x, "
          f"backprojection {t_ref_b / t_b:.2f}x)")
    assert t_f < t_ref_f and t_b < t_ref_b
    torch.cuda.empty_cache()


def test_reference_cuda_pixel_backprojection_fdk_scanner(cuda, oracle_lib):
    """pixel_3d's voxel-driven backprojection (the FDK body without its
    distance weight) on the FDK scanner: 256^3 at 1 mm, 360 views of 512 x
    384 at 1.2 mm, 600 / 1200 mm.  Element-wise on every 10th view against
    the reference's CUDA build and its host build (the source's operations;
    the voxels at the detector's edges, kept or dropped by Q11, are decided
    as the reference decides them); timed on all 360 views.  The reference's
    two builds place an edge voxel differently now and then (device cosf
    against the host's): on all views they differ by 1.9e-4 x max at one
    voxel, so the full-scan comparison asserts rel-L2 only."""
    n, nv, na, nbr, px, si, sd = 256, 360, 512, 384, 1.2, 600.0, 1200.0
    ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(30, 2), device=cuda).permute(2, 1, 0).contiguous()
    corner = (-n / 2.0,) * 3
    for views in (list(range(0, nv, 10)), list(range(nv))):
        a = ang[views]
        g = nb.ConeBeam((n, n, n), a, si, sd, na, px, nbr, px, size=(float(n),) * 3)
        sino = ops.cb_forward(vol, g, 0)
        d_ang = torch.from_numpy(a).to(cuda)
        ref, t_ref = _events(lambda: oracle_lib.ref_gpu_pixel_backproject(sino, (n, n, n), corner, (float(n),) * 3,
                                                                          d_ang, si, sd, na, px, 0.0, nbr, px, 0.0))
        mirror = nb.cc.pixel_3d.back_project_flat(sino, [n, n, n], list(corner), [float(n)] * 3, a, si, sd, na, px,
                                                  0.0, nbr, px, 0.0, n, n, n)
        r, m = rel(mirror.reshape(n, n, n), ref)
        out, t = _events(lambda: ops.fdk_backproject(sino, g, weight=False))
        assert torch.equal(out.reshape(-1), mirror.reshape(-1))
        if len(views) < nv:
            assert r <= 1e-5 and m <= 1e-4, (r, m)
            if oracle_lib.have_ref():
                host = oracle_lib.ref_pixel_backproject(sino.cpu().numpy(), a, (n, n, n), np.array(corner, np.float32),
                                                        np.array((float(n),) * 3, np.float32), si, sd, na, px, 0.0,
                                                        nbr, px, 0.0)
                r, m = rel(out, torch.from_numpy(host).to(cuda))
                assert r <= 1e-5 and m <= 1e-5, (r, m)
        else:
            assert r <= 1e-5, r
            print(f"\npixel_3d backprojection, 256^3 x 360 views: reference CUDA {t_ref:.1f} ms, library "
                  f"{t:.2f} ms ({t_ref / t:.1f}x)")
            assert t < t_ref
        del sino, ref, mirror, out


def test_reference_cuda_lor_pair(cuda, oracle_lib):
    """cpp/siddon's LOR pair on 1 Mi lines between random points of a ring of
    radius 300 mm around a 256^3 grid of 1 mm voxels (the reference launches
    32 CTAs of 1024 threads; the library walks the lines in lor_order).  The
    reference's CUDA build contracts its multiply-adds (nvcc's default), which
    moves a few lines' voxel boundaries against its own source order (the
    host build, -ffp-contract=off): the library follows the source order
    (parity bar against the host build) and must be as close to the CUDA
    build as the host build is."""
    if not oracle_lib.have_ref():
        pytest.skip("the reference's host build is absent")
    n, nl = 256, 2 ** 20
    rng = np.random.default_rng(19)
    phi1, phi2 = rng.uniform(0, 2 * np.pi, nl), rng.uniform(0, 2 * np.pi, nl)
    lors_np = np.stack([300 * np.cos(phi1), 300 * np.sin(phi1), rng.uniform(-100, 100, nl),
                        300 * np.cos(phi2), 300 * np.sin(phi2), rng.uniform(-100, 100, nl)]).astype(np.float32)
    lors = torch.from_numpy(lors_np).to(cuda)
    gen = torch.Generator(device=cuda).manual_seed(20)
    vol = torch.rand((n, n, n), device=cuda, generator=gen)
    vals = torch.rand(nl, device=cuda, generator=gen)
    shape, center, size = (n, n, n), (0.0, 0.0, 0.0), (float(n),) * 3
    og = oracle_lib.grid(shape, center, size)
    order = ops.lor_order(lors, shape, center, size)
    ref_f, t_ref_f = _events(lambda: oracle_lib.ref_gpu_lor(True, lors, shape, center, size, vol))
    out_f, t_f = _events(lambda: ops.lor_forward(lors, vol, shape, center, size, _lib.LOR_REF_FORWARD, order=order))
    host_f = torch.from_numpy(oracle_lib.ref_lor_forward(og, vol.cpu().numpy(), lors_np)).to(cuda)
    ref_b, t_ref_b = _events(lambda: oracle_lib.ref_gpu_lor(False, lors, shape, center, size, vals))
    out_b, t_b = _events(lambda: ops.lor_backward(lors, vals, shape, center, size, _lib.LOR_REF_BACKPROJECT,
                                                  order=order))
    host_b = torch.from_numpy(oracle_lib.ref_lor_backward(og, vals.cpu().numpy(), lors_np)).to(cuda)
    for out, ref, host in ((out_f, ref_f, host_f), (out_b, ref_b, host_b)):
        r, m = rel(out, host)
        assert r <= 1e-5 and m <= 1e-4, (r, m)
        rg, mg = rel(ref, host)                 # the reference's two builds
        ro, mo = rel(out, ref)
        assert ro <= rg + 1e-5 and mo <= mg + 1e-4, (ro, mo, rg, mg)
    print(f"\nLOR pair, 1 Mi lines through 256^3: reference CUDA forward {t_ref_f:.1f} ms, backprojection "
          f"{t_ref_b:.1f} ms; library (ordered walk) forward {t_f:.2f} ms, backprojection {t_b:.2f} ms "
          f"({t_ref_f / t_f:.1f}x, {t_ref_b / t_b:.1f}x)")
    assert t_f < t_ref_f and t_b < t_ref_b


def test_reference_cuda_distance_driven_backprojection(cuda, oracle_lib):
    """The distance-driven FDK backprojection (dist_3d_back_fdk.cu.cc) on 72
    views of the FDK scanner in voxel units (256^3, 512 x 384 bins of 1.2,
    source-axis 600, source-detector 1200), against the reference's CUDA
    kernel (a thread per bin, atomics into the x-fastest volume)."""
    n, nv, na, nbr, px, sad, sid = 256, 72, 512, 384, 1.2, 600.0, 1200.0
    ang = (np.linspace(0, 2 * np.pi, nv, endpoint=False)).astype(np.float32)
    proj = torch.rand((nv, nbr, na), device=cuda, generator=torch.Generator(device=cuda).manual_seed(21))
    d_ang = torch.from_numpy(ang).to(cuda)
    d_off = torch.zeros(nv, device=cuda)
    ref, t_ref = _events(lambda: oracle_lib.ref_gpu_dd_backproject(proj, (n, n, n), d_ang, d_off, sid, sad, na, px,
                                                                    0.0, nbr, px, 0.0))
    out, t = _events(lambda: ops.dd_backproject(proj, (n, n, n), ang, sad, sid, px, px))
    r, m = rel(out, ref)
    assert r <= 1e-5 and m <= 1e-4, (r, m)
    print(f"\ndistance-driven backprojection, 256^3 x 72 views: reference CUDA {t_ref:.1f} ms, library {t:.2f} ms "
          f"({t_ref / t:.1f}x)")
    assert t < t_ref


def test_reference_cuda_warp(cuda, oracle_lib):
    """The trilinear warp at the motion workload's size (256^3, a field of
    four sinusoids per component up to 5 voxels) against the reference's
    cpp/deform CUDA kernel."""
    n = 256
    gen = torch.Generator(device=cuda).manual_seed(6)
    img = torch.rand((n, n, n), device=cuda, generator=gen)
    z, y, x = torch.meshgrid(*[torch.arange(n, device=cuda, dtype=torch.float32)] * 3, indexing="ij")
    rng = np.random.default_rng(6)
    m = []
    for _ in range(3):
        f = torch.zeros_like(img)
        for _ in range(4):
            k, ph = rng.uniform(0.5, 3, 3) * 2 * np.pi / n, rng.uniform(0, 2 * np.pi)
            f += 1.25 * torch.sin(float(k[0]) * x + float(k[1]) * y + float(k[2]) * z + float(ph))
        m.append(f.contiguous())
    ref, t_ref = _events(lambda: oracle_lib.ref_gpu_deform(img, *m))
    out, t = _events(lambda: ops.warp_forward(img, *m))
    r, mx = rel(out, ref)
    assert r <= 1e-5 and mx <= 1e-4, (r, mx)
    print(f"\ntrilinear warp, 256^3: reference CUDA {t_ref:.3f} ms, library {t:.3f} ms ({t_ref / t:.1f}x)")

"""GPU: the library against the reference's own CUDA projector, built
unchanged by nvcc from the reference sources (oracle/_ref/libnefct_ref_gpu.so:
ProjectFlatKernel / BackProjectFlatKernel and their host launchers,
siddon.cu.cc:6-890) and run on the same GPU.

* parity: the library's forward and reference backprojection against the
  reference's CUDA kernels, element-wise, on the 64^3 workload at full size
  and on views of the 512^3 scan (rel-L2 <= 1e-5, max-abs <= 1e-4 x max);
* speed: the 512^3 scan's forward + backprojection through the reference's
  kernels beside the library's forward + exact transpose (the same
  intersections), both timed with CUDA events after a warm-up call.
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


def _events(fn):
    fn()                                      # warm-up (allocations, first launch)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


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

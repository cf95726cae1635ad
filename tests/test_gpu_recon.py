"""Iterative reconstruction loops over the device operators: SIRT and
conjugate gradients, run eagerly and as a replayed CUDA graph of one
iteration."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib, ops, recon

pytestmark = pytest.mark.gpu


def _problem(cuda):
    g = nb.ConeBeam((40, 40, 32), np.linspace(0, 2 * np.pi, 48, endpoint=False), 150.0, 300.0, 64, 1.4, 48, 1.4,
                    size=(40.0, 40.0, 32.0))
    vol = nb.ellipsoid_phantom(40, nb.random_ellipsoids(6, 7))[:, :, 4:36].permute(2, 1, 0).contiguous().to(cuda)
    b = ops.cb_forward(vol, g, _lib.LINE_INTEGRAL)
    return g, vol, b


@pytest.mark.parametrize("method", ["sirt", "cg"])
def test_graph_replay_matches_eager_loop(cuda, method):
    """The deterministic transpose makes every iteration reproducible, so the
    graph replays give the eager loop's result bit for bit."""
    g, vol, b = _problem(cuda)
    flags = _lib.LINE_INTEGRAL | _lib.DETERMINISTIC
    run = getattr(recon, method)
    eager = run(b, g, 6, flags)
    graphed = run(b, g, 6, flags, graph=True)
    torch.cuda.synchronize()
    assert torch.equal(eager, graphed)


@pytest.mark.parametrize("method", ["sirt", "cg"])
def test_iterations_reduce_the_residual(cuda, method):
    g, vol, b = _problem(cuda)
    res = []
    run = getattr(recon, method)
    run(b, g, 8, graph=True,
        callback=lambda it, x: res.append(float((ops.cb_forward(x, g, _lib.LINE_INTEGRAL) - b).norm())))
    assert len(res) == 8
    assert res[-1] < 0.5 * res[0]
    assert all(r1 <= r0 * 1.0001 for r0, r1 in zip(res, res[1:])) or method == "cg"


def _dropin_problem(oracle_lib):
    """A 32^3 phantom (2 mm voxels), 36 views, 64 x 48 detector at 2 mm,
    source-axis 200 mm, source-detector 400 mm; drop-in operators (numpy in
    and out) and the reference's own operators built for the host."""
    from nefct_b200 import functions as F
    n, vox, nv, na, nbr, px, si, sd = 32, 2.0, 36, 64, 48, 2.0, 200.0, 400.0
    ang = (np.linspace(0, 2 * np.pi, nv, endpoint=False) + 0.02).astype(np.float32)
    cfg = nb.ScannerConfig3D("flat", sd, si, nb.DetectorDirectAConfig(na, na * px), nb.DetectorDirectBConfig(nbr, nbr * px))
    size = [n * vox] * 3
    phantom = nb.ellipsoid_phantom(n, nb.random_ellipsoids(6, 8)).numpy()            # [x, y, z]
    og = oracle_lib.grid((n, n, n), (0, 0, 0), tuple(size))
    args = (si, sd, na, px, 0.5, nbr, px, 0.5)
    have = oracle_lib.have_ref()

    def ref_fwd(x_xyz):
        v = np.ascontiguousarray(x_xyz.transpose(2, 1, 0))
        s = oracle_lib.ref_cb_forward(og, v, ang, *args) if have else \
            oracle_lib.cb_forward(og, v, ang, *args, use_cosf=True)[0]
        return np.ascontiguousarray(s.transpose(2, 1, 0))                           # [na, nb, nv]

    def ref_bp(p_abv):
        s = np.ascontiguousarray(p_abv.transpose(2, 1, 0))
        v = oracle_lib.ref_cb_backward(og, s, ang, *args) if have else \
            oracle_lib.cb_backward(og, s, ang, *args, use_cosf=True)
        return np.ascontiguousarray(v.transpose(2, 1, 0))                           # [x, y, z]

    proj = nb.ProjectionSequence3D(ref_fwd(phantom), cfg, list(ang), np.zeros(nv, np.float32))
    project = F.Project3D(cfg, list(ang), None)
    back = F.BackProject3D(cfg, [n, n, n], vox)
    return dict(F=F, proj=proj, project=project, back=back, ref_fwd=ref_fwd, ref_bp=ref_bp, size=size, n=n)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_sart_iterates_vs_reference_operators(cuda, oracle_lib):
    """functions.SART over the drop-in Project3D / BackProject3D (GPU)
    against sart.py:29-39 restated in numpy over the reference's own
    forward and backprojection built for the host:
    x <- x + lambda * div_no_nan(BP(p - A x), emap), emap = BP(ones).
    The iterates agree to rel-L2 1e-5 after 1 and after 4 iterations."""
    P = _dropin_problem(oracle_lib)
    p = P["proj"].data
    emap_np = P["ref_bp"](np.ones_like(p))
    emap = P["back"](nb.ProjectionSequence3D(np.ones_like(p), P["proj"].scanner, P["proj"].angles,
                                             P["proj"].offsets))
    assert _rel(emap.data, emap_np) < 1e-5
    lam = 0.8
    x = np.zeros_like(emap_np)
    for it in range(4):
        bp = P["ref_bp"](p - P["ref_fwd"](x))
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = np.where(emap_np != 0, bp / np.where(emap_np != 0, emap_np, 1), 0).astype(np.float32)
        x = (x + ratio * np.float32(lam)).astype(np.float32)
        if it in (0, 3):
            ours = P["F"].SART(it + 1, lam, emap, P["project"], P["back"])(P["proj"])
            assert _rel(ours.data, x) < 1e-5, (it, _rel(ours.data, x))


def test_conjgrad_iterates_vs_reference_operators(cuda, oracle_lib):
    """functions.ConjGrad (no total-variation term) against
    conj_grad.py:37-62 restated in numpy over the reference's host-built
    operators: CG on BP(A x) = BP(p).  After 3 iterations the iterates
    agree to rel-L2 1e-4 (CG amplifies the float32 rounding of the two
    operator paths' summation orders)."""
    P = _dropin_problem(oracle_lib)
    p = P["proj"].data
    A = lambda v: P["ref_bp"](P["ref_fwd"](v))
    b = P["ref_bp"](p)
    x = np.zeros_like(b)
    r = b - A(x)
    d = r.copy()
    rsold = np.sum(r ** 2)
    for _ in range(3):
        Ad = A(d)
        alpha = rsold / np.sum(d * Ad)
        x = x + d * alpha
        r = r - Ad * alpha
        rsnew = np.sum(r ** 2)
        d = r + d * (rsnew / rsold)
        rsold = rsnew
    ours = P["F"].ConjGrad(3, P["project"], P["back"])(P["proj"])
    assert _rel(ours.data, x) < 1e-4, _rel(ours.data, x)


@pytest.mark.parametrize("graph", [False, True])
def test_cg_zero_right_hand_side_stays_finite(cuda, graph):
    """With b = 0 the residual is zero from the start: the step sizes are
    guarded (0 instead of 0/0), so the iterate stays at zero instead of
    turning into NaN, also inside the replayed graph."""
    g, vol, b = _problem(cuda)
    x = recon.cg(torch.zeros_like(b), g, 4, graph=graph)
    torch.cuda.synchronize()
    assert torch.isfinite(x).all() and float(x.abs().max()) == 0.0

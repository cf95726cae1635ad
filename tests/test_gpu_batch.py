"""GPU: batched uneven problems in one persistent launch (and a CUDA graph)
against per-problem calls of the same operators."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import ops
from nefct_b200.batch import BatchProjector
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


class _walk:
    """Context: the walk of both directions (0 thread per ray, 3 column
    warps); a batch plan fixes its walk when it is made."""

    def __init__(self, walk):
        self.walk = walk

    def __enter__(self):
        from nefct_b200 import autotune
        self.saved = autotune.current()
        autotune.apply(self.saved["rows"], self.saved["order"], self.walk)

    def __exit__(self, *exc):
        from nefct_b200 import autotune
        autotune.apply(self.saved["rows"], self.saved["order"], self.saved["walk"])


def _problems(dev):
    rng = np.random.default_rng(4)
    geoms = [
        nb.ConeBeam((40, 40, 40), np.linspace(0, 2 * np.pi, 30, endpoint=False), 120.0, 220.0, 70, 1.2, 50, 1.2,
                    size=(40.0,) * 3),
        nb.ConeBeam((24, 30, 20), np.linspace(0.3, 5.0, 17), 90.0, 170.0, 45, 1.5, 33, 1.1,
                    size=(24.0, 36.0, 20.0), center=(1.0, -0.5, 0.3)),                 # non-cubic voxels
        nb.ConeBeam((32, 32, 24), np.linspace(0, 2 * np.pi, 25, endpoint=False), 100.0, 200.0, 60, 0.012, 40, 1.0,
                    size=(32.0, 32.0, 24.0), det_kind="cyl"),
        nb.ConeBeam((16, 16, 16), np.linspace(0, np.pi, 9), 60.0, 110.0, 33, 1.0, 17, 1.0, size=(16.0,) * 3,
                    z_offsets=np.linspace(-2, 2, 9)),
        nb.ConeBeam((56, 48, 36), np.linspace(0, 2 * np.pi, 41, endpoint=False), 160.0, 300.0, 96, 1.3, 64, 1.3,
                    size=(56.0, 48.0, 36.0)),
    ]
    vols = [torch.from_numpy(rng.random(g.vol_shape, dtype=np.float32)).to(dev) for g in geoms]
    grads = [torch.from_numpy(rng.random(g.sino_shape, dtype=np.float32)).to(dev) for g in geoms]
    return geoms, vols, grads


@pytest.mark.parametrize("walk", [0, 3], ids=["thread-walk", "column-warps"])
@pytest.mark.parametrize("strategy", ["persistent", "per-problem"])
@pytest.mark.parametrize("flags", [0, nb._lib.LINE_INTEGRAL])
def test_batch_matches_per_problem(cuda, flags, strategy, walk):
    geoms, vols, grads = _problems(cuda)
    with _walk(walk):
        bp = BatchProjector(geoms, vols, grads=grads, flags=flags, strategy=strategy)
        bp.step()
        torch.cuda.synchronize()
        for g, v, gr, s, b in zip(geoms, vols, grads, bp.sinos, bp.backs):
            ref = ops.cb_forward(v, g, flags)
            assert torch.equal(s, ref)                   # same per-ray code: bitwise
            assert_parity(b.cpu().numpy(), ops.cb_backward(gr, g, flags).cpu().numpy())


@pytest.mark.parametrize("walk", [0, 3], ids=["thread-walk", "column-warps"])
@pytest.mark.parametrize("strategy", ["persistent", "per-problem"])
def test_batch_graph_replay(cuda, strategy, walk):
    geoms, vols, grads = _problems(cuda)
    with _walk(walk):
        bp = BatchProjector(geoms, vols, grads=grads, strategy=strategy)
        graph = bp.capture()
        for b in bp.backs:
            b.zero_()
        for s in bp.sinos:
            s.fill_(float("nan"))
        graph.replay()
        graph.replay()
        torch.cuda.synchronize()
        for g, v, gr, s, b in zip(geoms, vols, grads, bp.sinos, bp.backs):
            assert torch.equal(s, ops.cb_forward(v, g))
            assert_parity(b.cpu().numpy(), ops.cb_backward(gr, g).cpu().numpy())
        assert bp.tiles > 0


def test_batch_auto_strategy_times_both(cuda):
    geoms, vols, grads = _problems(cuda)
    bp = BatchProjector(geoms, vols, grads=grads)
    assert set(bp.timings) == {"persistent", "per-problem"} and bp.strategy in bp.timings


@pytest.mark.parametrize("strategy", ["persistent", "per-problem"])
def test_batch_vs_reference_build(cuda, oracle_lib, strategy):
    """Two problems of the batch (cubic flat 40^3 and a cylindrical detector
    over 32 x 32 x 24) against the reference's own kernels built for the
    host: the batched forward (reference forward flags) against
    ProjectFlat/CyliKernel, and the batched backward of a plan with the
    reference backprojection's flags against BackProjectFlat/CyliKernel of
    the same sinograms (the cylindrical one with the forward's sinogram
    layout, i.e. without Q8)."""
    geoms, vols, grads = _problems(cuda)
    pick = [0, 2]
    geoms, vols, grads = [geoms[i] for i in pick], [vols[i] for i in pick], [grads[i] for i in pick]
    for walk in (0, 3):
        with _walk(walk):
            fwd = BatchProjector(geoms, vols, flags=0, strategy=strategy)
            fwd.forward()
            bwd = BatchProjector(geoms, vols, grads=grads, flags=nb._lib.REF_BACKPROJECT, strategy=strategy)
            bwd.backward()
            torch.cuda.synchronize()
            for g, v, gr, s, b in zip(geoms, vols, grads, fwd.sinos, bwd.backs):
                og = oracle_lib.grid(g.shape, g.center, g.size)
                args = (g.angles, g.src_iso, g.src_det, g.na, g.da, g.a_shift, g.nb, g.db, g.b_shift)
                cyl = g.det_kind == "cyl"
                vn, yn = v.cpu().numpy(), gr.cpu().numpy()
                if oracle_lib.have_ref():
                    rs = oracle_lib.ref_cb_forward(og, vn, *args, cyl=cyl)
                    rb = oracle_lib.ref_cb_backward(og, yn, *args, cyl=False)
                else:
                    rs = oracle_lib.cb_forward(og, vn, *args, cyl=cyl, use_cosf=True)[0]
                    rb = oracle_lib.cb_backward(og, yn, *args, cyl=False, use_cosf=True)
                assert_parity(s.cpu().numpy(), rs)
                if not cyl:
                    assert_parity(b.cpu().numpy(), rb)


@pytest.mark.parametrize("strategy", ["persistent", "per-problem"])
def test_batch_autograd_function(cuda, strategy):
    """batch_project: the batched forward as a torch.autograd.Function; the
    gradient of sum_i ||A_i x_i - b_i||^2 / 2 comes from one batched
    transpose and matches per-problem autograd through nb.project.  The
    inputs and incoming gradients are read in place (the plan is pointed at
    them for the launch), and the plan is pointed back at its own tensors
    afterwards."""
    from nefct_b200.batch import batch_project
    geoms, vols, _ = _problems(cuda)
    targets = [ops.cb_forward(v * 0.5, g) for g, v in zip(geoms, vols)]
    xs = [v.clone().requires_grad_() for v in vols]
    own = [torch.rand_like(v) for v in vols]
    bp = BatchProjector(geoms, own, grads=[torch.empty_like(t) for t in targets], strategy=strategy)
    sinos = batch_project(bp, xs)
    for g, x, s_ in zip(geoms, xs, sinos):
        assert torch.equal(s_, ops.cb_forward(x.detach(), g))
    loss = sum(((s - t) ** 2).sum() / 2 for s, t in zip(sinos, targets))
    loss.backward()
    for g, x, t in zip(geoms, xs, targets):
        xr = x.detach().clone().requires_grad_()
        (((nb.project(xr, g) - t) ** 2).sum() / 2).backward()
        assert_parity(x.grad.cpu().numpy(), xr.grad.cpu().numpy())
    bp.forward()                                  # back on the plan's own volumes
    for g, v, s_ in zip(geoms, own, bp.sinos):
        assert torch.equal(s_, ops.cb_forward(v, g))


def test_batch_tile_shape_autotuning(cuda):
    """tune_rows=True times plans with 2, 4 and 8 rows (columns) per CTA under
    both strategies, keeps the fastest, restores the process-wide setting,
    and the tuned plan gives the single-problem results."""
    from nefct_b200 import autotune
    geoms, vols, grads = _problems(cuda)
    before = autotune.current()
    bp = BatchProjector(geoms, vols, grads=grads, tune_rows=True)
    assert autotune.current() == before
    assert bp.tuned_rows["rows"] in (2, 4, 8) and bp.strategy == bp.tuned_rows["strategy"]
    assert len(bp.tuned_rows["ms"]) == 6
    bp.step()
    torch.cuda.synchronize()
    for g, v, gr, s, b in zip(geoms, vols, grads, bp.sinos, bp.backs):
        assert torch.equal(s, ops.cb_forward(v, g))
        assert_parity(b.cpu().numpy(), ops.cb_backward(gr, g).cpu().numpy())

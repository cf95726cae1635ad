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

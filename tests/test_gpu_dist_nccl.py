"""GPU: the view-sharded projector over NCCL with the CUDA operators.

One GPU is available per run here, so the process group has one rank: the
NCCL all-reduce / all-gather run for real (on the GPU, through NCCL's
single-rank path) around the real kernels, with no rank waiting on
another.  The child process is spawned (a fresh CUDA context), joins the
group on 127.0.0.1 with a short timeout, and compares the sharded forward,
gather and transpose with the single-process operators."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(port, q):
    import datetime

    import torch.distributed as dist

    import nefct_b200 as nb
    from nefct_b200 import ops
    from nefct_b200.dist import ShardedProjector
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("NCCL_NVLS_ENABLE", "0")
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        dev = torch.device("cuda", 0)
        g = nb.ConeBeam((40, 36, 32), np.linspace(0, 2 * np.pi, 45, endpoint=False), 120.0, 240.0, 64, 1.4, 48, 1.4,
                        size=(40.0, 36.0, 32.0))
        gen = torch.Generator(device=dev).manual_seed(3)
        vol = torch.rand(g.vol_shape, device=dev, generator=gen)
        y = torch.rand(g.sino_shape, device=dev, generator=gen)
        sp = ShardedProjector(g, 0)
        full = sp.gather(sp.forward(vol))
        back = sp.backward(y[sp.views].contiguous())
        ref_f = ops.cb_forward(vol, g)
        ref_b = ops.cb_backward(y, g)
        torch.cuda.synchronize()
        q.put((bool(torch.equal(full, ref_f)),
               float((back.double() - ref_b.double()).norm() / ref_b.double().norm()),
               sp.world, sp.views.start, sp.views.stop))
    finally:
        dist.destroy_process_group()


def test_sharded_projector_nccl_single_rank(cuda):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_worker, args=(_free_port(), q))
    p.start()
    try:
        same_forward, rel_back, world, v0, v1 = q.get(timeout=240)
    finally:
        p.join(timeout=120)
    assert p.exitcode == 0
    assert world == 1 and (v0, v1) == (0, 45)
    assert same_forward                      # same kernels, same views: bitwise
    assert rel_back < 1e-6                   # atomic summation order only

"""CPU, world_size 2 (gloo): the view-sharded projector's host logic.

Each rank projects its block of views and the transpose sums the partial
volumes with an all-reduce.  The per-rank operator is the oracle (CPU), so
the test needs no GPU; the result must equal the single-process oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nefct_b200.dist import view_shard


def test_view_shard_partitions():
    for nv in (1, 7, 90, 360):
        for world in (1, 2, 3, 8):
            parts = [view_shard(nv, r, world) for r in range(world)]
            idx = np.concatenate([np.arange(nv)[p] for p in parts])
            np.testing.assert_array_equal(idx, np.arange(nv))
            sizes = [p.stop - p.start for p in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_ops():
    import oracle

    def fwd(vol, g, flags):
        og = oracle.grid(g.shape, g.center, g.size)
        out, _ = oracle.cb_forward(og, vol.numpy(), g.angles, g.src_iso, g.src_det, g.na, g.da, g.a_shift, g.nb,
                                   g.db, g.b_shift, flags=oracle.CB_FWD)
        return torch.from_numpy(out)

    def bwd(sino, g, flags):
        og = oracle.grid(g.shape, g.center, g.size)
        out = oracle.cb_backward(og, sino.numpy(), g.angles, g.src_iso, g.src_det, g.na, g.da, g.a_shift, g.nb,
                                 g.db, g.b_shift, flags=oracle.CB_FWD)
        return torch.from_numpy(out)

    return fwd, bwd


def _geom():
    import nefct_b200 as nb
    return nb.ConeBeam((20, 18, 16), np.linspace(0, 2 * np.pi, 13, endpoint=False), 80.0, 160.0, 30, 1.5, 24, 1.5)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from nefct_b200.dist import ShardedProjector
        fwd, bwd = _oracle_ops()
        g = _geom()
        sp = ShardedProjector(g, 0, forward_fn=fwd, backward_fn=bwd)
        vol = torch.from_numpy(np.random.default_rng(0).random(g.vol_shape, dtype=np.float32))
        sino_local = sp.forward(vol)
        full = sp.gather(sino_local)
        y = torch.from_numpy(np.random.default_rng(1).random(g.sino_shape, dtype=np.float32))
        back = sp.backward(y[sp.views].contiguous())
        q.put((rank, full.numpy(), back.numpy()))
    finally:
        dist.destroy_process_group()


def test_sharded_projector_two_ranks_matches_single_process():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fwd, bwd = _oracle_ops()
    g = _geom()
    vol = torch.from_numpy(np.random.default_rng(0).random(g.vol_shape, dtype=np.float32))
    y = torch.from_numpy(np.random.default_rng(1).random(g.sino_shape, dtype=np.float32))
    ref_full = fwd(vol, g, 0).numpy()
    ref_back = bwd(y, g, 0).numpy()
    for rank, full, back in res:
        np.testing.assert_array_equal(full, ref_full)
        np.testing.assert_allclose(back, ref_back, rtol=1e-5, atol=1e-6 * np.abs(ref_back).max())

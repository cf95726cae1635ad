"""GPU: the allocation-free forward projection (nefct_cb_forward_noalloc).

It exists for callers that may not allocate device memory -- a service that
reserves all GPU memory at start-up, a host framework that owns the memory
pool, a binding that only receives device pointers -- and so cannot supply
the workspace nefct_cb_forward needs.  Its scratch lives in a fixed array in
the library.  This test calls it through the C ABI twice in a row and checks
each result against nefct_cb_forward with a caller workspace: the two run
the same kernels, so the sinograms agree bit for bit (and within the parity
tolerance of the other tests a fortiori), for both walks.  The refusal of
grids larger than the fixed array happens before any CUDA call and is
tested on the CPU (tests/test_capi.py).  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import _lib
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


def _forward_with_workspace(lib, g, vol, stream):
    s = g.struct()
    n = lib.nefct_cb_workspace_bytes(C.byref(s), 0)
    ws = torch.empty(n, dtype=torch.uint8, device=vol.device)
    out = torch.empty(g.sino_shape, device=vol.device)
    _lib.check(lib.nefct_cb_forward(C.byref(s), vol.data_ptr(), out.data_ptr(), 0, ws.data_ptr(), n, stream))
    return out


@pytest.mark.parametrize("walk", [3, 0], ids=["column-warps", "thread-walk"])
def test_noalloc_forward_matches_workspace_forward_twice(cuda, walk):
    from nefct_b200 import autotune
    lib = _lib.load()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    g = nb.ConeBeam((96, 80, 64), np.linspace(0, 2 * np.pi, 45, endpoint=False), 300.0, 600.0, 160, 1.5, 96, 1.5,
                    size=(96.0, 80.0, 64.0), center=(0.5, -1.0, 0.25))
    gen = torch.Generator(device=cuda).manual_seed(11)
    saved = autotune.current()
    try:
        autotune.apply(saved["rows"], saved["order"], walk)
        for call in range(2):
            vol = torch.rand(g.vol_shape, device=cuda, generator=gen)
            ref = _forward_with_workspace(lib, g, vol, stream)
            out = torch.full(g.sino_shape, float("nan"), device=cuda)
            s = g.struct()
            _lib.check(lib.nefct_cb_forward_noalloc(C.byref(s), vol.data_ptr(), out.data_ptr(), 0, stream))
            torch.cuda.synchronize(cuda)
            assert torch.isfinite(out).all(), f"call {call}"
            assert_parity(out.cpu().numpy(), ref.cpu().numpy())
            assert torch.equal(out, ref), f"call {call}"
    finally:
        autotune.apply(saved["rows"], saved["order"], saved["walk"])

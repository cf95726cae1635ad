"""GPU: the allocation-free forward projection (nefct_cb_forward_noalloc).

It exists for callers that may not allocate device memory -- a service that
reserves all GPU memory at start-up, a host framework that owns the memory
pool, a binding that only receives device pointers -- and so cannot supply
the workspace nefct_cb_forward needs.  Its scratch lives in a fixed array in
the library.  This test calls it through the C ABI twice in a row and checks
each result against nefct_cb_forward with a caller workspace, and checks
that grids larger than the fixed array are refused before any GPU work.
This file is collected last.
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


def test_noalloc_forward_matches_workspace_forward_twice(cuda):
    lib = _lib.load()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    g = nb.ConeBeam((96, 80, 64), np.linspace(0, 2 * np.pi, 45, endpoint=False), 300.0, 600.0, 160, 1.5, 96, 1.5,
                    size=(96.0, 80.0, 64.0), center=(0.5, -1.0, 0.25))
    gen = torch.Generator(device=cuda).manual_seed(11)
    for call in range(2):
        vol = torch.rand(g.vol_shape, device=cuda, generator=gen)
        ref = _forward_with_workspace(lib, g, vol, stream)
        out = torch.full(g.sino_shape, float("nan"), device=cuda)
        s = g.struct()
        _lib.check(lib.nefct_cb_forward_noalloc(C.byref(s), vol.data_ptr(), out.data_ptr(), 0, stream))
        torch.cuda.synchronize(cuda)
        assert torch.isfinite(out).all(), f"call {call}"
        assert_parity(out.cpu().numpy(), ref.cpu().numpy())


def test_noalloc_refuses_grids_beyond_its_scratch(cuda):
    lib = _lib.load()
    g = nb.ConeBeam((256, 256, 256), [0.0], 600.0, 1200.0, 64, 1.0, 64, 1.0)
    s = g.struct()
    st = lib.nefct_cb_forward_noalloc(C.byref(s), C.c_void_p(256), C.c_void_p(256), 0, None)
    assert st == _lib.ERR_INVALID
    assert b"at most 8388608 voxels" in lib.nefct_last_error()

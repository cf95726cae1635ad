"""GPU parity of the distance-driven FDK backprojection (dist_3d_back_fdk)."""
import numpy as np
import pytest
import torch

import nefct_b200 as nb
from nefct_b200 import ops
from tests.golden.make_golden import (DD_AI, DD_BI, DD_DA, DD_DA_CYL, DD_DB, DD_GRID, DD_NA, DD_NB, DD_SAD,
                                      DD_SID)
from tests.test_gpu_siddon import assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_dd_vs_reference_fixtures(cuda, golden, cyl):
    """Against the reference's own kernel (host build), which evaluates the
    view and detector-angle trigonometry with cosf/sinf (here: the
    double-precision functions, rounded)."""
    key, da = ("dd/cyl", DD_DA_CYL) if cyl else ("dd/flat", DD_DA)
    proj = torch.from_numpy(golden["dd/proj"]).to(cuda)
    out = ops.dd_backproject(proj, DD_GRID, golden["angles"], DD_SAD, DD_SID, da, DD_DB, DD_AI, DD_BI,
                             "cyl" if cyl else "flat", golden["dd/off"])
    assert_parity(out.cpu().numpy(), golden[key])


@pytest.mark.parametrize("cyl", [False, True], ids=["flat", "cyl"])
def test_dd_vs_restatement_tight(cuda, oracle_lib, cyl):
    """Same trigonometry as the restatement: only the summation order of the
    reductions differs.  Views on both sides of the 45-degree switch of the
    driving axis, z offsets, a partial row tile (45 rows) and zero bins."""
    rng = np.random.default_rng(23)
    shape, na, nbins = (30, 26, 20), 37, 45
    ang = np.array([0.2, np.pi / 4 - 2e-3, np.pi / 4 + 2e-3, 1.9, 3.3, 5.0], np.float32)
    proj = rng.random((ang.size, nbins, na), dtype=np.float32)
    proj[2, 5:9] = 0
    off = rng.uniform(-2, 2, ang.size).astype(np.float32)
    sad, sid, da = 70.0, 150.0, (0.009 if cyl else 1.1)
    ref = oracle_lib.dd_backproject(proj, ang, shape, sid, sad, na, da, 0.2, nbins, 1.05, -0.3, cyl=cyl, off=off,
                                    use_cosf=False)
    out = ops.dd_backproject(torch.from_numpy(proj).to(cuda), shape, ang, sad, sid, da, 1.05, 0.2, -0.3,
                             "cyl" if cyl else "flat", off).cpu().numpy()
    assert_parity(out, ref, rel=1e-6, mabs=1e-5)


def test_dd_op_mirror_accumulates(cuda, golden):
    """back_project_flat_fdk_gpu adds into the caller's image, as the
    reference's host function does."""
    proj = torch.from_numpy(golden["dd/proj"]).to(cuda)
    nx, ny, nz = DD_GRID
    image = torch.ones((nx, ny, nz), device=cuda)
    out = nb.cc.distance_3d.back_project_flat_fdk_gpu(proj, DD_GRID, golden["dd/off"], golden["angles"],
                                                      proj.shape[0], DD_SID, DD_SAD, DD_DA, DD_AI, DD_NA, DD_DB,
                                                      DD_BI, DD_NB, image)
    assert out is image
    assert_parity(out.cpu().numpy().reshape(nz, ny, nx) - 1.0, golden["dd/flat"], rel=1e-5, mabs=1e-4)

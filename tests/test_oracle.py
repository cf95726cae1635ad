"""CPU: pin the oracle restatement against the reference itself.

The restatement (oracle/nefct_oracle.c) must reproduce the reference's own
device routines compiled for the host bit for bit, on the committed golden
fixtures (generated from the reference by tests/golden/make_golden.py) and,
where the reference build is present, on fresh seeded cases.
"""
import numpy as np
import pytest

from tests.golden.make_golden import AI, BI, CASES, DB, NA, NB, SRC_DET, SRC_ISO


def _args(da):
    return dict(src_iso=SRC_ISO, src_det=SRC_DET, na=NA, da=da, ai=AI, nb=NB, db=DB, bi=BI)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_forward_matches_golden_bitwise(oracle_lib, golden, case):
    name, grid, centre, size, cyl, da = case
    g = oracle_lib.grid(grid, centre, size)
    out, cnt = oracle_lib.cb_forward(g, golden[f"{name}/vol"], golden["angles"], cyl=cyl, use_cosf=True, **_args(da))
    np.testing.assert_array_equal(out, golden[f"{name}/fwd"])
    assert cnt == int(golden[f"{name}/count"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_backprojection_matches_golden_bitwise(oracle_lib, golden, case):
    name, grid, centre, size, cyl, da = case
    g = oracle_lib.grid(grid, centre, size)
    out = oracle_lib.cb_backward(g, golden[f"{name}/sino_in"], golden["angles"], cyl=cyl, q8=cyl,
                                 use_cosf=True, **_args(da))
    np.testing.assert_array_equal(out, golden[f"{name}/bp"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_forward_f64_matches_golden(oracle_lib, golden, case):
    name, grid, centre, size, cyl, da = case
    g = oracle_lib.grid(grid, centre, size)
    out, _ = oracle_lib.cb_forward(g, golden[f"{name}/vol"].astype(np.float64), golden["angles"], cyl=cyl,
                                   f64=True, **_args(da))
    ref = golden[f"{name}/fwd64"]
    # the golden FP64 run evaluates cos of the float angle in double as well
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_lor_pair_matches_golden(oracle_lib, golden):
    g = oracle_lib.grid((24, 20, 16), (0, 0, 0), (48.0, 40.0, 32.0))
    fwd, _ = oracle_lib.lor_forward(g, golden["lor/vol"], golden["lor/lors"])
    np.testing.assert_array_equal(fwd, golden["lor/fwd"])
    assert np.all(fwd[:5] == 0)          # Q4 rays
    bp = oracle_lib.lor_backward(g, golden["lor/vals"], golden["lor/lors"])
    np.testing.assert_allclose(bp, golden["lor/bp"], rtol=1e-6, atol=1e-6 * np.abs(golden["lor/bp"]).max())


def test_pixel_backprojection_matches_golden(oracle_lib, golden):
    corner = golden["pixel/corner"]
    for cyl, key, da in ((False, "pixel/flat", 2.5), (True, "pixel/cyl", 0.012)):
        out = oracle_lib.pixel_backproject(golden["pixel/sino"], golden["angles"], (24, 20, 16), corner,
                                           (48.0, 40.0, 32.0), SRC_ISO, SRC_DET, NA, da, 0.0, NB, DB, 0.0,
                                           cyl=cyl)
        np.testing.assert_allclose(out, golden[key], rtol=2e-6, atol=2e-6 * np.abs(golden[key]).max())


def test_deform_matches_golden_bitwise(oracle_lib, golden):
    out = oracle_lib.deform(golden["deform/img"], golden["deform/mx"], golden["deform/my"], golden["deform/mz"])
    np.testing.assert_array_equal(out, golden["deform/out"])


def test_known_answer_axis_ray(oracle_lib):
    """An axis-aligned ray through a uniform n^3 volume sums n * dx / L^2."""
    n = 8
    g = oracle_lib.grid((n, n, n), (0, 0, 0), (8.0, 8.0, 8.0))
    vol = np.ones((n, n, n), np.float32)
    lors = np.array([[-100.0], [0.3], [0.2], [100.0], [0.3], [0.2]], np.float32)
    out, cnt = oracle_lib.lor_forward(g, vol, lors, flags=oracle_lib.INV_L2)
    assert cnt == n
    np.testing.assert_allclose(out[0], n * 1.0 / 200.0 ** 2, rtol=1e-6)


@pytest.mark.skipif("not __import__('oracle').have_ref()")
def test_fresh_random_cases_bitwise(oracle_lib):
    """Seeded cases beyond the fixtures, against the reference build."""
    rng = np.random.default_rng(7)
    for trial in range(4):
        grid = tuple(int(v) for v in rng.integers(8, 28, 3))
        size = tuple(float(v) for v in np.array(grid) * rng.uniform(0.8, 2.5))
        centre = tuple(float(v) for v in rng.uniform(-3, 3, 3))
        vol = rng.random(grid[::-1], dtype=np.float32)
        ang = rng.uniform(0, 2 * np.pi, 7).astype(np.float32)
        na, nb = int(rng.integers(8, 40)), int(rng.integers(8, 30))
        da, db = float(rng.uniform(0.5, 3)), float(rng.uniform(0.5, 3))
        si, sd = float(rng.uniform(80, 200)), float(rng.uniform(250, 500))
        g = oracle_lib.grid(grid, centre, size)
        port, _ = oracle_lib.cb_forward(g, vol, ang, si, sd, na, da, 0.5, nb, db, 0.5, use_cosf=True)
        ref = oracle_lib.ref_cb_forward(g, vol, ang, si, sd, na, da, 0.5, nb, db, 0.5)
        np.testing.assert_array_equal(port, ref)
        sino = rng.random((7, nb, na), dtype=np.float32)
        pb = oracle_lib.cb_backward(g, sino, ang, si, sd, na, da, 0.5, nb, db, 0.5, use_cosf=True)
        rb = oracle_lib.ref_cb_backward(g, sino, ang, si, sd, na, da, 0.5, nb, db, 0.5)
        np.testing.assert_array_equal(pb, rb)


def test_reference_discretisation_vs_exact_siddon(oracle_lib, golden):
    """The reference's slab split differs from the exact path by the Q1
    pairing; the error against the FP64 exact oracle is stated, not zero."""
    name, grid, centre, size, cyl, da = CASES[0]
    g = oracle_lib.grid(grid, centre, size)
    ex = oracle_lib.cb_exact(g, golden[f"{name}/vol"], golden["angles"], **{k: v for k, v in _args(da).items()})
    ref = golden[f"{name}/fwd64"]
    rel = np.linalg.norm(ref - ex) / np.linalg.norm(ex)
    assert 1e-4 < rel < 3e-2


def test_warp_invert_oracle_composes_to_identity(oracle_lib):
    """The fixed-point inverse of a smooth small field satisfies
    inv(p) = -m(p + inv(p)) in the interior."""
    n = 24
    z, y, x = np.meshgrid(*[np.linspace(0, 1, n)] * 3, indexing="ij")
    m = [1.2 * np.sin(2 * np.pi * (x + 0.3 * y)), 0.8 * np.cos(2 * np.pi * z), 0.6 * np.sin(2 * np.pi * y)]
    m = [a.astype(np.float32) for a in m]
    inv = oracle_lib.warp_invert(*m, iters=30)
    # m(p + inv(p)) + inv(p) ~ 0 in the interior (the fixed point of the iteration)
    from scipy.ndimage import map_coordinates
    c = slice(4, n - 4)
    pz, py, px = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    pos = [pz + inv[2], py + inv[1], px + inv[0]]
    res = [map_coordinates(m[k], pos, order=1, mode="nearest") + inv[k] for k in range(3)]
    assert max(np.abs(r[c, c, c]).max() for r in res) < 1e-3


def test_dd_backprojection_matches_golden_bitwise(oracle_lib, golden):
    """Distance-driven FDK backprojection (dist_3d_back_fdk): the restatement
    against the reference's own kernel, flat and cylindrical."""
    from tests.golden.make_golden import (DD_AI, DD_BI, DD_DA, DD_DA_CYL, DD_DB, DD_GRID, DD_NA, DD_NB, DD_SAD,
                                          DD_SID)
    for key, cyl, da in (("dd/flat", False, DD_DA), ("dd/cyl", True, DD_DA_CYL)):
        out = oracle_lib.dd_backproject(golden["dd/proj"], golden["angles"], DD_GRID, DD_SID, DD_SAD, DD_NA, da,
                                        DD_AI, DD_NB, DD_DB, DD_BI, cyl=cyl, off=golden["dd/off"])
        np.testing.assert_array_equal(out, golden[key])


@pytest.mark.skipif("not __import__('oracle').have_ref()")
def test_dd_fresh_random_cases_bitwise(oracle_lib):
    """Seeded distance-driven cases (views on both sides of the 45-degree
    switch of the driving axis, z offsets, odd sizes) against the reference
    build."""
    rng = np.random.default_rng(17)
    for trial in range(3):
        shape = tuple(int(v) for v in rng.integers(6, 22, 3))
        nv, na, nb = 5, int(rng.integers(6, 30)), int(rng.integers(4, 20))
        ang = (np.array([0.1, np.pi / 4 - 1e-3, np.pi / 4 + 1e-3, 2.0, 4.0]) + 0.05 * trial).astype(np.float32)
        proj = rng.random((nv, nb, na), dtype=np.float32)
        off = rng.uniform(-2, 2, nv).astype(np.float32)
        sad, sid = float(rng.uniform(40, 80)), float(rng.uniform(100, 160))
        cyl = trial == 1
        da = float(rng.uniform(0.004, 0.01)) if cyl else float(rng.uniform(0.6, 1.6))
        args = (proj, ang, shape, sid, sad, na, da, float(rng.uniform(-0.5, 0.5)), nb, float(rng.uniform(0.6, 1.6)),
                float(rng.uniform(-0.5, 0.5)))
        ours = oracle_lib.dd_backproject(*args, cyl=cyl, off=off)
        ref = oracle_lib.ref_dd_backproject(*args, cyl=cyl, off=off)
        np.testing.assert_array_equal(ours, ref)
        assert np.abs(ref).max() > 0

"""Generates tests/golden/golden.npz from the reference itself.

Runs the reference's own device routines compiled for the host
(oracle/_ref/libnefct_ref.so, built by oracle/Makefile from the reference
sources) on small seeded inputs and stores inputs and outputs.  The tests
compare the oracle restatement (bit for bit) and the GPU kernels (within
tolerance) against these fixtures; they never need the reference checkout.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# Cone-beam cases: (name, grid (nx,ny,nz), centre, size, cyl, da)
CASES = [
    ("flat_iso", (24, 20, 16), (1.0, -0.5, 0.25), (48.0, 40.0, 32.0), False, 2.5),
    ("flat_aniso", (24, 20, 16), (-2.0, 1.5, 0.0), (48.0, 50.0, 48.0), False, 2.5),
    ("cyl_iso", (24, 20, 16), (0.5, 0.5, -1.0), (48.0, 40.0, 32.0), True, 0.012),
]
NV, NA, NB = 12, 40, 32
# distance-driven case (voxel units; SID = source-detector, SAD = source-axis there)
DD_GRID = (24, 20, 16)
DD_SID, DD_SAD = 200.0, 100.0
DD_NA, DD_DA, DD_DA_CYL, DD_AI = 40, 1.1, 0.011, 0.3
DD_NB, DD_DB, DD_BI = 28, 1.2, -0.2
DD_OFF = np.linspace(-1.5, 1.5, NV).astype(np.float32)
SRC_ISO, SRC_DET = 200.0, 400.0
AI, BI, DB = 0.5, 0.5, 2.0


def main() -> None:
    if not oracle.have_ref():
        oracle.build()
    rng = np.random.default_rng(20261203)
    out = {}
    angles = (np.arange(NV) * (2 * np.pi / NV) + 0.1).astype(np.float32)
    out["angles"] = angles
    for name, grid, centre, size, cyl, da in CASES:
        nx, ny, nz = grid
        vol = rng.random((nz, ny, nx), dtype=np.float32)
        sino = rng.random((NV, NB, NA), dtype=np.float32)
        g = oracle.grid(grid, centre, size)
        args = (SRC_ISO, SRC_DET, NA, da, AI, NB, DB, BI)
        out[f"{name}/vol"] = vol
        out[f"{name}/sino_in"] = sino
        out[f"{name}/fwd"] = oracle.ref_cb_forward(g, vol, angles, *args, cyl=cyl)
        out[f"{name}/bp"] = oracle.ref_cb_backward(g, sino, angles, *args, cyl=cyl)
        out[f"{name}/fwd64"] = oracle.ref_cb_forward(g, vol.astype(np.float64), angles.astype(np.float64),
                                                     *args, cyl=cyl, f64=True)
        _, cnt = oracle.cb_forward(g, vol, angles, *args, cyl=cyl, use_cosf=True)
        out[f"{name}/count"] = np.int64(cnt)
    # LOR pair (cpp/siddon): random chords through a 24x20x16 box
    grid, centre, size = (24, 20, 16), (0.0, 0.0, 0.0), (48.0, 40.0, 32.0)
    n = 600
    phi = rng.uniform(0, 2 * np.pi, n)
    p1 = np.stack([60 * np.cos(phi), 60 * np.sin(phi), rng.uniform(-20, 20, n)])
    p2 = np.stack([-60 * np.cos(phi) + rng.uniform(-15, 15, n), -60 * np.sin(phi) + rng.uniform(-15, 15, n),
                   rng.uniform(-20, 20, n)])
    lors = np.concatenate([p1, p2]).astype(np.float32)
    lors[:, :5] = np.array([[0, 0, 0, 3, 0, 0]], np.float32).T   # five short rays: Q4 skips them
    vol = rng.random((16, 20, 24), dtype=np.float32)
    vals = rng.random(n, dtype=np.float32)
    g = oracle.grid(grid, centre, size)
    out["lor/lors"] = lors
    out["lor/vol"] = vol
    out["lor/vals"] = vals
    fwd = oracle.ref_lor_forward(g, vol, lors)
    out["lor/fwd"] = fwd
    out["lor/bp"] = oracle.ref_lor_backward(g, vals, lors)
    # pixel_3d voxel-driven backprojection
    grid, size = (24, 20, 16), (48.0, 40.0, 32.0)
    corner = (-24.0 + 0.5, -20.0 - 0.5, -16.0 + 0.25)
    sino = rng.random((NV, NB, NA), dtype=np.float32)
    out["pixel/sino"] = sino
    out["pixel/corner"] = np.array(corner, np.float32)
    out["pixel/flat"] = oracle.ref_pixel_backproject(sino, angles, grid, corner, size, SRC_ISO, SRC_DET,
                                                     NA, 2.5, 0.0, NB, DB, 0.0)
    out["pixel/cyl"] = oracle.ref_pixel_backproject(sino, angles, grid, corner, size, SRC_ISO, SRC_DET,
                                                    NA, 0.012, 0.0, NB, DB, 0.0, cyl=True)
    # cpp/deform warp
    img = rng.random((18, 20, 22), dtype=np.float32)
    m = [rng.uniform(-3, 3, img.shape).astype(np.float32) for _ in range(3)]
    out["deform/img"] = img
    out["deform/mx"], out["deform/my"], out["deform/mz"] = m
    out["deform/out"] = oracle.ref_deform(img, *m)
    # distance-driven FDK backprojection (dist_3d_back_fdk): voxel units
    proj = rng.random((NV, DD_NB, DD_NA), dtype=np.float32)
    out["dd/proj"] = proj
    out["dd/off"] = DD_OFF
    for key, cyl, da in (("dd/flat", False, DD_DA), ("dd/cyl", True, DD_DA_CYL)):
        out[key] = oracle.ref_dd_backproject(proj, angles, DD_GRID, DD_SID, DD_SAD, DD_NA, da, DD_AI, DD_NB,
                                             DD_DB, DD_BI, cyl=cyl, off=DD_OFF)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in out.values()), "bytes raw")


if __name__ == "__main__":
    main()

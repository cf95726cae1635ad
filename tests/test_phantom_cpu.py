"""CPU: the phantom generator against the reference's own phantom code.

tests/golden/phantom.npz holds phantoms drawn by the reference's
nefct/data/sl_phantom.py (3-D branch, :109-148) -- the standard 3-D
Shepp-Logan table and a seeded table of random ellipsoids -- made by
tests/golden/make_phantom_golden.py.  The torch generator must reproduce
them bit for bit (same float64 arithmetic, same grid, same rounding to
float32)."""
import os

import numpy as np
import pytest

from nefct_b200 import data

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "phantom.npz")


@pytest.fixture(scope="module")
def fixtures():
    return dict(np.load(FIX))


@pytest.mark.parametrize("n", [24, 33])
def test_shepp_logan_3d_bitwise(fixtures, n):
    np.testing.assert_array_equal(data.phantom(n), fixtures[f"sl3d/{n}"])


@pytest.mark.parametrize("n", [24, 33])
def test_random_ellipsoids_bitwise(fixtures, n):
    out = data.ellipsoid_phantom(n, fixtures["rand/rows"]).numpy()
    np.testing.assert_array_equal(out, fixtures[f"rand/{n}"])


def test_bounding_box_evaluation_equals_full_grid():
    """Each ellipsoid is tested only on its bounding box; the sum equals the
    test over the whole grid for ellipsoids that touch the grid's faces."""
    import torch
    rows = data.random_ellipsoids(12, 5)
    rows[0, 1:7] = [0.9, 0.3, 0.5, 0.8, -0.7, 0.1]         # crosses the grid's faces
    n = 29
    g = torch.from_numpy(np.linspace(-1 + 2 / n, 1 - 2 / n, n))
    xg, yg, zg = g.view(-1, 1, 1), g.view(1, -1, 1), g.view(1, 1, -1)
    full = torch.zeros((n, n, n), dtype=torch.float64)
    for e in rows:
        A, a, b, c, x0, y0, z0, phi, theta, psi = [float(v) for v in e]
        al = data._rotation(phi, theta, psi)
        x = xg * al[0, 0] + yg * al[1, 0] + zg * al[2, 0]
        y = xg * al[0, 1] + yg * al[1, 1] + zg * al[2, 1]
        z = xg * al[0, 2] + yg * al[1, 2] + zg * al[2, 2]
        full += ((x - x0) ** 2 / a ** 2 + (y - y0) ** 2 / b ** 2 + (z - z0) ** 2 / c ** 2 <= 1).double() * A
    assert torch.equal(data.ellipsoid_phantom(n, rows), full.float())

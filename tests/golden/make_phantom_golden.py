"""Generates tests/golden/phantom.npz from the reference's own phantom code.

Loads nefct/data/sl_phantom.py from a reference checkout (NEFCT_REF, else
/root/reference) as a standalone module -- its only package import,
``from nefct import nef_class``, is satisfied by a stub, so the package's
HDF5 dependencies (deepdish, h5py) are not needed -- and stores the 3-D
phantoms it draws:

* ``sl3d/<n>``: phantom(n, 'shepp-logan-3d') for n in SIZES;
* ``rand/<n>``: the 3-D branch (sl_phantom.py:109-148) on a seeded table of
  10 random ellipsoids (``rand/rows``), handed to it through its phantom
  table lookup (its ``phantom`` refuses user tables that do not have 6
  columns, so 3-D tables reach the 3-D branch only that way).

    NEFCT_REF=<checkout> python tests/golden/make_phantom_golden.py
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SIZES = (24, 33)


def load_reference_phantom(ref: str):
    stub = types.ModuleType("nefct")
    stub.nef_class = lambda cls: cls
    saved = sys.modules.get("nefct")
    sys.modules["nefct"] = stub
    try:
        spec = importlib.util.spec_from_file_location("ref_sl_phantom",
                                                      os.path.join(ref, "nefct", "data", "sl_phantom.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        if saved is None:
            del sys.modules["nefct"]
        else:
            sys.modules["nefct"] = saved
    return mod


def random_rows(count: int, seed: int) -> np.ndarray:
    """Rows [A, a, b, c, x0, y0, z0, phi, theta, psi]: densities U[0.1, 1],
    semi-axes U[0.05, 0.4], centres U[-0.6, 0.6], angles U[0, 360)."""
    rng = np.random.default_rng(seed)
    rows = np.empty((count, 10))
    rows[:, 0] = rng.uniform(0.1, 1.0, count)
    rows[:, 1:4] = rng.uniform(0.05, 0.4, (count, 3))
    rows[:, 4:7] = rng.uniform(-0.6, 0.6, (count, 3))
    rows[:, 7:10] = rng.uniform(0.0, 360.0, (count, 3))
    return rows


def main() -> None:
    ref = os.environ.get("NEFCT_REF") or "/root/reference"
    mod = load_reference_phantom(ref)
    out = {}
    rows = random_rows(10, 11)
    out["rand/rows"] = rows
    for n in SIZES:
        out[f"sl3d/{n}"] = mod.phantom(n, "shepp-logan-3d")
        orig = mod._select_phantom
        mod._select_phantom = lambda name: [list(r) for r in rows]
        try:
            out[f"rand/{n}"] = mod.phantom(n, "user-3d")
        finally:
            mod._select_phantom = orig
    np.savez_compressed(os.path.join(HERE, "phantom.npz"), **out)
    print("wrote", os.path.join(HERE, "phantom.npz"))


if __name__ == "__main__":
    main()

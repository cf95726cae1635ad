"""Image and projection containers plus the ellipsoid phantom.

Mirrors nefct/data/image.py:25-96, nefct/data/projection.py:118-209 and the
3-D branch of nefct/data/sl_phantom.py:14-148.  ``data`` may be a numpy
array (as in the reference) or a torch tensor (kept on its device); the
index order is the reference's: images [nx, ny, nz], projections
[na, nb, nv].
"""
from __future__ import annotations

import numpy as np
import torch

from .base import nef_class
from .geometry import ScannerConfig3D

__all__ = ["Image", "Image3D", "Image3DT", "ProjectionSequence3D", "all_one_image", "all_zero_image",
           "phantom", "random_ellipsoids", "ellipsoid_phantom"]


def _shape(data) -> list:
    return [int(x) for x in data.shape]


class _ArithmeticMixin:
    """Elementwise arithmetic on ``data`` returning the same container type
    (nefct/ops/common/arithmetic_mixins.py:12-87)."""

    def _op(self, other, fn):
        o = other.data if hasattr(other, "data") else other
        return self.update(data=fn(self.data, o))

    def __add__(self, other): return self._op(other, lambda a, b: a + b)
    def __radd__(self, other): return self._op(other, lambda a, b: b + a)
    def __sub__(self, other): return self._op(other, lambda a, b: a - b)
    def __rsub__(self, other): return self._op(other, lambda a, b: b - a)
    def __mul__(self, other): return self._op(other, lambda a, b: a * b)
    def __rmul__(self, other): return self._op(other, lambda a, b: b * a)
    def __truediv__(self, other): return self._op(other, lambda a, b: a / b)
    def __neg__(self): return self.update(data=-self.data)


class _SaveLoadMixin:
    """obj.save(path) / Cls.load(path) (nefct/io/local_io_mixin.py:14-40),
    through nefct_b200.io."""

    def save(self, path: str) -> str:
        from .io import save
        return save(self, path)

    @classmethod
    def load(cls, path: str, partial=None):
        from .io import load
        return load(cls, path, partial)


@nef_class
class Image(_ArithmeticMixin, _SaveLoadMixin):
    data: object
    center: list
    size: list
    timestamps: object

    @property
    def shape(self):
        return _shape(self.data)

    @property
    def unit_size(self):
        return [s1 / s2 for s1, s2 in zip(self.size, self.shape)]

    @property
    def central_slices(self):
        s = self.shape
        return self.data[s[0] // 2], self.data[:, s[1] // 2], self.data[:, :, s[2] // 2]


@nef_class
class Image3D(Image):
    data: object
    center: list
    size: list
    timestamps: object


@nef_class
class Image3DT(Image):
    data: object
    center: list
    size: list
    timestamps: object = [0]

    def __getitem__(self, item):
        return Image3D(self.data[:, :, :, item], self.center, self.size, self.timestamps[item])


def all_one_image(shape: list, timestamps=None):
    if timestamps is None or np.isscalar(timestamps):
        return Image3D(np.ones(shape, np.float32), [0, 0, 0], list(shape))
    shape_ = list(shape) + [len(timestamps)]
    return Image3DT(np.ones(shape_, np.float32), [0, 0, 0], list(shape), timestamps=timestamps)


def all_zero_image(*args, **kwargs):
    return all_one_image(*args, **kwargs) * 0


@nef_class
class ProjectionSequence3D(_ArithmeticMixin, _SaveLoadMixin):
    data: object
    scanner: ScannerConfig3D
    angles: list
    offsets: list
    timestamps: list

    def __attrs_post_init__(self):
        n_view = self.data.shape[-1]
        if self.angles is None:
            object.__setattr__(self, "angles", [i * 2 * np.pi / n_view for i in range(n_view)])
        if self.offsets is None:
            object.__setattr__(self, "offsets", [0.0])
        if not isinstance(self.offsets, (list, np.ndarray)):
            object.__setattr__(self, "offsets", [self.offsets] * n_view)
        if self.timestamps is None:
            object.__setattr__(self, "timestamps", 0.0)
        if not isinstance(self.timestamps, (list, np.ndarray)):
            object.__setattr__(self, "timestamps", self.timestamps * np.arange(n_view))

    @property
    def shape(self):
        return _shape(self.data)

    @property
    def n_view(self):
        return self.data.shape[2]

    def source_position(self, ind: int):
        x0 = -self.scanner.SAD
        a = self.angles[ind]
        return x0 * np.cos(a), x0 * np.sin(a), 0.0


# ---------------- phantoms ----------------

def _rotation(phi, theta, psi):
    """Euler rotation of nefct/data/sl_phantom.py:130-139 (degrees in,
    converted as there: v * pi / 180)."""
    phi, theta, psi = (v * np.pi / 180 for v in (phi, theta, psi))
    cphi, sphi, cth, sth, cpsi, spsi = np.cos(phi), np.sin(phi), np.cos(theta), np.sin(theta), np.cos(psi), np.sin(psi)
    return np.array([[cpsi * cphi - cth * sphi * spsi, cpsi * sphi + cth * cphi * spsi, spsi * sth],
                     [-spsi * cphi - cth * sphi * cpsi, -spsi * sphi + cth * cphi * cpsi, cpsi * sth],
                     [sth * sphi, -sth * cphi, cth]])


def ellipsoid_phantom(n, ellipsoids, device=None, dtype=torch.float32) -> torch.Tensor:
    """Sum of ellipsoids on an n^3 grid, indexed [x, y, z] like the reference.

    Rows are [A, a, b, c, x0, y0, z0, phi, theta, psi] in the [-1, 1]^3 box;
    grid coordinates linspace(-1 + 2/n, 1 - 2/n, n) (sl_phantom.py:109-148).
    Evaluated in float64 with torch on ``device``.  Each ellipsoid is tested
    only on the grid points of its bounding box (widened by two points):
    the per-point arithmetic is the full-grid test's, and points outside the
    box fail it, so the sum is the same to the bit.
    """
    if np.isscalar(n):
        n = (int(n),) * 3
    dev = torch.device(device) if device is not None else torch.device("cpu")
    # numpy's linspace (the reference's grid, sl_phantom.py:114) to the bit
    rng = [torch.from_numpy(np.linspace(-1 + 2 / k, 1 - 2 / k, k)).to(dev) for k in n]
    p = torch.zeros(n, dtype=torch.float64, device=dev)
    for e in ellipsoids:
        A, a, b, c, x0, y0, z0, phi, theta, psi = [float(v) for v in e]
        al = _rotation(phi, theta, psi)
        # grid point q lies inside when u = al^T q is inside the axis-aligned
        # ellipsoid at (x0, y0, z0); q = al u spans centre +- half along each axis
        centre = al @ np.array([x0, y0, z0])
        half = np.sqrt((al * np.array([a, b, c])) ** 2 @ np.ones(3))
        box = []
        for ax in range(3):
            k = n[ax]
            step = (2 - 4 / k) / (k - 1) if k > 1 else 1.0
            lo = int(np.floor((centre[ax] - half[ax] - (-1 + 2 / k)) / step)) - 2
            hi = int(np.ceil((centre[ax] + half[ax] - (-1 + 2 / k)) / step)) + 3
            box.append(slice(max(lo, 0), min(hi, k)))
        if any(s.start >= s.stop for s in box):
            continue
        xg = rng[0][box[0]].view(-1, 1, 1)
        yg = rng[1][box[1]].view(1, -1, 1)
        zg = rng[2][box[2]].view(1, 1, -1)
        x = xg * al[0, 0] + yg * al[1, 0] + zg * al[2, 0]
        y = xg * al[0, 1] + yg * al[1, 1] + zg * al[2, 1]
        z = xg * al[0, 2] + yg * al[1, 2] + zg * al[2, 2]
        idx = (x - x0) ** 2 / a ** 2 + (y - y0) ** 2 / b ** 2 + (z - z0) ** 2 / c ** 2 <= 1
        p[box[0], box[1], box[2]] += idx.to(torch.float64) * A      # A in float64, as p[idx] += A
    return p.to(dtype)


def random_ellipsoids(count: int, seed: int) -> np.ndarray:
    """Seeded ellipsoid rows: centres U[-0.6, 0.6]^3, semi-axes U[0.05, 0.4],
    Euler angles U[0, 360) degrees, densities U[0.1, 1.0]."""
    rng = np.random.default_rng(seed)
    rows = np.empty((count, 10))
    rows[:, 0] = rng.uniform(0.1, 1.0, count)
    rows[:, 1:4] = rng.uniform(0.05, 0.4, (count, 3))
    rows[:, 4:7] = rng.uniform(-0.6, 0.6, (count, 3))
    rows[:, 7:10] = rng.uniform(0.0, 360.0, (count, 3))
    return rows


_SHEPP_LOGAN_3D = [[1, .6900, .920, .810, 0, 0, 0, 0, 0, 0],
                   [-.8, .6624, .874, .780, 0, -.0184, 0, 0, 0, 0],
                   [-.2, .1100, .310, .220, .22, 0, 0, -18, 0, 10],
                   [-.2, .1600, .410, .280, -.22, 0, 0, 18, 0, 10],
                   [.1, .2100, .250, .410, 0, .35, -.15, 0, 0, 0],
                   [.1, .0460, .046, .050, 0, .1, .25, 0, 0, 0],
                   [.1, .0460, .046, .050, 0, -.1, .25, 0, 0, 0],
                   [.1, .0460, .023, .050, -.08, -.605, 0, 0, 0, 0],
                   [.1, .0230, .023, .020, 0, -.606, 0, 0, 0, 0],
                   [.1, .0230, .046, .020, .06, -.605, 0, 0, 0, 0]]


def phantom(n=256, p_type="shepp-logan-3d", ellipses=None) -> np.ndarray:
    """3-D phantom as numpy float32 [n, n, n] (sl_phantom.py:14-148, 3-D branch)."""
    if ellipses is None:
        if p_type.lower() != "shepp-logan-3d":
            raise ValueError("only the 3-D phantom is provided; pass ellipses for others")
        ellipses = _SHEPP_LOGAN_3D
    elif np.shape(ellipses)[1] != 10:
        raise AssertionError("Wrong number of columns in user phantom")
    return ellipsoid_phantom(n, ellipses).numpy().astype(np.float32)

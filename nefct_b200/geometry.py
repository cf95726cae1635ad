"""Scanner and detector geometry, unchanged from the reference's API.

Mirrors nefct/geometry/detector_config.py:8-37 and
nefct/geometry/scanner_config.py:44-77 (3-D only; the 2-D fan-beam classes
are out of scope).  Naming follows the python side of the reference:
``SID`` is source -> detector, ``SAD`` source -> rotation axis,
``IAD = SID - SAD`` (scanner_config.py:12-24).  The CUDA kernels of the
reference name the two distances the other way round (quirk Q12);
``to_cone_beam`` does the conversion.
"""
from __future__ import annotations

import numpy as np

from .base import nef_class

__all__ = ["DetectorDirectAConfig", "DetectorDirectBConfig", "DetectorConfig", "ScannerConfig",
           "ScannerConfig3D", "cbct_a_detector", "cbct_b_detector", "cbct_3d_scanner",
           "cbct_3d_full_fan_scanner", "cbct_angles"]


@nef_class
class DetectorDirectAConfig:
    number: int
    size: float
    offset: float = 0.0

    @property
    def unit_size(self):
        return self.size / self.number

    @property
    def meshgrid(self):
        return (0.5 + np.arange(self.number)) * self.unit_size - self.size / 2 + self.offset


@nef_class
class DetectorDirectBConfig:
    number: int
    size: float
    offset: float = 0.0

    @property
    def unit_size(self):
        return self.size / self.number

    @property
    def meshgrid(self):
        return (0.5 + np.arange(self.number)) * self.unit_size - self.size / 2 + self.offset


@nef_class
class DetectorConfig:
    direct_a: DetectorDirectAConfig
    direct_b: DetectorDirectBConfig

    @property
    def shape(self):
        return [self.direct_a.number, self.direct_b.number]

    @property
    def size(self):
        return [self.direct_a.size, self.direct_b.size]

    @property
    def center(self):
        return [self.direct_a.offset, self.direct_b.offset]

    @property
    def unit_size(self):
        return [self.direct_a.unit_size, self.direct_b.unit_size]

    @property
    def meshgrid(self):
        return np.meshgrid(self.direct_a.meshgrid, self.direct_b.meshgrid, indexing="ij")


class ScannerConfig:
    pass


@nef_class
class ScannerConfig3D(ScannerConfig):
    mode: str
    SID: float
    SAD: float
    detector_a: DetectorDirectAConfig
    detector_b: DetectorDirectBConfig

    @property
    def IAD(self):
        return self.SID - self.SAD

    @property
    def positions(self):
        if self.mode == "flat" or self.mode.startswith("f"):
            x1 = np.zeros((self.detector_a.number, self.detector_b.number), np.float32) + self.SID - self.SAD
            y1 = np.kron(self.detector_a.meshgrid, [[1]] * self.detector_b.number).transpose()
            z1 = np.kron(self.detector_b.meshgrid, [[1]] * self.detector_a.number)
            return x1, y1, z1
        elif self.mode == "cylin" or self.mode.startswith("c"):
            ang = np.kron(self.detector_a.meshgrid, [[1]] * self.detector_b.number).transpose()
            x1 = self.SID * np.cos(ang) - self.SAD
            y1 = self.SID * np.sin(ang)
            z1 = np.kron(self.detector_b.meshgrid, [[1]] * self.detector_a.number)
            return x1, y1, z1
        elif "2d" in self.mode:
            raise ValueError("switch to ScannerConfig2D")
        raise NotImplementedError

    @property
    def is_flat(self) -> bool:
        return self.mode == "flat" or self.mode.startswith("f")


# presets of nefct/geometry/existing_geometry.py:9-16 (3-D ones)
cbct_a_detector = DetectorDirectAConfig(512, 0.388 * 1024, 147.44)
cbct_b_detector = DetectorDirectBConfig(512, 0.388 * 1024, 0)
cbct_3d_scanner = ScannerConfig3D("flat", 1500, 1000, cbct_a_detector, cbct_b_detector)
cbct_3d_full_fan_scanner = ScannerConfig3D("flat", 1500, 1000, cbct_a_detector.update(offset=0), cbct_b_detector)
cbct_angles = np.linspace(0, np.pi * 2, 599).astype(np.float32)

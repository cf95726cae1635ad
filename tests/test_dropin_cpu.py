"""CPU: host logic of the drop-in layer (geometry conversion, containers,
phantom) -- no GPU calls."""
import numpy as np
import pytest

import nefct_b200 as nb


def test_geometry_conversion_swaps_sid_sad():
    sc = nb.ScannerConfig3D("flat", 1000.0, 500.0, nb.DetectorDirectAConfig(128, 256.0, 4.0),
                            nb.DetectorDirectBConfig(96, 192.0, -2.0))
    g = nb.cone_beam(sc, [64, 64, 64], [0, 0, 0], [128, 128, 128], np.zeros(3), None)
    assert g.src_iso == 500.0 and g.src_det == 1000.0        # Q12
    assert g.da == 2.0 and g.db == 2.0
    # cell centres equal DetectorDirectAConfig.meshgrid
    a = (np.arange(128) + g.a_shift) * g.da - 128 * g.da / 2
    np.testing.assert_allclose(a, sc.detector_a.meshgrid, atol=1e-9)
    b = (np.arange(96) + g.b_shift) * g.db - 96 * g.db / 2
    np.testing.assert_allclose(b, sc.detector_b.meshgrid, atol=1e-9)
    assert g.z_offsets is None and g.det_kind == "flat"


def test_cylindrical_mode_and_offsets():
    sc = nb.ScannerConfig3D("cylin", 1000.0, 500.0, nb.DetectorDirectAConfig(64, 0.5),
                            nb.DetectorDirectBConfig(32, 64.0))
    g = nb.cone_beam(sc, [8, 8, 8], [0, 0, 0], [8, 8, 8], np.zeros(4), [0.0, 1.0, 2.0, 3.0])
    assert g.det_kind == "cyl"
    np.testing.assert_array_equal(g.z_offsets, [0, 1, 2, 3])


def test_projection_sequence_defaults():
    sc = nb.ScannerConfig3D("flat", 1000.0, 500.0, nb.DetectorDirectAConfig(4, 4.0), nb.DetectorDirectBConfig(3, 3.0))
    p = nb.ProjectionSequence3D(np.zeros((4, 3, 5)), sc)
    assert len(p.angles) == 5 and p.n_view == 5
    np.testing.assert_allclose(p.angles[1], 2 * np.pi / 5)
    assert p.offsets == [0.0]
    np.testing.assert_array_equal(p.timestamps, np.zeros(5))


def test_image_unit_size_and_arithmetic():
    img = nb.Image3D(np.ones((4, 6, 8), np.float32), [0, 0, 0], [8.0, 12.0, 16.0])
    assert img.unit_size == [2.0, 2.0, 2.0]
    assert img.shape == [4, 6, 8]
    two = img + img
    assert float(two.data.sum()) == 2 * 4 * 6 * 8
    assert isinstance(two, nb.Image3D)
    assert (img * 3).data.max() == 3


def test_phantom_shape_and_values():
    p = nb.phantom(32)
    assert p.shape == (32, 32, 32) and p.dtype == np.float32
    assert p.max() <= 1.0 + 1e-6
    r = nb.random_ellipsoids(10, 1)
    assert r.shape == (10, 10)
    np.testing.assert_array_equal(r, nb.random_ellipsoids(10, 1))
    q = nb.ellipsoid_phantom(16, r).numpy()
    assert q.sum() > 0


def test_nef_class_is_frozen_with_update():
    d = nb.DetectorDirectAConfig(10, 5.0)
    with pytest.raises(Exception):
        d.number = 3
    assert d.update(number=3).number == 3 and d.number == 10
    assert nb.DetectorDirectAConfig.keys() == ["number", "size", "offset"]

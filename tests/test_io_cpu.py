"""CPU: saving and loading the data and geometry classes (nefct_b200.io,
mirroring nefct/io/local_io_mixin.py and json_io_mixin.py), and
from_dict / astype (nefct/base/base.py:98-121)."""
import numpy as np
import pytest

import nefct_b200 as nb
from nefct_b200 import _lib


def _scanner():
    return nb.ScannerConfig3D("flat", 1200.0, 600.0, nb.DetectorDirectAConfig(64, 76.8),
                              nb.DetectorDirectBConfig(48, 57.6))


def test_image_save_load_round_trip(tmp_path):
    data = np.random.default_rng(1).random((6, 5, 4), dtype=np.float32)
    img = nb.Image3D(data, [0.5, -1.0, 2.0], [12.0, 10.0, 8.0])
    path = img.save(str(tmp_path / "img"))
    assert path.endswith(".npz")
    back = nb.Image3D.load(path)
    np.testing.assert_array_equal(back.data, data)
    assert list(back.center) == [0.5, -1.0, 2.0] and list(back.size) == [12.0, 10.0, 8.0]
    assert back.timestamps is None


def test_projection_with_nested_scanner_round_trip(tmp_path):
    sino = np.random.default_rng(2).random((64, 48, 7), dtype=np.float32)
    ang = list(np.linspace(0, 1, 7, dtype=np.float32))
    proj = nb.ProjectionSequence3D(sino, _scanner(), ang, np.zeros(7, np.float32))
    path = nb.save(proj, str(tmp_path / "p.npz"))
    back = nb.load(nb.ProjectionSequence3D, path)
    np.testing.assert_array_equal(back.data, sino)
    assert isinstance(back.scanner, nb.ScannerConfig3D)
    assert back.scanner.SID == 1200.0 and back.scanner.detector_a.number == 64
    np.testing.assert_array_equal(np.asarray(back.angles), np.asarray(ang))
    part = nb.load(nb.ScannerConfig3D, path, partial="/scanner")
    assert part.SAD == 600.0 and part.detector_b.unit_size == pytest.approx(57.6 / 48)


def test_hdf5_paths_are_refused(tmp_path):
    img = nb.Image3D(np.zeros((2, 2, 2), np.float32), [0, 0, 0], [2, 2, 2])
    with pytest.raises(_lib.NefctError, match="h5py"):
        img.save(str(tmp_path / "x.hdf5"))


def test_json_round_trip_and_data_rule(tmp_path):
    sc = _scanner()
    s = nb.json_dumps(sc)
    assert nb.json_loads(nb.ScannerConfig3D, s).detector_b.number == 48
    path = nb.json_dump(sc, str(tmp_path / "sc.json"))
    assert nb.json_load(nb.ScannerConfig3D, path).asdict(recurse=True) == sc.asdict(recurse=True)
    with pytest.raises(_lib.NefctError, match="dump data first"):
        nb.json_dumps(nb.Image3D(np.zeros((2, 2, 2)), [0, 0, 0], [2, 2, 2]))


def test_from_dict_and_astype():
    img = nb.Image3D(np.ones((2, 3, 4), np.float32), [0, 0, 0], [2, 3, 4])
    t = img.astype(nb.Image3DT)
    assert isinstance(t, nb.Image3DT) and t.size == [2, 3, 4]
    sc = nb.ScannerConfig3D.from_dict(_scanner().asdict(recurse=True))
    assert isinstance(sc.detector_a, nb.DetectorDirectAConfig)
    assert nb.Image3D.from_dict(None).data is None

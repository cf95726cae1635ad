"""Saving and loading the data and geometry classes.

Mirrors nefct/io/local_io_mixin.py:14-61 (``save`` / ``load`` and the
``save`` / ``load`` methods of the data classes) and
nefct/io/json_io_mixin.py:17-70 (``json_dump(s)`` / ``json_load(s)``).

The reference writes ``obj.asdict(recurse=True)`` with deepdish to HDF5.
Neither deepdish nor h5py (nor an HDF5 library) is a dependency of this
package, so ``save`` keeps the same dict tree in a numpy ``.npz``
archive: every array of the tree is one entry (its key the path of names
joined by '/'), and the rest of the tree (scalars, strings, lists, None,
nesting) is one JSON entry, ``__tree__``, in which arrays appear as
``{"__array__": key}``.  Paths ending in .hdf5 / .h5 are refused with an
error that says so.  ``load(cls, path)`` rebuilds the instance with
``cls.from_dict``; ``partial`` loads one sub-tree ('/a/b').
"""
from __future__ import annotations

import json

import numpy as np
import torch

from ._lib import ERR_INVALID, ERR_UNSUPPORTED, NefctError
from .base import NefBaseClass

__all__ = ["save", "load", "json_dump", "json_dumps", "json_load", "json_loads"]


def _to_numpy(v):
    if isinstance(v, torch.Tensor):
        return v.detach().cpu().numpy()
    return v


def _split(tree, prefix: str, arrays: dict):
    """The JSON-able skeleton of tree, arrays moved into `arrays`."""
    tree = _to_numpy(tree)
    if isinstance(tree, dict):
        return {str(k): _split(v, f"{prefix}/{k}", arrays) for k, v in tree.items()}
    if isinstance(tree, np.ndarray):
        key = prefix or "/"
        arrays[key] = tree
        return {"__array__": key}
    if isinstance(tree, (list, tuple)):
        if len(tree) and all(isinstance(_to_numpy(x), (np.ndarray, np.generic)) for x in tree):
            arr = np.asarray([_to_numpy(x) for x in tree])
            key = prefix or "/"
            arrays[key] = arr
            return {"__array__": key, "__list__": True}
        return [_split(v, f"{prefix}/{i}", arrays) for i, v in enumerate(tree)]
    if isinstance(tree, np.generic):
        return tree.item()
    if tree is None or isinstance(tree, (bool, int, float, str)):
        return tree
    raise NefctError(ERR_INVALID, f"cannot save a value of type {type(tree).__name__} at {prefix or '/'}")


def _join(skel, arrays):
    if isinstance(skel, dict):
        if "__array__" in skel:
            arr = arrays[skel["__array__"]]
            return list(arr) if skel.get("__list__") else arr
        return {k: _join(v, arrays) for k, v in skel.items()}
    if isinstance(skel, list):
        return [_join(v, arrays) for v in skel]
    return skel


def _check_path(path: str) -> None:
    if str(path).lower().endswith((".hdf5", ".h5")):
        raise NefctError(ERR_UNSUPPORTED, "HDF5 files need h5py/deepdish, which this environment does not "
                                          "provide; save to a .npz path instead")


def save(obj: NefBaseClass, path: str) -> str:
    """Writes obj.asdict(recurse=True) to path (.npz); returns the path."""
    _check_path(path)
    if not str(path).endswith(".npz"):
        path = f"{path}.npz"
    arrays: dict = {}
    skel = _split(obj.asdict(recurse=True), "", arrays)
    np.savez(path, __tree__=np.asarray(json.dumps(skel)), **arrays)
    return path


def load(cls: type, path: str, partial: str | None = None) -> NefBaseClass:
    """Instance of cls from a file written by save (partial: '/a/b' loads
    that sub-tree of the saved dict instead)."""
    _check_path(path)
    if not (isinstance(cls, type) and issubclass(cls, NefBaseClass)):
        raise NefctError(ERR_INVALID, "cls must be a nef_class")
    with np.load(path, allow_pickle=False) as f:
        arrays = {k: f[k] for k in f.files if k != "__tree__"}
        tree = _join(json.loads(str(f["__tree__"])), arrays)
    if partial:
        for name in partial.strip("/").split("/"):
            tree = tree[name]
    return cls.from_dict(tree)


def _jsonable(v):
    v = _to_numpy(v)
    if isinstance(v, dict):
        return {str(k): _jsonable(x) for k, x in v.items()}
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, (list, tuple)):
        return [_jsonable(x) for x in v]
    if isinstance(v, np.generic):
        return v.item()
    return v


def json_dumps(obj: NefBaseClass) -> str:
    """JSON of obj.asdict(recurse=True); array data must be dumped first
    (json_io_mixin.py:17-22)."""
    dct = obj.asdict(recurse=True)
    for key, val in dct.items():
        if key == "data" and not isinstance(val, str) and val is not None:
            raise NefctError(ERR_INVALID, "please dump data first")
    return json.dumps(_jsonable(dct))


def json_dump(obj: NefBaseClass, path: str) -> str:
    with open(path, "w") as fout:
        fout.write(json_dumps(obj))
    return path


def json_loads(cls: type, json_str: str) -> NefBaseClass:
    return cls.from_dict(json.loads(json_str))


def json_load(cls: type, path: str) -> NefBaseClass:
    with open(path) as fin:
        return json_loads(cls, fin.read())

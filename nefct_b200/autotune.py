"""Autotuner for the launch shape of the cone-beam Siddon kernels.

For a geometry signature (grid, views, detector, kind, flags) it times the
equivalent launch variants of include/nefct_b200.h's tuning table -- the walk
(one thread per ray, or one warp per 32 rows of a detector column), rows or
columns per CTA and the grid order -- on the current device with CUDA
events (forward + transpose, after a warm-up), applies the fastest with
nefct_tune_set and caches the choice in a JSON file
(``$NEFCT_TUNE_CACHE``, default ``~/.cache/nefct_b200/tune.json``).  Every
variant runs the same per-ray arithmetic in the same order (the atomic
transpose's summation order is never fixed).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading

import torch

from . import _lib, ops

_ROWS = (2, 4, 8)
_ORDERS = (0, 1)
_WALKS = (0, 1)
_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("NEFCT_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "nefct_b200",
                                                           "tune.json"))


def signature(geom: ops.ConeBeam, flags: int, device) -> str:
    name = torch.cuda.get_device_name(device)
    nv_bucket = 1 << max(0, (geom.nv - 1).bit_length())
    return (f"{name}|{geom.shape}|{geom.size}|nv~{nv_bucket}|{geom.na}x{geom.nb}|{geom.det_kind}|"
            f"{geom.src_iso:.1f}/{geom.src_det:.1f}|flags={flags}")


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db: dict) -> None:
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def apply(rows: int, order: int, walk: int | None = None) -> None:
    _lib.call("nefct_tune_set", _lib.TUNE_CB_ROWS, int(rows))
    _lib.call("nefct_tune_set", _lib.TUNE_CB_ORDER, int(order))
    if walk is not None:
        _lib.call("nefct_tune_set", _lib.TUNE_CB_WALK, int(walk))


def current() -> dict:
    lib = _lib.load()
    return {"rows": lib.nefct_tune_get(_lib.TUNE_CB_ROWS), "order": lib.nefct_tune_get(_lib.TUNE_CB_ORDER),
            "walk": lib.nefct_tune_get(_lib.TUNE_CB_WALK)}


def tune_cone_beam(geom: ops.ConeBeam, flags: int = 0, device=None, reps: int = 2, use_cache: bool = True) -> dict:
    """Picks and applies the fastest launch shape for forward + transpose of
    this geometry; returns {"rows", "order", "walk", "ms": {variant: ms}}."""
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = signature(geom, flags, device)
    with _lock:
        db = _load() if use_cache else {}
        if key in db and "walk" in db[key]:
            apply(db[key]["rows"], db[key]["order"], db[key]["walk"])
            return db[key]
        gen = torch.Generator(device=device).manual_seed(0)
        vol = torch.rand(geom.vol_shape, device=device, generator=gen)
        grad = torch.rand(geom.sino_shape, device=device, generator=gen)
        sino = torch.empty(geom.sino_shape, device=device)
        back = torch.empty(geom.vol_shape, device=device)
        # forward and transpose are timed separately for each walk; rows and
        # order are shared, the walk is chosen per direction
        times, best = {}, None
        for rows in _ROWS:
            for order in _ORDERS:
                t_dir = {}
                for walk in _WALKS:
                    apply(rows, order, 3 * walk)
                    for name, fn in (("fwd", lambda: ops.cb_forward(vol, geom, flags, out=sino)),
                                     ("bwd", lambda: ops.cb_backward(grad, geom, flags, out=back))):
                        fn()
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record()
                        for _ in range(reps):
                            fn()
                        e1.record()
                        e1.synchronize()
                        t_dir[(name, walk)] = e0.elapsed_time(e1) / reps
                wf = min(_WALKS, key=lambda w: t_dir[("fwd", w)])
                wb = min(_WALKS, key=lambda w: t_dir[("bwd", w)])
                for walk in _WALKS:
                    times[f"{rows}/{order}/{3 * walk}"] = t_dir[("fwd", walk)] + t_dir[("bwd", walk)]
                    times[f"{rows}/{order}/{3 * walk}/fwd"] = t_dir[("fwd", walk)]
                    times[f"{rows}/{order}/{3 * walk}/bwd"] = t_dir[("bwd", walk)]
                total = t_dir[("fwd", wf)] + t_dir[("bwd", wb)]
                if best is None or total < best[0]:
                    best = (total, rows, order, wf | (wb << 1))
        _, rows, order, walk = best
        apply(rows, order, walk)
        rec = {"rows": rows, "order": order, "walk": walk, "ms": times}
        if use_cache:
            db = _load()
            db[key] = rec
            _store(db)
        return rec

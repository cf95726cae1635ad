"""ctypes binding of libnefct_b200.so (the C ABI of include/nefct_b200.h).

The library is loaded lazily on first use.  There is no fallback: if the
shared object is missing or fails to load, every op raises NefctError.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libnefct_b200.so")

# status codes
OK, ERR_INVALID, ERR_CUDA, ERR_WORKSPACE, ERR_TIMEOUT, ERR_UNSUPPORTED = 0, 1, 2, 3, 4, 5

# walk flags (include/nefct_b200.h)
TIE_GT = 0x01
SKIP_SHORT = 0x02
NO_INV_L2 = 0x04
Q5 = 0x08
Q8_INDEX = 0x10
NO_TRANSPOSE = 0x20
DETERMINISTIC = 0x40
EXACT = 0x80
REF_FORWARD = 0
REF_BACKPROJECT = TIE_GT | SKIP_SHORT | NO_INV_L2
LINE_INTEGRAL = NO_INV_L2
LOR_REF_FORWARD = TIE_GT | SKIP_SHORT | Q5
LOR_REF_BACKPROJECT = TIE_GT | SKIP_SHORT | NO_INV_L2
FDK_NO_WEIGHT = 0x100

DET_FLAT, DET_CYL = 0, 1
TUNE_CB_ROWS, TUNE_CB_ORDER, TUNE_CB_WALK = 0, 1, 2
BATCH_PERSISTENT, BATCH_PER_PROBLEM = 0, 1
WIN_RAM_LAK, WIN_SHEPP_LOGAN, WIN_COSINE, WIN_HAMMING, WIN_HANN = 0, 1, 2, 3, 4
WINDOWS = {"ram-lak": WIN_RAM_LAK, "shepp-logan": WIN_SHEPP_LOGAN, "cosine": WIN_COSINE,
           "hamming": WIN_HAMMING, "hann": WIN_HANN}


class NefctError(RuntimeError):
    """A C-ABI call returned a non-zero status (or the library is missing)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"nefct_b200 status {status}: {message}")
        self.status = status


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float),
                ("sx", C.c_float), ("sy", C.c_float), ("sz", C.c_float)]


class CBGeom(C.Structure):
    _fields_ = [("grid", Grid), ("nv", C.c_int32),
                ("angles", C.POINTER(C.c_float)), ("z_offsets", C.POINTER(C.c_float)),
                ("src_iso", C.c_float), ("src_det", C.c_float),
                ("na", C.c_int32), ("da", C.c_float), ("a_shift", C.c_float),
                ("nb", C.c_int32), ("db", C.c_float), ("b_shift", C.c_float),
                ("det_kind", C.c_int32)]


class DDGeom(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("nv", C.c_int32),
                ("angles", C.POINTER(C.c_float)), ("z_offsets", C.POINTER(C.c_float)),
                ("src_iso", C.c_float), ("src_det", C.c_float),
                ("na", C.c_int32), ("da", C.c_float), ("a_offset", C.c_float),
                ("nb", C.c_int32), ("db", C.c_float), ("b_offset", C.c_float),
                ("det_kind", C.c_int32)]


class CBProblem(C.Structure):
    _fields_ = [("geom", CBGeom), ("vol", C.c_void_p), ("sino", C.c_void_p), ("grad", C.c_void_p),
                ("back", C.c_void_p)]


_vp = C.c_void_p
_i32 = C.c_int32
_u32 = C.c_uint32
_PROTOS = {
    "nefct_version": (C.c_char_p, []),
    "nefct_status_string": (C.c_char_p, [_i32]),
    "nefct_last_error": (C.c_char_p, []),
    "nefct_tune_set": (_i32, [_i32, _i32]),
    "nefct_tune_get": (_i32, [_i32]),
    "nefct_cb_workspace_bytes": (C.c_size_t, [C.POINTER(CBGeom), _u32]),
    "nefct_cb_forward": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_cb_backward": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_cb_forward_noalloc": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp]),
    "nefct_cb_forward_f64": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_cb_backward_f64": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_cb_count_intersections": (_i32, [C.POINTER(CBGeom), _u32, _vp, _vp]),
    "nefct_cb_batch_plan": (_i32, [C.POINTER(CBProblem), _i32, _u32, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]),
    "nefct_cb_batch_bind": (_i32, [_vp, _vp, C.c_size_t, _vp]),
    "nefct_cb_batch_forward": (_i32, [_vp, _vp]),
    "nefct_cb_batch_backward": (_i32, [_vp, _vp]),
    "nefct_cb_batch_tiles": (C.c_int64, [_vp]),
    "nefct_cb_batch_set_strategy": (_i32, [_vp, _i32]),
    "nefct_cb_batch_set_buffers": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "nefct_cb_batch_destroy": (None, [_vp]),
    "nefct_lor_forward": (_i32, [C.POINTER(Grid), _vp, C.c_int64, _vp, _vp, _u32, _vp]),
    "nefct_lor_backward": (_i32, [C.POINTER(Grid), _vp, C.c_int64, _vp, _vp, _u32, _vp]),
    "nefct_lor_order_keys": (_i32, [C.POINTER(Grid), _vp, C.c_int64, _vp, _vp]),
    "nefct_lor_forward_ordered": (_i32, [C.POINTER(Grid), _vp, C.c_int64, _vp, _vp, _vp, _u32, _vp]),
    "nefct_lor_backward_ordered": (_i32, [C.POINTER(Grid), _vp, C.c_int64, _vp, _vp, _vp, _u32, _vp]),
    "nefct_fdk_filter": (_i32, [C.POINTER(CBGeom), _vp, _vp, _i32, _i32, _vp]),
    "nefct_fdk_backproject": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp]),
    "nefct_fdk_workspace_bytes": (C.c_size_t, [C.POINTER(CBGeom)]),
    "nefct_fdk_backproject_ws": (_i32, [C.POINTER(CBGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_warp_forward": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "nefct_warp_adjoint": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "nefct_warp_grad_dvf": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
    "nefct_warp_invert": (_i32, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
    "nefct_warp_forward_f64": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "nefct_warp_adjoint_f64": (_i32, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "nefct_warp_grad_dvf_f64": (_i32, [_vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
    "nefct_dd_workspace_bytes": (C.c_size_t, [C.POINTER(DDGeom)]),
    "nefct_dd_backproject": (_i32, [C.POINTER(DDGeom), _vp, _vp, _vp, C.c_size_t, _vp]),
    "nefct_dd_forward": (_i32, [C.POINTER(DDGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_dd_backward": (_i32, [C.POINTER(DDGeom), _vp, _vp, _u32, _vp, C.c_size_t, _vp]),
    "nefct_dd_forward_f64": (_i32, [C.POINTER(DDGeom), _vp, _vp, _u32, _vp]),
    "nefct_dd_backward_f64": (_i32, [C.POINTER(DDGeom), _vp, _vp, _u32, _vp]),
    "nefct_probe_sink_floats": (C.c_size_t, [_i32]),
    "nefct_probe_l2_read": (_i32, [_vp, C.c_size_t, _i32, _i32, _vp, _vp]),
    "nefct_probe_l2_red": (_i32, [_vp, C.c_size_t, _i32, _i32, _vp]),
}

_lib: C.CDLL | None = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Loads the shared library (once).  Raises NefctError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise NefctError(-1, f"{LIB_PATH} is missing; build it with `python -m nefct_b200.build`")
            try:
                lib = C.CDLL(LIB_PATH)
            except OSError as e:
                raise NefctError(-1, f"cannot load {LIB_PATH}: {e}") from e
            for name, (res, args) in _PROTOS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def symbols() -> list[str]:
    return list(_PROTOS)


def check(status: int) -> None:
    if status != OK:
        lib = load()
        msg = lib.nefct_last_error().decode(errors="replace")
        raise NefctError(status, f"{lib.nefct_status_string(status).decode()}: {msg}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))

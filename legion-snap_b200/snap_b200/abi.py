"""ctypes binding of the C ABI declared in include/snap_b200.h.

The library is built in-tree (``snap_b200/libsnap_b200.so``).  There is no
fallback: if it is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libsnap_b200.so"

SNAP_OK = 0
STATUS = {0: "SNAP_OK", 1: "SNAP_ERR_BAD_ARG", 2: "SNAP_ERR_UNSUPPORTED", 3: "SNAP_ERR_OOM",
          4: "SNAP_ERR_DEVICE_TIMEOUT", 5: "SNAP_ERR_CUDA"}
SNAP_FP64, SNAP_FP32 = 0, 1

_dp = C.POINTER(C.c_double)


class SnapConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nang", C.c_int),
                ("ng", C.c_int), ("nmom", C.c_int), ("nmat", C.c_int), ("fixup", C.c_int),
                ("precision", C.c_int), ("hi", C.c_double), ("hj", C.c_double),
                ("hk", C.c_double), ("mu", _dp), ("eta", _dp), ("xi", _dp), ("w", _dp),
                ("ec", _dp)]


class SnapIterRecord(C.Structure):
    _fields_ = [("kind", C.c_int), ("time_step", C.c_int), ("outer", C.c_int),
                ("inner", C.c_int), ("converged", C.c_int), ("us", C.c_double)]


class SnapSolveInfo(C.Structure):
    _fields_ = [("epsi", C.c_double), ("iitm", C.c_int), ("oitm", C.c_int),
                ("inner_total", C.c_int), ("outer_total", C.c_int), ("converged", C.c_int),
                ("inners_per_outer", C.c_int * 1024), ("sweep_ms", C.c_double),
                ("total_ms", C.c_double), ("outers_lowp", C.c_int),
                ("records", C.POINTER(SnapIterRecord)), ("records_cap", C.c_int),
                ("records_len", C.c_int)]


class SnapTimeConfig(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("dt", C.c_double), ("vdelt", C.c_void_p),
                ("psi_t", C.c_void_p), ("psi_t_initialised", C.c_int), ("qim", C.c_void_p),
                ("qim_time_scaled", C.c_int)]


class SnapTiming(C.Structure):
    _fields_ = [("sweep_ms", C.c_double), ("sweep_calls", C.c_longlong),
                ("kernel_launches", C.c_longlong)]


class SnapError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


# (name, argtypes) of every entry point in include/snap_b200.h
_vp, _ip = C.c_void_p, C.POINTER(C.c_int)
SIGNATURES = {
    "snap_create": [C.POINTER(SnapConfig), C.c_int, C.POINTER(C.c_void_p)],
    "snap_destroy": [_vp],
    "snap_scratch_bytes": [_vp],
    "snap_expand_xs": [_vp, _vp, _vp, _vp, _vp],
    "snap_expand_scattering_xs": [_vp, _vp, _vp, _vp, _vp],
    "snap_calc_outer_source": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snap_calc_outer_source_tc": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snap_calc_outer_source_groups": [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp],
    "snap_calc_inner_source": [_vp, _vp, _vp, _vp, _vp, _vp],
    "snap_sweep": [_vp, _vp, _vp, _vp, _vp],
    "snap_test_convergence": [_vp, C.c_int, _vp, _vp, C.c_double, _ip, _vp],
    "snap_inner_iteration": [_vp, _vp, _vp, _vp, _vp, _vp, C.c_double, _ip, _vp],
    "snap_get_timing": [_vp, C.POINTER(SnapTiming), C.c_int],
    "snap_transport_solve": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(SnapSolveInfo), _vp],
    "snap_transport_solve_td": [_vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(SnapTimeConfig), _vp,
                                C.POINTER(SnapSolveInfo), _vp],
    "snap_record_forward": [_vp, _vp, _vp, _vp, _vp],
    "snap_adjoint_sweep": [_vp, _vp, _vp, _vp, _vp, _vp],
    "snap_adjoint_solve": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                           C.POINTER(SnapSolveInfo), _vp],
    "snap_sweep_noalloc": [C.POINTER(SnapConfig), _vp, _vp, _vp, _vp],
    "snap_inject_stall": [_vp, C.c_int],
    "snap_sweep_td": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snap_mms_init": [_vp, _vp, _vp, _vp, C.c_double, C.c_double, C.c_double, _vp, C.c_int,
                      C.c_double, C.c_double, _vp, _vp, _vp, _vp],
    "snap_mms_compare": [_vp, _vp, _vp, _vp, _vp],
    "snap_selftest_division": [C.c_int, _vp, _vp, C.c_longlong, _vp, _vp],
    "snap_last_error": [],
}

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library, failing loudly if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
        lib = C.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        lib.snap_scratch_bytes.restype = C.c_size_t
        lib.snap_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def check(status: int):
    if status != SNAP_OK:
        msg = load().snap_last_error()
        raise SnapError(status, msg.decode() if msg else "")

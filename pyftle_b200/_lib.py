"""ctypes binding of ``libpyftle_b200.so`` (the C ABI in ``include/pyftle_b200.h``).

The library is built in-tree by ``pyftle_b200/build.py``.  There is no
fallback: if the shared library is missing or CUDA is unavailable every entry
point raises, so nothing silently runs on the CPU.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyftle_b200.so")

FTLE_OK, FTLE_ERR_INVALID, FTLE_ERR_CUDA, FTLE_ERR_DEVICE, FTLE_ERR_UNSUPPORTED = range(5)
EULER, AB2, RK4 = 0, 1, 2
HOLD, BLEND = 0, 1
F64, F16, BF16, FX15, FX16 = 0, 1, 2, 3, 4

INTEGRATOR_CODES = {"euler": EULER, "ab2": AB2, "rk4": RK4}
STORAGE_CODES = {"fp64": F64, "fp16": F16, "bf16": BF16, "fx15": FX15, "fx16": FX16}
TIME_MODES = {"hold": HOLD, "blend": BLEND}

_c_dp = ctypes.c_void_p  # device pointers travel as plain addresses
_i32, _i64, _f64, _f32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_float


class FtleGrid(ctypes.Structure):
    """Mirror of ``ftle_grid``."""

    _fields_ = [("dim", _i32), ("n", _i32 * 3), ("origin", _f64 * 3), ("spacing", _f64 * 3),
                ("periodic", _i32), ("reserved", _i32)]


class FtleWindow(ctypes.Structure):
    """Mirror of ``ftle_window``."""

    _fields_ = [("grid", FtleGrid), ("snapshots", _c_dp), ("num_snapshots", _i32),
                ("storage", _i32), ("time_mode", _i32), ("periodic_time", _i32),
                ("snapshot_t0", _f64), ("snapshot_dt", _f64), ("first_snapshot", _i32),
                ("integrator", _i32), ("t0", _f64), ("h", _f64), ("num_steps", _i32),
                ("flags", _i32), ("positions", _c_dp), ("num_groups", _i64),
                ("map_period", _f64), ("ftle", _c_dp)]


class FtleFlow(ctypes.Structure):
    """Mirror of ``ftle_flow``."""

    _fields_ = [("kind", _i32), ("reserved", _i32), ("params", _f64 * 8)]


FLOW_DOUBLE_GYRE, FLOW_ABC = 0, 1
KEEP_POSITIONS = 1

# name -> (restype, argtypes)
SIGNATURES = {
    "ftle_version": (ctypes.c_int, []),
    "ftle_last_error": (ctypes.c_char_p, []),
    "ftle_stream_synchronize": (ctypes.c_int, [_c_dp]),
    "ftle_interp2d_vec_inplace": (ctypes.c_int, [_c_dp, _i32, _i32, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_interp3d_vec_inplace": (ctypes.c_int,
                                  [_c_dp, _i32, _i32, _i32, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_grid_interpolate": (ctypes.c_int,
                              [ctypes.POINTER(FtleGrid), _c_dp, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_grid_step": (ctypes.c_int, [ctypes.POINTER(FtleGrid), _c_dp, _i32, _f64, _c_dp, _i64,
                                      _c_dp, _i32, _c_dp]),
    "ftle_axpy": (ctypes.c_int, [_c_dp, _c_dp, _f64, _c_dp, _i64, _c_dp]),
    "ftle_ab2_update": (ctypes.c_int, [_c_dp, _f64, _c_dp, _c_dp, _i64, _c_dp]),
    "ftle_rk4_update": (ctypes.c_int, [_c_dp, _f64, _c_dp, _c_dp, _c_dp, _c_dp, _i64, _c_dp]),
    "ftle_flow_map_jacobian": (ctypes.c_int, [_i32, _c_dp, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_cauchy_green": (ctypes.c_int, [_i32, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_max_eigenvalue": (ctypes.c_int, [_i32, _c_dp, _i64, _c_dp, _c_dp]),
    "ftle_from_jacobian": (ctypes.c_int, [_i32, _c_dp, _i64, _f64, _c_dp, _c_dp]),
    "ftle_from_positions": (ctypes.c_int, [_i32, _c_dp, _c_dp, _i64, _f64, _c_dp, _c_dp]),
    "ftle_packed_snapshot_bytes": (ctypes.c_int64, [_i32, _i64, _i32, _i32]),
    "ftle_pack_snapshots": (ctypes.c_int, [_i32, _i64, _i32, _i32, _c_dp, _i32, _c_dp, _c_dp]),
    "ftle_window_run_f64": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _c_dp]),
    "ftle_gather_probe": (ctypes.c_int, [_c_dp, _i64, _i64, _i64, _i32, _i32, _i32,
                                         ctypes.c_uint32, _c_dp, _c_dp]),
    "ftle_gather_probe_loads": (_i64, [_i32, _i32]),
    "ftle_window_run_mixed": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _c_dp]),
    "ftle_window_workspace_bytes": (ctypes.c_int64, [ctypes.POINTER(FtleWindow)]),
    "ftle_window_run_mixed_chunked": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _c_dp, _i64,
                                                     _i32, _i32, _c_dp]),
    "ftle_window_run_mixed_chunked_static": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _i32,
                                                            _i32, _c_dp]),
    "ftle_analytic_window_run": (ctypes.c_int, [ctypes.POINTER(FtleFlow), _i32, _f64, _f64, _i32,
                                                _i32, _c_dp, _i64, _f64, _c_dp, _c_dp]),
    "ftle_windows_plan_bytes": (ctypes.c_int64, [ctypes.POINTER(FtleWindow), _i32]),
    "ftle_windows_plan": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _i32, _i32, _c_dp, _i64]),
    "ftle_windows_run_mixed": (ctypes.c_int, [ctypes.POINTER(FtleWindow), _i32, _c_dp, _i64,
                                              _i32, _c_dp]),
    # flow-map surrogate MLP (BF16 tensor-core kernels)
    "ftle_mlp_gemm": (ctypes.c_int, [_c_dp, _i32, _i32, _c_dp, _i32, _i32, _c_dp, _i32, _i32,
                                     _i32, _i32, _i32, _i32, _c_dp, _c_dp]),
    "ftle_mlp_linear": (ctypes.c_int, [_c_dp, _i32, _c_dp, _i32, _c_dp, _i32, _i32, _i32, _i32,
                                       _c_dp, _i32, _c_dp, _i32, _c_dp, _c_dp]),
    "ftle_mlp_gemm_dsilu": (ctypes.c_int, [_c_dp, _i32, _i32, _c_dp, _i32, _i32, _i32, _i32,
                                           _i32, _c_dp, _i32, _c_dp, _i32, _c_dp, _c_dp, _c_dp]),
    "ftle_mlp_features": (ctypes.c_int, [_c_dp, _i64, _c_dp, _i32, _c_dp, _c_dp, _c_dp, _c_dp]),
    "ftle_mlp_mse_grad": (ctypes.c_int, [_c_dp, _i32, _c_dp, _i32, _i64, _c_dp, _i32, _c_dp,
                                         _c_dp, _c_dp]),
    "ftle_mlp_adam": (ctypes.c_int, [_c_dp, _c_dp, _c_dp, _c_dp, _c_dp, _i64, _f32, _f32, _f32,
                                     _f32, _i32, _f32, _c_dp]),
    "ftle_mlp_jacobian_ftle": (ctypes.c_int, [_c_dp, _c_dp, _i32, _i64, _f64, _f64, _c_dp,
                                              _c_dp]),
    "ftle_mlp_apply_displacement": (ctypes.c_int, [_c_dp, _c_dp, _i32, _i64, _f64, _c_dp,
                                                   _c_dp]),
    "ftle_mlp_features3": (ctypes.c_int, [_c_dp, _i64, _c_dp, _i32, _c_dp, _c_dp, _c_dp, _c_dp,
                                          _c_dp]),
    "ftle_mlp_jacobian_ftle3": (ctypes.c_int, [_c_dp, _c_dp, _c_dp, _i32, _i64, _f64, _f64,
                                               _c_dp, _c_dp]),
    "ftle_mlp_apply_displacement3": (ctypes.c_int, [_c_dp, _c_dp, _i32, _i64, _f64, _c_dp,
                                                    _c_dp]),
    "ftle_surrogate_packed_bytes": (ctypes.c_int64, []),
    "ftle_surrogate_pack": (ctypes.c_int, [_c_dp, _c_dp, _c_dp, _c_dp, _c_dp, _c_dp, _c_dp]),
    "ftle_surrogate_ftle": (ctypes.c_int, [_c_dp, _i64, _f64, _c_dp, _c_dp, _c_dp, _f64, _f64,
                                           _c_dp, _c_dp, _c_dp, _c_dp]),
}

_lock = threading.Lock()
_lib = None


class FTLEError(RuntimeError):
    """Raised when a C-ABI entry point returns a non-zero status."""

    def __init__(self, status: int, name: str, message: str):
        super().__init__(f"{name} failed with status {status}: {message}")
        self.status = status


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the engine library (no fallback: a missing library is an error)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build the CUDA engine with `python -m pyftle_b200.build`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def call(name: str, *args) -> int:
    """Call an entry point and raise FTLEError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != FTLE_OK:
        msg = lib.ftle_last_error()
        raise FTLEError(rc, name, msg.decode() if msg else "")
    return rc

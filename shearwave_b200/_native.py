"""ctypes binding of the C ABI declared in include/shearwave_b200.h.

The shared library is built in-tree (``python -m shearwave_b200.build``) and
loaded from ``shearwave_b200/_lib``.  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libshearwave_b200.so"

SW_F32, SW_F64 = 0, 1
SW_PLAIN_F64, SW_MIXED_F32 = 0, 1
SW_OK, SW_EINVAL, SW_ECUDA, SW_ENONFINITE, SW_ERANGE, SW_EWORKSPACE, SW_ETIMEOUT = range(7)
# solve flag bits (sw_fdtd_desc.flags)
FLAG_NONFINITE, FLAG_TIMEOUT, FLAG_REFUSED = 1, 2, 4
# sw_tune_knob values that are not launch-shape knobs
SW_TUNE_WAIT_BUDGET = 5
SW_CG_CONVERGED = 1
CG_REASONS = {0: "running", 1: "converged", 2: "breakdown", 3: "nonfinite", 4: "max_iters",
              5: "early_exit"}

_vp, _i32, _i64, _f64, _sz = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_size_t


class CGStats(C.Structure):
    """sw_cg_stats."""

    _fields_ = [("iters", C.c_int32), ("reason", C.c_int32), ("rel", C.c_double),
                ("max_div", C.c_double)]

    def as_dict(self) -> dict:
        return {"iters": int(self.iters), "reason": CG_REASONS.get(self.reason, str(self.reason)),
                "rel": float(self.rel), "max_div": float(self.max_div)}


class ProjectJob(C.Structure):
    """sw_project_job."""

    _fields_ = [
        ("in_dtype", C.c_int32),
        ("fx", C.c_void_p), ("fy", C.c_void_p), ("fz", C.c_void_p),
        ("sx", C.c_int64), ("sy", C.c_int64), ("sz", C.c_int64),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dX", C.c_double), ("dY", C.c_double), ("dZ", C.c_double), ("tol", C.c_double),
        ("max_iters", C.c_int32),
        ("out", C.c_void_p),
        ("workspace", C.c_void_p),
        ("workspace_bytes", C.c_size_t),
    ]


class FdtdDesc(C.Structure):
    """sw_fdtd_desc (field order and types must match the header)."""

    _fields_ = [
        ("precision", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("pz", C.c_int32),
        ("n_steps", C.c_int32),
        ("dX", C.c_double), ("dY", C.c_double), ("dZ", C.c_double), ("dT", C.c_double),
        ("vel_damp", C.c_double),
        ("state", C.c_void_p * 3),
        ("coef_m", C.c_void_p), ("coef_e", C.c_void_p), ("inv_rho", C.c_void_p),
        ("patterns", C.c_void_p),
        ("n_patterns", C.c_int32),
        ("term_off", C.c_void_p), ("term_pat", C.c_void_p), ("term_scale", C.c_void_p),
        ("kahan", C.c_int32),
        ("snap_stride", C.c_int32),
        ("snaps", C.c_void_p),
        ("n_traces", C.c_int32),
        ("trace_cells", C.c_void_p),
        ("traces", C.c_void_p),
        ("flags", C.c_void_p),
        ("xchunk", C.c_int32),
        ("steps_per_pass", C.c_int32),
        ("kernel", C.c_int32),
        ("clock", C.c_void_p),
        ("queue", C.c_void_p),
        ("stall_test", C.c_int32),
    ]


_SIGNATURES = {
    "sw_abi_version": ([], C.c_int),
    "sw_last_error": ([], C.c_char_p),
    "sw_set_device": ([C.c_int], C.c_int),
    "sw_pitch": ([C.c_int], C.c_int),
    "sw_fdtd_desc_size": ([], _sz),
    "sw_launch_count": ([], C.c_uint64),
    "sw_host_enqueue_count": ([], C.c_uint64),
    "sw_arf_workspace_bytes": ([C.c_int64, C.c_int32], _sz),
    "sw_arf_envelope": ([C.c_int, _vp, C.c_int64, C.c_int32, _vp, _vp, _sz, _vp], C.c_int),
    "sw_arf_force": ([C.c_int, C.c_int, _vp, _vp, _vp, _vp, C.c_int64, C.c_int32, _vp, C.c_int32,
                      _vp, _vp, _vp, C.c_int64, C.c_double, C.c_int, _vp, _vp, _vp, _vp],
                     C.c_int),
    "sw_tune_set": ([C.c_int, C.c_int], C.c_int),
    "sw_tune_get": ([C.c_int], C.c_int),
    "sw_laplacian": ([C.c_int, _vp, _vp, C.c_int, C.c_int, C.c_int, _f64, _f64, _f64, _vp],
                     C.c_int),
    "sw_divergence": ([C.c_int, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _f64, _f64, _f64,
                       _vp], C.c_int),
    "sw_gradient": ([C.c_int, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, _f64, _f64, _f64,
                     _vp], C.c_int),
    "sw_project_workspace_bytes": ([C.c_int, C.c_int, C.c_int], _sz),
    "sw_project": ([C.c_int, _vp, _vp, _vp, _i64, _i64, _i64, C.c_int, C.c_int, C.c_int, _f64,
                    _f64, _f64, _f64, C.c_int, _vp, _vp, _sz, C.POINTER(CGStats), _vp], C.c_int),
    "sw_project_spectral_workspace_bytes": ([C.c_int, C.c_int, C.c_int], _sz),
    "sw_project_spectral": ([C.c_int, _vp, _vp, _vp, _i64, _i64, _i64, C.c_int, C.c_int,
                             C.c_int, _f64, _f64, _f64, _vp, _vp, _sz, C.POINTER(CGStats), _vp],
                            C.c_int),
    "sw_spectral_basis": ([C.c_int, _f64, _vp, _vp], C.c_int),
    "sw_project_noalloc_scratch_bytes": ([], _sz),
    "sw_project_noalloc": ([C.c_int, _vp, _vp, _vp, _i64, _i64, _i64, C.c_int, C.c_int,
                            C.c_int, _f64, _f64, _f64, _f64, C.c_int, _vp, C.POINTER(CGStats),
                            _vp], C.c_int),
    "sw_project_batch_table_bytes": ([C.c_int], _sz),
    "sw_project_batch": ([C.POINTER(ProjectJob), C.c_int, _vp, _sz, C.POINTER(CGStats), _vp],
                         C.c_int),
    "sw_fdtd_batch_table_bytes": ([C.c_int], _sz),
    "sw_fdtd_batch_steps": ([C.POINTER(FdtdDesc), C.POINTER(C.c_int32), C.c_int, _i32, _i32, _vp,
                             _sz, _vp], C.c_int),
    "sw_static_solve": ([C.c_int, _vp, _vp, _f64, _i64, _i64, _i64, C.c_int, C.c_int, C.c_int,
                         _f64, _f64, _f64, _f64, C.c_int, _vp, _vp, _sz, C.POINTER(CGStats), _vp],
                        C.c_int),
    "sw_convert": ([C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _i64, _i64, _i64,
                    _i64, _f64, C.c_int, _vp, _i64, _i64, _i64, _vp], C.c_int),
    "sw_fdtd_materials": ([C.POINTER(FdtdDesc), C.c_int, _vp, _f64, _vp, _f64, C.c_int, _vp,
                           _f64, _vp], C.c_int),
    "sw_fdtd_init": ([C.POINTER(FdtdDesc), _vp, _vp, _vp], C.c_int),
    "sw_fdtd_steps": ([C.POINTER(FdtdDesc), _i32, _i32, _vp], C.c_int),
    "sw_fdtd_finish": ([C.POINTER(FdtdDesc), _i32, _vp, _vp, _vp], C.c_int),
    "sw_fdtd_status": ([C.POINTER(FdtdDesc), C.POINTER(C.c_int32), _vp], C.c_int),
    "sw_fdtd_reproject": ([C.POINTER(FdtdDesc), _i32, _f64, C.c_int, _vp, _vp, _sz,
                           C.POINTER(CGStats), _vp], C.c_int),
    "sw_strain": ([C.c_int, _vp, _vp, _vp, _i64, _i64, _i64, C.c_int, C.c_int, C.c_int, _f64,
                   _f64, _f64, _vp, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "sw_strain_invariants": ([C.c_int, _vp, _i64, _vp, _vp, _vp, _vp, _vp], C.c_int),
}

_lib = None
_lock = threading.Lock()


class NativeError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, func: str, code: int, msg: str):
        super().__init__(f"{func} failed with status {code}: {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load (once) and return the shared library; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise ImportError(
                    f"shearwave_b200 CUDA library not found at {LIB_PATH}; "
                    "build it with `python -m shearwave_b200.build`"
                )
            lib = C.CDLL(str(LIB_PATH))
            for name, (args, res) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = res
            if lib.sw_abi_version() != 1:
                raise ImportError("shearwave_b200 library ABI version mismatch; rebuild it")
            if lib.sw_fdtd_desc_size() != C.sizeof(FdtdDesc):
                raise ImportError("sw_fdtd_desc layout differs between the library and ctypes")
            _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    """Names bound by this module (each must be exported by the library)."""
    return sorted(_SIGNATURES)


def call(name: str, *args) -> None:
    """Call entry point ``name`` and raise NativeError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != SW_OK:
        msg = lib.sw_last_error()
        raise NativeError(name, rc, msg.decode() if msg else "")


def launch_count() -> int:
    """Kernels launched by the library in this process so far."""
    return int(load().sw_launch_count())


def host_enqueue_count() -> int:
    """Host-side enqueue calls (kernel or graph launches) behind those kernels."""
    return int(load().sw_host_enqueue_count())

"""ctypes binding of libplamatrix_b200.so (the C ABI declared in include/plamatrix_b200.h).

The library is built in-tree by plamatrix_b200/build.py.  There is no fallback: if the
shared library is missing, importing the package's device API raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libplamatrix_b200.so")

PM_OK = 0
PM_INVALID_ARGUMENT = 1
PM_OUT_OF_RANGE = 2
PM_RUNTIME_ERROR = 3
PM_LOGIC_ERROR = 4
PM_OVERFLOW_ERROR = 5
PM_CUDA_ERROR = 6


class PlamatrixError(RuntimeError):
    """Base class; `status` is the PM_* code."""

    status = PM_RUNTIME_ERROR


class InvalidArgument(PlamatrixError, ValueError):
    status = PM_INVALID_ARGUMENT


class OutOfRange(PlamatrixError, IndexError):
    status = PM_OUT_OF_RANGE


class LogicError(PlamatrixError):
    status = PM_LOGIC_ERROR


class Overflow(PlamatrixError, OverflowError):
    status = PM_OVERFLOW_ERROR


class CudaError(PlamatrixError):
    status = PM_CUDA_ERROR


_EXCEPTIONS = {PM_INVALID_ARGUMENT: InvalidArgument, PM_OUT_OF_RANGE: OutOfRange, PM_RUNTIME_ERROR: PlamatrixError,
               PM_LOGIC_ERROR: LogicError, PM_OVERFLOW_ERROR: Overflow, PM_CUDA_ERROR: CudaError}

_lib = None

vp = C.c_void_p
i64 = C.c_int64
i32 = C.c_int
f64 = C.c_double
f32 = C.c_float


class SolverOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("use_jacobi", C.c_int), ("require_convergence", C.c_int)]


class SolverReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double)]


# name -> argtypes (restype int unless listed in _RESTYPES)
_SIGNATURES = {
    "pm_last_error": [],
    "pm_version": [],
    "pm_kernel_launches": [],
    "pm_device_malloc": [C.c_size_t, vp],
    "pm_device_free": [vp],
    "pm_copy_to_device": [vp, vp, C.c_size_t, vp],
    "pm_copy_to_host": [vp, vp, C.c_size_t, vp],
    "pm_device_name": [C.c_char_p, C.c_int],
    "pm_stream_synchronize": [vp],
    "pm_sparse_workspace_create": [vp],
    "pm_sparse_workspace_destroy": [vp],
    "pm_sparse_workspace_close": [vp],
    "pm_sparse_workspace_capacity": [vp],
    "pm_coo_to_csr_count_f32": [vp, vp, i64, i64, i64, vp, vp, vp],
    "pm_coo_to_csr_count_f64": [vp, vp, i64, i64, i64, vp, vp, vp],
    "pm_coo_to_csr_fill_f32": [vp, vp, i64, vp, vp, vp],
    "pm_coo_to_csr_fill_f64": [vp, vp, i64, vp, vp, vp],
    "pm_coo_to_csr_async_f32": [vp, vp, i64, i64, i64, vp, vp, vp, i64, vp, vp, vp],
    "pm_coo_to_csr_async_f64": [vp, vp, i64, i64, i64, vp, vp, vp, i64, vp, vp, vp],
    "pm_coo_status": [vp, C.c_char_p, vp],
    "pm_coo_to_csr_static_f32": [vp, i64, i64, i64, vp, vp, vp, i64, vp, vp, vp, vp],
    "pm_coo_to_csr_static_f64": [vp, i64, i64, i64, vp, vp, vp, i64, vp, vp, vp, vp],
    "pm_csr_create_f32": [vp, i64, i64, i64, vp, vp, vp, vp],
    "pm_csr_create_f64": [vp, i64, i64, i64, vp, vp, vp, vp],
    "pm_csr_destroy": [vp],
    "pm_csr_set_values": [vp, vp],
    "pm_csr_spmv_f32": [vp, vp, vp, vp],
    "pm_csr_spmv_f64": [vp, vp, vp, vp],
    "pm_solver_workspace_create": [vp],
    "pm_solver_workspace_destroy": [vp],
    "pm_solver_workspace_close": [vp],
    "pm_cg_f32": [vp, vp, vp, vp, vp, vp, vp],
    "pm_cg_f64": [vp, vp, vp, vp, vp, vp, vp],
    "pm_pcg_f32": [vp, vp, vp, vp, vp, vp, vp],
    "pm_pcg_f64": [vp, vp, vp, vp, vp, vp, vp],
    "pm_block_pcg_f32": [vp, vp, vp, vp, vp, vp, i64, vp, vp],
    "pm_block_pcg_f64": [vp, vp, vp, vp, vp, vp, i64, vp, vp],
}
_RESTYPES = {"pm_last_error": C.c_char_p, "pm_kernel_launches": C.c_longlong, "pm_sparse_workspace_destroy": None, "pm_csr_destroy": None,
             "pm_solver_workspace_destroy": None, "pm_sparse_workspace_capacity": C.c_size_t}


def register(name: str, argtypes, restype=C.c_int) -> None:
    """Declare a further entry point (used by the modules that add ABI surface)."""
    _SIGNATURES[name] = argtypes
    if restype is not C.c_int:
        _RESTYPES[name] = restype
    if _lib is not None:
        fn = getattr(_lib, name)
        fn.argtypes = argtypes
        fn.restype = restype


def library_path() -> str:
    return LIB_PATH


def load() -> C.CDLL:
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m plamatrix_b200.build` "
                              "(or __graft_entry__.build()) first; there is no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        for name, argtypes in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = lib
    return _lib


def call(name: str, *args) -> None:
    """Call an int-returning entry point and raise the mapped exception on failure."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != PM_OK:
        message = lib.pm_last_error().decode(errors="replace")
        raise _EXCEPTIONS.get(status, PlamatrixError)(message)


def declared_symbols(header: str | None = None) -> list:
    """Entry points declared (PM_API) in include/*.h."""
    import glob
    import re
    names = []
    for path in [header] if header else sorted(glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h"))):
        text = open(path).read()
        names += re.findall(r"PM_API\s+[A-Za-z_][A-Za-z0-9_ \*]*?\b(pm_[a-z0-9_]+)\s*\(", text)
    return names

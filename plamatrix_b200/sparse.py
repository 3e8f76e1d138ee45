"""Python mirror of the reference's sparse API for the device path
(include/plamatrix/sparse/{sparse_ops,iterative_solver}.h): COO -> CSR, SpMV, CG/PCG.

Device arrays are torch CUDA tensors (torch is used for device memory and streams
only); every computation runs in libplamatrix_b200.so through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _native as N


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _sfx(dtype: torch.dtype) -> str:
    if dtype == torch.float32:
        return "f32"
    if dtype == torch.float64:
        return "f64"
    raise N.InvalidArgument(f"unsupported scalar type {dtype}; expected float32 or float64")


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def _check_device(name: str, t: torch.Tensor, dtype=None):
    if not t.is_cuda:
        raise N.InvalidArgument(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise N.InvalidArgument(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise N.InvalidArgument(f"{name} must have dtype {dtype}, got {t.dtype}")


def _check_vector(name: str, t: torch.Tensor, dtype, size: int):
    """A contiguous CUDA vector of `dtype` with exactly `size` elements: the native calls take
    raw pointers and read or write `size` scalars through them."""
    _check_device(name, t, dtype)
    if t.numel() != size:
        raise N.InvalidArgument(f"{name} must have {size} elements, got {t.numel()}")


class SparseOpsWorkspace:
    """Grow-only, stream-bound scratch + deferred COO status (sparse_ops.h:13-77)."""

    def __init__(self):
        h = C.c_void_p()
        N.call("pm_sparse_workspace_create", C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        N.call("pm_sparse_workspace_close", self._h)

    def capacity_bytes(self) -> int:
        return int(N.load().pm_sparse_workspace_capacity(self._h))

    def check_status(self, operation: str = "cooToCsrAsync") -> int:
        """checkStatus(): raise the deferred error of the last conversion; return its nnz."""
        nnz = C.c_int64(0)
        N.call("pm_coo_status", self._h, operation.encode(), C.byref(nnz))
        return nnz.value

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_sparse_workspace_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


@dataclass
class CSRMatrix:
    """Device CSR with int64 row offsets / column indices (the reference's Index)."""

    rows: int
    cols: int
    row_offsets: torch.Tensor
    col_indices: torch.Tensor
    values: torch.Tensor

    @property
    def nnz(self) -> int:
        return int(self.values.numel())

    @staticmethod
    def empty(rows: int, cols: int, nnz: int, dtype=torch.float64, device="cuda") -> "CSRMatrix":
        return CSRMatrix(rows, cols, torch.zeros(rows + 1, dtype=torch.int64, device=device),
                         torch.empty(nnz, dtype=torch.int64, device=device), torch.empty(nnz, dtype=dtype, device=device))

    def cpu(self):
        return (self.row_offsets.cpu().numpy(), self.col_indices.cpu().numpy(), self.values.cpu().numpy())


def _coo_args(rows, cols, row_indices, col_indices, values):
    _check_device("row_indices", row_indices, torch.int64)
    _check_device("col_indices", col_indices, torch.int64)
    _check_device("values", values)
    if row_indices.numel() != col_indices.numel() or row_indices.numel() != values.numel():
        raise N.InvalidArgument("cooToCsr GPU triplet lengths must match")
    return _sfx(values.dtype), int(values.numel())


def coo_to_csr(rows: int, cols: int, row_indices: torch.Tensor, col_indices: torch.Tensor, values: torch.Tensor,
               workspace: SparseOpsWorkspace | None = None, stream=None) -> CSRMatrix:
    """Synchronous device cooToCsr (src/sparse/coo_to_csr.cu:536-561): count, sync, allocate, fill."""
    sfx, count = _coo_args(rows, cols, row_indices, col_indices, values)
    ws = workspace or SparseOpsWorkspace()
    s = _stream_handle(stream)
    N.call(f"pm_coo_to_csr_count_{sfx}", ws.handle, s, rows, cols, count, _ptr(row_indices), _ptr(col_indices),
           _ptr(values))
    torch.cuda.synchronize()
    nnz = ws.check_status("cooToCsr")
    out = CSRMatrix.empty(rows, cols, nnz, values.dtype, values.device)
    N.call(f"pm_coo_to_csr_fill_{sfx}", ws.handle, s, nnz, _ptr(out.row_offsets), _ptr(out.col_indices),
           _ptr(out.values))
    torch.cuda.synchronize()
    ws.check_status("cooToCsr")
    return out


def coo_to_csr_async(rows: int, cols: int, row_indices: torch.Tensor, col_indices: torch.Tensor,
                     values: torch.Tensor, output: CSRMatrix, workspace: SparseOpsWorkspace, stream=None) -> None:
    """cooToCsrAsync (sparse_ops.h:108-120): enqueue; sync then workspace.check_status()."""
    sfx, count = _coo_args(rows, cols, row_indices, col_indices, values)
    if output.rows != rows or output.cols != cols:
        raise N.PlamatrixError("cooToCsrAsync output dimensions do not match")
    N.call(f"pm_coo_to_csr_async_{sfx}", workspace.handle, _stream_handle(stream), rows, cols, count,
           _ptr(row_indices), _ptr(col_indices), _ptr(values), output.nnz, _ptr(output.row_offsets),
           _ptr(output.col_indices), _ptr(output.values))


class CsrOperand:
    """Validated device CSR operand (int32 structure copy) for SpMV and the solvers."""

    def __init__(self, matrix: CSRMatrix, stream=None):
        _check_device("values", matrix.values)
        sfx = _sfx(matrix.values.dtype)
        h = C.c_void_p()
        N.call(f"pm_csr_create_{sfx}", _stream_handle(stream), matrix.rows, matrix.cols, matrix.nnz,
               _ptr(matrix.row_offsets), _ptr(matrix.col_indices), _ptr(matrix.values), C.byref(h))
        self._h = h
        self.matrix = matrix
        self.sfx = sfx
        self.dtype = matrix.values.dtype

    @property
    def handle(self):
        return self._h

    def set_values(self, values: torch.Tensor) -> None:
        _check_vector("values", values, self.dtype, self.matrix.nnz)
        N.call("pm_csr_set_values", self._h, _ptr(values))
        self.matrix = CSRMatrix(self.matrix.rows, self.matrix.cols, self.matrix.row_offsets,
                                self.matrix.col_indices, values)

    def spmv(self, x: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        if x.numel() != self.matrix.cols:
            raise N.PlamatrixError(f"spmv dimension mismatch: CSR is {self.matrix.rows}x{self.matrix.cols}, "
                                   f"x has {x.numel()} rows")
        y = torch.empty(self.matrix.rows, dtype=x.dtype, device=x.device) if out is None else out
        if y.numel() != self.matrix.rows:
            raise N.PlamatrixError("spmv output dimension mismatch")
        _check_device("x", x, self.dtype)
        _check_device("out", y, self.dtype)
        N.call(f"pm_csr_spmv_{self.sfx}", self._h, _stream_handle(stream), _ptr(x), _ptr(y))
        return y

    KERNELS = {-1: "heuristic", 0: "row-group stream", 1: "1 lane/row", 2: "2 lanes/row", 4: "4 lanes/row",
               8: "8 lanes/row", 16: "16 lanes/row", 32: "32 lanes/row"}

    def autotune(self, x: torch.Tensor | None = None, y: torch.Tensor | None = None, stream=None) -> int:
        """Time every SpMV shape on this operand (x, y: the caller's vectors, random ones when
        omitted; y is overwritten) and keep the fastest; returns its code (see KERNELS)."""
        dt = self.matrix.values.dtype
        x = torch.randn(self.matrix.cols, dtype=dt, device="cuda") if x is None else x
        y = torch.empty(self.matrix.rows, dtype=dt, device="cuda") if y is None else y
        k = C.c_int(-1)
        N.call(f"pm_csr_autotune_{self.sfx}", self._h, _stream_handle(stream), _ptr(x), _ptr(y), C.byref(k))
        return k.value

    def set_kernel(self, kernel: int) -> None:
        N.call("pm_csr_set_kernel", self._h, int(kernel))

    def kernel(self) -> int:
        k, h = C.c_int(), C.c_int()
        N.call("pm_csr_kernel", self._h, C.byref(k), C.byref(h))
        return k.value

    def spmm(self, B: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """out = A B for column-major dense matrices (spmmAsync, sparse_ops.cu:762-818): B is
        (cols x k) and out (rows x k), each with strides (1, its row count), e.g.
        `dense_matrix(rows, k)`."""
        if B.dim() != 2 or out is not None and out.dim() != 2:
            raise N.InvalidArgument("spmm operands must be 2-D column-major tensors")
        y = dense_matrix(self.matrix.rows, B.shape[1], B.dtype, B.device) if out is None else out
        for name, t in (("input", B), ("output", y)):
            if t.numel() > 0 and t.shape[1] > 1 and t.stride() != (1, t.shape[0]):
                raise N.InvalidArgument(f"spmm {name} must be column-major (strides (1, rows))")
            if not t.is_cuda or t.dtype != self.dtype:
                raise N.InvalidArgument(f"spmm {name} must be a CUDA matrix of dtype {self.dtype}")
        N.call(f"pm_csr_spmm_{self.sfx}", self._h, _stream_handle(stream), B.shape[0], B.shape[1], _ptr(B),
               y.shape[0], y.shape[1], _ptr(y))
        return y

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_csr_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


def dense_matrix(rows: int, cols: int, dtype=torch.float64, device="cuda") -> torch.Tensor:
    """A (rows x cols) column-major device matrix, the reference's DenseMatrix layout."""
    return torch.empty((cols, rows), dtype=dtype, device=device).t()


def spmm(matrix, B: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    op = matrix if isinstance(matrix, CsrOperand) else CsrOperand(matrix, stream)
    return op.spmm(B, out, stream)


def spmv(matrix, x: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    op = matrix if isinstance(matrix, CsrOperand) else CsrOperand(matrix, stream)
    return op.spmv(x, out, stream)


@dataclass
class IterativeSolverOptions:
    max_iterations: int = 1000
    relative_tolerance: float = 1e-6
    absolute_tolerance: float = 0.0
    use_jacobi_preconditioner: bool = True
    require_convergence: bool = False

    def c(self) -> N.SolverOptions:
        return N.SolverOptions(self.max_iterations, self.relative_tolerance, self.absolute_tolerance,
                               int(self.use_jacobi_preconditioner), int(self.require_convergence))


class IterativeSolverWorkspace:
    def __init__(self):
        h = C.c_void_p()
        N.call("pm_solver_workspace_create", C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        N.call("pm_solver_workspace_close", self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_solver_workspace_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


def _solve(kind: str, matrix, rhs, solution, workspace, options, stream, blocks=None, block_size=0) -> dict:
    op = matrix if isinstance(matrix, CsrOperand) else CsrOperand(matrix, stream)
    _check_vector("rhs", rhs, op.dtype, op.matrix.rows)
    _check_vector("solution", solution, op.dtype, op.matrix.cols)
    if kind == "block_pcg":
        if block_size <= 0:
            raise N.InvalidArgument("block size must be positive")
        _check_vector("inverse_blocks", blocks, op.dtype, op.matrix.rows * int(block_size))
    ws = workspace or IterativeSolverWorkspace()
    opts = (options or IterativeSolverOptions()).c()
    rep = N.SolverReport()
    s = _stream_handle(stream)
    if kind == "block_pcg":
        N.call(f"pm_block_pcg_{op.sfx}", ws.handle, s, op.handle, _ptr(rhs), _ptr(solution), _ptr(blocks),
               block_size, C.byref(opts), C.byref(rep))
    else:
        N.call(f"pm_{kind}_{op.sfx}", ws.handle, s, op.handle, _ptr(rhs), _ptr(solution), C.byref(opts),
               C.byref(rep))
    return {"converged": bool(rep.converged), "iterations": rep.iterations,
            "initial_residual": rep.initial_residual, "final_residual": rep.final_residual}


def cg(matrix, rhs, solution, workspace=None, options=None, stream=None) -> dict:
    return _solve("cg", matrix, rhs, solution, workspace, options, stream)


def pcg(matrix, rhs, solution, workspace=None, options=None, stream=None) -> dict:
    return _solve("pcg", matrix, rhs, solution, workspace, options, stream)


def block_pcg(matrix, rhs, solution, inverse_blocks, block_size, workspace=None, options=None, stream=None) -> dict:
    return _solve("block_pcg", matrix, rhs, solution, workspace, options, stream, inverse_blocks, block_size)


# ---------------------------------------------------------------- fixed-iteration solves
for _suffix in ("f32", "f64"):
    for _kind in ("cg", "pcg"):
        N.register(f"pm_{_kind}_fixed_iterations_async_{_suffix}",
                   [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p])
N.register("pm_fixed_state_finalize", [C.c_void_p, C.c_void_p, C.c_void_p])
N.register("pm_csr_set_kernel", [C.c_void_p, C.c_int])
N.register("pm_csr_kernel", [C.c_void_p, C.c_void_p, C.c_void_p])
for _suffix in ("f32", "f64"):
    N.register(f"pm_csr_autotune_{_suffix}", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p])
    N.register(f"pm_csr_spmm_{_suffix}", [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64,
                                          C.c_int64, C.c_void_p])
N.register("pm_fixed_state_destroy", [C.c_void_p], None)


class AsyncIterativeSolverState:
    """AsyncIterativeSolverState (iterative_solver.h:68-91): the submitted fixed-iteration solve;
    finalize() after synchronising the stream (finalizeIterativeSolverReport)."""

    def __init__(self, handle, iterations: int):
        self._h = handle
        self.submitted_iterations = iterations

    def finalize(self, options: IterativeSolverOptions | None = None) -> dict:
        opts = (options or IterativeSolverOptions()).c()
        rep = N.SolverReport()
        N.call("pm_fixed_state_finalize", self._h, C.byref(opts), C.byref(rep))
        return {"converged": bool(rep.converged), "iterations": rep.iterations,
                "initial_residual": rep.initial_residual, "final_residual": rep.final_residual}

    def close(self) -> None:
        h, self._h = self._h, None
        if h is not None:
            N.load().pm_fixed_state_destroy(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_fixed_state_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


def _fixed(kind, matrix, rhs, solution, iterations, workspace, stream):
    op = matrix if isinstance(matrix, CsrOperand) else CsrOperand(matrix, stream)
    _check_vector("rhs", rhs, op.dtype, op.matrix.rows)
    _check_vector("solution", solution, op.dtype, op.matrix.cols)
    ws = workspace or IterativeSolverWorkspace()
    h = C.c_void_p()
    N.call(f"pm_{kind}_fixed_iterations_async_{op.sfx}", ws.handle, _stream_handle(stream), op.handle, _ptr(rhs),
           _ptr(solution), int(iterations), C.byref(h))
    st = AsyncIterativeSolverState(h, int(iterations))
    st._keep = (op, ws)  # the operand and workspace must outlive the submitted work
    return st


def cg_fixed_iterations_async(matrix, rhs, solution, iterations: int, workspace=None, stream=None):
    return _fixed("cg", matrix, rhs, solution, iterations, workspace, stream)


def pcg_fixed_iterations_async(matrix, rhs, solution, iterations: int, workspace=None, stream=None):
    return _fixed("pcg", matrix, rhs, solution, iterations, workspace, stream)

"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Two implementations share one Python surface:

* ``impl="orc"``: the plain-C restatement in ``oracle/oracle.c`` (always built);
* ``impl="ref"``: the reference's own CPU library, compiled from the reference
  sources into ``oracle/_ref/libplamatrix_ref.so`` by ``oracle/Makefile``.

Only the test-suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs use this module.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree the Makefile compiles from (absent on machines that only run the
# prebuilt checkers)
REF_SOURCE_ROOT = os.environ.get("PLAMATRIX_REFERENCE", "/root/reference")
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libplamatrix_ref.so")

STATUS_NAMES = {0: "ok", 1: "invalid_argument", 2: "out_of_range", 3: "runtime_error",
                4: "logic_error", 5: "overflow_error", 6: "no_memory"}

_i64p = C.POINTER(C.c_int64)


class CheckerError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.kind = STATUS_NAMES.get(status, str(status))
        self.message = message


def build() -> None:
    """Compile the oracle (and, when the reference tree is present, the reference library)."""
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


_libs: dict[str, C.CDLL] = {}


def available(impl: str) -> bool:
    return os.path.exists(ORACLE_SO if impl == "orc" else REF_SO)


def lib(impl: str = "orc") -> C.CDLL:
    if impl not in _libs:
        path = ORACLE_SO if impl == "orc" else REF_SO
        if not os.path.exists(path):
            build()
        handle = C.CDLL(path)
        err = handle.orc_last_error if impl == "orc" else handle.ref_last_error
        err.restype = C.c_char_p
        for name in ("ne_create_f32", "ne_create_f64"):
            getattr(handle, f"{impl}_{name}").restype = C.c_void_p
        _libs[impl] = handle
    return _libs[impl]


def _ptr(array: np.ndarray | None):
    if array is None:
        return None
    return C.c_void_p(array.ctypes.data)


def _check(impl: str, status: int) -> None:
    if status != 0:
        handle = lib(impl)
        err = handle.orc_last_error if impl == "orc" else handle.ref_last_error
        raise CheckerError(status, err().decode())


def _sfx(dtype) -> str:
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


def _ctype(dtype):
    return C.c_float if np.dtype(dtype) == np.float32 else C.c_double


# ---------------------------------------------------------------- COO -> CSR / SpMV / PCG
def coo_to_csr(rows: int, cols: int, r, c, v, impl: str = "orc"):
    r = np.ascontiguousarray(r, dtype=np.int64)
    c = np.ascontiguousarray(c, dtype=np.int64)
    v = np.ascontiguousarray(v)
    n = len(v)
    row_offsets = np.zeros(rows + 1, dtype=np.int64)
    out_cols = np.zeros(max(n, 1), dtype=np.int64)
    out_vals = np.zeros(max(n, 1), dtype=v.dtype)
    nnz = C.c_int64(0)
    fn = getattr(lib(impl), f"{impl}_coo_to_csr_{_sfx(v.dtype)}")
    _check(impl, fn(C.c_int64(rows), C.c_int64(cols), C.c_int64(n), _ptr(r), _ptr(c), _ptr(v),
                    _ptr(row_offsets), _ptr(out_cols), _ptr(out_vals), C.byref(nnz)))
    k = nnz.value
    return row_offsets, out_cols[:k].copy(), out_vals[:k].copy()


def csr_spmv(row_offsets, cols, vals, x, impl: str = "orc"):
    n = len(row_offsets) - 1
    y = np.zeros(n, dtype=vals.dtype)
    fn = getattr(lib(impl), f"{impl}_csr_spmv_{_sfx(vals.dtype)}")
    _check(impl, fn(C.c_int64(n), C.c_int64(len(x)), _ptr(row_offsets), _ptr(cols), _ptr(vals), _ptr(np.ascontiguousarray(x, vals.dtype)),
                    _ptr(y)))
    return y


def csr_spmm(row_offsets, cols, vals, n_cols, B, impl: str = "orc"):
    """output (rows x k) = CSR x B (n_cols x k); B and output column-major (numpy order="F")."""
    n = len(row_offsets) - 1
    B = np.asfortranarray(B, dtype=vals.dtype)
    k = B.shape[1]
    out = np.zeros((n, k), dtype=vals.dtype, order="F")
    fn = getattr(lib(impl), f"{impl}_csr_spmm_{_sfx(vals.dtype)}")
    _check(impl, fn(C.c_int64(n), C.c_int64(n_cols), _ptr(row_offsets), _ptr(cols), _ptr(vals), C.c_int64(k),
                    _ptr(B), _ptr(out)))
    return out


class SolverOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("use_jacobi", C.c_int),
                ("require_convergence", C.c_int)]


class SolverReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double)]


def pcg(row_offsets, cols, vals, rhs, x0=None, *, max_iterations=1000, relative_tolerance=1e-6,
        absolute_tolerance=0.0, use_jacobi=True, require_convergence=False, preconditioned=True,
        impl: str = "orc"):
    n = len(row_offsets) - 1
    x = np.zeros(n, dtype=vals.dtype) if x0 is None else np.array(x0, dtype=vals.dtype)
    opts = SolverOptions(max_iterations, relative_tolerance, absolute_tolerance, int(use_jacobi),
                         int(require_convergence))
    rep = SolverReport()
    fn = getattr(lib(impl), f"{impl}_pcg_{_sfx(vals.dtype)}")
    _check(impl, fn(C.c_int64(n), _ptr(row_offsets), _ptr(cols), _ptr(vals),
                    _ptr(np.ascontiguousarray(rhs, vals.dtype)), _ptr(x), C.byref(opts), C.c_int(int(preconditioned)),
                    C.byref(rep)))
    return x, {"converged": bool(rep.converged), "iterations": rep.iterations,
               "initial_residual": rep.initial_residual, "final_residual": rep.final_residual}


def huber(squared_norm: float, delta: float, dtype=np.float64, impl: str = "orc"):
    ct = _ctype(dtype)
    cost, weight = ct(0), ct(0)
    fn = getattr(lib(impl), f"{impl}_huber_{_sfx(dtype)}")
    fn.argtypes = [ct, ct, C.POINTER(ct), C.POINTER(ct)]
    _check(impl, fn(squared_norm, delta, C.byref(cost), C.byref(weight)))
    return cost.value, weight.value


# ---------------------------------------------------------------- normal equations / Schur
class SchurOptions(C.Structure):
    _fields_ = [("backend", C.c_int), ("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("minimum_diagonal", C.c_double),
                ("use_initial_guess", C.c_int)]


class OrcSchurReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual_norm", C.c_double),
                ("final_residual_norm", C.c_double), ("message", C.c_char * 128)]


class RefSchurReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual_norm", C.c_double),
                ("final_residual_norm", C.c_double), ("pattern_reused", C.c_int),
                ("pattern_build_count", C.c_int64), ("linear_solve_seconds", C.c_double),
                ("total_seconds", C.c_double), ("message", C.c_char * 128)]


BACKENDS = {"cpu": 0, "dense_cpu": 1}


class NormalEquations:
    """BlockNormalEquations<Scalar> held by the oracle ("orc") or the reference ("ref")."""

    def __init__(self, P, L, bp, bl, dtype=np.float64, impl: str = "orc"):
        self.impl, self.dtype = impl, np.dtype(dtype)
        self.P, self.L, self.bp, self.bl = P, L, bp, bl
        self._lib = lib(impl)
        self._sfx = _sfx(dtype)
        create = getattr(self._lib, f"{impl}_ne_create_{self._sfx}")
        create.restype = C.c_void_p
        self._h = create(C.c_int64(P), C.c_int64(L), C.c_int64(bp), C.c_int64(bl))
        if not self._h:
            err = self._lib.orc_last_error if impl == "orc" else self._lib.ref_last_error
            raise CheckerError(1, err().decode())
        self._ct = _ctype(dtype)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            getattr(self._lib, f"{self.impl}_ne_destroy_{self._sfx}")(C.c_void_p(h))
            self._h = None

    def _fn(self, name):
        return getattr(self._lib, f"{self.impl}_{name}_{self._sfx}")

    def add_residual(self, primaries, primary_jacobians, eliminated, eliminated_jacobian, residual,
                     weight=1.0):
        """primaries: list of ints (may be empty); eliminated: int or -1."""
        prim = np.ascontiguousarray(primaries, dtype=np.int64)
        pj = np.ascontiguousarray(primary_jacobians if len(prim) else np.zeros(1), dtype=self.dtype)
        ej = np.ascontiguousarray(eliminated_jacobian if eliminated_jacobian is not None else np.zeros(1),
                                  dtype=self.dtype)
        r = np.ascontiguousarray(residual, dtype=self.dtype)
        fn = self._fn("ne_add_residual")
        _check(self.impl, fn(C.c_void_p(self._h), C.c_int64(len(prim)), _ptr(prim), _ptr(pj),
                             C.c_int64(eliminated), _ptr(ej) if eliminated_jacobian is not None else None,
                             _ptr(r), C.c_int64(len(r)), self._ct(weight)))

    def add_observations(self, obs_p, obs_l, jp, jl, r, huber_delta):
        obs_p = np.ascontiguousarray(obs_p, dtype=np.int64)
        obs_l = np.ascontiguousarray(obs_l, dtype=np.int64)
        jp = np.ascontiguousarray(jp, dtype=self.dtype)
        jl = np.ascontiguousarray(jl, dtype=self.dtype)
        r = np.ascontiguousarray(r, dtype=self.dtype)
        m = r.shape[1] if r.ndim == 2 else 1
        fn = self._fn("ne_add_observations")
        _check(self.impl, fn(C.c_void_p(self._h), C.c_int64(len(obs_p)), C.c_int64(m), _ptr(obs_p), _ptr(obs_l),
                             _ptr(jp), _ptr(jl), _ptr(r), self._ct(huber_delta)))

    def merge_from(self, other: "NormalEquations"):
        _check(self.impl, self._fn("ne_merge")(C.c_void_p(self._h), C.c_void_p(other._h)))

    def counts(self):
        cc, pc = C.c_int64(0), C.c_int64(0)
        self._fn("ne_counts")(C.c_void_p(self._h), C.byref(cc), C.byref(pc))
        return cc.value, pc.value

    def export(self) -> dict:
        cc, pc = self.counts()
        P, L, bp, bl, dt = self.P, self.L, self.bp, self.bl, self.dtype
        out = {
            "primary_diagonal": np.zeros((P, bp, bp), dt), "eliminated_diagonal": np.zeros((L, bl, bl), dt),
            "primary_gradient": np.zeros((P, bp), dt), "eliminated_gradient": np.zeros((L, bl), dt),
            "adjacency_offsets": np.zeros(L + 1, np.int64), "cross_primary": np.zeros(max(cc, 1), np.int64),
            "cross_values": np.zeros((max(cc, 1), bp, bl), dt), "primary_cross_row": np.zeros(max(pc, 1), np.int64),
            "primary_cross_col": np.zeros(max(pc, 1), np.int64),
            "primary_cross_values": np.zeros((max(pc, 1), bp, bp), dt),
        }
        self._fn("ne_export")(C.c_void_p(self._h), *[_ptr(out[k]) for k in (
            "primary_diagonal", "eliminated_diagonal", "primary_gradient", "eliminated_gradient",
            "adjacency_offsets", "cross_primary", "cross_values", "primary_cross_row", "primary_cross_col",
            "primary_cross_values")])
        out["cross_primary"] = out["cross_primary"][:cc]
        out["cross_values"] = out["cross_values"][:cc]
        out["primary_cross_row"] = out["primary_cross_row"][:pc]
        out["primary_cross_col"] = out["primary_cross_col"][:pc]
        out["primary_cross_values"] = out["primary_cross_values"][:pc]
        return out

    def solve(self, damping, backend="cpu", max_iterations=100, relative_tolerance=1e-8,
              absolute_tolerance=1e-12, minimum_diagonal=1e-12, initial_guess=None):
        P, L, bp, bl = self.P, self.L, self.bp, self.bl
        opts = SchurOptions(BACKENDS[backend], max_iterations, relative_tolerance, absolute_tolerance,
                            minimum_diagonal, int(initial_guess is not None))
        dp = np.zeros(P * bp, self.dtype) if initial_guess is None else np.array(initial_guess, self.dtype)
        dl = np.zeros(L * bl, self.dtype)
        rep = OrcSchurReport() if self.impl == "orc" else RefSchurReport()
        _check(self.impl, self._fn("schur_solve")(C.c_void_p(self._h), self._ct(damping), C.byref(opts),
                                                  _ptr(dp), _ptr(dl), C.byref(rep)))
        report = {k: getattr(rep, k) for k, _ in rep._fields_}
        report["message"] = rep.message.decode()
        report["converged"] = bool(rep.converged)
        return dp, dl, report

    def schur_system(self, damping, minimum_diagonal=1e-12, with_preconditioner=True):
        """(row_offsets, col_indices, values, rhs[, preconditioner_inverse]) of the reduced system."""
        P, bp = self.P, self.bp
        n = P * bp
        if self.impl == "orc":
            nnz, blocks = C.c_int64(0), C.c_int64(0)
            _check("orc", self._fn("schur_pattern_nnz")(
                C.c_void_p(self._h), C.byref(nnz), C.byref(blocks)))
            ro = np.zeros(n + 1, np.int64)
            ci = np.zeros(max(nnz.value, 1), np.int64)
            vals = np.zeros(max(nnz.value, 1), self.dtype)
            rhs = np.zeros(max(n, 1), self.dtype)
            pre = np.zeros((max(P, 1), bp, bp), self.dtype) if with_preconditioner else None
            _check("orc", self._fn("schur_system")(C.c_void_p(self._h), self._ct(damping), self._ct(minimum_diagonal),
                                                  _ptr(ro), _ptr(ci), _ptr(vals), _ptr(rhs), _ptr(pre)))
            k = nnz.value
            out = (ro, ci[:k], vals[:k], rhs[:n])
            return out + ((pre[:P],) if with_preconditioner else ())
        # reference: size query first (values NULL), then the real call
        nnz = C.c_int64(0)
        _check("ref", self._fn("schur_system")(C.c_void_p(self._h), self._ct(damping), self._ct(minimum_diagonal),
                                              C.byref(nnz), None, None, None, None))
        ro = np.zeros(n + 1, np.int64)
        ci = np.zeros(max(nnz.value, 1), np.int64)
        vals = np.zeros(max(nnz.value, 1), self.dtype)
        rhs = np.zeros(max(n, 1), self.dtype)
        _check("ref", self._fn("schur_system")(C.c_void_p(self._h), self._ct(damping), self._ct(minimum_diagonal),
                                              C.byref(nnz), _ptr(ro), _ptr(ci), _ptr(vals), _ptr(rhs)))
        k = nnz.value
        return ro, ci[:k], vals[:k], rhs[:n]


def normal_equations_from_observations(problem: dict, dtype=np.float64, impl: str = "orc") -> NormalEquations:
    """Accumulate a synthetic observation problem (plamatrix_b200.workloads layout) in array order."""
    ne = NormalEquations(problem["P"], problem["L"], problem["bp"], problem["bl"], dtype=dtype, impl=impl)
    ne.add_observations(problem["obs_primary"], problem["obs_eliminated"], problem["jp"], problem["jl"],
                        problem["residual"], problem["huber_delta"])
    return ne


# ---------------------------------------------------------------- learned block-Jacobi correction
MLP_IN, MLP_HIDDEN, MLP_OUT = 25, 128, 21


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def mlp_param_count() -> int:
    fn = lib("orc").orc_mlp_param_count
    fn.restype = C.c_int64
    return int(fn())


def mlp_features(block_row_ptr, block_col, blocks) -> np.ndarray:
    """25 features per block row of a 6x6 block-CSR matrix (blocks: B x 36, row-major)."""
    ro = np.ascontiguousarray(block_row_ptr, np.int64)
    bc = np.ascontiguousarray(block_col, np.int64)
    bl = _f64(blocks).reshape(-1, 36)
    P = len(ro) - 1
    out = np.zeros((max(P, 1), MLP_IN))
    _check("orc", lib("orc").orc_mlp_features(C.c_int64(P), _ptr(ro), _ptr(bc), _ptr(bl), _ptr(out)))
    return out[:P]


def mlp_forward(features, params, bf16: bool = False) -> dict:
    f = _f64(features).reshape(-1, MLP_IN)
    w = _f64(params)
    P = f.shape[0]
    cache = {k: np.zeros((max(P, 1), MLP_HIDDEN)) for k in ("z1", "h1", "z2", "h2")}
    out = np.zeros((max(P, 1), MLP_OUT))
    _check("orc", lib("orc").orc_mlp_forward(C.c_int64(P), _ptr(f), _ptr(w), C.c_int(int(bf16)), _ptr(cache["z1"]),
                                             _ptr(cache["h1"]), _ptr(cache["z2"]), _ptr(cache["h2"]), _ptr(out)))
    cache = {k: v[:P] for k, v in cache.items()}
    cache["out"] = out[:P]
    return cache


def mlp_loss_grad(diag_blocks, out, x, b):
    d = _f64(diag_blocks).reshape(-1, 36)
    o = _f64(out).reshape(-1, MLP_OUT)
    P = d.shape[0]
    loss = C.c_double(0.0)
    dout = np.zeros((max(P, 1), MLP_OUT))
    _check("orc", lib("orc").orc_mlp_loss_grad(C.c_int64(P), _ptr(d), _ptr(o), _ptr(_f64(x)), _ptr(_f64(b)),
                                               C.byref(loss), _ptr(dout)))
    return loss.value, dout[:P]


def mlp_probe_loss_grad(diag_blocks, out, v, sv):
    """||(I - M S) v||^2 / ||v||^2 for the corrected block preconditioner M, given sv = S v."""
    d = _f64(diag_blocks).reshape(-1, 36)
    o = _f64(out).reshape(-1, MLP_OUT)
    P = d.shape[0]
    loss = C.c_double(0.0)
    dout = np.zeros((max(P, 1), MLP_OUT))
    _check("orc", lib("orc").orc_mlp_probe_loss_grad(C.c_int64(P), _ptr(d), _ptr(o), _ptr(_f64(v)), _ptr(_f64(sv)),
                                                     C.byref(loss), _ptr(dout)))
    return loss.value, dout[:P]


def mlp_backward(features, params, cache: dict, dout, bf16: bool = False) -> np.ndarray:
    f = _f64(features).reshape(-1, MLP_IN)
    P = f.shape[0]
    grads = np.zeros(mlp_param_count())
    _check("orc", lib("orc").orc_mlp_backward(C.c_int64(P), _ptr(f), _ptr(_f64(params)), C.c_int(int(bf16)),
                                              _ptr(_f64(cache["z1"])), _ptr(_f64(cache["h1"])),
                                              _ptr(_f64(cache["z2"])), _ptr(_f64(cache["h2"])),
                                              _ptr(_f64(dout)), _ptr(grads)))
    return grads


def mlp_preconditioner(diag_blocks, out) -> np.ndarray:
    d = _f64(diag_blocks).reshape(-1, 36)
    P = d.shape[0]
    minv = np.zeros((max(P, 1), 36))
    _check("orc", lib("orc").orc_mlp_preconditioner(C.c_int64(P), _ptr(d), _ptr(_f64(out)), _ptr(minv)))
    return minv[:P]

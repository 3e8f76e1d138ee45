"""Python mirror of the reference's optimisation API for the device path
(include/plamatrix/optimization/block_schur.h): BlockNormalEquations state on the device,
Huber-weighted accumulation of device observations, solveDampedSchurComplement with a
reusable SchurComplementSolverWorkspace.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .sparse import _ptr, _stream_handle

vp, i64 = C.c_void_p, C.c_int64


class SchurOptions(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("relative_tolerance", C.c_double),
                ("absolute_tolerance", C.c_double), ("minimum_diagonal", C.c_double),
                ("use_initial_guess", C.c_int), ("precision", C.c_int), ("tolerance_rule", C.c_int),
                ("check_true_residual", C.c_int), ("inner_relative_tolerance", C.c_double),
                ("max_refinements", C.c_int), ("learned", C.c_void_p), ("stagnation_window", C.c_int),
                ("linear_backend", C.c_int)]


class SchurReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual_norm", C.c_double),
                ("final_residual_norm", C.c_double), ("true_relative_residual", C.c_double),
                ("pattern_reused", C.c_int), ("mixed_precision_used", C.c_int), ("refinement_steps", C.c_int),
                ("pattern_ms", C.c_double), ("eliminated_inverse_ms", C.c_double), ("assembly_ms", C.c_double),
                ("solve_ms", C.c_double), ("back_substitution_ms", C.c_double), ("total_ms", C.c_double),
                ("message", C.c_char * 128), ("learned_used", C.c_int), ("learned_fallback", C.c_int),
                ("learned_iterations", C.c_int)]


for _sfx, _ct in (("f32", C.c_float), ("f64", C.c_double)):
    N.register(f"pm_ne_upload_{_sfx}", [vp, vp, vp, vp, vp, vp, i64, vp, vp, vp, i64, vp, vp, vp])
    N.register(f"pm_ne_download_{_sfx}", [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp])
    N.register(f"pm_ne_accumulate_observations_{_sfx}", [vp, vp, i64, i64, vp, vp, vp, vp, vp, _ct])
    N.register(f"pm_schur_solve_{_sfx}", [vp, vp, vp, _ct, vp, vp, vp, vp])
    N.register(f"pm_schur_export_{_sfx}", [vp, vp, vp, vp, vp, vp, vp])
N.register("pm_ne_create", [i64, i64, i64, i64, C.c_int, vp])
N.register("pm_ne_destroy", [vp], None)
N.register("pm_ne_counts", [vp, vp, vp, vp])
N.register("pm_ne_check_observations", [vp, vp, vp])
N.register("pm_schur_workspace_create", [vp])
N.register("pm_schur_workspace_destroy", [vp], None)
N.register("pm_schur_workspace_close", [vp])
N.register("pm_schur_pattern_build_count", [vp], C.c_int64)
N.register("pm_schur_dims", [vp, vp, vp, vp])
N.register("pm_schur_spmv_f32", [vp, vp, vp, vp])
N.register("pm_schur_assembly_shape_count", [], C.c_int)
N.register("pm_schur_set_assembly_shape", [vp, C.c_int])
N.register("pm_schur_assembly_shape_info", [C.c_int, vp, vp])
N.register("pm_schur_assembly_shape", [vp, vp])
N.register("pm_schur_autotune_assembly", [vp, vp, vp, C.c_int, vp, vp, vp])
N.register("pm_schur_spmv_f64", [vp, vp, vp, vp])

PRECISION = {"native": 0, "mixed": 1, "mixed_fp32_assembly": 2}


LINEAR_BACKEND = {"pcg": 0, "dense": 1}
DENSE_MAX_UNKNOWNS = 16384  # PM_DENSE_MAX_UNKNOWNS


@dataclass
class SchurComplementSolverOptions:
    """SchurComplementSolverOptions<Scalar> (block_schur.h:31-47) plus device-path knobs."""

    max_iterations: int = 100
    relative_tolerance: float = 1e-8
    absolute_tolerance: float = 1e-12
    minimum_diagonal: float = 1e-12
    use_initial_guess: bool = False
    precision: str = "native"
    tolerance_rule: str = "cpu"      # "cpu": abs + rel*||r0||; "max": max(abs, rel*||r0||)
    check_true_residual: bool = True
    inner_relative_tolerance: float = 1e-4
    max_refinements: int = 8
    learned: "LearnedPreconditioner | None" = None  # no counterpart in the reference
    stagnation_window: int = 25
    linear_backend: str = "pcg"  # "pcg" (Cpu / Cuda backends) or "dense" (DenseCpu: device Cholesky)

    def c(self) -> SchurOptions:
        return SchurOptions(self.max_iterations, self.relative_tolerance, self.absolute_tolerance,
                            self.minimum_diagonal, int(self.use_initial_guess), PRECISION[self.precision],
                            0 if self.tolerance_rule == "cpu" else 1, int(self.check_true_residual),
                            self.inner_relative_tolerance, self.max_refinements,
                            self.learned.handle if self.learned is not None else None, self.stagnation_window,
                            LINEAR_BACKEND[self.linear_backend])


def _dtype_info(dtype):
    dt = np.dtype(dtype)
    if dt == np.float32:
        return "f32", 4, torch.float32, C.c_float
    if dt == np.float64:
        return "f64", 8, torch.float64, C.c_double
    raise N.InvalidArgument(f"unsupported scalar type {dtype}")


class DeviceNormalEquations:
    """Device-resident BlockNormalEquations<Scalar>."""

    def __init__(self, P: int, L: int, bp: int, bl: int, dtype=np.float64):
        self.sfx, size, self.tdtype, self.ct = _dtype_info(dtype)
        self.dtype = np.dtype(dtype)
        self.P, self.L, self.bp, self.bl = P, L, bp, bl
        h = C.c_void_p()
        N.call("pm_ne_create", P, L, bp, bl, size, C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_ne_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None

    def counts(self):
        cc, pc, ver = C.c_int64(), C.c_int64(), C.c_int64()
        N.call("pm_ne_counts", self._h, C.byref(cc), C.byref(pc), C.byref(ver))
        return cc.value, pc.value, ver.value

    def upload(self, state: dict, stream=None) -> None:
        """state: the dict layout of oracle.NormalEquations.export() (host numpy arrays)."""
        dt = self.dtype
        arr = {k: np.ascontiguousarray(v, dtype=(np.int64 if v.dtype.kind in "iu" else dt)) for k, v in state.items()}
        C_ = len(arr["cross_primary"])
        PC = len(arr["primary_cross_row"])
        hp = lambda a: C.c_void_p(a.ctypes.data) if a.size else None  # noqa: E731
        N.call(f"pm_ne_upload_{self.sfx}", self._h, _stream_handle(stream), hp(arr["primary_diagonal"]),
               hp(arr["eliminated_diagonal"]), hp(arr["primary_gradient"]), hp(arr["eliminated_gradient"]), C_,
               hp(arr["adjacency_offsets"]), hp(arr["cross_primary"]), hp(arr["cross_values"]), PC,
               hp(arr["primary_cross_row"]), hp(arr["primary_cross_col"]), hp(arr["primary_cross_values"]))

    def download(self, stream=None) -> dict:
        cc, pc, _ = self.counts()
        P, L, bp, bl, dt = self.P, self.L, self.bp, self.bl, self.dtype
        out = {"primary_diagonal": np.zeros((P, bp, bp), dt), "eliminated_diagonal": np.zeros((L, bl, bl), dt),
               "primary_gradient": np.zeros((P, bp), dt), "eliminated_gradient": np.zeros((L, bl), dt),
               "adjacency_offsets": np.zeros(L + 1, np.int64), "cross_primary": np.zeros(max(cc, 1), np.int64),
               "cross_values": np.zeros((max(cc, 1), bp, bl), dt), "primary_cross_row": np.zeros(max(pc, 1), np.int64),
               "primary_cross_col": np.zeros(max(pc, 1), np.int64),
               "primary_cross_values": np.zeros((max(pc, 1), bp, bp), dt)}
        hp = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
        N.call(f"pm_ne_download_{self.sfx}", self._h, _stream_handle(stream), *[hp(out[k]) for k in (
            "primary_diagonal", "eliminated_diagonal", "primary_gradient", "eliminated_gradient",
            "adjacency_offsets", "cross_primary", "cross_values", "primary_cross_row", "primary_cross_col",
            "primary_cross_values")])
        for k in ("cross_primary", "cross_values"):
            out[k] = out[k][:cc]
        for k in ("primary_cross_row", "primary_cross_col", "primary_cross_values"):
            out[k] = out[k][:pc]
        return out

    def check_observations(self, stream=None) -> None:
        """Raise InvalidArgument when the last accumulation met a residual whose squared norm is
        not finite (evaluateHuberLoss, robust_loss.h:31-35); synchronises the stream."""
        bad = C.c_int64(-1)
        N.call("pm_ne_check_observations", self._h, _stream_handle(stream), C.byref(bad))

    def accumulate_observations(self, obs_primary: torch.Tensor, obs_eliminated: torch.Tensor, jp: torch.Tensor,
                                jl: torch.Tensor, residual: torch.Tensor, huber_delta: float, stream=None) -> None:
        count = int(obs_primary.numel())
        m = int(residual.numel() // max(count, 1)) if count else 1
        for name, t, dt in (("obs_primary", obs_primary, torch.int64), ("obs_eliminated", obs_eliminated, torch.int64),
                            ("jp", jp, self.tdtype), ("jl", jl, self.tdtype), ("residual", residual, self.tdtype)):
            if not t.is_cuda or not t.is_contiguous() or t.dtype != dt:
                raise N.InvalidArgument(f"{name} must be a contiguous CUDA tensor of dtype {dt}")
        N.call(f"pm_ne_accumulate_observations_{self.sfx}", self._h, _stream_handle(stream), count, m,
               _ptr(obs_primary), _ptr(obs_eliminated), _ptr(jp), _ptr(jl), _ptr(residual), self.ct(huber_delta))


class SchurComplementSolverWorkspace:
    """Reusable Schur pattern + device buffers (block_schur.h:81-169)."""

    def __init__(self):
        h = C.c_void_p()
        N.call("pm_schur_workspace_create", C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def pattern_build_count(self) -> int:
        return int(N.load().pm_schur_pattern_build_count(self._h))

    def close(self) -> None:
        N.call("pm_schur_workspace_close", self._h)

    def dims(self):
        n, nnz, b = C.c_int64(), C.c_int64(), C.c_int64()
        N.call("pm_schur_dims", self._h, C.byref(n), C.byref(nnz), C.byref(b))
        return n.value, nnz.value, b.value

    @staticmethod
    def assembly_shape_count() -> int:
        """Number of launch shapes of the upper-block assembly pass."""
        return int(N.load().pm_schur_assembly_shape_count())

    @staticmethod
    def assembly_shape_info(shape: int) -> tuple:
        """(pair streams, lanes per pair) of an assembly launch shape."""
        streams, split = C.c_int(), C.c_int()
        N.call("pm_schur_assembly_shape_info", int(shape), C.byref(streams), C.byref(split))
        return streams.value, split.value

    @property
    def assembly_shape(self) -> int:
        shape = C.c_int()
        N.call("pm_schur_assembly_shape", self._h, C.byref(shape))
        return shape.value

    @assembly_shape.setter
    def assembly_shape(self, shape: int) -> None:
        N.call("pm_schur_set_assembly_shape", self._h, int(shape))

    def autotune_assembly(self, equations, repeats: int = 3, stream=None) -> dict:
        """Time every assembly launch shape on the system this workspace last solved (`equations`),
        keep the fastest; the workspace then needs a new solve before export / spmv."""
        count = self.assembly_shape_count()
        shape, best = C.c_int(), C.c_double()
        per = (C.c_double * count)()
        N.call("pm_schur_autotune_assembly", self._h, _stream_handle(stream), equations.handle, int(repeats),
               C.byref(shape), C.byref(best), per)
        return {"shape": shape.value, "ms": best.value, "shape_ms": [per[k] for k in range(count)]}

    def spmv(self, x: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """y = S x on the last assembled reduced system."""
        sfx = "f32" if x.dtype == torch.float32 else "f64"
        y = torch.empty_like(x) if out is None else out
        N.call(f"pm_schur_spmv_{sfx}", self._h, _stream_handle(stream), _ptr(x), _ptr(y))
        return y

    def export(self, dtype=torch.float64, stream=None) -> dict:
        """Last assembled reduced system in the reference's scalar-CSR layout."""
        n, nnz, blocks = self.dims()
        ro = torch.empty(n + 1, dtype=torch.int64, device="cuda")
        ci = torch.empty(nnz, dtype=torch.int64, device="cuda")
        v = torch.empty(nnz, dtype=dtype, device="cuda")
        rhs = torch.empty(n, dtype=torch.float64, device="cuda")
        bp2 = nnz // max(blocks, 1)
        P = n // max(int(round(bp2 ** 0.5)), 1) if blocks else 0
        pre = torch.empty(max(P * bp2, 1), dtype=torch.float64, device="cuda")
        sfx = "f32" if dtype == torch.float32 else "f64"
        N.call(f"pm_schur_export_{sfx}", self._h, _stream_handle(stream), _ptr(ro), _ptr(ci), _ptr(v), _ptr(rhs),
               _ptr(pre))
        torch.cuda.synchronize()
        return {"row_offsets": ro, "col_indices": ci, "values": v, "rhs": rhs, "preconditioner": pre}

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_schur_workspace_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


def solve_damped_schur_complement(equations: DeviceNormalEquations, damping: float,
                                  options: SchurComplementSolverOptions | None = None,
                                  workspace: SchurComplementSolverWorkspace | None = None,
                                  primary_step: torch.Tensor | None = None,
                                  eliminated_step: torch.Tensor | None = None, stream=None):
    """solveDampedSchurComplement (block_schur.cpp:54-459) on the device.

    Returns (primary_step, eliminated_step, report dict)."""
    opts = options or SchurComplementSolverOptions()
    ws = workspace or SchurComplementSolverWorkspace()
    n, m = equations.P * equations.bp, equations.L * equations.bl
    dt = equations.tdtype
    dp = primary_step if primary_step is not None else torch.zeros(max(n, 1), dtype=dt, device="cuda")
    dl = eliminated_step if eliminated_step is not None else torch.zeros(max(m, 1), dtype=dt, device="cuda")
    for name, t, size in (("primary_step", dp, n), ("eliminated_step", dl, m)):
        # the native solve writes `size` scalars through the pointer
        if not t.is_cuda or not t.is_contiguous() or t.dtype != dt or t.numel() < size:
            raise N.InvalidArgument(f"{name} must be a contiguous CUDA tensor of dtype {dt} with at least "
                                    f"{size} elements")
    rep = SchurReport()
    N.call(f"pm_schur_solve_{equations.sfx}", ws.handle, _stream_handle(stream), equations.handle,
           equations.ct(damping), C.byref(opts.c()), _ptr(dp), _ptr(dl), C.byref(rep))
    report = {k: getattr(rep, k) for k, _ in rep._fields_}
    report["message"] = rep.message.decode()
    report["converged"] = bool(rep.converged)
    report["pattern_reused"] = bool(rep.pattern_reused)
    report["mixed_precision_used"] = bool(rep.mixed_precision_used)
    report["learned_used"] = bool(rep.learned_used)
    report["learned_fallback"] = bool(rep.learned_fallback)
    return dp[:n], dl[:m], report


# ---------------------------------------------------------------- learned block Jacobi
N.register("pm_mlp_param_count", [], C.c_int64)
N.register("pm_mlp_create", [C.c_uint64, vp])
N.register("pm_mlp_destroy", [vp], None)
N.register("pm_mlp_get_params", [vp, vp])
N.register("pm_mlp_set_params", [vp, vp])
N.register("pm_mlp_forward", [vp, vp, vp])
N.register("pm_mlp_train_step", [vp, vp, vp, vp, vp, C.c_double, vp])
N.register("pm_mlp_inspect", [vp, vp, vp, vp, vp])
N.register("pm_mlp_set_wait_limit", [vp, i64])
N.register("pm_mlp_train_probe_step", [vp, vp, vp, vp, vp, C.c_double, vp])


class LearnedPreconditioner:
    """Per-block-row network correcting the block-Jacobi Cholesky factors of the reduced system
    (no counterpart in the reference; see pm_mlp_* in include/plamatrix_b200.h).  Pass it as
    SchurComplementSolverOptions(learned=...); train it on solved systems with train_step."""

    IN, HIDDEN, OUT = 25, 128, 21

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        N.call("pm_mlp_create", C.c_uint64(seed), C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    @staticmethod
    def param_count() -> int:
        return int(N.load().pm_mlp_param_count())

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        N.call("pm_mlp_get_params", self._h, C.c_void_p(out.ctypes.data))
        return out

    def set_params(self, params: np.ndarray) -> None:
        a = np.ascontiguousarray(params, np.float32)
        if a.size != self.param_count():
            raise N.InvalidArgument("parameter vector has the wrong length")
        N.call("pm_mlp_set_params", self._h, C.c_void_p(a.ctypes.data))

    def set_wait_limit(self, polls: int) -> None:
        """Polls of a GEMM operand-stage wait before it gives up (default 2^20); see
        pm_mlp_set_wait_limit."""
        N.call("pm_mlp_set_wait_limit", self._h, C.c_int64(polls))

    def forward(self, workspace: "SchurComplementSolverWorkspace", stream=None) -> dict:
        N.call("pm_mlp_forward", self._h, workspace.handle, _stream_handle(stream))
        return self.inspect()

    def train_step(self, workspace: "SchurComplementSolverWorkspace", x: torch.Tensor, b: torch.Tensor,
                   learning_rate: float = 1e-3, stream=None) -> float:
        """Loss of the last assembled system in `workspace` for its solution x and right-hand side
        b (device FP64, n = 6P); with learning_rate > 0 one Adam step follows."""
        if x.dtype != torch.float64 or b.dtype != torch.float64 or not (x.is_cuda and b.is_cuda):
            raise N.InvalidArgument("x and b must be float64 CUDA tensors")
        loss = C.c_double(0.0)
        N.call("pm_mlp_train_step", self._h, workspace.handle, _stream_handle(stream), _ptr(x), _ptr(b),
               C.c_double(learning_rate), C.byref(loss))
        return loss.value

    def train_probe_step(self, workspace: "SchurComplementSolverWorkspace", v: torch.Tensor, sv: torch.Tensor,
                         learning_rate: float = 1e-3, stream=None) -> float:
        """Loss ||(I - M S) v||^2 / ||v||^2 of the last assembled system in `workspace` along the probe
        v, given sv = S v (device FP64, n = 6P); with learning_rate > 0 one Adam step follows."""
        if v.dtype != torch.float64 or sv.dtype != torch.float64 or not (v.is_cuda and sv.is_cuda):
            raise N.InvalidArgument("v and sv must be float64 CUDA tensors")
        loss = C.c_double(0.0)
        N.call("pm_mlp_train_probe_step", self._h, workspace.handle, _stream_handle(stream), _ptr(v), _ptr(sv),
               C.c_double(learning_rate), C.byref(loss))
        return loss.value

    def inspect(self) -> dict:
        rows = C.c_int64(0)
        N.call("pm_mlp_inspect", self._h, C.byref(rows), None, None, None)
        P = rows.value
        feats = np.zeros((max(P, 1), self.IN), np.float32)
        outs = np.zeros((max(P, 1), self.OUT), np.float32)
        grads = np.zeros(self.param_count(), np.float32)
        N.call("pm_mlp_inspect", self._h, C.byref(rows), C.c_void_p(feats.ctypes.data),
               C.c_void_p(outs.ctypes.data), C.c_void_p(grads.ctypes.data))
        return {"features": feats[:P], "outputs": outs[:P], "gradients": grads}

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_mlp_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


# ---------------------------------------------------------------- batched independent systems
class BatchedSystemReport(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("learned_fallback", C.c_int),
                ("breakdown", C.c_int), ("initial_residual_norm", C.c_double), ("final_residual_norm", C.c_double),
                ("time_ms", C.c_double)]


N.register("pm_schur_batched_solve_f64", [vp, vp, vp, C.c_double, vp, i64, vp, vp, vp, vp, vp])


def pack_observation_systems(problems: list) -> dict:
    """One union observation problem (block-diagonal) from independent ones: system s gets the
    primary blocks [primary_offsets[s], primary_offsets[s+1]) and its own eliminated blocks."""
    P_off = np.cumsum([0] + [p["P"] for p in problems]).astype(np.int64)
    L_off = np.cumsum([0] + [p["L"] for p in problems]).astype(np.int64)
    first = problems[0]
    for p in problems:
        if (p["bp"], p["bl"], p["m"]) != (first["bp"], first["bl"], first["m"]):
            raise N.InvalidArgument("batched systems must share block and residual sizes")
    cat = lambda key: np.ascontiguousarray(np.concatenate([p[key] for p in problems]))  # noqa: E731
    return {
        "P": int(P_off[-1]), "L": int(L_off[-1]), "bp": first["bp"], "bl": first["bl"], "m": first["m"],
        "huber_delta": first["huber_delta"],
        "obs_primary": np.ascontiguousarray(np.concatenate([p["obs_primary"] + P_off[i] for i, p in enumerate(problems)])),
        "obs_eliminated": np.ascontiguousarray(
            np.concatenate([p["obs_eliminated"] + L_off[i] for i, p in enumerate(problems)])),
        "jp": cat("jp"), "jl": cat("jl"), "residual": cat("residual"),
        "primary_offsets": P_off, "eliminated_offsets": L_off,
    }


def solve_batched_schur_complement(equations: DeviceNormalEquations, damping: float, primary_offsets,
                                   options: SchurComplementSolverOptions | None = None,
                                   workspace: SchurComplementSolverWorkspace | None = None, stream=None):
    """Independent systems accumulated into one block-diagonal `equations` (double), solved together.
    Returns (primary_step, eliminated_step, summary report, list of per-system report dicts)."""
    if equations.dtype != np.float64:
        raise N.InvalidArgument("batched solves run on double normal equations")
    opts = options or SchurComplementSolverOptions()
    ws = workspace or SchurComplementSolverWorkspace()
    offs = np.ascontiguousarray(primary_offsets, np.int64)
    systems = len(offs) - 1
    n, m = equations.P * equations.bp, equations.L * equations.bl
    dp = torch.zeros(max(n, 1), dtype=torch.float64, device="cuda")
    dl = torch.zeros(max(m, 1), dtype=torch.float64, device="cuda")
    rep = SchurReport()
    per = (BatchedSystemReport * max(systems, 1))()
    N.call("pm_schur_batched_solve_f64", ws.handle, _stream_handle(stream), equations.handle, C.c_double(damping),
           C.byref(opts.c()), systems, C.c_void_p(offs.ctypes.data), _ptr(dp), _ptr(dl), C.byref(rep), per)
    report = {k: getattr(rep, k) for k, _ in rep._fields_}
    report["message"] = rep.message.decode()
    report["converged"] = bool(rep.converged)
    systems_out = [{k: getattr(per[s], k) for k, _ in BatchedSystemReport._fields_} for s in range(systems)]
    return dp[:n], dl[:m], report, systems_out

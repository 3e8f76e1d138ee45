"""The C-ABI library builds for sm_100a, loads without a GPU and exports every entry
point that include/*.h declares (no device compute here)."""
import ctypes as C
import os
import subprocess

import pytest

from plamatrix_b200 import _native as N


@pytest.fixture(scope="module")
def lib():
    from plamatrix_b200 import build
    build.build()
    return N.load()


def test_every_declared_symbol_is_exported(lib):
    declared = N.declared_symbols()
    assert len(declared) > 20
    out = subprocess.run(["nm", "-D", "--defined-only", N.library_path()], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [name for name in declared if name not in exported]
    assert not missing, missing
    for name in declared:
        assert hasattr(lib, name)


def test_library_is_built_for_sm100a_only(lib):
    """The build recipe compiles every translation unit and the link for sm_100a and nothing else."""
    from plamatrix_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert not any("arch=" in flag or flag.startswith("-arch") for flag in build.FLAGS)
    assert os.path.getmtime(N.library_path()) >= max(os.path.getmtime(s) for s in build._sources())


def test_host_side_argument_checks(lib):
    ws = C.c_void_p()
    assert lib.pm_sparse_workspace_create(C.byref(ws)) == 0
    # an unused workspace has no pending status
    nnz = C.c_int64(-1)
    assert lib.pm_coo_status(ws, b"cooToCsrAsync", C.byref(nnz)) == 0 and nnz.value == 0
    # metadata is rejected before any device work
    status = lib.pm_coo_to_csr_count_f64(ws, None, -1, 4, 0, None, None, None)
    assert status == N.PM_INVALID_ARGUMENT
    assert b"non-negative" in lib.pm_last_error()
    status = lib.pm_coo_to_csr_count_f64(ws, None, 4, 1 << 33, 0, None, None, None)
    assert status == N.PM_OVERFLOW_ERROR
    with pytest.raises(N.InvalidArgument):
        N.call("pm_coo_to_csr_count_f32", None, None, 1, 1, 0, None, None, None)
    lib.pm_sparse_workspace_destroy(ws)
    opts = N.SolverOptions(-1, 1e-6, 0.0, 1, 0)
    rep = N.SolverReport()
    sw = C.c_void_p()
    assert lib.pm_solver_workspace_create(C.byref(sw)) == 0
    assert lib.pm_cg_f64(sw, None, None, None, None, C.byref(opts), C.byref(rep)) == N.PM_INVALID_ARGUMENT
    lib.pm_solver_workspace_destroy(sw)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No CPU fallback: without the built library every entry point raises instead of computing."""
    from plamatrix_b200 import _native as N
    from plamatrix_b200 import schur as SC

    monkeypatch.setattr(N, "_lib", None)
    monkeypatch.setattr(N, "LIB_PATH", str(tmp_path / "libplamatrix_b200.so"))
    with pytest.raises(ImportError, match="no CPU fallback"):
        N.load()
    with pytest.raises(ImportError, match="no CPU fallback"):
        SC.SchurComplementSolverWorkspace()


def test_assembly_shape_table(lib):
    """The assembly launch shapes are host-side data: readable without a GPU."""
    count = lib.pm_schur_assembly_shape_count()
    assert count >= 2
    seen = set()
    for k in range(count):
        streams, split = C.c_int(), C.c_int()
        assert lib.pm_schur_assembly_shape_info(k, C.byref(streams), C.byref(split)) == 0
        assert split.value in (2, 4) and streams.value * split.value <= 32
        seen.add((streams.value, split.value))
    assert len(seen) == count
    streams, split = C.c_int(), C.c_int()
    assert lib.pm_schur_assembly_shape_info(count, C.byref(streams), C.byref(split)) != 0
    assert lib.pm_schur_set_assembly_shape(None, 0) != 0

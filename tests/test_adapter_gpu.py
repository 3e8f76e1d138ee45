"""The C++ drop-in header (include/plamatrix_b200_adapter.hpp) on the reference's own types: the
test binary tests/adapter/adapter_test.cpp, compiled against the reference headers and linked
with the reference's CPU library and libplamatrix_b200.so by oracle/Makefile (target `adapter`),
compares solveDampedSchurComplement, cooToCsr and blockPcg through the adapter (on the device)
with the reference's CPU implementations of the same calls."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "adapter_test")


def test_adapter_builds_against_the_reference_headers():
    """CPU: the header compiles against the reference's headers and links (where the reference
    tree is present; elsewhere the prebuilt binary is used as is)."""
    import oracle
    if os.path.isdir(os.path.join(oracle.REF_SOURCE_ROOT, "include")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "adapter"], check=True)
    if not os.path.exists(BINARY):
        pytest.skip("reference tree absent and no prebuilt adapter test binary")
    assert os.access(BINARY, os.X_OK)


@pytest.mark.gpu
def test_adapter_matches_the_reference_on_its_own_types():
    assert os.path.exists(BINARY), "oracle/_ref/adapter_test was not built"
    res = subprocess.run([BINARY], capture_output=True, text=True, timeout=600)
    print(res.stdout)
    fails = [line for line in res.stdout.splitlines() if line.startswith("FAIL")]
    assert res.returncode == 0 and not fails, res.stdout + res.stderr
    assert "ADAPTER OK" in res.stdout
    assert sum(line.startswith("PASS") for line in res.stdout.splitlines()) >= 25

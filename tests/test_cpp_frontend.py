"""The C++ front end (include/loom_b200.hpp): Loom kernel types bound to the
compiled kernels by IR digest and run through function / hybrid_function /
stream, as Loom's CUDA backend test runs vm::cuda::function and
vm::cuda::stream (Loom src/tests/vm.cu:43-88).

The program is built from the Loom headers (tests/cpp/build_vm_test.py); on
a machine without them the prebuilt binary is used, and without either the
tests are skipped.
"""

from __future__ import annotations

import pathlib
import subprocess
import sys

import pytest

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "cpp"))

import build_vm_test  # noqa: E402


@pytest.fixture(scope="module")
def program():
    exe = build_vm_test.build()
    if exe is None or not exe.exists():
        pytest.skip("C++ front-end test program not built (no Loom headers here)")
    return exe


def test_kernel_types_bind_by_digest(program):
    """Every kernel type of the test binds to the kernel compiled from its IR
    (no GPU needed: binding reads only the registry)."""
    r = subprocess.run([str(program), "--bind-only"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    names = [ln.split()[0] for ln in r.stdout.splitlines()]
    assert names == ["increment_i32", "fac_u32", "union_f32", "union_cmov_f32", "jmp4_f32", "lshift_u32", "rshift_u32"]


@pytest.mark.gpu
@pytest.mark.parametrize("numruns,seed", [(1000, 0), (4096, 7)])
def test_vm_cu_suite(program, numruns, seed):
    r = subprocess.run(
        [str(program), "-n", str(numruns), "-s", str(seed)], capture_output=True, text=True, timeout=300
    )
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
    assert r.stdout.count("PASS") == 15, r.stdout

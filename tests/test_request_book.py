"""The serving loop's failure bookkeeping (cancel, watchdog, hand-out of
failed tickets; loom_b200/csrc/request_book.hpp) compiled with g++ and run
on the host: it holds no CUDA, so its logic is tested without a GPU.  The
ABI entry points that use it refuse a NULL server without touching one."""

import pathlib
import shutil
import subprocess

import pytest

from loom_b200 import api

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_request_book_logic(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    exe = tmp_path / "request_book_test"
    src = ROOT / "tests" / "cpp" / "request_book_test.cpp"
    subprocess.run(
        [gxx, "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{ROOT / 'loom_b200' / 'csrc'}", str(src), "-o", str(exe)],
        check=True,
        timeout=120,
    )
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


def test_server_calls_refuse_a_null_server():
    L = api.lib()
    n = api.ctypes.c_uint32()
    assert L.loom_b200_server_cancel(None, 1) == api.ERR_INVALID
    assert L.loom_b200_server_set_timeout(None, 10) == api.ERR_INVALID
    assert L.loom_b200_server_failed(None, None, None, 0, api.ctypes.byref(n)) == api.ERR_INVALID

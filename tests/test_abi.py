"""The C-ABI library: loads, exports what include/loom_b200.h declares, and
describes every kernel exactly as its IR does (CPU only; no compute)."""

import pathlib
import re

import pytest

from loom_b200 import api
from loom_b200.codegen import ir

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "loom_b200.h").read_text()
    return sorted(set(re.findall(r"\b(loom_b200_[a-z_]+)\s*\(", text)))


def test_header_declares_the_abi():
    assert "loom_b200_create" in declared_functions()
    assert set(declared_functions()) == set(api.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = api.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_version():
    assert api.lib().loom_b200_version() == 1


def test_registry_matches_ir():
    names = set(api.kernels())
    assert names == set(ir.available())
    for n in sorted(names):
        k = ir.load(n)
        info = api.info(n)
        assert info.ir_digest == k.digest(), n
        assert info.num_blocks == k.num_blocks
        assert [t for _, t in info.inputs] == [t for _, t, _ in k.inputs]
        assert [t for _, t in info.outputs] == [t for _, t, _ in k.outputs]
        assert info.block_instrs == k.instr_counts()
        assert info.state_size == sum(r.nbytes for r in k.regs)


def test_find_by_structural_digest():
    """The C++ front end binds a kernel type by the digest of its IR: every
    compiled kernel is found under its own digest, and digests are unique."""
    import ctypes

    L = api.lib()
    digests = {}
    for n in api.kernels():
        d = ir.load(n).digest()
        assert re.fullmatch(r"[0-9a-f]{16}", d), d
        assert d not in digests, (n, digests.get(d))
        digests[d] = n
        p = ctypes.POINTER(api.KernelInfoC)()
        assert L.loom_b200_kernel_find_digest(d.encode(), ctypes.byref(p)) == 0
        assert p.contents.name.decode() == n
    p = ctypes.POINTER(api.KernelInfoC)()
    assert L.loom_b200_kernel_find_digest(b"0000000000000000", ctypes.byref(p)) == api.ERR_NOT_FOUND


def test_unknown_kernel_is_not_found():
    with pytest.raises(api.LoomError) as e:
        api.info("no_such_kernel")
    assert e.value.code == api.ERR_NOT_FOUND


def test_generated_sources_are_current():
    from loom_b200.codegen import emit_cuda

    gen = ROOT / "loom_b200" / "csrc" / "gen"
    for n in ir.available():
        assert (gen / f"{n}.cu").read_text() == emit_cuda.generate(ir.load(n)), n
    assert (gen / "registry.cu").read_text() == emit_cuda.generate_registry(ir.available())


def test_liveness_of_fib():
    k = ir.load("fib_u64")
    live_in, _ = k.liveness()
    names = {r.idx: r.name for r in k.regs}
    assert {names[r] for r in live_in[0]} == {"n"}
    assert {names[r] for r in live_in[1]} == {"n"}
    assert {names[r] for r in live_in[2]} == {"n", "p", "c", "i"}


def test_create_without_device_fails_cleanly():
    from conftest import cuda_available

    if cuda_available():
        pytest.skip("a device is visible")
    with pytest.raises(api.LoomError) as e:
        api.Function("fib_u64", 16)
    assert e.value.code in (api.ERR_NO_DEVICE, api.ERR_CUDA)


def test_server_create_without_device_fails_cleanly():
    from conftest import cuda_available

    if cuda_available():
        pytest.skip("a device is visible")
    with pytest.raises(api.LoomError) as e:
        api.Server("collatz_u64", ring_threads=1 << 10)
    assert e.value.code in (api.ERR_NO_DEVICE, api.ERR_CUDA)


def test_server_rejects_bad_configuration():
    """Checked before any device call: ring size not a power of two, no
    request slots, a relocated word outside the header."""
    for kw in (dict(ring_threads=1000), dict(ring_threads=1 << 10, max_requests=0),
               dict(ring_threads=1 << 10, header_words=4, reloc_word=4)):
        with pytest.raises(api.LoomError) as e:
            api.Server("collatz_u64", **kw)
        assert e.value.code == api.ERR_INVALID, kw

"""loom_b200_launch_static: the regrouping engine for callers that cannot
allocate device memory at the point of the call (a plugin whose host's
caching allocator already holds the free memory, code that must not stall on
cudaMalloc).  The engine's workspace lives in a fixed device array inside the
library instead.

The GPU tests call the entry point through the C ABI (ctypes, device columns
from torch) twice in a row and compare every output with the handle-based
entry point, loom_b200_launch_device, bit for bit, as every engine test does.
This file sorts last, so a run that stops at the first failure has already
run every other test; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from loom_b200 import api
from oracle import oracle as O


def _launch_struct(kernel, inputs, outputs, n, starts=None, table=None):
    """Builds loom_b200_launch from device tensors; an input is a tensor or
    one of the forms api.Instance / api.LocalIota / api.Iota."""
    ins = (api.InputC * max(1, len(inputs)))()
    for i, a in enumerate(inputs):
        if a is api.Instance:
            ins[i] = api.InputC(None, api.IN_INSTANCE, 0, 0)
        elif a is api.LocalIota:
            ins[i] = api.InputC(None, api.IN_LOCAL_IOTA, 0, 0)
        elif a is api.Iota:
            ins[i] = api.InputC(None, api.IN_IOTA, 0, 0)
        else:
            ins[i] = api.InputC(a.data_ptr(), api.IN_ARRAY, 0, 0)
    outs = (ctypes.c_void_p * len(outputs))(*[o.data_ptr() for o in outputs])
    L = api.LaunchC()
    L.inputs = ins
    L.outputs = outs
    L.n = n
    L.instance_starts = None if starts is None else starts.data_ptr()
    L.num_instances = 0 if starts is None else starts.numel() - 1
    L.table = None if table is None else table.data_ptr()
    L.table_words = 0 if table is None else table.numel()
    return L, (ins, outs)


def _static(kernel, inputs, outputs, n, starts=None, table=None, opts=None):
    import torch

    L, keep = _launch_struct(kernel, inputs, outputs, n, starts, table)
    status = ctypes.c_uint32(0)
    rc = api.lib().loom_b200_launch_static(
        kernel.encode(),
        ctypes.byref(L),
        None if opts is None else ctypes.byref(opts),
        torch.cuda.current_stream().cuda_stream,
        ctypes.byref(status),
    )
    del keep
    return rc, status.value


def _existing(kernel, inputs, outputs, n, starts=None, table=None):
    """The same launch through a handle (the entry point that allocates)."""
    import torch

    with api.Function(kernel, 0, "regroup") as f:
        L, keep = _launch_struct(kernel, inputs, outputs, n, starts, table)
        api.check(api.lib().loom_b200_launch_device(f._h, ctypes.byref(L), torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        f.sync()
        del keep


@pytest.mark.gpu
def test_static_collatz_matches_launch_device_twice():
    import torch

    for call, seed in enumerate((3, 4)):
        x = O.uniform_int(seed, 200_000, 1, 1 << 40)
        d_x = torch.from_numpy(x.view(np.int64)).cuda()
        want = torch.empty(len(x), dtype=torch.int32, device="cuda")
        got = torch.full((len(x),), -1, dtype=torch.int32, device="cuda")
        _existing("collatz_u64", [d_x], [want], len(x))
        rc, status = _static("collatz_u64", [d_x], [got], len(x))
        assert (rc, status) == (api.OK, 0), f"call {call}: rc {rc} status {status:#x}"
        assert torch.equal(got, want), f"call {call}: {(got != want).sum().item()} threads differ"
        assert np.array_equal(want.cpu().numpy().view(np.uint32), O.val_collatz(x))


@pytest.mark.gpu
def test_static_path_tracer_matches_launch_device_twice(golden, golden_extra):
    """The batched path-tracing fixture (several scenes in one launch, table
    and instance offsets on the device), with a population small enough that
    inputs are admitted in many rounds."""
    import torch

    ins, _ = golden("sphere_pt_f32")
    extra = golden_extra("sphere_pt_f32")
    n = len(ins[0])
    table = torch.from_numpy(extra["table"].view(np.int32)).cuda()
    starts = torch.from_numpy(extra["starts"].view(np.int64)).cuda()
    forms = [api.Instance, api.LocalIota]
    want = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3)]
    _existing("sphere_pt_f32", forms, want, n, starts, table)
    opts = api.Opts()
    opts.population = 4096
    for call in range(2):
        got = [torch.full((n,), float("nan"), dtype=torch.float32, device="cuda") for _ in range(3)]
        rc, status = _static("sphere_pt_f32", forms, got, n, starts, table, opts if call else None)
        assert (rc, status) == (api.OK, 0), f"call {call}: rc {rc} status {status:#x}"
        for g, w in zip(got, want):
            assert torch.equal(g.view(torch.int32), w.view(torch.int32)), f"call {call}: outputs differ"


@pytest.mark.gpu
def test_static_device_status_then_clean_call():
    """A launch that stops at its round limit reports the device status
    (LOOM_B200_ERR_DEVICE with the STEP_LIMIT bit in *status_out); the next
    call starts from cleared control words and equals the handle-based launch
    bit for bit, although the shared array still holds the stopped launch's
    parked threads."""
    import torch

    x = O.uniform_int(9, 100_000, 1, 1 << 40)
    d_x = torch.from_numpy(x.view(np.int64)).cuda()
    out = torch.empty(len(x), dtype=torch.int32, device="cuda")
    opts = api.Opts()
    opts.population = 4096  # many rounds are needed ...
    opts.max_steps = 1  # ... and the engine may run one
    rc, status = _static("collatz_u64", [d_x], [out], len(x), opts=opts)
    assert rc == api.ERR_DEVICE
    assert status & api.STATUS_STEP_LIMIT
    want = torch.empty(len(x), dtype=torch.int32, device="cuda")
    got = torch.full((len(x),), -1, dtype=torch.int32, device="cuda")
    _existing("collatz_u64", [d_x], [want], len(x))
    rc, status = _static("collatz_u64", [d_x], [got], len(x), opts=None)
    assert (rc, status) == (api.OK, 0), f"rc {rc} status {status:#x}"
    assert torch.equal(got, want)


def test_static_refuses_what_the_array_cannot_hold():
    """Sizes beyond the fixed array are refused before anything runs (no GPU
    needed): a population whose queue state exceeds the array, and more
    threads than 32-bit thread ids can name."""
    limit = 64 << 20
    ins = (api.InputC * 2)(api.InputC(None, api.IN_IOTA, 0, 0), api.InputC(None, api.IN_IOTA, 0, 0))
    # output pointers are never dereferenced: every call below is refused first
    outs = (ctypes.c_void_p * 3)(16, 16, 16)
    L = api.LaunchC()
    L.inputs = ins
    L.outputs = outs
    L.n = 1 << 30
    opts = api.Opts()
    # sphere_pt_f32 keeps 2832 queue bytes per thread in flight, twice over
    # (both round parities): this population needs twice the array
    opts.population = limit // 2832
    rc = api.lib().loom_b200_launch_static(b"sphere_pt_f32", ctypes.byref(L), ctypes.byref(opts), None, None)
    assert rc == api.ERR_BUDGET
    L.n = 1 << 32
    rc = api.lib().loom_b200_launch_static(b"collatz_u64", ctypes.byref(L), None, None, None)
    assert rc == api.ERR_INVALID
    rc = api.lib().loom_b200_launch_static(b"no_such_kernel", ctypes.byref(L), None, None, None)
    assert rc == api.ERR_NOT_FOUND

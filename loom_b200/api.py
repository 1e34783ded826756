"""Python binding of libloom_b200 (the C ABI in include/loom_b200.h).

Mirrors the call shapes of Loom's backends:

* ``Function(kernel, n)(*inputs)`` is ``vm::cuda::function<K>(n)(inputs...)``
  (Loom src/vm/cuda.hpp:1406-1462): input columns in, output columns out, in
  input order;
* ``Function.run_device`` launches on device columns (torch tensors or raw
  pointers) without synchronising, for callers that keep data resident.

There is no CPU fallback: if the CUDA library is missing or no device is
visible, construction raises.
"""

from __future__ import annotations

import ctypes
import pathlib
from typing import Dict, List, Optional, Sequence, Tuple, Union

import numpy as np

import os

# LOOM_B200_LIB selects another build of the library (e.g. one with more
# kernels compiled in); default: the in-tree build
LIB_PATH = pathlib.Path(
    os.environ.get("LOOM_B200_LIB", pathlib.Path(__file__).resolve().parent / "libloom_b200.so")
)

PLAIN = 0
REGROUP = 1

OK = 0
ERR_INVALID = -1
ERR_NOT_FOUND = -2
ERR_CUDA = -3
ERR_OOM = -4
ERR_DEVICE = -5
ERR_BUDGET = -6
ERR_NO_DEVICE = -7
ERR_CANCELLED = -8
ERR_TIMEOUT = -9

IN_ARRAY = 0
IN_IOTA = 1
IN_BROADCAST = 2
IN_LOCAL_IOTA = 3
IN_INSTANCE = 4

STATUS_STEP_LIMIT = 1
STATUS_ASSERT_FP = 2
STATUS_QUEUE_OVERRUN = 4
STATUS_BARRIER_TIMEOUT = 8
PERIOD_UNBOUNDED = 0xFFFFFFFF  # opts.period: schedule 2 never parks

TYPE_NAMES = ["b8", "i8", "u8", "i16", "u16", "i32", "u32", "i64", "u64", "f32", "f64"]
F32, F64 = 9, 10  # enum loom_b200_type
NP_TYPE = {
    "b8": np.uint8,
    "i8": np.int8,
    "u8": np.uint8,
    "i16": np.int16,
    "u16": np.uint16,
    "i32": np.int32,
    "u32": np.uint32,
    "i64": np.int64,
    "u64": np.uint64,
    "f32": np.float32,
    "f64": np.float64,
}


class LoomError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libloom_b200 error {code}: {msg}")
        self.code = code


class KernelInfoC(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char_p),
        ("ir_digest", ctypes.c_char_p),
        ("num_inputs", ctypes.c_uint32),
        ("num_outputs", ctypes.c_uint32),
        ("input_types", ctypes.POINTER(ctypes.c_int)),
        ("output_types", ctypes.POINTER(ctypes.c_int)),
        ("input_names", ctypes.POINTER(ctypes.c_char_p)),
        ("output_names", ctypes.POINTER(ctypes.c_char_p)),
        ("num_blocks", ctypes.c_uint32),
        ("num_regs", ctypes.c_uint32),
        ("state_size", ctypes.c_uint32),
        ("state_cols", ctypes.c_uint32),
        ("block_instrs", ctypes.POINTER(ctypes.c_uint32)),
        ("block_live_bytes", ctypes.POINTER(ctypes.c_uint32)),
    ]


class Opts(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_uint32),
        ("block_size", ctypes.c_uint32),
        ("utr_lanes", ctypes.c_uint32),
        ("period", ctypes.c_uint32),
        ("burst", ctypes.c_uint32),
        ("spread_lanes", ctypes.c_uint32),
        ("no_refill", ctypes.c_uint32),
        ("graph", ctypes.c_uint32),
        ("population", ctypes.c_uint64),
        ("max_steps", ctypes.c_uint64),
        ("profile", ctypes.c_uint32),
        ("no_prefetch", ctypes.c_uint32),
        ("ctas_per_sm", ctypes.c_uint32),
        ("fault_phantom_ctas", ctypes.c_uint32),
        ("barrier_spins", ctypes.c_uint64),
        ("cost_model", ctypes.c_uint32),
        ("schedule", ctypes.c_uint32),
        ("host_chunks", ctypes.c_uint32),
        ("max_regs", ctypes.c_uint32),
        ("plain_below", ctypes.c_uint64),
        ("defer_lanes", ctypes.c_uint32),
        ("bulk_restore", ctypes.c_uint32),
        ("spin_iters", ctypes.c_uint32),
        ("refill_lanes", ctypes.c_uint32),
    ]


class StatsC(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64),
        ("threads", ctypes.c_uint64),
        ("thread_instr", ctypes.c_uint64),
        ("warp_instr", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
        ("parks", ctypes.c_uint64),
        ("state_bytes", ctypes.c_uint64),
        ("status", ctypes.c_uint32),
        ("grid", ctypes.c_uint32),
        ("ms", ctypes.c_double),
        ("graph_captures", ctypes.c_uint64),
        ("graph_launches", ctypes.c_uint64),
    ]


class InputC(ctypes.Structure):
    _fields_ = [
        ("ptr", ctypes.c_void_p),
        ("form", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("value", ctypes.c_uint64),
    ]


class LaunchC(ctypes.Structure):
    _fields_ = [
        ("inputs", ctypes.POINTER(InputC)),
        ("outputs", ctypes.POINTER(ctypes.c_void_p)),
        ("n", ctypes.c_uint64),
        ("instance_starts", ctypes.c_void_p),
        ("num_instances", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("table", ctypes.c_void_p),
        ("table_words", ctypes.c_uint64),
    ]


class MeanC(ctypes.Structure):
    _fields_ = [
        ("group", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("instance_group", ctypes.POINTER(ctypes.c_uint32)),
    ]


class BudgetC(ctypes.Structure):
    _fields_ = [("limit", ctypes.c_uint64), ("used", ctypes.c_uint64)]


class Budget:
    """A device-memory budget for the thread state of admitted requests
    (loom_b200_budget), shared by the servers created with it."""

    def __init__(self, limit_bytes: int):
        self.c = BudgetC(int(limit_bytes), 0)

    @property
    def limit(self) -> int:
        return int(self.c.limit)

    @property
    def used(self) -> int:
        return int(self.c.used)


class ServerCfgC(ctypes.Structure):
    _fields_ = [
        ("ring_threads", ctypes.c_uint64),
        ("table_words", ctypes.c_uint64),
        ("header_words", ctypes.c_uint32),
        ("reloc_word", ctypes.c_int32),
        ("max_requests", ctypes.c_uint32),
        ("slice_rounds", ctypes.c_uint32),
        ("forms", ctypes.POINTER(ctypes.c_uint32)),
        ("budget", ctypes.POINTER(BudgetC)),
    ]


class RequestC(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint64),
        ("inputs", ctypes.POINTER(ctypes.c_void_p)),
        ("outputs", ctypes.POINTER(ctypes.c_void_p)),
        ("header", ctypes.POINTER(ctypes.c_uint32)),
        ("body", ctypes.POINTER(ctypes.c_uint32)),
        ("body_words", ctypes.c_uint64),
    ]


class ServerStatsC(ctypes.Structure):
    _fields_ = [
        (f, ctypes.c_uint64)
        for f in (
            "submitted",
            "admitted",
            "completed",
            "threads",
            "slices",
            "rounds",
            "queued",
            "in_flight",
            "unreported",
            "device_bytes",
            "thread_instr",
            "warp_instr",
        )
    ] + [
        ("status", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("budget_waits", ctypes.c_uint64),
        ("held_bytes", ctypes.c_uint64),
        ("busy_ms", ctypes.c_double),
        ("slice_t0_ns", ctypes.c_uint64),
        ("slice_t1_ns", ctypes.c_uint64),
    ]


class Iota:
    """Input column = thread index."""


class LocalIota:
    """Input column = thread index within its instance."""


class Instance:
    """Input column = index of the thread's instance."""


class Broadcast:
    """Input column = one value for every thread."""

    def __init__(self, value, type_name: str):
        self.value = value
        self.type_name = type_name

    def bits(self) -> int:
        a = np.array([self.value], dtype=NP_TYPE[self.type_name])
        b = np.zeros(8, dtype=np.uint8)
        b[: a.itemsize] = a.view(np.uint8)
        return int(b.view(np.uint64)[0])


_lib = None

# every symbol include/loom_b200.h declares
EXPORTS = [
    "loom_b200_version",
    "loom_b200_error_string",
    "loom_b200_kernel_count",
    "loom_b200_kernel_get",
    "loom_b200_kernel_find",
    "loom_b200_kernel_find_digest",
    "loom_b200_kernel_reg_caps",
    "loom_b200_create",
    "loom_b200_destroy",
    "loom_b200_set_opts",
    "loom_b200_get_opts",
    "loom_b200_run_host",
    "loom_b200_run_device",
    "loom_b200_launch_device",
    "loom_b200_launch_host",
    "loom_b200_launch_host_mean",
    "loom_b200_group_mean",
    "loom_b200_sync",
    "loom_b200_get_stats",
    "loom_b200_reset_stats",
    "loom_b200_device_bytes",
    "loom_b200_get_block_stats",
    "loom_b200_kernel_queues",
    "loom_b200_parked_counts",
    "loom_b200_parked_dump",
    "loom_b200_launch_static",
    "loom_b200_server_create",
    "loom_b200_server_destroy",
    "loom_b200_server_submit",
    "loom_b200_server_step",
    "loom_b200_server_launch",
    "loom_b200_server_get_stats",
    "loom_b200_server_cancel",
    "loom_b200_server_set_timeout",
    "loom_b200_server_failed",
]


def lib() -> ctypes.CDLL:
    """Load libloom_b200.so (fails loudly when it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m loom_b200.build` "
            "(there is no CPU fallback)"
        )
    L = ctypes.CDLL(str(LIB_PATH))
    vp = ctypes.c_void_p
    L.loom_b200_version.restype = ctypes.c_int
    L.loom_b200_error_string.restype = ctypes.c_char_p
    L.loom_b200_error_string.argtypes = [ctypes.c_int]
    L.loom_b200_kernel_count.restype = ctypes.c_int
    L.loom_b200_kernel_get.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.POINTER(KernelInfoC))]
    L.loom_b200_kernel_find.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(KernelInfoC))]
    L.loom_b200_kernel_find_digest.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(KernelInfoC))]
    L.loom_b200_kernel_reg_caps.argtypes = [
        ctypes.c_char_p,
        ctypes.POINTER(ctypes.c_uint32),
        ctypes.c_uint32,
        ctypes.POINTER(ctypes.c_uint32),
    ]
    L.loom_b200_create.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(Opts), ctypes.POINTER(vp)]
    L.loom_b200_destroy.argtypes = [vp]
    L.loom_b200_set_opts.argtypes = [vp, ctypes.POINTER(Opts)]
    L.loom_b200_get_opts.argtypes = [vp, ctypes.POINTER(Opts)]
    L.loom_b200_run_host.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_uint64]
    L.loom_b200_run_device.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_uint64, vp]
    L.loom_b200_launch_device.argtypes = [vp, ctypes.POINTER(LaunchC), vp]
    L.loom_b200_launch_host.argtypes = [vp, ctypes.POINTER(LaunchC)]
    L.loom_b200_launch_host_mean.argtypes = [vp, ctypes.POINTER(LaunchC), ctypes.POINTER(MeanC)]
    L.loom_b200_group_mean.argtypes = [ctypes.c_uint32, vp, vp, ctypes.c_uint64, ctypes.c_uint32, vp]
    L.loom_b200_sync.argtypes = [vp]
    L.loom_b200_get_stats.argtypes = [vp, ctypes.POINTER(StatsC)]
    L.loom_b200_reset_stats.argtypes = [vp]
    L.loom_b200_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.loom_b200_get_block_stats.argtypes = [
        vp,
        ctypes.POINTER(ctypes.c_uint64),
        ctypes.POINTER(ctypes.c_uint64),
        ctypes.c_uint32,
    ]
    L.loom_b200_kernel_queues.argtypes = [
        ctypes.c_char_p,
        ctypes.POINTER(ctypes.c_uint32),
        ctypes.POINTER(ctypes.POINTER(QueueLayoutC)),
    ]
    L.loom_b200_parked_counts.argtypes = [
        vp,
        ctypes.POINTER(ctypes.c_uint32),
        ctypes.c_uint32,
        ctypes.POINTER(ctypes.c_uint32),
    ]
    L.loom_b200_parked_dump.argtypes = [
        vp,
        ctypes.c_uint32,
        ctypes.POINTER(vp),
        ctypes.POINTER(ctypes.c_uint32),
        ctypes.c_uint64,
        ctypes.POINTER(ctypes.c_uint64),
    ]
    L.loom_b200_server_create.argtypes = [
        ctypes.c_char_p,
        ctypes.POINTER(Opts),
        ctypes.POINTER(ServerCfgC),
        vp,
        ctypes.POINTER(vp),
    ]
    L.loom_b200_server_destroy.argtypes = [vp]
    L.loom_b200_server_submit.argtypes = [vp, ctypes.POINTER(RequestC), ctypes.POINTER(ctypes.c_uint64)]
    L.loom_b200_server_launch.argtypes = [vp, ctypes.c_uint32]
    L.loom_b200_server_step.argtypes = [
        vp,
        ctypes.POINTER(ctypes.c_uint64),
        ctypes.c_uint32,
        ctypes.POINTER(ctypes.c_uint32),
    ]
    L.loom_b200_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStatsC)]
    L.loom_b200_server_cancel.argtypes = [vp, ctypes.c_uint64]
    L.loom_b200_server_set_timeout.argtypes = [vp, ctypes.c_uint64]
    L.loom_b200_server_failed.argtypes = [
        vp,
        ctypes.POINTER(ctypes.c_uint64),
        ctypes.POINTER(ctypes.c_int32),
        ctypes.c_uint32,
        ctypes.POINTER(ctypes.c_uint32),
    ]
    L.loom_b200_launch_static.argtypes = [
        ctypes.c_char_p,
        ctypes.POINTER(LaunchC),
        ctypes.POINTER(Opts),
        vp,
        ctypes.POINTER(ctypes.c_uint32),
    ]
    _lib = L
    return L


def check(code: int) -> int:
    if code != OK:
        msg = lib().loom_b200_error_string(code)
        raise LoomError(code, msg.decode() if msg else "?")
    return code


class KernelInfo:
    def __init__(self, c: KernelInfoC):
        self.name = c.name.decode()
        self.ir_digest = c.ir_digest.decode()
        self.inputs = [
            (c.input_names[i].decode(), TYPE_NAMES[c.input_types[i]]) for i in range(c.num_inputs)
        ]
        self.outputs = [
            (c.output_names[i].decode(), TYPE_NAMES[c.output_types[i]])
            for i in range(c.num_outputs)
        ]
        self.num_blocks = c.num_blocks
        self.num_regs = c.num_regs
        self.state_size = c.state_size
        self.state_cols = c.state_cols
        self.block_instrs = [c.block_instrs[i] for i in range(c.num_blocks)]
        self.block_live_bytes = [c.block_live_bytes[i] for i in range(c.num_blocks)]

    def __repr__(self):
        return f"KernelInfo({self.name}, in={self.inputs}, out={self.outputs}, blocks={self.num_blocks})"


def kernels() -> List[str]:
    L = lib()
    out = []
    for i in range(L.loom_b200_kernel_count()):
        p = ctypes.POINTER(KernelInfoC)()
        check(L.loom_b200_kernel_get(i, ctypes.byref(p)))
        out.append(p.contents.name.decode())
    return out


class QueueLayoutC(ctypes.Structure):
    _fields_ = [
        ("block", ctypes.c_uint32),
        ("context", ctypes.c_int32),
        ("num_cols", ctypes.c_uint32),
        ("regs", ctypes.POINTER(ctypes.c_uint32)),
        ("types", ctypes.POINTER(ctypes.c_int)),
        ("names", ctypes.POINTER(ctypes.c_char_p)),
    ]


def queues(kernel: str) -> List[Dict]:
    """The regrouping engine's work queues of `kernel` (static tables of the
    library): block, dispatch context (-1: the block's own queue) and the
    registers a parked thread carries, as (index, name, type)."""
    nq = ctypes.c_uint32()
    p = ctypes.POINTER(QueueLayoutC)()
    check(lib().loom_b200_kernel_queues(kernel.encode(), ctypes.byref(nq), ctypes.byref(p)))
    out = []
    for q in range(nq.value):
        c = p[q]
        cols = [(c.regs[i], c.names[i].decode(), TYPE_NAMES[c.types[i]]) for i in range(c.num_cols)]
        out.append({"queue": q, "block": c.block, "context": c.context, "cols": cols})
    return out


def group_mean(inp, out, rows: int, group: int, stream=None) -> None:
    """Per-group means of one device float column (loom_b200_group_mean):
    out[r] = mean of inp[r * group : (r + 1) * group], summed in order."""
    t = {4: F32, 8: F64}[inp.element_size()] if hasattr(inp, "element_size") else F32
    s = getattr(stream, "cuda_stream", stream)
    check(lib().loom_b200_group_mean(t, _ptr(inp), _ptr(out), rows, group, s))


def reg_caps(kernel: str) -> List[int]:
    """Register caps compiled for the kernel's megakernel, default first."""
    caps = (ctypes.c_uint32 * 16)()
    n = ctypes.c_uint32()
    check(lib().loom_b200_kernel_reg_caps(kernel.encode(), caps, 16, ctypes.byref(n)))
    return [int(caps[i]) for i in range(min(16, n.value))]


def info(kernel: str) -> KernelInfo:
    p = ctypes.POINTER(KernelInfoC)()
    check(lib().loom_b200_kernel_find(kernel.encode(), ctypes.byref(p)))
    return KernelInfo(p.contents)


def make_opts(
    mode: Union[int, str] = PLAIN,
    block_size: int = 0,
    utr_lanes: int = 0,
    period: int = 0,
    burst: int = 0,
    spread_lanes: int = 0,
    refill: bool = True,
    population: int = 0,
    max_steps: int = 0,
    profile: bool = False,
    prefetch: bool = True,
    ctas_per_sm: int = 0,
    fault_phantom_ctas: int = 0,
    barrier_spins: int = 0,
    graph: bool = False,
    cost_model: bool = False,
    schedule: int = 0,
    host_chunks: int = 0,
    max_regs: int = 0,
    plain_below: int = 0,
    defer_lanes: int = 0,
    bulk_restore: bool = False,
    spin_iters: int = 0,
    refill_lanes: int = 0,
) -> Opts:
    if isinstance(mode, str):
        mode = {"plain": PLAIN, "regroup": REGROUP}[mode]
    return Opts(
        mode=mode,
        block_size=block_size,
        utr_lanes=utr_lanes,
        period=period,
        burst=burst,
        spread_lanes=spread_lanes,
        no_refill=0 if refill else 1,
        graph=1 if graph else 0,
        population=population,
        max_steps=max_steps,
        profile=1 if profile else 0,
        no_prefetch=0 if prefetch else 1,
        ctas_per_sm=ctas_per_sm,
        fault_phantom_ctas=fault_phantom_ctas,
        barrier_spins=barrier_spins,
        cost_model=1 if cost_model else 0,
        schedule=int(schedule),
        host_chunks=int(host_chunks),
        max_regs=int(max_regs),
        plain_below=int(plain_below),
        defer_lanes=int(defer_lanes),
        bulk_restore=1 if bulk_restore else 0,
        spin_iters=int(spin_iters),
        refill_lanes=int(refill_lanes),
    )


def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(f"cannot take a pointer of {type(x)}")


class Function:
    """A kernel bound to a device, a capacity and launch options."""

    def __init__(self, kernel: str, capacity: int, mode: Union[int, str] = PLAIN, **opts):
        self.kernel = kernel
        self.info = info(kernel)
        self.capacity = int(capacity)
        o = make_opts(mode, **opts)
        h = ctypes.c_void_p()
        check(lib().loom_b200_create(kernel.encode(), self.capacity, ctypes.byref(o), ctypes.byref(h)))
        self._h = h

    # -------------------------------------------------------------- options
    def set_opts(self, mode: Union[int, str] = PLAIN, **opts) -> None:
        o = make_opts(mode, **opts)
        check(lib().loom_b200_set_opts(self._h, ctypes.byref(o)))

    def get_opts(self) -> Dict[str, int]:
        o = Opts()
        check(lib().loom_b200_get_opts(self._h, ctypes.byref(o)))
        return {f: getattr(o, f) for f, _ in Opts._fields_}

    # -------------------------------------------------------------- runs
    def __call__(self, *inputs: Optional[np.ndarray], n: Optional[int] = None):
        """Host arrays in, host arrays out (blocking).  ``None`` = iota."""
        ins = []
        for a, (_, t) in zip(inputs, self.info.inputs):
            ins.append(None if a is None else np.ascontiguousarray(a, dtype=NP_TYPE[t]))
        if len(ins) != len(self.info.inputs):
            raise ValueError(f"{self.kernel} takes {len(self.info.inputs)} input columns")
        if n is None:
            sized = [a for a in ins if a is not None]
            if not sized:
                raise ValueError("n is required when every input is iota")
            n = len(sized[0])
        outs = [np.empty(n, dtype=NP_TYPE[t]) for _, t in self.info.outputs]
        pin = (ctypes.c_void_p * max(1, len(ins)))(*[_ptr(a) for a in ins])
        pout = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        check(lib().loom_b200_run_host(self._h, pin, pout, n))
        return outs[0] if len(outs) == 1 else tuple(outs)

    def run_host_ptrs(self, inputs: Sequence, outputs: Sequence, n: int) -> None:
        """Host pointers (e.g. pinned torch tensors) in and out, blocking."""
        pin = (ctypes.c_void_p * max(1, len(inputs)))(*[_ptr(a) for a in inputs])
        pout = (ctypes.c_void_p * len(outputs))(*[_ptr(o) for o in outputs])
        check(lib().loom_b200_run_host(self._h, pin, pout, n))

    def run_device(self, inputs: Sequence, outputs: Sequence, n: int, stream=None) -> None:
        """Device columns in and out; asynchronous on `stream` (cudaStream_t
        handle or torch.cuda.Stream; None = the CUDA default stream)."""
        pin = (ctypes.c_void_p * max(1, len(inputs)))(*[_ptr(a) for a in inputs])
        pout = (ctypes.c_void_p * len(outputs))(*[_ptr(o) for o in outputs])
        s = getattr(stream, "cuda_stream", stream)
        check(lib().loom_b200_run_device(self._h, pin, pout, n, s))

    def _launch_struct(self, inputs, outputs, n, instance_starts, table):
        ins = (InputC * max(1, len(inputs)))()
        keep = []
        for i, (a, (_, t)) in enumerate(zip(inputs, self.info.inputs)):
            if a is None or a is Iota or isinstance(a, Iota):
                ins[i] = InputC(None, IN_IOTA, 0, 0)
            elif a is LocalIota or isinstance(a, LocalIota):
                ins[i] = InputC(None, IN_LOCAL_IOTA, 0, 0)
            elif a is Instance or isinstance(a, Instance):
                ins[i] = InputC(None, IN_INSTANCE, 0, 0)
            elif isinstance(a, Broadcast):
                ins[i] = InputC(None, IN_BROADCAST, 0, a.bits())
            else:
                if isinstance(a, np.ndarray):
                    a = np.ascontiguousarray(a, dtype=NP_TYPE[t])
                    keep.append(a)
                ins[i] = InputC(_ptr(a), IN_ARRAY, 0, 0)
        outs = (ctypes.c_void_p * len(outputs))(*[_ptr(o) for o in outputs])
        L = LaunchC()
        L.inputs = ins
        L.outputs = outs
        L.n = n
        L.instance_starts = _ptr(instance_starts)
        L.num_instances = 0 if instance_starts is None else len(instance_starts) - 1
        L.table = _ptr(table)
        L.table_words = 0 if table is None else len(table)
        keep += [ins, outs, instance_starts, table]
        return L, keep

    def launch_host(self, inputs, n: int, instance_starts=None, table=None):
        """General blocking launch on host arrays; inputs may be arrays or
        Iota / LocalIota / Instance / Broadcast.  Returns output arrays."""
        outs = [np.empty(n, dtype=NP_TYPE[t]) for _, t in self.info.outputs]
        if instance_starts is not None:
            instance_starts = np.ascontiguousarray(instance_starts, dtype=np.uint64)
        if table is not None:
            table = np.ascontiguousarray(table, dtype=np.uint32)
        L, keep = self._launch_struct(inputs, outs, n, instance_starts, table)
        check(lib().loom_b200_launch_host(self._h, ctypes.byref(L)))
        del keep
        return outs[0] if len(outs) == 1 else tuple(outs)

    def launch_host_mean(self, inputs, n: int, group: int = 0, instance_group=None, instance_starts=None,
                         table=None, outputs=None):
        """`launch_host` whose outputs are per-group means (loom_b200_launch_host_mean):
        one row per `group` consecutive threads, or per instance_group[i]
        threads of instance i.  `outputs` may be given (host arrays or
        pointers of the row count); returns them."""
        if instance_starts is not None:
            instance_starts = np.ascontiguousarray(instance_starts, dtype=np.uint64)
        if table is not None:
            table = np.ascontiguousarray(table, dtype=np.uint32)
        ig = None
        if instance_group is not None:
            ig = np.ascontiguousarray(instance_group, dtype=np.uint32)
            starts = np.asarray(instance_starts, dtype=np.uint64)
            rows = int(((starts[1:] - starts[:-1]) // ig).sum())
        else:
            rows = n // group if group else 0
        if outputs is None:
            outputs = [np.empty(rows, dtype=NP_TYPE[t]) for _, t in self.info.outputs]
        L, keep = self._launch_struct(inputs, outputs, n, instance_starts, table)
        M = MeanC(group, 0, None if ig is None else ig.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        check(lib().loom_b200_launch_host_mean(self._h, ctypes.byref(L), ctypes.byref(M)))
        del keep
        return outputs

    def launch_device(self, inputs, outputs, n: int, instance_starts=None, table=None, stream=None):
        """General asynchronous launch; every array is device memory (torch
        tensors or raw pointers)."""
        L, keep = self._launch_struct(inputs, outputs, n, instance_starts, table)
        s = getattr(stream, "cuda_stream", stream)
        check(lib().loom_b200_launch_device(self._h, ctypes.byref(L), s))
        del keep

    def sync(self) -> None:
        check(lib().loom_b200_sync(self._h))

    def stats(self, raise_on_device_error: bool = False) -> Dict[str, float]:
        s = StatsC()
        check(lib().loom_b200_get_stats(self._h, ctypes.byref(s)))
        d = {f: getattr(s, f) for f, _ in StatsC._fields_}
        d["lane_efficiency"] = (
            s.thread_instr / (32.0 * s.warp_instr) if s.warp_instr else float("nan")
        )
        if raise_on_device_error and s.status:
            raise LoomError(ERR_DEVICE, f"device status {s.status:#x}")
        return d

    def reset_stats(self) -> None:
        check(lib().loom_b200_reset_stats(self._h))

    def device_bytes(self) -> int:
        """Device memory the handle holds (columns, queues, control words)."""
        b = ctypes.c_uint64()
        check(lib().loom_b200_device_bytes(self._h, ctypes.byref(b)))
        return int(b.value)

    def block_stats(self) -> List[Dict[str, float]]:
        """Per basic block over the profiled launches since the last reset:
        VM instructions (thread and warp sums) and lane efficiency."""
        nb = self.info.num_blocks
        ti = (ctypes.c_uint64 * nb)()
        wi = (ctypes.c_uint64 * nb)()
        check(lib().loom_b200_get_block_stats(self._h, ti, wi, nb))
        return [
            {
                "block": b,
                "thread_instr": ti[b],
                "warp_instr": wi[b],
                "lane_efficiency": ti[b] / (32.0 * wi[b]) if wi[b] else float("nan"),
            }
            for b in range(nb)
        ]

    def parked(self, max_rows: int = 1 << 20) -> List[Dict]:
        """The threads the last regrouping launch left parked (see
        `loom_b200_parked_dump`): per non-empty queue its block, context,
        row count, thread ids (low 32 bits) and one array per live
        register, by register name."""
        qs = queues(self.kernel)
        counts = (ctypes.c_uint32 * max(1, len(qs)))()
        nq = ctypes.c_uint32()
        check(lib().loom_b200_parked_counts(self._h, counts, len(qs), ctypes.byref(nq)))
        out = []
        for q in qs:
            n = min(int(counts[q["queue"]]), max_rows)
            if n == 0:
                continue
            arrs = [np.empty(n, dtype=NP_TYPE[t]) for _, _, t in q["cols"]]
            ptrs = (ctypes.c_void_p * max(1, len(arrs)))(*[a.ctypes.data for a in arrs])
            tids = np.empty(n, dtype=np.uint32)
            got = ctypes.c_uint64()
            check(
                lib().loom_b200_parked_dump(
                    self._h,
                    q["queue"],
                    ptrs,
                    tids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                    n,
                    ctypes.byref(got),
                )
            )
            k = int(got.value)
            regs = {name: a[:k] for (_, name, _), a in zip(q["cols"], arrs)}
            out.append(dict(queue=q["queue"], block=q["block"], context=q["context"], rows=k, tid=tids[:k], regs=regs))
        return out

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().loom_b200_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Continuous batching of requests of one kernel (loom_b200_server_*).

    ``forms`` gives the form of each kernel input (array inputs come with
    every request; IOTA / LOCAL_IOTA / INSTANCE are computed on the device).
    A request may carry a table header (``header_words`` words, the
    INSTANCE form gives its slot) and a body whose table position the server
    adds to header word ``reloc_word``.
    """

    FORM = {"array": IN_ARRAY, "iota": IN_IOTA, "local_iota": IN_LOCAL_IOTA, "instance": IN_INSTANCE}

    def __init__(
        self,
        kernel: str,
        ring_threads: int,
        max_requests: int = 1024,
        slice_rounds: int = 4,
        forms: Optional[Sequence[str]] = None,
        header_words: int = 0,
        reloc_word: int = -1,
        table_words: int = 0,
        stream=None,
        budget: Optional[Budget] = None,
        **opts,
    ):
        self.info = info(kernel)
        self._h = ctypes.c_void_p()
        fs = [self.FORM[f] for f in forms] if forms else [IN_ARRAY] * len(self.info.inputs)
        self._forms = (ctypes.c_uint32 * max(1, len(fs)))(*fs)
        self.forms = fs
        self.budget = budget  # kept alive while the server points to it
        cfg = ServerCfgC(ring_threads, table_words, header_words, reloc_word, max_requests, slice_rounds, self._forms,
                         None if budget is None else ctypes.pointer(budget.c))
        o = make_opts("regroup", **opts)
        s = getattr(stream, "cuda_stream", stream)
        check(lib().loom_b200_server_create(kernel.encode(), ctypes.byref(o), ctypes.byref(cfg), s, ctypes.byref(self._h)))
        self.header_words = header_words
        self._live: Dict[int, tuple] = {}
        self._done = (ctypes.c_uint64 * max(1, max_requests))()
        self._max = max(1, max_requests)

    def submit(self, n: int, inputs: Sequence = (), outputs: Optional[Sequence] = None, header=None, body=None) -> int:
        """Queues a request of n threads; returns its ticket.  Array inputs
        and outputs are host arrays (numpy or pinned torch tensors) that
        stay referenced until the request completes; outputs default to new
        numpy arrays, returned by ``result``."""
        if outputs is None:
            outputs = [np.empty(n, dtype=NP_TYPE[t]) for _, t in self.info.outputs]
        ins = []
        it = iter(inputs)
        for f, (_, t) in zip(self.forms, self.info.inputs):
            if f == IN_ARRAY:
                a = next(it)
                if isinstance(a, np.ndarray):
                    a = np.ascontiguousarray(a, dtype=NP_TYPE[t])
                ins.append(a)
            else:
                ins.append(None)
        pin = (ctypes.c_void_p * max(1, len(ins)))(*[_ptr(a) for a in ins])
        pout = (ctypes.c_void_p * len(outputs))(*[_ptr(o) for o in outputs])
        hdr = None if header is None else np.ascontiguousarray(header, dtype=np.uint32)
        bod = None if body is None else np.ascontiguousarray(body, dtype=np.uint32)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        r = RequestC(
            n,
            pin,
            pout,
            None if hdr is None else hdr.ctypes.data_as(u32p),
            None if bod is None else bod.ctypes.data_as(u32p),
            0 if bod is None else len(bod),
        )
        t = ctypes.c_uint64()
        check(lib().loom_b200_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        self._live[t.value] = (ins, outputs, hdr, bod, pin, pout)
        return t.value

    def launch(self, ctas_per_sm: int = 0) -> None:
        """Admits and starts the next slice without waiting for it
        (loom_b200_server_launch); the next ``step`` completes it."""
        check(lib().loom_b200_server_launch(self._h, int(ctas_per_sm)))

    def step(self) -> List[int]:
        """Admits, runs one slice (or completes the one ``launch`` started),
        returns the tickets that completed."""
        k = ctypes.c_uint32()
        check(lib().loom_b200_server_step(self._h, self._done, self._max, ctypes.byref(k)))
        return [self._done[i] for i in range(k.value)]

    def result(self, ticket: int):
        """Outputs of a completed request (and forgets it)."""
        outs = self._live.pop(ticket)[1]
        return outs[0] if len(outs) == 1 else tuple(outs)

    def cancel(self, ticket: int) -> bool:
        """Cancels a request (``loom_b200_server_cancel``): a queued one at
        once, one in flight when its threads have finished.  False when the
        ticket is not pending."""
        return lib().loom_b200_server_cancel(self._h, ticket) == OK

    def set_timeout(self, seconds: float) -> None:
        """Host-side watchdog: requests not completed `seconds` after their
        submission are cancelled with ERR_TIMEOUT (0: off)."""
        check(lib().loom_b200_server_set_timeout(self._h, int(round(seconds * 1e6))))

    def failed(self) -> List[tuple]:
        """(ticket, code) of the requests cancelled or timed out since the
        last call; their arrays are released."""
        out = []
        t = (ctypes.c_uint64 * 64)()
        c = (ctypes.c_int32 * 64)()
        k = ctypes.c_uint32()
        while True:
            check(lib().loom_b200_server_failed(self._h, t, c, 64, ctypes.byref(k)))
            for i in range(k.value):
                out.append((t[i], c[i]))
                self._live.pop(t[i], None)
            if k.value < 64:
                return out

    def stats(self) -> Dict[str, int]:
        st = ServerStatsC()
        check(lib().loom_b200_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStatsC._fields_ if f != "pad"}

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().loom_b200_server_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

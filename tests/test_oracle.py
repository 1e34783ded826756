"""The oracle pinned against Loom's own scalar backend (CPU only).

tests/golden/*.npz hold outputs of vm::bse::function<K> compiled from the Loom
headers (tests/golden/make_golden.py); the C restatement of bse must
reproduce every one of them bit for bit, and the numpy restatements of Loom's
validators (src/tests/programs.hpp:290-389) must agree with both.
"""

import pathlib

import numpy as np
import pytest

from loom_b200.codegen import ir
from oracle import oracle as O

KERNELS = ir.available()


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


# Loom's own path tracers run up to 64 adaptive samples per pixel: the C
# restatement checks a seeded subset of their 1600 pixels to stay fast.
SUBSET = {"pt_const_40": 160, "pt2_const_40": 160, "pt_const_512": 160, "pt2_const_512": 160,
          "primary_const_256": 160, "primary_const_b20_256": 160}


@pytest.mark.parametrize("name", KERNELS)
def test_interp_matches_golden(name, golden, golden_extra):
    ins, outs = golden(name)
    if name in SUBSET:
        idx = np.sort(O.uniform_int(3, SUBSET[name], 0, len(ins[0]) - 1).astype(np.int64))
        ins = [a[idx] for a in ins]
        outs = [a[idx] for a in outs]
    got = O.Interp(name).run(ins, table=golden_extra(name).get("table"))
    assert len(got) == len(outs)
    for g, o in zip(got, outs):
        assert np.array_equal(_bits(g), _bits(o)), name


def test_golden_fixture_for_every_kernel():
    d = pathlib.Path(__file__).parent / "golden"
    # macro_kat.npz holds known answers beside the macro kernels' fixtures
    assert {p.stem for p in d.glob("*.npz")} - {"macro_kat"} == set(KERNELS)


def test_val_fib_matches_golden(golden):
    (n,), (c,) = golden("fib_u64")
    assert np.array_equal(O.val_fib(n), c)
    # Loom README.md:113-128 example values
    assert int(O.val_fib(np.array([90], dtype=np.uint64))[0]) == 2880067194370816120


def test_val_collatz_matches_golden(golden):
    (n,), (s,) = golden("collatz_u64")
    assert np.array_equal(O.val_collatz(n), s)
    known = {1: 0, 2: 1, 3: 7, 6: 8, 7: 16, 27: 111, 97: 118, 837799: 524}
    for k, v in known.items():
        assert int(O.val_collatz(np.array([k], dtype=np.uint64))[0]) == v


def test_val_fac_and_jmp4(golden):
    (a,), (r,) = golden("fac_u64")
    assert np.array_equal(O.val_fac(a), r)
    (i,), (j,) = golden("jmp4_u64")
    assert np.array_equal(O.val_jmp4(i), j)


def _logical(f):
    return lambda *a: f(*[np.asarray(x) != 0 for x in a]).astype(np.asarray(a[0]).dtype)


# the validator of each Loom test program, as Loom's test pairs them
# (src/tests/vm.cpp:277-327: val_* of programs.hpp:290-389 and std functors)
VALIDATORS = {
    "increment": O.val_inc,
    "union_cmov": O.val_union2,
    "union": O.val_union1,
    "bit_and": np.bitwise_and,
    "bit_or": np.bitwise_or,
    "bit_xor": np.bitwise_xor,
    "bit_not": O.val_bit_not,
    "bool_and": _logical(np.logical_and),
    "bool_or": _logical(np.logical_or),
    "bool_not": _logical(np.logical_not),
    "lshift": O.val_lshift,
    "rshift": O.val_rshift,
}


@pytest.mark.parametrize(
    "name", [k for k in KERNELS if any(k.startswith(p + "_") for p in VALIDATORS)]
)
def test_loom_validators_match_golden(name, golden):
    """Loom's own validators agree with bse's outputs in every fixture of
    the test programs they cover."""
    prefix = next(p for p in VALIDATORS if name.startswith(p + "_"))
    ins, (out,) = golden(name)
    want = VALIDATORS[prefix](*ins)
    assert want.dtype == out.dtype, (want.dtype, out.dtype)
    assert np.array_equal(want, out), name


def test_interp_out_of_table_parmjump_halts():
    # jmp4: values outside the 4-entry table leave the thread unchanged,
    # like bse's switch without a matching case (bse.hpp:192-198)
    i = np.array([0, 1, 2, 3, 4, 9, 200], dtype=np.uint32)
    (o,) = O.Interp("jmp4_f32").run([i])
    assert o.tolist() == [1, 3, 7, 11, 4, 9, 200]


def test_interp_step_limit():
    # fib of 2^64 - 1 loops while i <= n, i.e. forever: the guard must end it
    with pytest.raises(RuntimeError):
        O.Interp("fib_u64").run([np.array([2**64 - 1], dtype=np.uint64)], max_steps=1000)


def test_interp_instruction_counts():
    # fib(n) for n >= 2: START (3) + work (4) + (n - 1) loop iterations (6)
    n = np.array([0, 1, 2, 10], dtype=np.uint64)
    (_,), cnt = O.Interp("fib_u64").run([n], count_instr=True)
    assert cnt.tolist() == [3, 3, 3 + 4 + 6, 3 + 4 + 6 * 9]


@pytest.mark.skipif(not O.ref_available(), reason="Loom bse runner not built here")
def test_interp_matches_loom_bse_fresh_inputs():
    import kernel_domains as D

    for name in ["fib_u64", "collatz_u64", "arithmetic_f32", "union_cmov_f64", "slt_inv_u32"]:
        k = ir.load(name)
        ins = D.inputs_for(name, 3000, 99, [t for _, t, _ in k.inputs])
        a = O.Interp(name).run(ins)
        b = O.ref_run(name, ins, 3000, threads=2)
        for x, y in zip(a, b):
            assert np.array_equal(_bits(x), _bits(y)), name


def test_splitmix_stream_is_fixed():
    # SplitMix64 reference values for seed 0 (Steele et al. 2014)
    z = O.splitmix64(0, 3)
    assert z.tolist() == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_workload_inputs_match_the_oracle_stream():
    """The bench's input generator (loom_b200.inputs) and the oracle's give
    the same arrays, so both sides of every parity check read equal inputs."""
    from loom_b200 import inputs as I

    for seed, n, lo, hi in ((1, 1000, 1, (1 << 32) - 1), (5, 777, 0, 93), (9, 100, 3, (1 << 63) + 5)):
        assert np.array_equal(I.uniform_int(seed, n, lo, hi), O.uniform_int(seed, n, lo, hi))


RNG_KERNELS = {"rotl32_u32": 1, "threefry_u32": 2, "canonical_f32": 1, "bump_u32": 2}
LINAL_KERNELS = {"cross_f32": 3, "norm_f32": 3}


def _kat():
    return np.load(pathlib.Path(__file__).resolve().parent / "golden" / "macro_kat.npz")


@pytest.mark.parametrize("name", sorted(RNG_KERNELS))
def test_rng_macros_match_loom_cpp_functions(name, golden):
    """The RNG macros of the path tracers (one kernel each) give the known
    answers of Loom's plain C++ functions (src/common/random.hpp: rotl32,
    threefry2x32r32<0xdead, 0xbeef>, gen_canonical, bump_ctr) on the
    fixture's inputs, exactly, in Loom's scalar backend (the golden outputs)
    and in the C restatement; tests/golden/make_macro_kat.py wrote the
    answers."""
    kat = _kat()
    ins, outs = golden(name)
    got = O.Interp(name).run(ins)
    for j in range(RNG_KERNELS[name]):
        want = kat[f"{name}_out{j}"]
        assert np.array_equal(np.ascontiguousarray(outs[j]).view(np.uint32), want), f"{name} golden out{j}"
        assert np.array_equal(np.ascontiguousarray(got[j]).view(np.uint32), want), f"{name} interp out{j}"


def almost_equal(a: np.ndarray, b: np.ndarray, ulp: int) -> np.ndarray:
    """Loom's loom::almost_equal (src/common/math.hpp:252-274) in float32:
    |a - b| <= epsilon * |a + b| * ulp, or |a - b| below the smallest normal
    float.  Differences and sums are rounded to float32 as in the C++."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        amb = np.abs(a - b)
        apb = np.abs(a + b)
        eps = np.finfo(np.float32).eps
        bound = (eps * apb).astype(np.float32) * np.float32(ulp)
        return (amb <= bound) | (amb < np.finfo(np.float32).tiny)


@pytest.mark.parametrize("name", sorted(LINAL_KERNELS))
def test_vector_macros_match_loom_cpp_functions(name, golden):
    """The vector macros of the sphere path tracer (vec3_cross, vec3_norm)
    against Loom's C++ cross and normalize (src/common/linal.hpp) with the
    check of Loom's own test: every component almost_equal at ulp = 30, for
    at least 99 % of the inputs (src/tests/vm_linal.cpp:77, 100-156: a fuzzy
    test with a 1 % failure allowance over ulp_cmp).  The two round differently (the
    macro multiplies by a reciprocal square root), so the bound, not bit
    equality, is the check; bse and the C restatement agree exactly."""
    kat = _kat()
    ins, outs = golden(name)
    got = O.Interp(name).run(ins)
    ok = np.ones(len(ins[0]), dtype=bool)
    for j in range(LINAL_KERNELS[name]):
        want = kat[f"{name}_out{j}"].view(np.float32)
        ok &= almost_equal(outs[j], want, 30)
        assert np.array_equal(np.ascontiguousarray(got[j]).view(np.uint32), np.ascontiguousarray(outs[j]).view(np.uint32))
    assert ok.mean() >= 0.99, f"{name}: {ok.mean():.4f} almost_equal at ulp 30"


def test_almost_equal_restatement():
    one = np.float32(1.0)
    up = lambda x, k: np.float32(x) + np.float32(k) * np.spacing(np.float32(x))  # noqa: E731
    # 1.0 and 1.0 + 30 ulp: |a-b| = 30 eps <= eps * (2 + 30 eps) * 30
    assert almost_equal(np.array([one]), np.array([up(1.0, 30)]), 30)[0]
    assert not almost_equal(np.array([one]), np.array([up(1.0, 61)]), 30)[0]
    # tiny values of opposite sign: their difference is below the smallest
    # normal float, so Loom's check passes although the bit patterns are far apart
    tiny = np.nextafter(np.float32(0.0), np.float32(1.0))
    assert almost_equal(np.array([-tiny]), np.array([tiny]), 30)[0]
    assert not almost_equal(np.array([np.float32(-1.0)]), np.array([one]), 30)[0]

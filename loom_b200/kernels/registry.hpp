// -*- C++ -*-
/// @file registry.hpp
/// @brief The Loom kernels compiled into libloom_b200.
///
/// LOOM_B200_KERNELS(X) expands X(name, type) once per kernel.  The same list
/// drives the IR extractor (kernel type -> text IR -> CUDA) and the scalar
/// oracle runner, so every kernel name means the same program on both sides.
///
/// The reference's own test programs (Loom src/tests/programs.hpp) are
/// included unchanged: they are the kernels Loom's backends are tested on
/// (src/tests/vm.cpp:266-328, src/tests/vm.cu:76-86); so are its path-tracing
/// kernels (src/smallpt/vm/pt.hpp), at the configurations of its published
/// benchmarks (src/benchmarks/pt.cpp:30-35).
#pragma once

#include <smallpt/vm/pt.hpp>
#include <tests/programs.hpp>

#include "collatz.hpp"
#include "linal_tests.hpp"
#include "rng_tests.hpp"
#include "sphere_pt.hpp"

#include <cstdint>

namespace loom::vm::b200::kernels
{
using std::int16_t;
using std::int32_t;
using std::int64_t;
using std::int8_t;
using std::uint16_t;
using std::uint32_t;
using std::uint64_t;
using std::uint8_t;
} // namespace loom::vm::b200::kernels

// clang-format off
#define LOOM_B200_KERNELS(X)                                                   \
    /* workloads */                                                            \
    X(fib_u64,            fib_test<std::uint64_t>)                             \
    X(fib_u32,            fib_test<std::uint32_t>)                             \
    X(collatz_u64,        loom::vm::b200::kernels::collatz<std::uint64_t>)     \
    X(sphere_pt_f32,      loom::vm::b200::kernels::sphere_pt<float>)           \
    /* Loom's own path tracers (src/smallpt/vm/pt.hpp:1259-1729) at the  */    \
    /* 40x40 configurations of its published benchmark results: 64      */    \
    /* samples, blur 1, depth 2, threshold 1e-4 (v1) and 1e-3 (v2)       */    \
    X(pt_const_40,        loom::vm::pt_const<float, loom::vm::constants<CS(40), CS(0.0001), CS(64), CS(1), CS(2)>>) \
    X(pt2_const_40,       loom::vm::pt2_const<float, loom::vm::constants<CS(40), CS(0.001), CS(64), CS(1), CS(2)>>) \
    /* the same programs at 512x512 pixels, enough threads to fill a GPU */    \
    X(pt_const_512,       loom::vm::pt_const<float, loom::vm::constants<CS(512), CS(0.0001), CS(64), CS(1), CS(2)>>) \
    X(pt2_const_512,      loom::vm::pt2_const<float, loom::vm::constants<CS(512), CS(0.001), CS(64), CS(1), CS(2)>>) \
    /* Loom's primary-ray tracer (pt.hpp:1369-1420) at the configuration */    \
    /* of its benchmark (src/benchmarks/primary.cpp:33): 256x256 pixels, */    \
    /* 64 samples per pixel, blur 1 and 20 (CMakeLists.txt:420)          */    \
    X(primary_const_256,  loom::vm::primary_const<float, loom::vm::constants<CS(256), CS(0.1), CS(64), CS(1)>>) \
    X(primary_const_b20_256, loom::vm::primary_const<float, loom::vm::constants<CS(256), CS(0.1), CS(64), CS(20)>>) \
    /* the path tracers' RNG macros, one kernel each (rng_tests.hpp)   */    \
    X(rotl32_u32,         loom::vm::b200::kernels::rotl32_k)                   \
    X(threefry_u32,       loom::vm::b200::kernels::threefry_k)                 \
    X(canonical_f32,      loom::vm::b200::kernels::canonical_k<float>)         \
    X(bump_u32,           loom::vm::b200::kernels::bump_k)                     \
    /* and its vector macros (linal_tests.hpp)                         */    \
    X(cross_f32,          loom::vm::b200::kernels::cross_k<float>)             \
    X(norm_f32,           loom::vm::b200::kernels::norm_k<float>)              \
    /* Loom test programs (src/tests/programs.hpp) */                          \
    X(increment_i32,      increment<std::int32_t>)                             \
    X(increment_u8,       increment<std::uint8_t>)                             \
    X(increment_i16,      increment<std::int16_t>)                             \
    X(increment_u64,      increment<std::uint64_t>)                            \
    X(fac_u32,            fac_test<std::uint32_t>)                             \
    X(fac_u64,            fac_test<std::uint64_t>)                             \
    X(union_f32,          union_test<float>)                                   \
    X(union_f64,          union_test<double>)                                  \
    X(union_cmov_f32,     union_cmov_test<float>)                              \
    X(union_cmov_f64,     union_cmov_test<double>)                             \
    X(jmp4_f32,           jmp4_test<float>)                                    \
    X(jmp4_u64,           jmp4_test<std::uint64_t>)                            \
    X(jmp4_u16,           jmp4_test<std::uint16_t>)                            \
    X(bit_and_u32,        bit_and_test<std::uint32_t>)                         \
    X(bit_or_u64,         bit_or_test<std::uint64_t>)                          \
    X(bit_xor_u16,        bit_xor_test<std::uint16_t>)                         \
    X(bit_not_u8,         bit_not_test<std::uint8_t>)                          \
    X(bit_not_u32,        bit_not_test<std::uint32_t>)                         \
    X(bool_and_u32,       bool_and_test<std::uint32_t>)                        \
    X(bool_or_u64,        bool_or_test<std::uint64_t>)                         \
    X(bool_not_u8,        bool_not_test<std::uint8_t>)                         \
    X(lshift_u16,         lshift_test<std::uint16_t>)                          \
    X(lshift_u32,         lshift_test<std::uint32_t>)                          \
    X(lshift_u64,         lshift_test<std::uint64_t>)                          \
    X(rshift_u16,         rshift_test<std::uint16_t>)                          \
    X(rshift_u32,         rshift_test<std::uint32_t>)                          \
    X(rshift_u64,         rshift_test<std::uint64_t>)                          \
    X(abs_f32,            abs_test<float>)                                     \
    X(trunc_f32,          trunc_test<float>)                                   \
    X(ceilfloor_f32,      ceilfloor<float>)                                    \
    X(minmax_f32,         minmax_test<float>)                                  \
    X(minmax_f64,         minmax_test<double>)                                 \
    X(arithmetic_f32,     arithmetic_test<float>)                              \
    X(arithmetic_f64,     arithmetic_test<double>)                             \
    X(sin_cos_f32,        sin_cos_test<float>)                                 \
    X(sqrt_f32,           sqrt_test<float>)                                    \
    X(rsqrt_f32,          rsqrt_test<float>)                                   \
    X(sct_inv_u32,        sct_inv_test<std::uint32_t>)                         \
    X(slt_inv_u32,        slt_inv_test<std::uint32_t>)
// clang-format on

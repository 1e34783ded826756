// -*- C++ -*-
/// @file rng_tests.hpp
/// @brief The random-number macros of Loom's path tracers as kernels of
/// their own, so that each is pinned against Loom's plain C++ version.
///
/// Loom tests its RNG macros the same way (src/tests/vm_smallpt.cpp:38-54,
/// 326-378): one kernel per macro, run on the scalar backend and compared
/// with the C++ function of src/common/random.hpp.  These kernels call the
/// same macros (src/vm/lib/random.hpp) with the same arguments, so the
/// device code the path tracers run is checked piece by piece:
///
///   rotl32_u32      vm::rotl32          vs loom::rotl32          (random.hpp:32)
///   threefry_u32    vm::threefry2x32r32 vs threefry2x32r32<k0,k1> (random.hpp:62-80),
///                   keys 0xdead, 0xbeef, k2 = 0x1bd11bda ^ k0 ^ k1
///   canonical_f32   vm::gen_canonical   vs loom::gen_canonical   (random.hpp:87)
///   bump_u32        vm::bump_ctr        vs loom::bump_ctr        (random.hpp:95)
#pragma once

#include <vm/core.hpp>
#include <vm/lib/random.hpp>
#include <vm/macros.hpp>
#include <vm/operators.hpp>

#include <concepts>
#include <cstdint>

namespace loom::vm::b200::kernels
{
inline constexpr std::uint32_t kThreefryK0 = 0xdead;
inline constexpr std::uint32_t kThreefryK1 = 0xbeef;
inline constexpr std::uint32_t kThreefryK2 = 0x1bd11bda ^ kThreefryK0 ^ kThreefryK1;
static_assert(kThreefryK2 == 0x1bd17b98);

// clang-format off
KERNEL(rotl32_k, VAR(std::uint32_t, x), VAR(std::uint32_t, n))
    INSERT_MACRO(vm::rotl32, CS(x), CS(n), CS(dst), CS(tmp))
KERNEL_END(VAR(std::uint32_t, dst));

KERNEL(threefry_k, VAR(std::uint32_t, c0), VAR(std::uint32_t, c1))
    INSERT_MACRO(vm::threefry2x32r32, CS(c0), CS(c1), CS(0xdead), CS(0xbeef), CS(0x1bd17b98), CS(tmp1), CS(tmp2))
KERNEL_END(VAR(std::uint32_t, c0), VAR(std::uint32_t, c1));

template <std::floating_point T>
KERNEL(canonical_k, VAR(std::uint32_t, x))
    INSERT_TMACRO(vm::gen_canonical, CS(x))
TKERNEL_END1(x);

KERNEL(bump_k, VAR(std::uint32_t, c0), VAR(std::uint32_t, c1), VAR(std::uint32_t, i))
    INSERT_MACRO(vm::bump_ctr, CS(c0), CS(c1), CS(i), CS(tmp1), CS(tmp2), CS(tmp3))
KERNEL_END(VAR(std::uint32_t, c0), VAR(std::uint32_t, c1));
// clang-format on
} // namespace loom::vm::b200::kernels

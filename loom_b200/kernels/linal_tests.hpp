// -*- C++ -*-
/// @file linal_tests.hpp
/// @brief The vector macros of the sphere path tracer as kernels of their
/// own, so that each is checked against Loom's plain C++ version.
///
/// Loom tests its linear-algebra macros this way (src/tests/vm_linal.cpp:
/// 25-57, 82-156): one kernel per macro on the scalar backend against the
/// C++ functions of src/common/linal.hpp, within 30 ulp for at least 99 % of
/// the inputs (the macro and the C++ function round differently: the macro
/// normalises with a reciprocal square root, the function divides by the
/// length).  These kernels call the same macros (src/vm/lib/linal.hpp):
///
///   cross_f32   vm::vec3_cross   vs loom::cross      (linal.hpp:1430)
///   norm_f32    vm::vec3_norm    vs loom::normalize  (linal.hpp:1461)
#pragma once

#include <vm/core.hpp>
#include <vm/lib/linal.hpp>
#include <vm/macros.hpp>
#include <vm/operators.hpp>

#include <concepts>

namespace loom::vm::b200::kernels
{
// clang-format off
template <std::floating_point T>
TKERNEL6(cross_k, x0, x1, x2, y0, y1, y2)
    INSERT_TMACRO(vm::vec3_cross, CS(z), CS(x), CS(y), CS(t1))
TKERNEL_END3(z0, z1, z2);

template <std::floating_point T>
TKERNEL3(norm_k, v0, v1, v2)
    INSERT_TMACRO(vm::vec3_norm, CS(v), CS(l))
TKERNEL_END3(v0, v1, v2);
// clang-format on
} // namespace loom::vm::b200::kernels

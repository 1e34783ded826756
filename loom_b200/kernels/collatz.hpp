// -*- C++ -*-
/// @file collatz.hpp
/// @brief Collatz stopping time written in the Loom kernel language.
///
/// Loom ships no Collatz kernel; this one follows the description of the
/// divergent-loop benchmark: input n (u64, n >= 1), loop
/// n = (n even) ? n >> 1 : 3n + 1 until n == 1, output the number of steps as
/// u32.  The loop body is branch-free (cmov), so threads differ only in their
/// trip count: the divergence that PC regrouping targets.
///
/// Prettified IR:
///   %kernel collatz n:u64
///       mov @u32 steps 0
///       le  @u64 cmp n 1
///       jmp cmp 0: loop 1: HALT
///   loop:
///       band @u64 odd n 1
///       rshift @u64 half n 1
///       mul @u64 up n 3
///       add @u64 up up 1
///       cmov @u64 n odd up half
///       add @u32 steps steps 1
///       ne  @u64 cmp n 1
///       jmp cmp 0: HALT 1: loop
///   %endkernel steps:u32
#pragma once

#include <vm/core.hpp>
#include <vm/macros.hpp>
#include <vm/operators.hpp>

#include <concepts>
#include <cstdint>

namespace loom::vm::b200::kernels
{
// clang-format off
template <std::unsigned_integral T, typename S = std::uint32_t>
KERNEL(collatz, TVAR(n))
    MOV(VAR(S, steps), VAR(S, 0)),
    TLE(cmp, n, 1),
    IPJMP2(cmp, loop, HALT),
    LABEL(loop),
    IBAND(odd, n, 1),
    IRSHFT(half, n, 1),
    TMUL(up, n, 3),
    TADD(up, up, 1),
    TCMOV(n, odd, up, half),
    ADD(S, steps, steps, 1),
    TNEQ(cmp, n, 1),
    IPJMP2(cmp, HALT, loop)
KERNEL_END(VAR(S, steps));
// clang-format on
} // namespace loom::vm::b200::kernels

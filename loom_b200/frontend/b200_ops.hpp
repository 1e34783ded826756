// -*- C++ -*-
/// @file b200_ops.hpp
/// @brief Loom language extension used by the B200 kernels: a read-only
/// table lookup op.
///
/// Loom has no load instruction: a kernel is a pure function of its inputs
/// (Loom README.md:103-107).  Per-instance data such as a scene (sphere
/// positions, materials, camera, resolution) therefore has to come from
/// somewhere that is constant for the whole launch.  `ops::tab<T>` is a pure
/// Compute functor (Loom src/vm/core.hpp:74-82 accepts any invocable): it maps
/// a u32 word index to the 32-bit word stored there, read as T.  The table is
/// bound per launch: the scalar backend reads it through a thread-local
/// pointer set by the caller (`bind_table`), the B200 engines lower the op to
/// a read-only global load of the table handed to the launch.
#pragma once

#include <vm/core.hpp>
#include <vm/macros.hpp>

#include <concepts>
#include <cstdint>
#include <cstring>

namespace loom::vm::b200
{
/// Table the scalar backend reads for ops::tab in this host thread.
inline thread_local const std::uint32_t* g_table_words = nullptr;

/// Binds `words` as the table of the Loom kernels run by this host thread.
inline void
bind_table(const std::uint32_t* words) noexcept
{
    g_table_words = words;
}

namespace ops
{
/// @brief Read-only table lookup: word `idx` of the launch's table as T.
template <typename T>
    requires(sizeof(T) == 4 && std::is_trivially_copyable_v<T>)
struct tab
{
    T
    operator()(const std::uint32_t idx) const noexcept
    {
        T v;
        std::memcpy(&v, g_table_words + idx, sizeof(T));
        return v;
    }
};
} // namespace ops
} // namespace loom::vm::b200

// clang-format off
/// dst (float) <- table word idx read as float
#define TABF_CS(DST, IDX) \
    loom::vm::Compute<loom::vm::b200::ops::tab<float>, VAR_CS(float, DST), VAR_CS(std::uint32_t, IDX)>
#define TABF(DST, IDX) TABF_CS(CS(DST), CS(IDX))
/// dst (u32) <- table word idx
#define TABU_CS(DST, IDX) \
    loom::vm::Compute<loom::vm::b200::ops::tab<std::uint32_t>, VAR_CS(std::uint32_t, DST), VAR_CS(std::uint32_t, IDX)>
#define TABU(DST, IDX) TABU_CS(CS(DST), CS(IDX))
// clang-format on

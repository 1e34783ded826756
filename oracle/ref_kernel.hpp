// Loom's own scalar backend, vm::bse::function<K> (Loom src/vm/bse.hpp:616-649),
// over a slice of threads: the part of the reference runner that is compiled
// once per registry kernel (oracle/build_ref.py).
//
// TEST AND BASELINE INFRASTRUCTURE ONLY (see ref_runner.cpp).
#pragma once

#include <vm/bse.hpp>

#include "../loom_b200/kernels/registry.hpp"

#include <cstdint>
#include <cstring>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace loom_ref
{
template <typename T>
struct is_tuple : std::false_type
{
};
template <typename... Ts>
struct is_tuple<std::tuple<Ts...>> : std::true_type
{
};

template <typename K, std::size_t I>
using in_t = loom::vm::vartype<loom::typelist::at<I, typename K::input_vars>>;
template <typename K, std::size_t O>
using out_t = loom::vm::vartype<loom::typelist::at<O, typename K::output_vars>>;

template <typename K, std::size_t I>
in_t<K, I>
input(const void* const* in, std::uint64_t t)
{
    using T = in_t<K, I>;
    return in[I] ? static_cast<const T*>(in[I])[t] : static_cast<T>(t);
}

template <typename K, std::size_t... I, std::size_t... O>
void
run_slice(const void* const*   in,
          void* const*         out,
          std::uint64_t        b,
          std::uint64_t        e,
          const std::uint32_t* table,
          std::index_sequence<I...>,
          std::index_sequence<O...>)
{
    loom::vm::b200::bind_table(table); // the tab extension of this thread
    loom::vm::bse::function<K> f;
    for(std::uint64_t t = b; t < e; ++t)
    {
        const auto r = f(input<K, I>(in, t)...);
        if constexpr(is_tuple<std::remove_cvref_t<decltype(r)>>::value)
            ((static_cast<out_t<K, O>*>(out[O])[t] = std::get<O>(r)), ...);
        else
            static_cast<out_t<K, 0>*>(out[0])[t] = r;
    }
}

template <typename K>
void
run_kernel(const void* const*   in,
           void* const*         out,
           std::uint64_t        n,
           int                  threads,
           const std::uint32_t* table)
{
    constexpr std::size_t ni = loom::typelist::length<typename K::input_vars>;
    constexpr std::size_t no = loom::typelist::length<typename K::output_vars>;
    if(threads < 1) threads = 1;
    if(static_cast<std::uint64_t>(threads) > n) threads = n ? static_cast<int>(n) : 1;
    std::vector<std::thread> pool;
    const std::uint64_t      chunk = (n + threads - 1) / threads;
    for(int w = 0; w < threads; ++w)
    {
        const std::uint64_t b = w * chunk;
        const std::uint64_t e = b + chunk < n ? b + chunk : n;
        if(b >= e) break;
        pool.emplace_back(
            [=]()
            {
                run_slice<K>(in,
                             out,
                             b,
                             e,
                             table,
                             std::make_index_sequence<ni>{},
                             std::make_index_sequence<no>{});
            });
    }
    for(auto& t: pool) t.join();
}
} // namespace loom_ref


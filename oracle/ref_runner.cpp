// Runner around Loom's own scalar backend, vm::bse::function<K>
// (Loom src/vm/bse.hpp:616-649), for every kernel of the B200 registry.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  Compiled from the Loom headers
// where they lie (oracle/build_ref.py); the resulting oracle/_ref/
// libloomref.so is the checker for golden fixtures and the timed CPU
// reference arm of bench.py.  Nothing in the product links it.
//
// C ABI:
//   int loom_ref_run(const char* kernel, const void* const* inputs,
//                    void* const* outputs, uint64_t n, int threads,
//                    const uint32_t* table)
// runs bse on threads [0, n) split into `threads` contiguous slices (one
// std::thread each, as Loom's demo spreads pixels over cores,
// src/smallpt/vm/vm.cpp:66-70).  A NULL input column means "iota".
#include <vm/bse.hpp>

#include "../loom_b200/kernels/registry.hpp"

#include <cstdint>
#include <cstring>
#include <thread>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace
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
} // namespace

extern "C" int
loom_ref_run(const char*          kernel,
             const void* const*   inputs,
             void* const*         outputs,
             std::uint64_t        n,
             int                  threads,
             const std::uint32_t* table)
{
#define LOOM_REF_CASE(NAME, ...)                                         \
    if(std::strcmp(kernel, #NAME) == 0)                                  \
    {                                                                    \
        run_kernel<__VA_ARGS__>(inputs, outputs, n, threads, table);     \
        return 0;                                                        \
    }
    LOOM_B200_KERNELS(LOOM_REF_CASE)
#undef LOOM_REF_CASE
    return -2;
}

extern "C" int
loom_ref_has(const char* kernel)
{
#define LOOM_REF_HAS(NAME, ...) \
    if(std::strcmp(kernel, #NAME) == 0) return 1;
    LOOM_B200_KERNELS(LOOM_REF_HAS)
#undef LOOM_REF_HAS
    return 0;
}

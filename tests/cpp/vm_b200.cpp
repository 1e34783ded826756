// B200 form of Loom's CUDA backend test (Loom src/tests/vm.cu:43-88): the
// same kernel types, input distributions and validation functions
// (src/tests/programs.hpp:292-387), run through the C++ front end
// (include/loom_b200.hpp) in both engines and through the stream protocol.
//
// Loom's harness (common/test.hpp) needs range-v3 and {fmt}, which are not
// part of the Loom sources, so this program carries a small harness of its
// own with the same shape: a column of random inputs per test, the kernel
// run once over the column, the outputs compared with the scalar validation
// function element by element (in input order; Loom sorts both sides first
// because its streams return outputs permuted, which this front end does
// not).  Built by tests/cpp/build_vm_test.py, run by
// tests/test_cpp_frontend.py.
#include <loom_b200.hpp>

#include <tests/programs.hpp>

#include <bit>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <utility>
#include <vector>

using namespace loom;
using namespace vm;

using incr_int     = increment<int>;
using fac_unsigned = fac_test<unsigned>;
using sut          = union_test<float>;
using cut          = union_cmov_test<float>;
using jmp4_float   = jmp4_test<float>;
using lshift_u     = lshift_test<unsigned>;
using rshift_u     = rshift_test<unsigned>;

namespace
{
struct Track
{
    int passed = 0, failed = 0;

    void
    check(bool ok, const std::string& name)
    {
        std::printf("%s %s\n", ok ? "PASS" : "FAIL", name.c_str());
        ++(ok ? passed : failed);
    }

    int
    ret_code() const
    {
        std::printf("%d passed, %d failed\n", passed, failed);
        return failed ? 1 : 0;
    }
};

/// Equality that treats NaN as equal to NaN bit patterns alike (the union
/// tests move raw float bits).
template <typename T>
bool
same(const T& a, const T& b)
{
    if constexpr(std::is_floating_point_v<T>)
        return std::bit_cast<std::conditional_t<sizeof(T) == 4, std::uint32_t, std::uint64_t>>(a)
            == std::bit_cast<std::conditional_t<sizeof(T) == 4, std::uint32_t, std::uint64_t>>(b);
    else
        return a == b;
}

/// One column per generator component; `call` maps the columns to outputs.
template <typename G, typename Call, typename Val>
bool
run_case(std::size_t n, G& g, Call&& call, Val&& val)
{
    using sample = decltype(g());
    std::vector<sample> in(n);
    for(auto& x: in) x = g();
    if constexpr(requires(sample s) { s.first; })
    {
        std::vector<decltype(in[0].first)>  a(n);
        std::vector<decltype(in[0].second)> b(n);
        for(std::size_t i = 0; i < n; ++i) std::tie(a[i], b[i]) = in[i];
        const auto out = call(a, b);
        if(out.size() != n) return false;
        for(std::size_t i = 0; i < n; ++i)
            if(!same(out[i], static_cast<std::remove_cvref_t<decltype(out[i])>>(val(a[i], b[i]))))
                return false;
        return true;
    }
    else
    {
        const auto out = call(in);
        if(out.size() != n) return false;
        for(std::size_t i = 0; i < n; ++i)
            if(!same(out[i], static_cast<std::remove_cvref_t<decltype(out[i])>>(val(in[i]))))
                return false;
        return true;
    }
}

/// Loom's StreamWrapper (src/tests/stream_wrapper.hpp:33-78) in plain
/// loops: set_inputs, step, exchange until the input is used up, step until
/// done, collect the rest.
template <typename S, typename In>
auto
drive_stream(S& s, const In& input)
{
    std::vector<output_type<typename S::program>> out;
    auto step = [&]() { s(); s.sort(); };
    auto it = s.set_inputs(input);
    step();
    while(it != input.end())
    {
        const auto exs = s.exchange(std::ranges::subrange(it, input.end()));
        it += exs.size();
        for(const auto& e: exs) out.push_back(std::get<0>(e));
        step();
    }
    while(!s.done()) step();
    for(const auto& e: s.get_output_zipped()) out.push_back(std::get<0>(e));
    return out;
}
} // namespace

int
main(int argc, char* argv[])
{
    unsigned nr = 1000, seed = 0;
    for(int i = 1; i < argc; ++i)
    {
        const std::string flag = argv[i];
        if(flag == "--bind-only")
        {
            // binds every kernel type to its compiled code (no GPU needed)
            for(const auto* info: {b200::detail::lookup<incr_int>(),
                                   b200::detail::lookup<fac_unsigned>(),
                                   b200::detail::lookup<sut>(),
                                   b200::detail::lookup<cut>(),
                                   b200::detail::lookup<jmp4_float>(),
                                   b200::detail::lookup<lshift_u>(),
                                   b200::detail::lookup<rshift_u>()})
                std::printf("%s %s\n", info->name, info->ir_digest);
            return 0;
        }
        if(i + 1 >= argc) break;
        if(flag == "-n" || flag == "--numruns") nr = std::strtoul(argv[++i], nullptr, 10);
        else if(flag == "-s" || flag == "--seed") seed = std::strtoul(argv[++i], nullptr, 10);
    }
    Track          track;
    const unsigned vector_size = std::bit_floor(nr);
    const unsigned stream_size = vector_size >> 1;
    std::mt19937   rng{seed};

    std::uniform_int_distribution<int>      d_int(2, 10);
    std::uniform_int_distribution<unsigned> d_ui(0, 10), d_u3(0, 3);
    auto g_int   = [&]() { return d_int(rng); };
    auto g_ui    = [&]() { return d_ui(rng); };
    auto g_u3    = [&]() { return d_u3(rng); };
    auto g_float = [&]() { return std::generate_canonical<float, 10>(rng); };
    auto g_shift = [&]() { return std::pair(g_ui(), g_ui()); };

    auto test_function = [&]<Kernel K>(K, auto& g, auto val, const char* name)
    {
        b200::function<K> plain(vector_size);
        track.check(run_case(vector_size, g, [&](const auto&... c) { return plain(c...); }, val),
                    std::string("B200 plain ") + name);
        b200::hybrid_function<K> regroup(vector_size);
        track.check(run_case(vector_size, g, [&](const auto&... c) { return regroup(c...); }, val),
                    std::string("B200 regroup ") + name);
    };

    auto test_stream = [&]<Kernel K>(K, auto& g, auto val, const char* name)
    {
        b200::stream<K> stream(stream_size);
        track.check(run_case(vector_size, g, [&](const auto& in) { return drive_stream(stream, in); }, val),
                    std::string("B200 ") + name);
    };

    test_function(incr_int{}, g_int, ::val_inc, "increment int");
    test_function(fac_unsigned{}, g_ui, ::val_fac, "factorial unsigned");
    test_function(sut{}, g_float, ::val_union1, "simple union");
    test_function(cut{}, g_float, ::val_union2, "complex union");
    test_function(jmp4_float{}, g_u3, ::val_jmp4, "jump4");
    test_function(lshift_u{}, g_shift, ::val_lshift, "left shift");
    test_function(rshift_u{}, g_shift, ::val_rshift, "right shift");
    test_stream(fac_unsigned{}, g_ui, ::val_fac, "stream factorial unsigned");

    return track.ret_code();
}

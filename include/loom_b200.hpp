// -*- C++ -*-
/// @file loom_b200.hpp
/// @brief C++ front end of the B200 backend: Loom's backend call shapes on
/// top of the C ABI (loom_b200.h).
///
/// Loom picks a backend by template alias and every backend offers the same
/// shapes (Loom src/vm/cuda.hpp:1581-1586, src/vm/simd.hpp:4294-4335):
///
///   vm::cuda::function<K> f(n);  auto out = f(inputs...);
///   vm::cuda::stream<K>   s(n);  set_inputs / operator() / sort / exchange /
///                                done / get_output_zipped
///
/// This header gives the same shapes for B200:
///
///   loom::vm::b200::function<K>         plain engine (one CUDA thread per
///                                       Loom thread, hardware reconvergence)
///   loom::vm::b200::hybrid_function<K>  regrouping engine (persistent
///                                       megakernel, warps re-formed by PC)
///   loom::vm::b200::stream<K>           the stream protocol over the
///                                       regrouping engine
///
/// A kernel type is bound to its compiled code by the structural digest of
/// its IR (ir_emit.hpp), so `K` must be one of the kernels compiled into
/// libloom_b200 (loom_b200/kernels/registry.hpp); otherwise construction
/// aborts with a message, as Loom's own ASSERT does.  Like Loom's backends
/// the calls are noexcept: a failing CUDA call or a device status bit aborts
/// with the library's message (use `run` for a status code instead).
///
/// Include paths: this directory, loom_b200/frontend and Loom's src and
/// ext/include; link libloom_b200.so.
#pragma once

#include <vm/core.hpp>

#include "ir_emit.hpp"
#include "loom_b200.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iterator>
#include <ranges>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace loom::vm::b200
{
namespace detail
{
template <typename T>
constexpr int
type_code() noexcept
{
    if constexpr(std::is_same_v<T, bool>) return LOOM_B200_B8;
    else if constexpr(std::is_floating_point_v<T>)
        return sizeof(T) == 4 ? LOOM_B200_F32 : LOOM_B200_F64;
    else if constexpr(std::is_signed_v<T>)
        return sizeof(T) == 1 ? LOOM_B200_I8
             : sizeof(T) == 2 ? LOOM_B200_I16
             : sizeof(T) == 4 ? LOOM_B200_I32
                              : LOOM_B200_I64;
    else
        return sizeof(T) == 1 ? LOOM_B200_U8
             : sizeof(T) == 2 ? LOOM_B200_U16
             : sizeof(T) == 4 ? LOOM_B200_U32
                              : LOOM_B200_U64;
}

[[noreturn]] inline void
fail(const char* what, int code) noexcept
{
    std::fprintf(stderr,
                 "loom_b200: %s: %s (%d)\n",
                 what,
                 loom_b200_error_string(code),
                 code);
    std::abort();
}

template <typename T>
struct is_tuple : std::false_type
{
};
template <typename... Ts>
struct is_tuple<std::tuple<Ts...>> : std::true_type
{
};

template <Kernel K, std::size_t I>
using in_t = vartype<typelist::at<I, typename K::input_vars>>;
template <Kernel K, std::size_t O>
using out_t = vartype<typelist::at<O, typename K::output_vars>>;

template <Kernel K>
inline constexpr std::size_t num_in = typelist::length<typename K::input_vars>;
template <Kernel K>
inline constexpr std::size_t num_out = typelist::length<typename K::output_vars>;

/// The compiled kernel whose IR matches K (looked up once per type).
template <Kernel K>
const loom_b200_kernel_info*
lookup() noexcept
{
    static const loom_b200_kernel_info* info = []() noexcept
    {
        const std::string                  d = ir::digest<K>();
        const loom_b200_kernel_info*       p = nullptr;
        const int rc = loom_b200_kernel_find_digest(d.c_str(), &p);
        if(rc != LOOM_B200_OK)
        {
            std::fprintf(stderr,
                         "loom_b200: kernel %.*s (IR digest %s) is not compiled into "
                         "libloom_b200\n",
                         static_cast<int>(K::nameview.size()),
                         K::nameview.data(),
                         d.c_str());
            std::abort();
        }
        // the signature must agree with the type, column by column
        bool ok = p->num_inputs == num_in<K> && p->num_outputs == num_out<K>;
        [&]<std::size_t... I, std::size_t... O>(std::index_sequence<I...>,
                                                std::index_sequence<O...>) noexcept
        {
            ok = ok && ((p->input_types[I] == type_code<in_t<K, I>>()) && ...);
            ok = ok && ((p->output_types[O] == type_code<out_t<K, O>>()) && ...);
        }(std::make_index_sequence<num_in<K>>{}, std::make_index_sequence<num_out<K>>{});
        if(!ok)
        {
            std::fprintf(stderr, "loom_b200: column types of %s disagree\n", p->name);
            std::abort();
        }
        return p;
    }();
    return info;
}

/// One input argument: a range (its elements, one per thread) or a single
/// value (broadcast to every thread), as Loom's cuda::MemoryFacade accepts
/// (src/vm/cuda.hpp:1094-1131).
template <typename T, typename Arg>
struct input_column
{
    std::vector<T>  data;
    loom_b200_input spec{};

    input_column(const Arg& a, std::size_t n) noexcept
    {
        if constexpr(std::ranges::input_range<Arg>)
        {
            data.reserve(n);
            for(auto it = std::ranges::begin(a);
                it != std::ranges::end(a) && data.size() < n;
                ++it)
                data.push_back(static_cast<T>(*it));
            data.resize(n);
            spec.ptr  = data.data();
            spec.form = LOOM_B200_IN_ARRAY;
        }
        else
        {
            const T v = static_cast<T>(a);
            std::uint64_t bits = 0;
            std::memcpy(&bits, &v, sizeof(T));
            spec.form  = LOOM_B200_IN_BROADCAST;
            spec.value = bits;
        }
    }
};
} // namespace detail

/// @brief A Loom kernel on B200 with a fixed capacity, in the plain or the
/// regrouping form.
template <Kernel K, unsigned Mode>
class basic_function
{
    loom_b200_handle*            h_ = nullptr;
    std::size_t                  n_ = 0;
    const loom_b200_kernel_info* info_;

    template <std::size_t O>
    using out_t = detail::out_t<K, O>;

  public:
    using program = K;

    explicit basic_function(std::size_t n, loom_b200_opts opts = {}) noexcept :
        n_(n), info_(detail::lookup<K>())
    {
        opts.mode    = Mode;
        const int rc = loom_b200_create(info_->name, n, &opts, &h_);
        if(rc != LOOM_B200_OK) detail::fail("create", rc);
    }

    basic_function(const basic_function&)            = delete;
    basic_function& operator=(const basic_function&) = delete;

    ~basic_function() { loom_b200_destroy(h_); }

    std::size_t
    size() const noexcept
    {
        return n_;
    }

    loom_b200_handle*
    handle() const noexcept
    {
        return h_;
    }

    /// Runs the kernel on `n` threads (default: the capacity).  Each argument
    /// is a range (one element per thread) or a value for every thread.
    /// Returns the output columns, in input order: one std::vector per
    /// output variable, a tuple of them when there are several (like
    /// cuda::MemoryFacade::get_outputs, src/vm/cuda.hpp:1133-1148).
    template <typename... Args>
        requires(sizeof...(Args) == detail::num_in<K>)
    auto
    operator()(const Args&... args) noexcept
    {
        auto out    = make_outputs(n_);
        const int rc = run(out, n_, args...);
        if(rc != LOOM_B200_OK) detail::fail("run", rc);
        if constexpr(detail::num_out<K> == 1)
            return std::move(std::get<0>(out));
        else
            return out;
    }

    auto
    make_outputs(std::size_t n) const
    {
        return [&]<std::size_t... O>(std::index_sequence<O...>)
        {
            return std::tuple<std::vector<out_t<O>>...>(std::vector<out_t<O>>(n)...);
        }(std::make_index_sequence<detail::num_out<K>>{});
    }

    /// Status-code variant of operator(): fills `out` (from make_outputs).
    template <typename Out, typename... Args>
    int
    run(Out& out, std::size_t n, const Args&... args) noexcept
    {
        if(n > n_) return LOOM_B200_ERR_INVALID;
        return [&]<std::size_t... I, std::size_t... O>(std::index_sequence<I...>,
                                                       std::index_sequence<O...>)
        {
            std::tuple<detail::input_column<detail::in_t<K, I>, Args>...> cols(
                detail::input_column<detail::in_t<K, I>, Args>(args, n)...);
            loom_b200_input ins[detail::num_in<K> + 1] = {std::get<I>(cols).spec...};
            void*           outs[] = {static_cast<void*>(std::get<O>(out).data())...};
            loom_b200_launch L{};
            L.inputs  = ins;
            L.outputs = outs;
            L.n       = n;
            return loom_b200_launch_host(h_, &L);
        }(std::make_index_sequence<detail::num_in<K>>{},
                 std::make_index_sequence<detail::num_out<K>>{});
    }

    loom_b200_stats
    stats() noexcept
    {
        loom_b200_stats s{};
        loom_b200_get_stats(h_, &s);
        return s;
    }
};

/// Plain engine: vm::cuda::function<K>(n) on B200.
template <Kernel K>
using function = basic_function<K, LOOM_B200_PLAIN>;

/// Regrouping engine: the B200 form of vm::simd::hybrid_function<K>.
template <Kernel K>
using hybrid_function = basic_function<K, LOOM_B200_REGROUP>;

/// @brief Loom's stream protocol (src/vm/bve.hpp:1105-1270,
/// src/vm/cuda.hpp:1468-1578) over the regrouping engine.
///
/// set_inputs takes up to `n` inputs; operator() runs them to completion on
/// the device (regrouping and the exchange of halted threads for new inputs
/// happen inside the megakernel, so sort() has nothing left to do);
/// exchange(range) returns as many finished outputs as it takes new inputs;
/// get_output_zipped returns the rest once done().  Outputs come back in
/// input order (Loom's streams return them permuted).
template <Kernel K>
class stream
{
    using in_tuple  = typelist::to<input_types<K>, std::tuple>;
    using out_tuple = typelist::to<output_types<K>, std::tuple>;

    hybrid_function<K>    f_;
    std::vector<in_tuple> loaded_;   // inputs waiting for operator()
    std::deque<out_tuple> finished_; // outputs not handed out yet

    template <typename Elem>
    static in_tuple
    as_tuple(const Elem& e) noexcept
    {
        if constexpr(detail::is_tuple<Elem>::value)
            return in_tuple(e);
        else
            return in_tuple(e);
    }

    template <typename It, typename End>
    It
    load(It it, End end, std::size_t k) noexcept
    {
        for(; it != end && k > 0; ++it, --k) loaded_.push_back(as_tuple(*it));
        return it;
    }

  public:
    using program = K;

    explicit stream(std::size_t n, loom_b200_opts opts = {}) noexcept : f_(n, opts) {}

    template <std::ranges::input_range Input>
    auto
    set_inputs(Input&& input) noexcept
    {
        loaded_.clear();
        return load(std::ranges::begin(input), std::ranges::end(input), f_.size());
    }

    void
    operator()() noexcept
    {
        const std::size_t n = loaded_.size();
        if(n == 0) return;
        auto out = f_.make_outputs(n);
        const int rc = [&]<std::size_t... I>(std::index_sequence<I...>)
        {
            std::tuple<std::vector<detail::in_t<K, I>>...> cols;
            ((std::get<I>(cols).reserve(n)), ...);
            for(const auto& t: loaded_) ((std::get<I>(cols).push_back(std::get<I>(t))), ...);
            return f_.run(out, n, std::get<I>(cols)...);
        }(std::make_index_sequence<detail::num_in<K>>{});
        if(rc != LOOM_B200_OK) detail::fail("stream", rc);
        for(std::size_t i = 0; i < n; ++i)
            finished_.push_back([&]<std::size_t... O>(std::index_sequence<O...>)
                                { return out_tuple(std::get<O>(out)[i]...); }(
                                    std::make_index_sequence<detail::num_out<K>>{}));
        loaded_.clear();
    }

    bool
    sort() noexcept
    {
        return true;
    }

    bool
    done() const noexcept
    {
        return loaded_.empty();
    }

    /// Takes up to as many new inputs as there are finished outputs and
    /// returns that many outputs.
    template <std::ranges::input_range Input>
    auto
    exchange(Input&& input) noexcept
    {
        const std::size_t room = std::min(finished_.size(), f_.size() - loaded_.size());
        const std::size_t before = loaded_.size();
        load(std::ranges::begin(input), std::ranges::end(input), room);
        const std::size_t k = loaded_.size() - before;
        std::vector<out_tuple> ret(finished_.begin(), finished_.begin() + k);
        finished_.erase(finished_.begin(), finished_.begin() + k);
        return ret;
    }

    auto
    get_output_zipped() noexcept
    {
        std::vector<out_tuple> ret(finished_.begin(), finished_.end());
        finished_.clear();
        return ret;
    }
};
} // namespace loom::vm::b200

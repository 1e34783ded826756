// Minimal stand-in for the fast_float library's from_chars interface.
//
// Loom's common/string.hpp includes <fast_float/fast_float.h> only for its
// run-time number reader (read_number_fn), which the kernel IR never calls:
// IR literals go through Loom's own constexpr parser (s2n).  This header
// forwards fast_float::from_chars to std::from_chars so that the Loom headers
// compile with g++ and libstdc++ without the third-party dependency.
#pragma once

#include <charconv>
#include <system_error>

namespace fast_float
{
enum class chars_format
{
    scientific = 1,
    fixed      = 2,
    hex        = 4,
    general    = 3
};

template <typename T>
struct from_chars_result_t
{
    const char* ptr;
    std::errc   ec;
};

template <typename T>
    requires std::is_integral_v<T>
from_chars_result_t<T>
from_chars(const char* first, const char* last, T& value, int base = 10) noexcept
{
    auto r = std::from_chars(first, last, value, base);
    return {r.ptr, r.ec};
}

template <typename T>
    requires std::is_floating_point_v<T>
from_chars_result_t<T>
from_chars(const char*  first,
           const char*  last,
           T&           value,
           chars_format fmt = chars_format::general) noexcept
{
    std::chars_format f = std::chars_format::general;
    switch(fmt)
    {
    case chars_format::scientific: f = std::chars_format::scientific; break;
    case chars_format::fixed: f = std::chars_format::fixed; break;
    case chars_format::hex: f = std::chars_format::hex; break;
    default: break;
    }
    auto r = std::from_chars(first, last, value, f);
    return {r.ptr, r.ec};
}
} // namespace fast_float

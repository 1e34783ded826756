// Loom's plain C++ functions behind the path tracers' VM macros, over raw
// input columns: the random-number functions of src/common/random.hpp and
// the vector functions of src/common/linal.hpp.  They are the known answers
// the macro kernels' golden outputs are checked against, as Loom's own
// tests compare them (src/tests/vm_smallpt.cpp:349-378,
// src/tests/vm_linal.cpp:82-156).  Built and run by make_macro_kat.py; not
// part of the product.
//
//   macro_kat <function> <n>  reads the kernel's input columns from stdin
//   (n little-endian 32-bit words each, one column after the other) and
//   writes its output columns to stdout the same way.
#include <common/functional.hpp>
#include <common/linal.hpp>
#include <common/random.hpp>

#include <array>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace
{
std::vector<std::uint32_t>
read_column(std::size_t n)
{
    std::vector<std::uint32_t> v(n);
    if(std::fread(v.data(), sizeof(std::uint32_t), n, stdin) != n) v.clear();
    return v;
}

void
write_column(const std::vector<std::uint32_t>& v)
{
    std::fwrite(v.data(), sizeof(std::uint32_t), v.size(), stdout);
}
} // namespace

int
main(int argc, char** argv)
{
    if(argc != 3) return 2;
    const std::string  fn = argv[1];
    const std::size_t  n  = std::stoull(argv[2]);
    if(fn == "rotl32")
    {
        const auto x = read_column(n), k = read_column(n);
        if(x.size() != n || k.size() != n) return 3;
        std::vector<std::uint32_t> d(n);
        for(std::size_t i = 0; i < n; ++i) d[i] = loom::rotl32(x[i], k[i]);
        write_column(d);
    }
    else if(fn == "threefry")
    {
        const auto a = read_column(n), b = read_column(n);
        if(a.size() != n || b.size() != n) return 3;
        std::vector<std::uint32_t> c0(n), c1(n);
        for(std::size_t i = 0; i < n; ++i)
        {
            const auto r = loom::threefry2x32r32<0xdead, 0xbeef>(std::array<std::uint32_t, 2>{a[i], b[i]});
            c0[i]        = r[0];
            c1[i]        = r[1];
        }
        write_column(c0);
        write_column(c1);
    }
    else if(fn == "canonical")
    {
        const auto x = read_column(n);
        if(x.size() != n) return 3;
        std::vector<std::uint32_t> d(n);
        for(std::size_t i = 0; i < n; ++i)
        {
            const float f = loom::gen_canonical(x[i]);
            std::memcpy(&d[i], &f, sizeof f);
        }
        write_column(d);
    }
    else if(fn == "bump")
    {
        const auto a = read_column(n), b = read_column(n), k = read_column(n);
        if(a.size() != n || b.size() != n || k.size() != n) return 3;
        std::vector<std::uint32_t> c0(n), c1(n);
        for(std::size_t i = 0; i < n; ++i)
        {
            const auto r = loom::bump_ctr(std::array<std::uint32_t, 2>{a[i], b[i]}, k[i]);
            c0[i]        = r[0];
            c1[i]        = r[1];
        }
        write_column(c0);
        write_column(c1);
    }
    else if(fn == "cross" || fn == "norm")
    {
        using Vec3f      = loom::Vector<float, 3, std::array>;
        const int    nin = fn == "cross" ? 6 : 3;
        std::vector<std::vector<float>> in(nin);
        for(auto& c: in)
        {
            const auto w = read_column(n);
            if(w.size() != n) return 3;
            c.resize(n);
            std::memcpy(c.data(), w.data(), n * sizeof(float));
        }
        std::vector<std::uint32_t> o[3];
        for(auto& c: o) c.resize(n);
        for(std::size_t i = 0; i < n; ++i)
        {
            const Vec3f a{in[0][i], in[1][i], in[2][i]};
            const Vec3f r = fn == "cross" ? Vec3f(loom::cross(a, Vec3f{in[3][i], in[4][i], in[5][i]}))
                                          : Vec3f(loom::normalize(a));
            for(int j = 0; j < 3; ++j)
            {
                const float f = r[j];
                std::memcpy(&o[j][i], &f, sizeof f);
            }
        }
        for(const auto& c: o) write_column(c);
    }
    else
        return 2;
    return 0;
}

// Runner around Loom's own scalar backend, vm::bse::function<K>
// (Loom src/vm/bse.hpp:616-649), for every kernel of the B200 registry.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY.  Compiled from the Loom headers
// where they lie (oracle/build_ref.py); the resulting oracle/_ref/
// libloomref.so writes the golden fixtures, checks results in the tests and
// is the timed CPU reference arm of bench.py.  Nothing in the product links
// it.
//
// C ABI:
//   int loom_ref_run(const char* kernel, const void* const* inputs,
//                    void* const* outputs, uint64_t n, int threads,
//                    const uint32_t* table)
// runs bse on threads [0, n) split into `threads` contiguous slices (one
// std::thread each, as Loom's demo spreads pixels over cores,
// src/smallpt/vm/vm.cpp:66-70).  A NULL input column means "iota".
//
// This file is the dispatcher; each kernel's bse instantiation lives in its
// own object (ref_kernel.hpp, one generated translation unit per kernel),
// so the large kernels compile in parallel.
#include "../loom_b200/kernels/registry.hpp"

#include <cstdint>
#include <cstring>

#define LOOM_REF_DECL(NAME, ...)                                                     \
    extern "C" int loom_ref_run_##NAME(const void* const*, void* const*, std::uint64_t, \
                                       int, const std::uint32_t*);
LOOM_B200_KERNELS(LOOM_REF_DECL)
#undef LOOM_REF_DECL

extern "C" int
loom_ref_run(const char*          kernel,
             const void* const*   inputs,
             void* const*         outputs,
             std::uint64_t        n,
             int                  threads,
             const std::uint32_t* table)
{
#define LOOM_REF_CASE(NAME, ...)                                                   \
    if(std::strcmp(kernel, #NAME) == 0)                                            \
        return loom_ref_run_##NAME(inputs, outputs, n, threads, table);
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

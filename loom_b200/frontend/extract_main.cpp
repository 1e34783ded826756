// IR extractor: writes <outdir>/<name>.lir for every kernel of the registry.
//
// Built and run on a machine that has the Loom headers (LOOM_REF_DIR); the
// resulting .lir files are the only input the CUDA code generator needs.
#include "ir_emit.hpp"

#include "../kernels/registry.hpp"

#include <cstdio>
#include <fstream>
#include <string>

int
main(int argc, char* argv[])
{
    if(argc < 2)
    {
        std::fprintf(stderr, "usage: %s <outdir> [name...]\n", argv[0]);
        return 2;
    }
    const std::string outdir = argv[1];
    auto wanted = [&](const char* name)
    {
        if(argc == 2) return true;
        for(int i = 2; i < argc; ++i)
            if(std::string(argv[i]) == name) return true;
        return false;
    };
    int n = 0;
#define LOOM_B200_EMIT(NAME, ...)                                        \
    if(wanted(#NAME))                                                    \
    {                                                                    \
        std::ofstream f(outdir + "/" #NAME ".lir");                      \
        f << loom::vm::b200::ir::emit<__VA_ARGS__>(#NAME);               \
        if(!f) return 1;                                                 \
        ++n;                                                             \
    }
    LOOM_B200_KERNELS(LOOM_B200_EMIT)
#undef LOOM_B200_EMIT
    std::printf("wrote %d kernel IR files to %s\n", n, outdir.c_str());
    return 0;
}

// `rrgsim <work_dir> [--resume <iteration>]`: the solver executable
// (solver/app/src/rrgsim.cu:12-62); --resume continues from dump/S_{iteration:>5d}.bin.
// Device and arithmetic come from the environment: RRGSIM_DEVICE (default 0) and
// RRGSIM_PRECISION = fp32 (default) | mixed | fp64.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "rrg.h"

int main(int argc, const char** argv) {
    bool resume = false;
    unsigned long long resume_iter = 0;
    if (argc == 4 && !std::strcmp(argv[2], "--resume")) {
        char* end = nullptr;
        resume_iter = std::strtoull(argv[3], &end, 10);
        resume = end && *end == '\0' && argv[3][0] != '\0';
    }
    if (argc < 2 || (argc > 2 && !resume)) {
        std::fprintf(stderr, "usage: rrgsim <work_dir> [--resume <iteration>]\n");
        return 1;
    }
    int device = 0;
    if (const char* d = std::getenv("RRGSIM_DEVICE")) device = std::atoi(d);
    int precision = RRG_PREC_FP32;
    if (const char* p = std::getenv("RRGSIM_PRECISION")) {
        if (!std::strcmp(p, "mixed")) precision = RRG_PREC_MIXED;
        else if (!std::strcmp(p, "fp64")) precision = RRG_PREC_FP64;
        else if (std::strcmp(p, "fp32") != 0) {
            std::fprintf(stderr, "RRGSIM_PRECISION must be fp32, mixed or fp64\n");
            return 1;
        }
    }
    const rrg_status s = resume ? rrg_run_resume(argv[1], resume_iter, device, precision)
                                : rrg_run(argv[1], device, precision);
    if (s != RRG_OK) {
        std::fprintf(stderr, "rrgsim: %s\n", rrg_last_error(nullptr));
        return 1;
    }
    return 0;
}

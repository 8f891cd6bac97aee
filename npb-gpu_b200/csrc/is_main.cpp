// is_main.cpp -- `is`, a drop-in for the reference benchmark binary is.<CLASS>
// (GMAP/NPB-GPU CUDA/IS/is.cu main, :335-505) on top of libcgb's C ABI.
//
//   is S|W|A|B|C|D          an NPB class (is.cu:86-140)
//   options: --device D  --json (one JSON result line instead of the report)
//
// Like the reference it runs one untimed ranking pass, times the ten ranking
// passes with their partial checks, then checks the full sort; verification
// needs all 5 x 10 partial checks and the full check (is.cu:477) and Mop/s is
// 10 x the keys over the time (is.cu:484).  The time is the device time of
// the ten passes.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/cgb.h"

namespace {

struct IsClass {
    char name;
    int total_log2, max_log2;
};

const IsClass kClasses[] = {{'S', 16, 11}, {'W', 20, 16}, {'A', 23, 19}, {'B', 25, 21}, {'C', 27, 23}, {'D', 31, 27}};

constexpr int kIterations = 10;
constexpr long long kPassed = 5 * kIterations + 1;

void usage() { std::fprintf(stderr, "usage: is S|W|A|B|C|D [--device D] [--json]\n"); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        usage();
        return 2;
    }
    const IsClass *P = nullptr;
    for (const auto &c : kClasses)
        if (argv[1][0] == c.name && argv[1][1] == '\0') P = &c;
    if (!P) {
        usage();
        return 2;
    }
    int device = 0, json = 0;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--json") json = 1;
        else {
            usage();
            return 2;
        }
    }
    cgb_is *s = nullptr;
    long long passed = 0;
    double ms = 0.0;
    int st = cgb_is_create(device, P->name, P->total_log2, P->max_log2, &s);
    if (!st) st = cgb_is_run(s, &passed, &ms);
    if (s) cgb_is_destroy(s);
    if (st) {
        std::fprintf(stderr, "is: run failed: %s (%s)\n", cgb_status_string(st), cgb_last_error());
        return 1;
    }
    const bool ok = passed == kPassed;
    const double keys = double(1LL << P->total_log2), t = ms / 1e3;
    const double mops = t > 0 ? kIterations * keys / t / 1e6 : 0.0;
    if (json) {
        std::printf("{\"class\": \"%c\", \"keys\": %.0f, \"max_key\": %lld, \"passed\": %lld, \"seconds\": %.9g, "
                    "\"mops\": %.6g, \"verified\": %s}\n",
                    P->name, keys, 1LL << P->max_log2, passed, t, mops, ok ? "true" : "false");
        return ok ? 0 : 1;
    }
    std::printf("\n\n NAS Parallel Benchmarks 4.1 - IS Benchmark (B200 sm_100a build)\n\n");
    std::printf(" Size:  %.0f  (class %c)\n", keys, P->name);
    std::printf(" Iterations:   %d\n", kIterations);
    std::printf("\n\n IS Benchmark Completed\n");
    std::printf(" class_npb       =                        %c\n", P->name);
    std::printf(" Size            =             %12.0f\n", keys);
    std::printf(" Iterations      =             %12d\n", kIterations);
    std::printf(" Time in seconds =             %12.6f\n", t);
    std::printf(" Mop/s total     =             %12.2f\n", mops);
    std::printf(" Operation type  = %24s\n", "keys ranked");
    std::printf(" Verification    =             %12s\n", ok ? "SUCCESSFUL" : "UNSUCCESSFUL");
    std::printf(" Checks passed   =             %12lld of %lld\n", passed, kPassed);
    return ok ? 0 : 1;
}

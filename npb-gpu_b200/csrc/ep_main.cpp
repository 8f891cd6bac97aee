// ep_main.cpp -- `ep`, a drop-in for the reference benchmark binary ep.<CLASS>
// (GMAP/NPB-GPU CUDA/EP/ep.cu main, :114-275) on top of libcgb's C ABI.
//
//   ep S|W|A|B|C|D|E        an NPB class (setparams.cpp:826-845: m = 24 .. 40)
//   options: --device D  --json (one JSON result line instead of the report)
//
// Like the reference it reports the number of pairs accepted, the two sums
// and the ten annulus counts, verifies the sums at relative 1e-8
// (ep.cu:189-218) and reports Mop/s as 2^(m+1) random numbers over the
// time (ep.cu:219); the time is the kernel's device time.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/cgb.h"

namespace {

struct EpClass {
    char name;
    int m;
    double sx, sy;
};

// ep.cu:189-212
const EpClass kClasses[] = {
    {'S', 24, -3.247834652034740e+3, -6.958407078382297e+3},
    {'W', 25, -2.863319731645753e+3, -6.320053679109499e+3},
    {'A', 28, -4.295875165629892e+3, -1.580732573678431e+4},
    {'B', 30, 4.033815542441498e+4, -2.660669192809235e+4},
    {'C', 32, 4.764367927995374e+4, -8.084072988043731e+4},
    {'D', 36, 1.982481200946593e+5, -1.020596636361769e+5},
    {'E', 40, -5.319717441530e+05, -3.688834557731e+05},
};

void usage() { std::fprintf(stderr, "usage: ep S|W|A|B|C|D|E [--device D] [--json]\n"); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        usage();
        return 2;
    }
    const EpClass *P = nullptr;
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
    double sx = 0.0, sy = 0.0, q[10] = {}, ms = 0.0;
    const int st = cgb_ep_run(device, P->m, &sx, &sy, q, &ms);
    if (st) {
        std::fprintf(stderr, "ep: run failed: %s (%s)\n", cgb_status_string(st), cgb_last_error());
        return 1;
    }
    double gc = 0.0;
    for (double c : q) gc += c;
    const double t = ms / 1e3;
    const double sx_err = std::fabs((sx - P->sx) / P->sx), sy_err = std::fabs((sy - P->sy) / P->sy);
    const bool ok = sx_err <= 1.0e-8 && sy_err <= 1.0e-8;
    const double mops = t > 0 ? std::pow(2.0, P->m + 1) / t / 1e6 : 0.0;
    if (json) {
        std::printf("{\"class\": \"%c\", \"m\": %d, \"sx\": %.17g, \"sy\": %.17g, \"pairs\": %.0f, "
                    "\"seconds\": %.9g, \"mops\": %.6g, \"verified\": %s, \"sx_err\": %.6g, \"sy_err\": %.6g}\n",
                    P->name, P->m, sx, sy, gc, t, mops, ok ? "true" : "false", sx_err, sy_err);
        return ok ? 0 : 1;
    }
    std::printf("\n\n NAS Parallel Benchmarks 4.1 - EP Benchmark (B200 sm_100a build)\n\n");
    std::printf(" Number of random numbers generated: %15.0f\n", std::pow(2.0, P->m + 1));
    std::printf("\n EP Benchmark Results:\n\n");
    std::printf(" CPU Time =%10.4f\n", t);
    std::printf(" N = 2^%5d\n", P->m);
    std::printf(" No. Gaussian Pairs = %15.0f\n", gc);
    std::printf(" Sums = %25.15e %25.15e\n", sx, sy);
    std::printf(" Counts: \n");
    for (int i = 0; i < 10; i++) std::printf("%3d%15.0f\n", i, q[i]);
    std::printf("\n\n EP Benchmark Completed\n");
    std::printf(" class_npb       =                        %c\n", P->name);
    std::printf(" Size            =             %12.0f\n", std::pow(2.0, P->m + 1));
    std::printf(" Time in seconds =             %12.6f\n", t);
    std::printf(" Mop/s total     =             %12.2f\n", mops);
    std::printf(" Operation type  = %24s\n", "Random numbers generated");
    std::printf(" Verification    =             %12s\n", ok ? "SUCCESSFUL" : "UNSUCCESSFUL");
    return ok ? 0 : 1;
}

// mg_main.cpp -- `mg`, a drop-in for the reference benchmark binary mg.<CLASS>
// (GMAP/NPB-GPU CUDA/MG/mg.cu main, :356-623) on top of libcgb's C ABI.
//
//   mg S|W|A|B|C|D        an NPB class (setparams.cpp:697-731 parameters)
//   options: --nit I (another iteration count: no verification)
//            --device D  --json (one JSON result line instead of the report)
//
// Like the reference it builds the grids and the right-hand side (zran3),
// runs one untimed pass of the timed region (the reference runs one
// untimed iteration, mg.cu:465-479), then the timed region (mg.cu:486-517)
// from u = 0, verifies the final residual norm against the class's value at
// relative 1e-8 (mg.cu:526-552), and reports time and Mop/s with the
// reference's operation count, 58 nit n^3 (mg.cu:554-559).  The time is the
// device time of the timed region.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/cgb.h"

namespace {

struct MgClass {
    char name;
    int lt, nit, smoother;
    double verify;
};

// NPB MG classes (setparams.cpp:697-731) and verification norms (mg.cu:528-543)
const MgClass kClasses[] = {
    {'S', 5, 4, 0, 0.5307707005734e-04},  {'W', 7, 4, 0, 0.6467329375339e-05},
    {'A', 8, 4, 0, 0.2433365309069e-05},  {'B', 8, 20, 1, 0.1800564401355e-05},
    {'C', 9, 20, 1, 0.5706732285740e-06}, {'D', 10, 50, 1, 0.1583275060440e-09},
};

int fail(int st, const char *what)
{
    std::fprintf(stderr, "mg: %s failed: %s (%s)\n", what, cgb_status_string(st), cgb_last_error());
    return 1;
}

void usage() { std::fprintf(stderr, "usage: mg S|W|A|B|C|D [--nit I] [--device D] [--json]\n"); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        usage();
        return 2;
    }
    const MgClass *P = nullptr;
    for (const auto &c : kClasses)
        if (argv[1][0] == c.name && argv[1][1] == '\0') P = &c;
    if (!P) {
        usage();
        return 2;
    }
    int nit = P->nit, device = 0, json = 0;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        if ((a == "--nit" || a == "--device") && i + 1 < argc) {
            const int v = std::atoi(argv[++i]);
            (a == "--nit" ? nit : device) = v;
        } else if (a == "--json") {
            json = 1;
        } else {
            usage();
            return 2;
        }
    }
    if (nit < 1) {
        usage();
        return 2;
    }
    const bool verify = nit == P->nit;  // another count has no reference value
    cgb_mg *g = nullptr;
    int st = cgb_mg_create(device, P->lt, P->smoother, &g);
    if (st) return fail(st, "create");
    double rnm2 = 0.0, rnmu = 0.0, ms = 0.0;
    st = cgb_mg_run(g, nit, nullptr, nullptr, nullptr);  // untimed pass
    if (!st) st = cgb_mg_run(g, nit, &rnm2, &rnmu, &ms);
    cgb_mg_destroy(g);
    if (st) return fail(st, "run");

    const int n = 1 << P->lt;
    const double t = ms / 1e3, nn = double(n) * n * n;
    const double mops = t > 0 ? 58.0 * nit * nn * 1e-6 / t : 0.0;
    const double err = std::fabs(rnm2 - P->verify) / P->verify;
    const bool ok = verify && err <= 1.0e-8;
    if (json) {
        std::printf("{\"class\": \"%c\", \"n\": %d, \"nit\": %d, \"rnm2\": %.17g, \"rnmu\": %.17g, "
                    "\"seconds\": %.9g, \"mops\": %.6g, \"verified\": %s, \"rel_err\": %.6g}\n",
                    P->name, n, nit, rnm2, rnmu, t, mops, verify ? (ok ? "true" : "false") : "null",
                    verify ? err : -1.0);
        return verify && !ok ? 1 : 0;
    }
    std::printf("\n\n NAS Parallel Benchmarks 4.1 - MG Benchmark (B200 sm_100a build)\n\n");
    std::printf(" Size: %3dx%3dx%3d (class_npb %1c)\n", n, n, n, P->name);
    std::printf(" Iterations: %3d\n", nit);
    std::printf(" Benchmark completed\n");
    if (!verify) {
        std::printf(" Problem size unknown\n");
        std::printf(" NO VERIFICATION PERFORMED\n");
    } else if (ok) {
        std::printf(" VERIFICATION SUCCESSFUL\n");
        std::printf(" L2 Norm is %20.13e\n", rnm2);
        std::printf(" Error is   %20.13e\n", err);
    } else {
        std::printf(" VERIFICATION FAILED\n");
        std::printf(" L2 Norm is             %20.13e\n", rnm2);
        std::printf(" The correct L2 Norm is %20.13e\n", P->verify);
    }
    std::printf("\n\n MG Benchmark Completed\n");
    std::printf(" class_npb       =                        %c\n", P->name);
    std::printf(" Size            =             %4dx%4dx%4d\n", n, n, n);
    std::printf(" Iterations      =             %12d\n", nit);
    std::printf(" Time in seconds =             %12.6f\n", t);
    std::printf(" Mop/s total     =             %12.2f\n", mops);
    std::printf(" Operation type  = %24s\n", "floating point");
    std::printf(" Verification    =             %12s\n",
                !verify ? "NOT PERFORMED" : ok ? "SUCCESSFUL" : "UNSUCCESSFUL");
    return verify && !ok ? 1 : 0;
}

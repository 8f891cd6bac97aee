// ft_main.cpp -- `ft`, a drop-in for the reference benchmark binary ft.<CLASS>
// (GMAP/NPB-GPU CUDA/FT/ft.cu main, :335-505) on top of libcgb's C ABI.
//
//   ft S|W|A|B|C|D          an NPB class (setparams.cpp:797-803)
//   options: --device D  --json (one JSON result line instead of the report)
//
// Like the reference it prints each iteration's checksum (ft.cu:412-414),
// verifies them at relative 1e-12 against the class's values (ft.cu:1638-
// 1830) and reports Mop/s by the reference's operation count (ft.cu:418-
// 424); the time is the device time of main's timed region.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cgb.h"

namespace {

struct FtClass {
    char name;
    int nx, ny, nz, niter;
    const double *sums;  // 2 niter: real, imaginary
};

// ft.cu:1655-1810, the first iterations' checksums of each class (the
// driver checks every iteration the class has)
const double kS[] = {5.546087004964E+02, 4.845363331978E+02, 5.546385409189E+02, 4.865304269511E+02,
                     5.546148406171E+02, 4.883910722336E+02, 5.545423607415E+02, 4.901273169046E+02,
                     5.544255039624E+02, 4.917475857993E+02, 5.542683411902E+02, 4.932597244941E+02};
const double kW[] = {5.673612178944E+02, 5.293246849175E+02, 5.631436885271E+02, 5.282149986629E+02,
                     5.594024089970E+02, 5.270996558037E+02, 5.560698047020E+02, 5.260027904925E+02,
                     5.530898991250E+02, 5.249400845633E+02, 5.504159734538E+02, 5.239212247086E+02};
const double kA[] = {5.046735008193E+02, 5.114047905510E+02, 5.059412319734E+02, 5.098809666433E+02,
                     5.069376896287E+02, 5.098144042213E+02, 5.077892868474E+02, 5.101336130759E+02,
                     5.085233095391E+02, 5.104914655194E+02, 5.091487099959E+02, 5.107917842803E+02};
const double kB[] = {5.177643571579E+02, 5.077803458597E+02, 5.154521291263E+02, 5.088249431599E+02,
                     5.146409228649E+02, 5.096208912659E+02, 5.142378756213E+02, 5.101023387619E+02,
                     5.139626667737E+02, 5.103976610617E+02, 5.137423460082E+02, 5.105948019802E+02,
                     5.135547056878E+02, 5.107404165783E+02, 5.133910925466E+02, 5.108576573661E+02,
                     5.132470705390E+02, 5.109577278523E+02, 5.131197729984E+02, 5.110460304483E+02,
                     5.130070319283E+02, 5.111252433800E+02, 5.129070537032E+02, 5.111968077718E+02,
                     5.128182883502E+02, 5.112616233064E+02, 5.127393733383E+02, 5.113203605551E+02,
                     5.126691062020E+02, 5.113735928093E+02, 5.126064276004E+02, 5.114218460548E+02,
                     5.125504076570E+02, 5.114656139760E+02, 5.125002331720E+02, 5.115053595966E+02,
                     5.124551951846E+02, 5.115415130407E+02, 5.124146770029E+02, 5.115744692211E+02};
const double kC[] = {5.195078707457E+02, 5.149019699238E+02, 5.155422171134E+02, 5.127578201997E+02,
                     5.144678022222E+02, 5.122251847514E+02, 5.140150594328E+02, 5.121090289018E+02,
                     5.137550426810E+02, 5.121143685824E+02, 5.135811056728E+02, 5.121496764568E+02,
                     5.134569343165E+02, 5.121870921893E+02, 5.133651975661E+02, 5.122193250322E+02,
                     5.132955192805E+02, 5.122454735794E+02, 5.132410471738E+02, 5.122663649603E+02,
                     5.131971141679E+02, 5.122830879827E+02, 5.131605205716E+02, 5.122965869718E+02,
                     5.131290734194E+02, 5.123075927445E+02, 5.131012720314E+02, 5.123166486553E+02,
                     5.130760908195E+02, 5.123241541685E+02, 5.130528295923E+02, 5.123304037599E+02,
                     5.130310107773E+02, 5.123356167976E+02, 5.130103090133E+02, 5.123399592211E+02,
                     5.129905029333E+02, 5.123435588985E+02, 5.129714421109E+02, 5.123465164008E+02};
const double kD[] = {5.122230065252E+02, 5.118534037109E+02, 5.120463975765E+02, 5.117061181082E+02,
                     5.119865766760E+02, 5.117096364601E+02, 5.119518799488E+02, 5.117373863950E+02,
                     5.119269088223E+02, 5.117680347632E+02, 5.119082416858E+02, 5.117967875532E+02,
                     5.118943814638E+02, 5.118225281841E+02, 5.118842385057E+02, 5.118451629348E+02,
                     5.118769435632E+02, 5.118649119387E+02, 5.118718203448E+02, 5.118820803844E+02,
                     5.118683569061E+02, 5.118969781011E+02, 5.118661708593E+02, 5.119098918835E+02,
                     5.118649768950E+02, 5.119210777066E+02, 5.118645605626E+02, 5.119307604484E+02,
                     5.118647586618E+02, 5.119391362671E+02, 5.118654451572E+02, 5.119463757241E+02,
                     5.118665212451E+02, 5.119526269238E+02, 5.118679083821E+02, 5.119580184108E+02,
                     5.118695433664E+02, 5.119626617538E+02, 5.118713748264E+02, 5.119666538138E+02,
                     5.118733606701E+02, 5.119700787219E+02, 5.118754661974E+02, 5.119730095953E+02,
                     5.118776626738E+02, 5.119755100241E+02, 5.118799262314E+02, 5.119776353561E+02,
                     5.118822370068E+02, 5.119794338060E+02};

const FtClass kClasses[] = {
    {'S', 64, 64, 64, 6, kS},       {'W', 128, 128, 32, 6, kW},     {'A', 256, 256, 128, 6, kA},
    {'B', 512, 256, 256, 20, kB},   {'C', 512, 512, 512, 20, kC},   {'D', 2048, 1024, 1024, 25, kD},
};

void usage() { std::fprintf(stderr, "usage: ft S|W|A|B|C|D [--device D] [--json]\n"); }

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        usage();
        return 2;
    }
    const FtClass *P = nullptr;
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
    std::vector<double> sums(2 * P->niter);
    cgb_ft *f = nullptr;
    double ms = 0.0, warm = 0.0;
    int st = cgb_ft_create(device, P->nx, P->ny, P->nz, &f);
    // the reference runs the problem once untimed first (ft.cu:354-368)
    if (!st) st = cgb_ft_run(f, P->niter, nullptr, &warm);
    if (!st) st = cgb_ft_run(f, P->niter, sums.data(), &ms);
    if (f) cgb_ft_destroy(f);
    if (st) {
        std::fprintf(stderr, "ft: run failed: %s (%s)\n", cgb_status_string(st), cgb_last_error());
        return 1;
    }
    double worst = 0.0;
    for (int i = 0; i < P->niter; i++) {
        const std::complex<double> s(sums[2 * i], sums[2 * i + 1]), r(P->sums[2 * i], P->sums[2 * i + 1]);
        worst = std::max(worst, std::abs((s - r) / r));
    }
    const bool ok = worst <= 1.0e-12;
    const double t = ms / 1e3, nt = double(P->nx) * P->ny * P->nz;
    const double mflops = t > 0 ? 1.0e-6 * nt *
                                      (14.8157 + 7.19641 * std::log(nt) +
                                       (5.23518 + 7.21113 * std::log(nt)) * P->niter) / t
                                : 0.0;
    if (json) {
        std::printf("{\"class\": \"%c\", \"nx\": %d, \"ny\": %d, \"nz\": %d, \"niter\": %d, \"seconds\": %.9g, "
                    "\"mops\": %.6g, \"verified\": %s, \"max_rel_err\": %.6g, \"last_checksum\": [%.17g, %.17g]}\n",
                    P->name, P->nx, P->ny, P->nz, P->niter, t, mflops, ok ? "true" : "false", worst,
                    sums[2 * P->niter - 2], sums[2 * P->niter - 1]);
        return ok ? 0 : 1;
    }
    std::printf("\n\n NAS Parallel Benchmarks 4.1 - FT Benchmark (B200 sm_100a build)\n\n");
    std::printf(" Size                : %4dx%4dx%4d\n", P->nx, P->ny, P->nz);
    std::printf(" Iterations                  :%7d\n\n", P->niter);
    for (int i = 0; i < P->niter; i++)
        std::printf("T = %5d     Checksum = %22.12e %22.12e\n", i + 1, sums[2 * i], sums[2 * i + 1]);
    std::printf(" Result verification %s\n", ok ? "successful" : "failed");
    std::printf(" class_npb = %c\n", P->name);
    std::printf("\n\n FT Benchmark Completed\n");
    std::printf(" class_npb       =                        %c\n", P->name);
    std::printf(" Size            =           %4dx%4dx%4d\n", P->nx, P->ny, P->nz);
    std::printf(" Iterations      =             %12d\n", P->niter);
    std::printf(" Time in seconds =             %12.6f\n", t);
    std::printf(" Mop/s total     =             %12.2f\n", mflops);
    std::printf(" Operation type  = %24s\n", "floating point");
    std::printf(" Verification    =             %12s\n", ok ? "SUCCESSFUL" : "UNSUCCESSFUL");
    return ok ? 0 : 1;
}

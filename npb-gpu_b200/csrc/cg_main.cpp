// cg_main.cpp -- `cg`, a drop-in for the reference benchmark binary cg.<CLASS>
// (GMAP/NPB-GPU CUDA/CG/cg.cu main(), :337-645) on top of libcgb's C ABI.
//
//   cg S|W|A|B|C|D|E        an NPB class (setparams.cpp:751-785 parameters)
//   cg U --n N --nonzer K --niter I --shift S [--seed X]   custom sizes
//   options: --mode fp64|tol|mixed|learned  --tol T  --cgitmax M
//            --weights FILE (learned mode: network weights, raw FP32; default
//            the trained weights shipped beside the package, npbcg/lp_weights.f32)
//            --device D  --json (one JSON result line instead of the report)
//            --spmv row|sliced (SpMV plan; default: the autotuner's choice)
//            --gpu-makea (generate the matrix with cgb_makea_device)
//            --ranks K (the row-partitioned solver: the rows split into K
//            blocks, each generated on the device, all K ranks driven from
//            this process on one GPU; the reference algorithm only.  Class E
//            always runs this way: its 6.4e9 entries overflow the int32 row
//            pointers of one CSR, cg.cu:81, so it takes the fewest blocks of
//            fewer than 2^31 entries each)
//
// Like the reference it generates the matrix (makea), runs the timed inverse
// power iteration, prints the per-iteration "||r||  zeta" lines in the
// reference format (cg.cu:515-516), verifies zeta against the class's value
// at relative 1e-10 (cg.cu:534-552), and reports time and Mop/s with the
// reference's operation count (cg.cu:553-561).  The timed region is the
// device time of the outer loop; matrix generation and upload are outside
// it, as in the reference (cg.cu:490-522).
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cgb.h"

namespace {

struct ClassParams {
    char name;
    int n, nonzer, niter;
    double shift, zeta_verify;
};

// NPB CG classes and verification zetas (cg.cu:373-396).
const ClassParams kClasses[] = {
    {'S', 1400, 7, 15, 10.0, 8.5971775078648},
    {'W', 7000, 8, 15, 12.0, 10.362595087124},
    {'A', 14000, 11, 15, 20.0, 17.130235054029},
    {'B', 75000, 13, 75, 60.0, 22.712745482631},
    {'C', 150000, 15, 75, 110.0, 28.973605592845},
    {'D', 1500000, 21, 100, 500.0, 52.514532105794},
    {'E', 9000000, 26, 100, 1500.0, 77.522164599383},
};

int fail(int st, const char *what)
{
    std::fprintf(stderr, "cg: %s failed: %s (%s)\n", what, cgb_status_string(st), cgb_last_error());
    return 1;
}

void usage()
{
    std::fprintf(stderr,
                 "usage: cg S|W|A|B|C|D|E | cg U --n N --nonzer K --niter I --shift S [--seed X]\n"
                 "          [--mode fp64|tol|mixed|learned] [--tol T] [--cgitmax M]\n"
                 "          [--weights FILE] [--device D] [--json] [--gpu-makea]\n"
                 "          [--spmv row|sliced] [--ranks K]\n");
}

// The weights shipped with the package: <dir of this binary>/../npbcg/lp_weights.f32.
std::string default_weights()
{
    char buf[4096];
    const ssize_t len = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    if (len <= 0) return "lp_weights.f32";
    std::string exe(buf, size_t(len));
    const size_t slash = exe.rfind('/');
    const std::string dir = slash == std::string::npos ? "." : exe.substr(0, slash);
    return dir + "/../npbcg/lp_weights.f32";
}

// Learned mode: loads the network weights, infers G for this matrix and
// installs F = G / sqrt(delta) in the session.
int attach_learned(cgb_session *s, const std::string &path, int device, int n,
                   const std::vector<int> &rowstr, const std::vector<int> &colidx,
                   const std::vector<double> &a)
{
    const int count = cgb_gnn_param_count();
    std::vector<float> w(static_cast<size_t>(count));
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        std::fprintf(stderr, "cg: cannot open weights %s\n", path.c_str());
        return 1;
    }
    const size_t got = std::fread(w.data(), sizeof(float), w.size(), f);
    const bool extra = std::fgetc(f) != EOF;
    std::fclose(f);
    if (got != w.size() || extra) {
        std::fprintf(stderr, "cg: %s holds no %d FP32 weights\n", path.c_str(), count);
        return 1;
    }
    cgb_gnn *m = nullptr;
    cgb_gnn_graph *g = nullptr;
    int st = cgb_gnn_create(device, 0u, &m);
    if (!st) st = cgb_gnn_set_params(m, w.data(), count);
    if (!st) st = cgb_gnn_graph_create(m, n, rowstr.data(), colidx.data(), a.data(), &g);
    if (!st) st = cgb_gnn_attach(m, g, s);
    if (g) cgb_gnn_graph_destroy(g);
    if (m) cgb_gnn_destroy(m);
    return st ? fail(st, "learned preconditioner") : 0;
}

// The row-partitioned solve: K row blocks generated on the device, one
// untimed outer step (as the reference's untimed iteration, cg.cu:453-482),
// then the timed niter steps.  Fills the traces, the device milliseconds
// and the stored entries.
int run_partitioned(const ClassParams &P, double seed, int K, int cgitmax, int device,
                    std::vector<double> &zeta, std::vector<double> &rnorm, double *ms,
                    long long *nnz)
{
    std::vector<cgb_part *> parts(size_t(K), nullptr);
    int st = CGB_OK;
    *nnz = 0;
    for (int r = 0; r < K && !st; r++) {
        st = cgb_part_create_generated(device, P.n, P.nonzer, 0.1, P.shift, seed, K, r, nullptr, &parts[r]);
        long long k = 0;
        if (!st) st = cgb_part_info(parts[r], nullptr, nullptr, &k);
        *nnz += k;
    }
    if (!st) st = cgb_part_group_power_iterate(parts.data(), K, 1, P.shift, cgitmax, nullptr, nullptr, nullptr);
    if (!st)
        st = cgb_part_group_power_iterate(parts.data(), K, P.niter, P.shift, cgitmax, zeta.data(),
                                          rnorm.data(), ms);
    const int failed = st;
    for (cgb_part *p : parts)
        if (p) cgb_part_destroy(p);
    return failed ? fail(failed, "partitioned solve") : 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        usage();
        return 2;
    }
    ClassParams P{'U', 0, 0, 0, 0.0, 0.0};
    const char cls = argv[1][0];
    bool known = false;
    for (const auto &c : kClasses)
        if (c.name == cls) {
            P = c;
            known = true;
        }
    if (!known && cls != 'U') {
        usage();
        return 2;
    }
    double seed = 314159265.0, tol = 1e-12;
    std::string weights;
    int mode = CGB_MODE_FP64, cgitmax = 25, device = 0, json = 0, gpu_makea = 0, spmv = 0, ranks = 0;
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](void) -> const char * {
            if (i + 1 >= argc) {
                usage();
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--n") P.n = std::atoi(next());
        else if (a == "--nonzer") P.nonzer = std::atoi(next());
        else if (a == "--niter") P.niter = std::atoi(next());
        else if (a == "--shift") P.shift = std::atof(next());
        else if (a == "--seed") seed = std::atof(next());
        else if (a == "--tol") tol = std::atof(next());
        else if (a == "--cgitmax") cgitmax = std::atoi(next());
        else if (a == "--device") device = std::atoi(next());
        else if (a == "--json") json = 1;
        else if (a == "--gpu-makea") gpu_makea = 1;
        else if (a == "--ranks") ranks = std::atoi(next());
        else if (a == "--spmv") {
            const std::string k = next();
            if (k == "row") spmv = 1;
            else if (k == "sliced") spmv = 2;
            else {
                usage();
                return 2;
            }
        }
        else if (a == "--weights") weights = next();
        else if (a == "--mode") {
            const std::string m = next();
            if (m == "fp64") mode = CGB_MODE_FP64;
            else if (m == "tol") mode = CGB_MODE_FP64_TOL;
            else if (m == "mixed") mode = CGB_MODE_MIXED;
            else if (m == "learned") mode = CGB_MODE_MIXED_LEARNED;
            else {
                usage();
                return 2;
            }
        } else {
            usage();
            return 2;
        }
    }
    if (P.n < 2 || P.nonzer < 1 || P.niter < 1) {
        usage();
        return 2;
    }
    // a custom size or another seed has no verification value (cg.cu:548-551)
    const bool verify = known && seed == 314159265.0;
    const long long cap = cgb_nz_bound(P.n, P.nonzer);
    if (ranks == 0 && cap > 0x7fffffffLL) ranks = int((cap + 0x7ffffffeLL) / 0x7fffffffLL);
    if (ranks < 0 || (ranks > 0 && mode != CGB_MODE_FP64)) {
        std::fprintf(stderr, "cg: --ranks K >= 1 runs the reference algorithm (--mode fp64) only\n");
        return 2;
    }

    double device_ms = 0.0, zeta_last = 0.0, rnorm_last = 0.0;
    int total_inner = 0, kind = 0, panels = 0;
    long long nnz = 0;
    std::vector<double> zeta(P.niter), rnorm(P.niter);
    if (ranks > 0) {
        if (run_partitioned(P, seed, ranks, cgitmax, device, zeta, rnorm, &device_ms, &nnz)) return 1;
        zeta_last = zeta[P.niter - 1];
        rnorm_last = rnorm[P.niter - 1];
        total_inner = P.niter * cgitmax;
        kind = 4;  // plan_kind 4: row blocks (panels = their count)
        panels = ranks;
    } else {
        std::vector<int> rowstr(P.n + 1), colidx(cap);
        std::vector<double> a(cap);
        int st = gpu_makea ? cgb_makea_device(device, P.n, P.nonzer, 0.1, P.shift, seed, rowstr.data(),
                                              colidx.data(), a.data(), cap, &nnz)
                           : cgb_makea(P.n, P.nonzer, 0.1, P.shift, seed, rowstr.data(), colidx.data(),
                                       a.data(), cap, &nnz);
        if (st) return fail(st, "makea");

        cgb_options opt;
        cgb_default_options(&opt);
        opt.device = device;
        opt.spmv_kernel = spmv;
        cgb_session *s = nullptr;
        st = cgb_create(P.n, rowstr.data(), colidx.data(), a.data(), &opt, &s);
        if (st) return fail(st, "create");
        if (mode == CGB_MODE_MIXED_LEARNED &&
            attach_learned(s, weights.empty() ? default_weights() : weights, device, P.n, rowstr,
                           colidx, a) != 0) {
            cgb_destroy(s);
            return 1;
        }

        cgb_solve_params sp;
        cgb_default_solve_params(&sp);
        sp.niter = P.niter;
        sp.shift = P.shift;
        sp.mode = mode;
        sp.cgitmax = cgitmax;
        sp.tol = tol;
        // one untimed solve first, as the reference does one untimed iteration (cg.cu:453-482)
        cgb_solve_result res;
        st = cgb_power_iterate(s, &sp, nullptr, nullptr, nullptr, nullptr, &res);
        if (st) return fail(st, "power_iterate (warm-up)");
        std::vector<int> iters(P.niter);
        st = cgb_power_iterate(s, &sp, zeta.data(), rnorm.data(), iters.data(), nullptr, &res);
        if (st) return fail(st, "power_iterate");
        // the plan the autotuner chose: row (1) or sliced (2, 3 with the L2
        // prefetch), and the sliced walk's row panels
        int lpr = 0, grid = 0, block = 0, prec_panels = 0;
        long long smem = 0, entries = 0;
        if (cgb_plan_info(s, &kind, &lpr, &grid, &block, &smem, &entries) ||
            cgb_plan_panels(s, &panels, &prec_panels))
            kind = panels = 0;
        cgb_destroy(s);
        device_ms = res.device_ms;
        zeta_last = res.zeta;
        rnorm_last = res.rnorm;
        total_inner = res.total_inner;
    }

    const double t = device_ms / 1e3;
    const double nz1 = double(P.nonzer) * (P.nonzer + 1);
    const double mops =
        t > 0 ? 2.0 * P.niter * P.n * (3.0 + nz1 + 25.0 * (5.0 + nz1) + 3.0) / t / 1e6 : 0.0;
    const double err = verify ? std::fabs(zeta_last - P.zeta_verify) / P.zeta_verify : -1.0;
    const bool ok = verify && err <= 1.0e-10;

    if (json) {
        std::printf("{\"class\": \"%c\", \"n\": %d, \"nonzer\": %d, \"niter\": %d, \"shift\": %.17g, "
                    "\"nnz\": %lld, \"mode\": %d, \"zeta\": %.17g, \"rnorm\": %.17g, "
                    "\"seconds\": %.9g, \"mops\": %.6g, \"inner_total\": %d, \"verified\": %s, "
                    "\"rel_err\": %.6g, \"plan_kind\": %d, \"panels\": %d}\n",
                    P.name, P.n, P.nonzer, P.niter, P.shift, nnz, mode, zeta_last, rnorm_last, t,
                    mops, total_inner, verify ? (ok ? "true" : "false") : "null", err, kind,
                    panels);
        return verify && !ok ? 1 : 0;
    }
    std::printf("\n\n NAS Parallel Benchmarks 4.1 - CG Benchmark (B200 sm_100a build)\n\n");
    std::printf(" Size: %11d\n", P.n);
    std::printf(" Iterations: %5d\n", P.niter);
    std::printf("\n   iteration           ||r||                 zeta\n");
    for (int it = 0; it < P.niter; it++)
        std::printf("    %5d       %20.14e%20.13e\n", it + 1, rnorm[it], zeta[it]);
    std::printf(" Benchmark completed\n");
    if (verify) {
        if (ok) {
            std::printf(" VERIFICATION SUCCESSFUL\n");
            std::printf(" Zeta is    %20.13e\n", zeta_last);
            std::printf(" Error is   %20.13e\n", err);
        } else {
            std::printf(" VERIFICATION FAILED\n");
            std::printf(" Zeta                %20.13e\n", zeta_last);
            std::printf(" The correct zeta is %20.13e\n", P.zeta_verify);
        }
    } else {
        std::printf(" Problem size unknown\n");
        std::printf(" NO VERIFICATION PERFORMED\n");
    }
    static const char *mode_names[] = {"FP64 fixed", "FP64 tolerance", "FP32 SpMV + FP64 refinement",
                                       "mixed + learned preconditioner"};
    std::printf("\n\n CG Benchmark Completed\n");
    std::printf(" class_npb       =                        %c\n", P.name);
    std::printf(" Size            =             %12d\n", P.n);
    std::printf(" Iterations      =             %12d\n", P.niter);
    std::printf(" Time in seconds =             %12.6f\n", t);
    std::printf(" Mop/s total     =             %12.2f\n", mops);
    std::printf(" Operation type  = %24s\n", "floating point");
    if (!verify) std::printf(" Verification    =            NOT PERFORMED\n");
    else std::printf(" Verification    =             %12s\n", ok ? "SUCCESSFUL" : "UNSUCCESSFUL");
    std::printf(" Mode            = %s\n", mode_names[mode & 3]);
    std::printf(" Inner CG steps  =             %12d\n", total_inner);
    std::printf(" Nonzeros        =             %12lld\n", nnz);
    if (ranks > 0) std::printf(" Row blocks      =             %12d\n", ranks);
    return verify && !ok ? 1 : 0;
}

/*
 * ref_harness.cu -- wraps the reference's own CG code as a shared library.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle of the tests and the CPU baseline, never the
 * product).  Compiled by oracle/Makefile straight from the reference
 * sources where they lie (CUDA/CG/cg.cu and CUDA/common/*.cpp|.cu of
 * GMAP/NPB-GPU); nothing of the reference is copied into this repository.
 * One library per NPB class, because cg.cu sizes its arrays from
 * compile-time NA / NONZER (cg.cu:81-122).  Outputs go to oracle/_ref/.
 *
 * Exported entry points (extern "C"):
 *   ref_info        class parameters the library was built with
 *   ref_makea       the reference makea() at a chosen LCG seed
 *                   (seed, discarded first draw as main() does, cg.cu:405-408)
 *   ref_conj_grad   one call of the reference CPU conj_grad (cg.cu:653-801)
 *                   on the last generated matrix
 *   ref_power       the reference outer loop (cg.cu:485-520) driven by the
 *                   CPU conj_grad: per-step zeta and rnorm, wall seconds
 *   ref_set_matrix  loads a CSR (the generator's, produced elsewhere bit for
 *                   bit) into the reference's arrays instead of ref_makea
 *   ref_power_gpu   the same loop as the reference times it on the GPU
 *                   (cg.cu:489-522: setup_gpu, then conj_grad_gpu and the
 *                   gpu_kernel_ten / eleven norms, release_gpu after): an
 *                   informative comparator of the GPU arm, compiled with the
 *                   reference's device flags (make.def OPTIMIZATIONS)
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#define main npb_cg_reference_main
#include "CG/cg.cu"
#undef main

static int g_nnz = -1;

static double harness_now()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

extern "C" void ref_info(int *na, int *nonzer, int *niter, double *shift, double *rcond,
                         long long *nz_bound)
{
    *na = NA;
    *nonzer = NONZER;
    *niter = NITER;
    *shift = SHIFT;
    *rcond = RCOND;
    *nz_bound = (long long)NZ;
}

/* Generate the matrix with the reference makea at LCG seed `seed`
 * (314159265 for the NPB classes).  Copies the CSR out when the
 * pointers are non-NULL; returns nnz. */
extern "C" int ref_makea(double seed, int *rowstr_out, int *colidx_out, double *a_out)
{
    firstrow = 0;
    lastrow = NA - 1;
    firstcol = 0;
    lastcol = NA - 1;
    naa = NA;
    nzz = NZ;
    tran = seed;
    amult = 1220703125.0;
    (void)randlc(&tran, amult);
    makea(naa, nzz, a, colidx, rowstr, firstrow, lastrow, firstcol, lastcol, arow,
          (int(*)[NONZER + 1])(void *)acol, (double(*)[NONZER + 1])(void *)aelt, iv);
    for (int j = 0; j < lastrow - firstrow + 1; j++)
        for (int k = rowstr[j]; k < rowstr[j + 1]; k++)
            colidx[k] = colidx[k] - firstcol;
    g_nnz = rowstr[NA];
    if (rowstr_out)
        memcpy(rowstr_out, rowstr, sizeof(int) * (NA + 1));
    if (colidx_out)
        memcpy(colidx_out, colidx, sizeof(int) * (size_t)g_nnz);
    if (a_out)
        memcpy(a_out, a, sizeof(double) * (size_t)g_nnz);
    return g_nnz;
}

/* Loads rowstr (NA+1), colidx and a (nnz entries) into the reference's
 * arrays, as ref_makea leaves them; returns nnz, or -1 when it exceeds NZ. */
extern "C" int ref_set_matrix(const int *rowstr_in, const int *colidx_in, const double *a_in)
{
    const int nnz = rowstr_in[NA];
    if (nnz < 0 || (long long)nnz > (long long)NZ)
        return -1;
    firstrow = 0;
    lastrow = NA - 1;
    firstcol = 0;
    lastcol = NA - 1;
    memcpy(rowstr, rowstr_in, sizeof(int) * (NA + 1));
    memcpy(colidx, colidx_in, sizeof(int) * (size_t)nnz);
    memcpy(a, a_in, sizeof(double) * (size_t)nnz);
    g_nnz = nnz;
    return nnz;
}

/* One reference conj_grad on the last generated matrix.  x_in has NA
 * entries (entry NA is set to 1.0 as main() does); z, r, p, q receive NA
 * entries each.  Returns -1 when no matrix was generated yet. */
extern "C" int ref_conj_grad(const double *x_in, double *z_out, double *r_out, double *p_out,
                             double *q_out, double *rnorm)
{
    if (g_nnz < 0)
        return -1;
    for (int i = 0; i < NA; i++)
        x[i] = x_in[i];
    x[NA] = 1.0;
    conj_grad(colidx, rowstr, x, z, a, p, q, r, rnorm);
    if (z_out) memcpy(z_out, z, sizeof(double) * NA);
    if (r_out) memcpy(r_out, r, sizeof(double) * NA);
    if (p_out) memcpy(p_out, p, sizeof(double) * NA);
    if (q_out) memcpy(q_out, q, sizeof(double) * NA);
    return 0;
}

/* The reference outer loop with the CPU conj_grad (cg.cu:485-520 with
 * conj_grad in place of conj_grad_gpu): x = 1, niter steps.  Returns the
 * wall seconds of the loop; traces may be NULL. */
extern "C" double ref_power(int niter, double *zeta_trace, double *rnorm_trace)
{
    if (g_nnz < 0)
        return -1.0;
    double rnorm = 0.0, zeta = 0.0;
    for (int i = 0; i < NA + 1; i++)
        x[i] = 1.0;
    double t0 = harness_now();
    for (int it = 1; it <= niter; it++) {
        conj_grad(colidx, rowstr, x, z, a, p, q, r, &rnorm);
        double norm_temp1 = 0.0, norm_temp2 = 0.0;
        for (int j = 0; j < lastcol - firstcol + 1; j++) {
            norm_temp1 = norm_temp1 + x[j] * z[j];
            norm_temp2 = norm_temp2 + z[j] * z[j];
        }
        norm_temp2 = 1.0 / sqrt(norm_temp2);
        zeta = SHIFT + 1.0 / norm_temp1;
        for (int j = 0; j < lastcol - firstcol + 1; j++)
            x[j] = norm_temp2 * z[j];
        if (zeta_trace) zeta_trace[it - 1] = zeta;
        if (rnorm_trace) rnorm_trace[it - 1] = rnorm;
    }
    return harness_now() - t0;
}

/* The reference's GPU outer loop (cg.cu:489-522): x = 1, setup_gpu() (the
 * uploads, outside the timed region as in main), niter steps of
 * conj_grad_gpu + gpu_kernel_ten / gpu_kernel_eleven, release_gpu().
 * Returns the wall seconds of the loop (the reference's own timer brackets
 * the same region); traces may be NULL. */
extern "C" double ref_power_gpu(int niter, double *zeta_trace, double *rnorm_trace)
{
    if (g_nnz < 0)
        return -1.0;
    for (int i = 0; i < NA + 1; i++)
        x[i] = 1.0;
    for (int j = 0; j < lastcol - firstcol + 1; j++) {
        q[j] = 0.0;
        z[j] = 0.0;
        r[j] = 0.0;
        p[j] = 0.0;
    }
    setup_gpu();
    cudaDeviceSynchronize();
    double t0 = harness_now();
    for (int it = 1; it <= niter; it++) {
        double rnorm = 0.0, norm_temp1 = 0.0, norm_temp2 = 0.0;
        conj_grad_gpu(&rnorm);
        gpu_kernel_ten(&norm_temp1, &norm_temp2);
        norm_temp2 = 1.0 / sqrt(norm_temp2);
        if (zeta_trace) zeta_trace[it - 1] = SHIFT + 1.0 / norm_temp1;
        if (rnorm_trace) rnorm_trace[it - 1] = rnorm;
        gpu_kernel_eleven(norm_temp2);
    }
    cudaDeviceSynchronize();
    const double secs = harness_now() - t0;
    release_gpu();
    return secs;
}

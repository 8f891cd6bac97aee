/*
 * ref_mg_harness.cu -- wraps the reference's own MG code as a shared library.
 *
 * TEST INFRASTRUCTURE ONLY (a checker of the tests and a comparator of the
 * bench, never the product).  Compiled by oracle/Makefile straight from the
 * reference sources where they lie (CUDA/MG/mg.cu and CUDA/common of
 * GMAP/NPB-GPU); nothing of the reference is copied into this repository.
 * One library per NPB class, because mg.cu sizes its arrays from
 * compile-time parameters (mg.cu:64-69).  Outputs go to oracle/_ref/.
 *
 * Exported entry points (extern "C"):
 *   ref_mg_info   lt and nit the library was built with
 *   ref_mg_cpu    main's set-up (mg.cu:386-447) and its timed sequence run
 *                 with the reference's serial CPU operators (resid, norm2u3,
 *                 nit x (mg3P, resid), norm2u3 -- the functions main's
 *                 untimed start-up iteration uses); final norms, wall
 *                 seconds, and the finest u and r
 *   ref_mg_gpu    the same set-up, then the reference's timed GPU region
 *                 exactly as main runs it (mg.cu:486-517: setup_gpu, then
 *                 resid_gpu, norm2u3_gpu, nit x (mg3P_gpu, resid_gpu),
 *                 norm2u3_gpu, release_gpu after), compiled with the
 *                 reference's device flags: an informative comparator
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#define main npb_mg_reference_main
#include "MG/mg.cu"
#undef main

static double harness_now()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* main's parameters and coefficients, its setup, zero3 and zran3 (the
 * state main has when it enters the timed region, mg.cu:386-447). */
static void mg_prepare(double a[4], double c[4], int *n1, int *n2, int *n3, int *nit)
{
    lt = LT_DEFAULT;
    *nit = NIT_DEFAULT;
    nx[lt] = NX_DEFAULT;
    ny[lt] = NY_DEFAULT;
    nz[lt] = NZ_DEFAULT;
    for (int i = 0; i <= 7; i++) debug_vec[i] = DEBUG_DEFAULT;
    a[0] = -8.0 / 3.0;
    a[1] = 0.0;
    a[2] = 1.0 / 6.0;
    a[3] = 1.0 / 12.0;
    const bool small = (NX_DEFAULT == 32 || NX_DEFAULT == 128 || (NX_DEFAULT == 256 && NIT_DEFAULT == 4));
    if (small) {
        c[0] = -3.0 / 8.0;
        c[1] = +1.0 / 32.0;
        c[2] = -1.0 / 64.0;
        c[3] = 0.0;
    } else {
        c[0] = -3.0 / 17.0;
        c[1] = +1.0 / 33.0;
        c[2] = -1.0 / 61.0;
        c[3] = 0.0;
    }
    lb = 1;
    int k = lt;
    setup(n1, n2, n3, k);
    zero3(u, *n1, *n2, *n3);
    zran3(v, *n1, *n2, *n3, nx[lt], ny[lt], k);
}

extern "C" void ref_mg_info(int *lt_out, int *nit_out)
{
    *lt_out = LT_DEFAULT;
    *nit_out = NIT_DEFAULT;
}

extern "C" int ref_mg_cpu(double *rnm2, double *rnmu, double *seconds, double *u_out, double *r_out)
{
    double a[4], c[4];
    int n1, n2, n3, nit;
    mg_prepare(a, c, &n1, &n2, &n3, &nit);
    const int k = lt;
    const double t0 = harness_now();
    resid(u, v, r, n1, n2, n3, a, k);
    norm2u3(r, n1, n2, n3, rnm2, rnmu, nx[lt], ny[lt], nz[lt]);
    for (int it = 1; it <= nit; it++) {
        mg3P(u, v, r, a, c, n1, n2, n3, k);
        resid(u, v, r, n1, n2, n3, a, k);
    }
    norm2u3(r, n1, n2, n3, rnm2, rnmu, nx[lt], ny[lt], nz[lt]);
    *seconds = harness_now() - t0;
    const size_t cells = (size_t)n1 * n2 * n3;
    if (u_out) memcpy(u_out, u, sizeof(double) * cells);
    if (r_out) memcpy(r_out, r, sizeof(double) * cells);
    return 0;
}

extern "C" int ref_mg_gpu(double *rnm2, double *rnmu, double *seconds)
{
    double a[4], c[4];
    int n1, n2, n3, nit;
    mg_prepare(a, c, &n1, &n2, &n3, &nit);
    setup_gpu(a, c);
    const int k = lt;
    const double t0 = harness_now();
    resid_gpu(u_device, v_device, r_device, n1, n2, n3, a_device, k);
    norm2u3_gpu(r_device, n1, n2, n3, rnm2, rnmu, nx[lt], ny[lt], nz[lt]);
    for (int it = 1; it <= nit; it++) {
        mg3P_gpu(u_device, v_device, r_device, a_device, c_device, n1, n2, n3, k);
        resid_gpu(u_device, v_device, r_device, n1, n2, n3, a_device, k);
    }
    norm2u3_gpu(r_device, n1, n2, n3, rnm2, rnmu, nx[lt], ny[lt], nz[lt]);
    *seconds = harness_now() - t0;
    release_gpu();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

/*
 * ep_oracle.c -- CPU oracle for the NPB EP path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle of the tests, never the
 * product: only tests/, __graft_entry__.smoke() and the cpu_baseline legs of
 * bench.py may load liboracle.so.  libcgb.so neither links nor calls anything
 * here.
 *
 * It restates, in plain C, the EP benchmark of the GMAP/NPB-GPU reference
 * (paths relative to that project, CUDA/EP/ep.cu):
 *   - an = A^(2^(MK+1)) by repeated squaring   :147-153
 *   - batch kk's seed S * an^kk                 :304-312
 *   - per batch 2 NK uniforms (vranlc), pairs mapped to (-1, 1)^2,
 *     accepted when x1^2 + x2^2 <= 1, Gaussian deviates
 *     (x1, x2) * sqrt(-2 log t / t), counts in square annuli by
 *     max(|t3|, |t4|), sums sx, sy              :314-340
 *   - class table (M: S 24, W 25, A 28, B 30, C 32, D 36, E 40;
 *     setparams.cpp:826-845) and verification sums (:189-212), epsilon 1e-8
 * with randlc / vranlc of CUDA/common/c_randdp.cpp:84-190 (orc_randlc, the
 * same 23-bit split arithmetic).  Sums run batch by batch, pair by pair; the
 * reference's GPU code adds per-thread sums with atomics, in no fixed order.
 * Pinned against the reference's verification sums (tests/test_ep_oracle.py).
 */
#include <math.h>
#include <stdlib.h>
#include <time.h>

double orc_randlc(double *x, double a); /* cg_oracle.c */

#define EP_MK 16
#define EP_NK (1 << EP_MK)
#define EP_NQ 10
#define EP_A 1220703125.0
#define EP_S 271828183.0

/* EP with 2^m pairs (m >= EP_MK): sx, sy, the ten annulus counts q, and
 * the wall seconds of the pair loop (nullable). */
int orc_ep_run(int m, double *sx_out, double *sy_out, double *q_out, double *seconds)
{
    if (m < EP_MK || m > 40) return 1;
    double *x = malloc(sizeof(double) * 2 * EP_NK);
    if (!x) return 2;
    double an = EP_A;
    for (int i = 0; i < EP_MK + 1; i++) (void)orc_randlc(&an, an);
    double q[EP_NQ] = {0}, sx = 0.0, sy = 0.0;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    const long long nn = 1LL << (m - EP_MK);
    for (long long kk = 0; kk < nn; kk++) {
        /* seed S * an^kk by the binary digits of kk */
        double s = EP_S, t2 = an;
        for (long long k = kk; k != 0; k /= 2) {
            if (k % 2 == 1) (void)orc_randlc(&s, t2);
            (void)orc_randlc(&t2, t2);
        }
        for (int i = 0; i < 2 * EP_NK; i++) x[i] = orc_randlc(&s, EP_A);
        for (int i = 0; i < EP_NK; i++) {
            const double x1 = 2.0 * x[2 * i] - 1.0;
            const double x2 = 2.0 * x[2 * i + 1] - 1.0;
            const double t = x1 * x1 + x2 * x2;
            if (t <= 1.0) {
                const double f = sqrt(-2.0 * log(t) / t);
                const double t3 = x1 * f, t4 = x2 * f;
                const int l = (int)fmax(fabs(t3), fabs(t4));
                q[l] += 1.0;
                sx += t3;
                sy += t4;
            }
        }
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    free(x);
    *sx_out = sx;
    *sy_out = sy;
    for (int i = 0; i < EP_NQ; i++) q_out[i] = q[i];
    if (seconds) *seconds = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    return 0;
}

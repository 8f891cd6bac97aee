/*
 * mg_oracle.c -- CPU oracle for the NPB MG V-cycle path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle of the tests, never the
 * product: only tests/, __graft_entry__.smoke() and the cpu_baseline legs of
 * bench.py may load liboracle.so.  libcgb.so neither links nor calls anything
 * here.
 *
 * It restates, in plain C, the serial MG algorithm of the GMAP/NPB-GPU
 * reference (paths relative to that project, CUDA/MG/mg.cu):
 *   - setup             :1921-1975  (levels k = 1..lt, m_k = 2^k + 2 a side)
 *   - zero3             :2118-2130
 *   - zran3             :2175-2303  (LCG fill, ten largest -> +1, ten smallest -> -1)
 *   - bubble            :626-680    (the candidate lists, kept sorted)
 *   - power             :1363-1380
 *   - vranlc / randlc   CUDA/common/c_randdp.cpp:84-114, :140-190
 *   - comm3             :687-716    (periodic ghost layer)
 *   - resid             :1572-1625  (r = v - A u, 27-point, a[1] = 0)
 *   - psinv             :1395-1440  (u = u + C r, c[3] = 0)
 *   - rprj3             :1724-1790  (full-weighting restriction)
 *   - interp            :836-890    (trilinear prolongation, the m > 3 branch)
 *   - norm2u3           :1201-1230
 *   - mg3P              :1078-1133  (one V-cycle)
 *   - main's timed loop :498-508    (resid, norm; nit x (mg3P, resid); norm)
 * and the coefficients of main (:422-442): a = (-8/3, 0, 1/6, 1/12); the
 * smoother c = (-3/8, 1/32, -1/64, 0) for classes S, W, A and
 * (-3/17, 1/33, -1/61, 0) above.
 *
 * Every sum is formed in the reference's order and no multiply-add is fused
 * (gcc -ffp-contract=off), so the grids follow the reference's serial code
 * operation for operation; parity is pinned against the verification norms
 * of mg.cu:528-543 (tests/test_mg_oracle.py).  Grids are cubes of side m,
 * index (i3 * m + i2) * m + i1, i1 fastest.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

double orc_randlc(double *x, double a); /* cg_oracle.c */

#define MG_MM 10

static size_t at(int m, int i3, int i2, int i1)
{
    return ((size_t)i3 * m + i2) * m + i1;
}

/* Ghost layer of a side-m cube from the interior, axis by axis (:687-716). */
void orc_mg_comm3(int m, double *u)
{
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i2 = 1; i2 < m - 1; i2++) {
            u[at(m, i3, i2, 0)] = u[at(m, i3, i2, m - 2)];
            u[at(m, i3, i2, m - 1)] = u[at(m, i3, i2, 1)];
        }
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i1 = 0; i1 < m; i1++) {
            u[at(m, i3, 0, i1)] = u[at(m, i3, m - 2, i1)];
            u[at(m, i3, m - 1, i1)] = u[at(m, i3, 1, i1)];
        }
    for (int i2 = 0; i2 < m; i2++)
        for (int i1 = 0; i1 < m; i1++) {
            u[at(m, 0, i2, i1)] = u[at(m, m - 2, i2, i1)];
            u[at(m, m - 1, i2, i1)] = u[at(m, 1, i2, i1)];
        }
}

/* r = v - A u on the interior, then comm3(r); r may be v (:1572-1625). */
void orc_mg_resid(int m, const double *u, const double *v, double *r, const double a[4])
{
    double *u1 = malloc(sizeof(double) * m), *u2 = malloc(sizeof(double) * m);
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i2 = 1; i2 < m - 1; i2++) {
            for (int i1 = 0; i1 < m; i1++) {
                u1[i1] = u[at(m, i3, i2 - 1, i1)] + u[at(m, i3, i2 + 1, i1)] +
                         u[at(m, i3 - 1, i2, i1)] + u[at(m, i3 + 1, i2, i1)];
                u2[i1] = u[at(m, i3 - 1, i2 - 1, i1)] + u[at(m, i3 - 1, i2 + 1, i1)] +
                         u[at(m, i3 + 1, i2 - 1, i1)] + u[at(m, i3 + 1, i2 + 1, i1)];
            }
            for (int i1 = 1; i1 < m - 1; i1++)
                r[at(m, i3, i2, i1)] = v[at(m, i3, i2, i1)] - a[0] * u[at(m, i3, i2, i1)] -
                                       a[2] * (u2[i1] + u1[i1 - 1] + u1[i1 + 1]) -
                                       a[3] * (u2[i1 - 1] + u2[i1 + 1]);
        }
    free(u1);
    free(u2);
    orc_mg_comm3(m, r);
}

/* u = u + C r on the interior, then comm3(u) (:1395-1440). */
void orc_mg_psinv(int m, const double *r, double *u, const double c[4])
{
    double *r1 = malloc(sizeof(double) * m), *r2 = malloc(sizeof(double) * m);
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i2 = 1; i2 < m - 1; i2++) {
            for (int i1 = 0; i1 < m; i1++) {
                r1[i1] = r[at(m, i3, i2 - 1, i1)] + r[at(m, i3, i2 + 1, i1)] +
                         r[at(m, i3 - 1, i2, i1)] + r[at(m, i3 + 1, i2, i1)];
                r2[i1] = r[at(m, i3 - 1, i2 - 1, i1)] + r[at(m, i3 - 1, i2 + 1, i1)] +
                         r[at(m, i3 + 1, i2 - 1, i1)] + r[at(m, i3 + 1, i2 + 1, i1)];
            }
            for (int i1 = 1; i1 < m - 1; i1++)
                u[at(m, i3, i2, i1)] = u[at(m, i3, i2, i1)] + c[0] * r[at(m, i3, i2, i1)] +
                                       c[1] * (r[at(m, i3, i2, i1 - 1)] + r[at(m, i3, i2, i1 + 1)] + r1[i1]) +
                                       c[2] * (r2[i1] + r1[i1 - 1] + r1[i1 + 1]);
        }
    free(r1);
    free(r2);
    orc_mg_comm3(m, u);
}

/* s (side mj) = restriction of r (side mk = 2 mj - 2), then comm3(s)
 * (:1724-1790, the mk > 3 case: d = 1). */
void orc_mg_rprj3(int mk, const double *r, int mj, double *s)
{
    double *x1 = malloc(sizeof(double) * mk), *y1 = malloc(sizeof(double) * mk);
    for (int j3 = 1; j3 < mj - 1; j3++) {
        const int i3 = 2 * j3 - 1;
        for (int j2 = 1; j2 < mj - 1; j2++) {
            const int i2 = 2 * j2 - 1;
            for (int j1 = 1; j1 < mj; j1++) {
                const int i1 = 2 * j1 - 1;
                x1[i1] = r[at(mk, i3 + 1, i2, i1)] + r[at(mk, i3 + 1, i2 + 2, i1)] +
                         r[at(mk, i3, i2 + 1, i1)] + r[at(mk, i3 + 2, i2 + 1, i1)];
                y1[i1] = r[at(mk, i3, i2, i1)] + r[at(mk, i3 + 2, i2, i1)] +
                         r[at(mk, i3, i2 + 2, i1)] + r[at(mk, i3 + 2, i2 + 2, i1)];
            }
            for (int j1 = 1; j1 < mj - 1; j1++) {
                const int i1 = 2 * j1 - 1;
                const double y2 = r[at(mk, i3, i2, i1 + 1)] + r[at(mk, i3 + 2, i2, i1 + 1)] +
                                  r[at(mk, i3, i2 + 2, i1 + 1)] + r[at(mk, i3 + 2, i2 + 2, i1 + 1)];
                const double x2 = r[at(mk, i3 + 1, i2, i1 + 1)] + r[at(mk, i3 + 1, i2 + 2, i1 + 1)] +
                                  r[at(mk, i3, i2 + 1, i1 + 1)] + r[at(mk, i3 + 2, i2 + 1, i1 + 1)];
                s[at(mj, j3, j2, j1)] =
                    0.5 * r[at(mk, i3 + 1, i2 + 1, i1 + 1)] +
                    0.25 * (r[at(mk, i3 + 1, i2 + 1, i1)] + r[at(mk, i3 + 1, i2 + 1, i1 + 2)] + x2) +
                    0.125 * (x1[i1] + x1[i1 + 2] + y2) + 0.0625 * (y1[i1] + y1[i1 + 2]);
            }
        }
    }
    free(x1);
    free(y1);
    orc_mg_comm3(mj, s);
}

/* u (side mk = 2 mj - 2) += prolongation of z (side mj) (:836-890, the
 * branch for sides > 3, which every level of a power-of-two grid takes). */
void orc_mg_interp(int mj, const double *z, int mk, double *u)
{
    double *z1 = malloc(sizeof(double) * mj), *z2 = malloc(sizeof(double) * mj),
           *z3 = malloc(sizeof(double) * mj);
    for (int i3 = 0; i3 < mj - 1; i3++)
        for (int i2 = 0; i2 < mj - 1; i2++) {
            for (int i1 = 0; i1 < mj; i1++) {
                z1[i1] = z[at(mj, i3, i2 + 1, i1)] + z[at(mj, i3, i2, i1)];
                z2[i1] = z[at(mj, i3 + 1, i2, i1)] + z[at(mj, i3, i2, i1)];
                z3[i1] = z[at(mj, i3 + 1, i2 + 1, i1)] + z[at(mj, i3 + 1, i2, i1)] + z1[i1];
            }
            for (int i1 = 0; i1 < mj - 1; i1++) {
                double *p = &u[at(mk, 2 * i3, 2 * i2, 2 * i1)];
                p[0] = p[0] + z[at(mj, i3, i2, i1)];
                p[1] = p[1] + 0.5 * (z[at(mj, i3, i2, i1 + 1)] + z[at(mj, i3, i2, i1)]);
            }
            for (int i1 = 0; i1 < mj - 1; i1++) {
                double *p = &u[at(mk, 2 * i3, 2 * i2 + 1, 2 * i1)];
                p[0] = p[0] + 0.5 * z1[i1];
                p[1] = p[1] + 0.25 * (z1[i1] + z1[i1 + 1]);
            }
            for (int i1 = 0; i1 < mj - 1; i1++) {
                double *p = &u[at(mk, 2 * i3 + 1, 2 * i2, 2 * i1)];
                p[0] = p[0] + 0.5 * z2[i1];
                p[1] = p[1] + 0.25 * (z2[i1] + z2[i1 + 1]);
            }
            for (int i1 = 0; i1 < mj - 1; i1++) {
                double *p = &u[at(mk, 2 * i3 + 1, 2 * i2 + 1, 2 * i1)];
                p[0] = p[0] + 0.25 * z3[i1];
                p[1] = p[1] + 0.125 * (z3[i1] + z3[i1 + 1]);
            }
        }
    free(z1);
    free(z2);
    free(z3);
}

/* sqrt(sum r^2 / n^3) and max |r| over the interior (:1201-1230). */
void orc_mg_norm2u3(int m, const double *r, double *rnm2, double *rnmu)
{
    const int n = m - 2;
    double s = 0.0, mx = 0.0;
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i2 = 1; i2 < m - 1; i2++)
            for (int i1 = 1; i1 < m - 1; i1++) {
                const double x = r[at(m, i3, i2, i1)];
                s = s + x * x;
                if (fabs(x) > mx) mx = fabs(x);
            }
    *rnm2 = sqrt(s / ((double)n * n * n));
    *rnmu = mx;
}

/* A^n mod 2^46 by squaring, the LCG's own multiply (:1363-1380). */
static double lcg_power(double a, long long n)
{
    double result = 1.0, base = a;
    while (n != 0) {
        if (n % 2 == 1) (void)orc_randlc(&result, base);
        (void)orc_randlc(&base, base);
        n /= 2;
    }
    return result;
}

/* Keeps list[0..MM) sorted with the extreme at the end: a new candidate
 * replaces entry 0, then moves up while it beats its neighbour (:626-680).
 * larger: 1 for the largest values (ascending list), 0 for the smallest. */
static void sift(double *val, int (*pos)[3], int larger)
{
    for (int i = 0; i < MG_MM - 1; i++) {
        const int swap = larger ? (val[i] > val[i + 1]) : (val[i] < val[i + 1]);
        if (!swap) return;
        double t = val[i];
        val[i] = val[i + 1];
        val[i + 1] = t;
        for (int d = 0; d < 3; d++) {
            int q = pos[i][d];
            pos[i][d] = pos[i + 1][d];
            pos[i + 1][d] = q;
        }
    }
}

/* v = 0 except +1 at the ten largest and -1 at the ten smallest of the
 * LCG's values laid over the interior (seed 314159265, multiplier 5^13,
 * value of interior point (i1, i2, i3) = draw 1 + (i1-1) + n (i2-1) +
 * n^2 (i3-1)), then comm3 (:2175-2303).  plus / minus (nullable) receive
 * the (i1, i2, i3) of the +1 / -1 points in list order. */
void orc_mg_zran3(int m, double *v, int *plus, int *minus)
{
    const int n = m - 2;
    const double amult = 1220703125.0; /* 5^13 */
    const double a1 = lcg_power(amult, n), a2 = lcg_power(amult, (long long)n * n);
    memset(v, 0, sizeof(double) * (size_t)m * m * m);
    double x0 = 314159265.0;
    (void)orc_randlc(&x0, 1.0); /* the reference's start offset is A^0 for one process */
    for (int i3 = 1; i3 <= n; i3++) {
        double x1 = x0;
        for (int i2 = 1; i2 <= n; i2++) {
            double xx = x1;
            for (int i1 = 1; i1 <= n; i1++) v[at(m, i3, i2, i1)] = orc_randlc(&xx, amult);
            (void)orc_randlc(&x1, a1);
        }
        (void)orc_randlc(&x0, a2);
    }
    double hi[MG_MM], lo[MG_MM];
    int hp[MG_MM][3], lp[MG_MM][3];
    for (int i = 0; i < MG_MM; i++) {
        hi[i] = 0.0;
        lo[i] = 1.0;
        for (int d = 0; d < 3; d++) hp[i][d] = lp[i][d] = 0;
    }
    for (int i3 = 1; i3 < m - 1; i3++)
        for (int i2 = 1; i2 < m - 1; i2++)
            for (int i1 = 1; i1 < m - 1; i1++) {
                const double x = v[at(m, i3, i2, i1)];
                if (x > hi[0]) {
                    hi[0] = x;
                    hp[0][0] = i1;
                    hp[0][1] = i2;
                    hp[0][2] = i3;
                    sift(hi, hp, 1);
                }
                if (x < lo[0]) {
                    lo[0] = x;
                    lp[0][0] = i1;
                    lp[0][1] = i2;
                    lp[0][2] = i3;
                    sift(lo, lp, 0);
                }
            }
    memset(v, 0, sizeof(double) * (size_t)m * m * m);
    /* -1 points first, then +1 (:2292-2297); every candidate is real here
     * (values lie strictly inside (0, 1)) */
    for (int i = MG_MM - 1; i >= 0; i--) v[at(m, lp[i][2], lp[i][1], lp[i][0])] = -1.0;
    for (int i = MG_MM - 1; i >= 0; i--) v[at(m, hp[i][2], hp[i][1], hp[i][0])] = +1.0;
    for (int i = 0; i < MG_MM; i++)
        for (int d = 0; d < 3; d++) {
            if (plus) plus[3 * i + d] = hp[i][d];
            if (minus) minus[3 * i + d] = lp[i][d];
        }
    orc_mg_comm3(m, v);
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* The benchmark on a 2^lt cube: u = 0, v = zran3, then main's timed
 * region -- resid, norm, nit x (mg3P, resid), norm -- with the smoother of
 * set `smoother` (0: classes S/W/A, 1: the others).  rnm2 / rnmu of the
 * final residual; u_out / r_out (nullable, (2^lt + 2)^3 doubles) the top
 * grids; *seconds the wall time of the timed region (nullable). */
int orc_mg_run(int lt, int nit, int smoother, double *rnm2, double *rnmu, double *u_out,
               double *r_out, double *seconds)
{
    if (lt < 2 || lt > 11 || nit < 0) return 1;
    const double a[4] = {-8.0 / 3.0, 0.0, 1.0 / 6.0, 1.0 / 12.0};
    const double ca[4] = {-3.0 / 8.0, 1.0 / 32.0, -1.0 / 64.0, 0.0};
    const double cb[4] = {-3.0 / 17.0, 1.0 / 33.0, -1.0 / 61.0, 0.0};
    const double *c = smoother ? cb : ca;
    double *u[12] = {0}, *r[12] = {0}, *v = NULL;
    int m[12];
    int st = 0;
    for (int k = 1; k <= lt; k++) {
        m[k] = (1 << k) + 2;
        const size_t cells = (size_t)m[k] * m[k] * m[k];
        u[k] = calloc(cells, sizeof(double));
        r[k] = calloc(cells, sizeof(double));
        if (!u[k] || !r[k]) st = 2;
    }
    const size_t top = (size_t)m[lt] * m[lt] * m[lt];
    v = calloc(top, sizeof(double));
    if (!v) st = 2;
    if (!st) {
        orc_mg_zran3(m[lt], v, NULL, NULL);
        const double t0 = now_s();
        double s2, su;
        orc_mg_resid(m[lt], u[lt], v, r[lt], a);
        orc_mg_norm2u3(m[lt], r[lt], &s2, &su);
        for (int it = 0; it < nit; it++) {
            for (int k = lt; k >= 2; k--) orc_mg_rprj3(m[k], r[k], m[k - 1], r[k - 1]);
            memset(u[1], 0, sizeof(double) * (size_t)m[1] * m[1] * m[1]);
            orc_mg_psinv(m[1], r[1], u[1], c);
            for (int k = 2; k <= lt - 1; k++) {
                memset(u[k], 0, sizeof(double) * (size_t)m[k] * m[k] * m[k]);
                orc_mg_interp(m[k - 1], u[k - 1], m[k], u[k]);
                orc_mg_resid(m[k], u[k], r[k], r[k], a);
                orc_mg_psinv(m[k], r[k], u[k], c);
            }
            orc_mg_interp(m[lt - 1], u[lt - 1], m[lt], u[lt]);
            orc_mg_resid(m[lt], u[lt], v, r[lt], a);
            orc_mg_psinv(m[lt], r[lt], u[lt], c);
            orc_mg_resid(m[lt], u[lt], v, r[lt], a);
        }
        orc_mg_norm2u3(m[lt], r[lt], rnm2, rnmu);
        if (seconds) *seconds = now_s() - t0;
        if (u_out) memcpy(u_out, u[lt], sizeof(double) * top);
        if (r_out) memcpy(r_out, r[lt], sizeof(double) * top);
    }
    for (int k = 1; k <= lt; k++) {
        free(u[k]);
        free(r[k]);
    }
    free(v);
    return st;
}

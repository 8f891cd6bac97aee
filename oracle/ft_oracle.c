/*
 * ft_oracle.c -- CPU oracle for the NPB FT path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle of the tests, never the
 * product: only tests/, __graft_entry__.smoke() and the cpu_baseline legs of
 * bench.py may load liboracle.so.  libcgb.so neither links nor calls anything
 * here.
 *
 * It restates, in plain C, the FT benchmark of the GMAP/NPB-GPU reference
 * (paths relative to that project, CUDA/FT/ft.cu):
 *   - initial conditions :1188-1227  element e = x + nx y + nx ny z holds the
 *                        LCG's draws 2e+1 (real) and 2e+2 (imaginary) after
 *                        the seed 314159265 (multiplier 5^13; the planes'
 *                        seeds by ipow46 :1369-1398, vranlc :1834-1857)
 *   - index map          :1166-1186  twiddle = exp(AP (i'^2 + j'^2 + k'^2)),
 *                        i' the signed frequency, AP = -4 alpha pi^2
 *   - roots table        :1280-1310  u[ln + i] = exp(i pi i / ln)
 *   - cfftz / fftz2      :963-1057   the radix-2 Stockham transform of one
 *                        line (is = 1: sum x_j exp(+2 pi i jk/n); is = -1:
 *                        exp(-...)), unnormalised, natural order
 *   - fft                :1258-1278  dir 1: x, y, z lines with is = 1;
 *                        dir -1: z, y, x lines with is = -1
 *   - evolve             :1245-1256  u0 *= twiddle, u1 = u0
 *   - checksum           :1124-1153  the sum of u1 at (j mod nx, 3j mod ny,
 *                        5j mod nz), j = 1 .. 1024, over nx ny nz
 *   - main               :335-420    forward transform of the initial
 *                        conditions, then niter x (evolve, inverse
 *                        transform, checksum)
 * Arrays are interleaved (real, imaginary) doubles, x fastest.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

double orc_randlc(double *x, double a); /* cg_oracle.c */

#define FT_SEED 314159265.0
#define FT_MULT 1220703125.0
#define FT_ALPHA 1.0e-6
#define FT_PI 3.141592653589793238
#define FT_AP (-4.0 * FT_ALPHA * FT_PI * FT_PI)
#define FT_POINTS 1024

/* a^exponent mod 2^46 by the reference's halving (ft.cu:1369-1398) */
static double ipow46(double a, long long exponent)
{
    if (exponent == 0) return 1.0;
    double q = a, r = 1.0;
    long long n = exponent;
    while (n > 1) {
        if ((n / 2) * 2 == n) {
            orc_randlc(&q, q);
            n /= 2;
        } else {
            orc_randlc(&r, q);
            n -= 1;
        }
    }
    orc_randlc(&r, q);
    return r;
}

void orc_ft_initial(int nx, int ny, int nz, double *u)
{
    double start = FT_SEED;
    orc_randlc(&start, ipow46(FT_MULT, 0));
    const double an = ipow46(FT_MULT, 2LL * nx * ny);
    for (int z = 0; z < nz; z++) {
        if (z > 0) orc_randlc(&start, an);
        double x0 = start;
        for (int y = 0; y < ny; y++) {
            double *row = u + 2 * ((size_t)y * nx + (size_t)z * nx * ny);
            for (int i = 0; i < 2 * nx; i++) row[i] = orc_randlc(&x0, FT_MULT);
        }
    }
}

void orc_ft_indexmap(int nx, int ny, int nz, double *tw)
{
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const int kk = ((k + nz / 2) % nz) - nz / 2, jj = ((j + ny / 2) % ny) - ny / 2;
                const int ii = ((i + nx / 2) % nx) - nx / 2;
                const int kj2 = jj * jj + kk * kk;
                tw[i + (size_t)j * nx + (size_t)k * nx * ny] = exp(FT_AP * (double)(ii * ii + kj2));
            }
}

static int ilog2i(int n)
{
    int m = 0;
    while ((1 << m) < n) m++;
    return m;
}

/* u[2 (ln + i)] = cos, sin (i pi / ln) for every level ln < n (ft.cu:1280-1310) */
static void roots(int n, double *u)
{
    const int m = ilog2i(n);
    u[0] = (double)m;
    u[1] = 0.0;
    int ku = 2, ln = 1;
    for (int j = 1; j <= m; j++) {
        const double t = FT_PI / ln;
        for (int i = 0; i < ln; i++) {
            const double ti = i * t;
            u[2 * (i + ku - 1)] = cos(ti);
            u[2 * (i + ku - 1) + 1] = sin(ti);
        }
        ku += ln;
        ln *= 2;
    }
}

/* one radix-2 Stockham stage l of an n = 2^m line, x -> y (ft.cu:1004-1057) */
static void fftz2(int is, int l, int m, int n, const double *u, const double *x, double *y)
{
    const int n1 = n / 2, lk = 1 << (l - 1), li = 1 << (m - l), lj = 2 * lk, ku = li;
    for (int i = 0; i < li; i++) {
        const int i11 = i * lk, i12 = i11 + n1, i21 = i * lj, i22 = i21 + lk;
        const double ur = u[2 * (ku + i)], ui = is >= 1 ? u[2 * (ku + i) + 1] : -u[2 * (ku + i) + 1];
        for (int k = 0; k < lk; k++) {
            const double x11r = x[2 * (i11 + k)], x11i = x[2 * (i11 + k) + 1];
            const double x21r = x[2 * (i12 + k)], x21i = x[2 * (i12 + k) + 1];
            y[2 * (i21 + k)] = x11r + x21r;
            y[2 * (i21 + k) + 1] = x11i + x21i;
            y[2 * (i22 + k)] = ur * (x11r - x21r) - ui * (x11i - x21i);
            y[2 * (i22 + k) + 1] = ur * (x11i - x21i) + ui * (x11r - x21r);
        }
    }
}

/* the line transform in x (y: scratch) (ft.cu:963-1002) */
static void cfftz(int is, int m, int n, const double *u, double *x, double *y)
{
    for (int l = 1; l <= m; l += 2) {
        fftz2(is, l, m, n, u, x, y);
        if (l == m) {
            memcpy(x, y, sizeof(double) * 2 * (size_t)n);
            return;
        }
        fftz2(is, l + 1, m, n, u, y, x);
    }
}

/* every line along `axis` (0 x, 1 y, 2 z) transformed in place */
static void cffts(int is, int axis, int nx, int ny, int nz, const double *u, double *a)
{
    const int dims[3] = {nx, ny, nz};
    const int n = dims[axis], m = ilog2i(n);
    const size_t stride = axis == 0 ? 1 : axis == 1 ? (size_t)nx : (size_t)nx * ny;
    double *x = malloc(sizeof(double) * 2 * (size_t)n), *y = malloc(sizeof(double) * 2 * (size_t)n);
    for (int c = 0; c < nz; c++)
        for (int b = 0; b < ny; b++)
            for (int a0 = 0; a0 < nx; a0++) {
                const int idx[3] = {a0, b, c};
                if (idx[axis] != 0) continue; /* one line per start point */
                const size_t base = (size_t)a0 + (size_t)b * nx + (size_t)c * nx * ny;
                for (int k = 0; k < n; k++) {
                    x[2 * k] = a[2 * (base + k * stride)];
                    x[2 * k + 1] = a[2 * (base + k * stride) + 1];
                }
                cfftz(is, m, n, u, x, y);
                for (int k = 0; k < n; k++) {
                    a[2 * (base + k * stride)] = x[2 * k];
                    a[2 * (base + k * stride) + 1] = x[2 * k + 1];
                }
            }
    free(x);
    free(y);
}

/* the 3-D transform in place: dir 1 (x, y, z; is = 1), dir -1 (z, y, x; is = -1) */
void orc_ft_fft3d(int dir, int nx, int ny, int nz, double *a)
{
    int maxdim = nx > ny ? nx : ny;
    if (nz > maxdim) maxdim = nz;
    double *u = malloc(sizeof(double) * 2 * (size_t)maxdim);
    roots(maxdim, u);
    if (dir == 1) {
        cffts(1, 0, nx, ny, nz, u, a);
        cffts(1, 1, nx, ny, nz, u, a);
        cffts(1, 2, nx, ny, nz, u, a);
    } else {
        cffts(-1, 2, nx, ny, nz, u, a);
        cffts(-1, 1, nx, ny, nz, u, a);
        cffts(-1, 0, nx, ny, nz, u, a);
    }
    free(u);
}

/* The benchmark; sums: 2 niter doubles (real, imaginary per iteration);
 * u1_out (nullable): the last inverse transform, 2 nx ny nz doubles.
 * Returns 0, or -1 when out of memory. */
int orc_ft_run(int nx, int ny, int nz, int niter, double *sums, double *u1_out)
{
    const size_t nt = (size_t)nx * ny * nz;
    double *u0 = malloc(sizeof(double) * 2 * nt), *u1 = malloc(sizeof(double) * 2 * nt);
    double *tw = malloc(sizeof(double) * nt);
    if (!u0 || !u1 || !tw) {
        free(u0);
        free(u1);
        free(tw);
        return -1;
    }
    orc_ft_indexmap(nx, ny, nz, tw);
    orc_ft_initial(nx, ny, nz, u1);
    memcpy(u0, u1, sizeof(double) * 2 * nt);
    orc_ft_fft3d(1, nx, ny, nz, u0);
    for (int it = 1; it <= niter; it++) {
        for (size_t e = 0; e < nt; e++) {
            u0[2 * e] *= tw[e];
            u0[2 * e + 1] *= tw[e];
        }
        memcpy(u1, u0, sizeof(double) * 2 * nt);
        orc_ft_fft3d(-1, nx, ny, nz, u1);
        double cr = 0.0, ci = 0.0;
        for (int j = 1; j <= FT_POINTS; j++) {
            const size_t e = (size_t)(j % nx) + (size_t)(3 * j % ny) * nx + (size_t)(5 * j % nz) * nx * ny;
            cr += u1[2 * e];
            ci += u1[2 * e + 1];
        }
        sums[2 * (it - 1)] = cr / (double)nt;
        sums[2 * (it - 1) + 1] = ci / (double)nt;
    }
    if (u1_out) memcpy(u1_out, u1, sizeof(double) * 2 * nt);
    free(u0);
    free(u1);
    free(tw);
    return 0;
}

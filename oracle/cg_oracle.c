/*
 * cg_oracle.c -- CPU oracle for the NPB CG inverse-power-iteration path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle of the tests, never the product:
 * only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs
 * of bench.py may load liboracle.so.  The shipped library (libcgb.so) neither
 * links nor calls anything here, and fails loudly when its CUDA code is
 * missing instead of falling back to this file.
 *
 * It restates, in plain C, the algorithm of the GMAP/NPB-GPU reference
 * (paths relative to that project):
 *   - randlc            CUDA/common/c_randdp.cpp:84-114
 *   - icnvrt            CUDA/CG/cg.cu:1272-1274
 *   - sprnvc            CUDA/CG/cg.cu:1798-1833
 *   - vecset            CUDA/CG/cg.cu:1841-1857
 *   - makea             CUDA/CG/cg.cu:1303-1368 (+ the discarded draw of main, cg.cu:406-408)
 *   - sparse            CUDA/CG/cg.cu:1611-1785
 *   - conj_grad         CUDA/CG/cg.cu:653-801
 *   - outer loop        CUDA/CG/cg.cu:458-520 (zeta = shift + 1/(x.z); x = z/||z||)
 *   - OpenMP variant    the same conj_grad with `omp parallel for` + reductions
 *                       (the reference ships no OpenMP CG; this is a restatement)
 *
 * Parity is pinned: tests compare this file with the reference's own code
 * compiled into oracle/_ref/ (CSR hash, zeta traces) and with the
 * verification zetas hard-coded in CUDA/CG/cg.cu:373-396.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp -shared -fPIC (see oracle/Makefile).
 * No FMA contraction: the generator's arithmetic must round exactly like the
 * reference's separate multiply and add.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2
#define ORC_ECAP 3

/* ------------------------------------------------------------------ */
/* LCG: x <- a*x mod 2^46, evaluated with 23-bit halves held in
 * doubles; returns x * 2^-46.  Follows c_randdp.cpp:84-114 step by step
 * (every intermediate is an exact integer below 2^53).                */
double orc_randlc(double *x, double a)
{
    const double two_m23 = 1.0 / 8388608.0;          /* 2^-23 */
    const double two_23 = 8388608.0;                 /* 2^23  */
    const double two_m46 = two_m23 * two_m23;        /* 2^-46 */
    const double two_46 = two_23 * two_23;           /* 2^46  */

    double a_hi = (double)(int)(two_m23 * a);
    double a_lo = a - two_23 * a_hi;
    double x_hi = (double)(int)(two_m23 * (*x));
    double x_lo = (*x) - two_23 * x_hi;
    double cross = a_hi * x_lo + a_lo * x_hi;         /* < 2^47 */
    double cross_hi = (double)(int)(two_m23 * cross);
    double cross_lo = cross - two_23 * cross_hi;      /* cross mod 2^23 */
    double full = two_23 * cross_lo + a_lo * x_lo;    /* < 2^47 */
    double wrap = (double)(int)(two_m46 * full);
    *x = full - two_46 * wrap;                        /* mod 2^46 */
    return two_m46 * (*x);
}

/* ------------------------------------------------------------------ */
/* One sparse random vector: `nz` distinct 1-based positions in 1..n,
 * each with a uniform value; rejected draws (position > n or repeated)
 * still consume two LCG numbers.  cg.cu:1798-1833 (+ icnvrt :1272).   */
static void orc_sprnvc(int n, int nz, int nn1, double *v, int *iv,
                       double *tran, double amult)
{
    int have = 0;
    while (have < nz) {
        double value = orc_randlc(tran, amult);
        double where = orc_randlc(tran, amult);
        int pos = (int)(nn1 * where) + 1;
        if (pos > n)
            continue;
        int dup = 0;
        for (int t = 0; t < have; t++)
            if (iv[t] == pos) { dup = 1; break; }
        if (dup)
            continue;
        v[have] = value;
        iv[have] = pos;
        have++;
    }
}

/* Force element `pos` (1-based) of the sparse vector to `val`,
 * appending it when absent.  cg.cu:1841-1857.                          */
static void orc_vecset(double *v, int *iv, int *nzv, int pos, double val)
{
    int found = 0;
    for (int t = 0; t < *nzv; t++)
        if (iv[t] == pos) { v[t] = val; found = 1; }
    if (!found) {
        v[*nzv] = val;
        iv[*nzv] = pos;
        (*nzv)++;
    }
}

/* Upper bound on the CSR length the reference allocates: NZ = n(nonzer+1)^2
 * (cg.cu:81).                                                          */
long long orc_nz_bound(int n, int nonzer)
{
    return (long long)n * (nonzer + 1) * (nonzer + 1);
}

/* ------------------------------------------------------------------ */
/* makea + sparse.  `seed` is the LCG state main() starts from
 * (314159265 for every NPB class, cg.cu:405); the first draw is thrown
 * away exactly as main() does (cg.cu:406-408).  Writes 0-based CSR with
 * sorted, unique columns; returns the number of stored entries through
 * *nnz_out.  Duplicate (row, col) contributions are summed in the order
 * the reference's insertion loop meets them (vector i, then nza, then
 * nzrow; cg.cu:1696-1756).                                            */
int orc_makea(int n, int nonzer, double rcond, double shift, double seed,
              int *rowstr, int *colidx, double *a, long long cap,
              long long *nnz_out)
{
    if (n < 1 || nonzer < 1 || nonzer >= n)
        return ORC_EINVAL;
    const double amult = 1220703125.0;
    double tran = seed;
    (void)orc_randlc(&tran, amult);              /* discarded, cg.cu:408 */

    int nn1 = 1;                                  /* cg.cu:1327-1330 */
    do { nn1 *= 2; } while (nn1 < n);

    const int w = nonzer + 1;
    int *arow = (int *)malloc(sizeof(int) * (size_t)n);
    int *acol = (int *)malloc(sizeof(int) * (size_t)n * w);
    double *aelt = (double *)malloc(sizeof(double) * (size_t)n * w);
    double *vc = (double *)malloc(sizeof(double) * (size_t)w);
    int *ivc = (int *)malloc(sizeof(int) * (size_t)w);
    if (!arow || !acol || !aelt || !vc || !ivc) {
        free(arow); free(acol); free(aelt); free(vc); free(ivc);
        return ORC_ENOMEM;
    }
    for (int i = 0; i < n; i++) {                 /* cg.cu:1336-1346 */
        int nzv = nonzer;
        orc_sprnvc(n, nzv, nn1, vc, ivc, &tran, amult);
        orc_vecset(vc, ivc, &nzv, i + 1, 0.5);
        arow[i] = nzv;
        for (int t = 0; t < nzv; t++) {
            acol[(size_t)i * w + t] = ivc[t] - 1;
            aelt[(size_t)i * w + t] = vc[t];
        }
    }
    free(vc);
    free(ivc);

    /* Slots per row: row j receives arow[i] candidates from every vector
     * i that contains j (cg.cu:1649-1662).                             */
    long long *slot = (long long *)calloc((size_t)n + 1, sizeof(long long));
    int *used = (int *)calloc((size_t)n, sizeof(int));
    if (!slot || !used) {
        free(slot); free(used); free(arow); free(acol); free(aelt);
        return ORC_ENOMEM;
    }
    for (int i = 0; i < n; i++)
        for (int t = 0; t < arow[i]; t++)
            slot[acol[(size_t)i * w + t] + 1] += arow[i];
    for (int j = 0; j < n; j++)
        slot[j + 1] += slot[j];
    long long total = slot[n];
    int *scol = (int *)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    double *sval = (double *)malloc(sizeof(double) * (size_t)(total > 0 ? total : 1));
    if (!scol || !sval) {
        free(scol); free(sval); free(slot); free(used);
        free(arow); free(acol); free(aelt);
        return ORC_ENOMEM;
    }

    /* Ordered insertion with duplicate summation (cg.cu:1694-1756).
     * size runs geometrically from 1 down to rcond: size *= ratio after
     * each vector, ratio = rcond^(1/n) from the host libm.             */
    double size = 1.0;
    const double ratio = pow(rcond, 1.0 / (double)n);
    for (int i = 0; i < n; i++) {
        for (int s = 0; s < arow[i]; s++) {
            int row = acol[(size_t)i * w + s];
            double scale = size * aelt[(size_t)i * w + s];
            int *rc = scol + slot[row];
            double *rv = sval + slot[row];
            for (int u = 0; u < arow[i]; u++) {
                int col = acol[(size_t)i * w + u];
                double va = aelt[(size_t)i * w + u] * scale;
                if (col == row && row == i) {
                    va = va + rcond;              /* (va + rcond) - shift, */
                    va = va - shift;              /* left to right          */
                }
                /* first position whose column is >= col */
                int k = 0;
                while (k < used[row] && rc[k] < col)
                    k++;
                if (k < used[row] && rc[k] == col) {
                    rv[k] = rv[k] + va;
                } else {
                    for (int m = used[row]; m > k; m--) {
                        rc[m] = rc[m - 1];
                        rv[m] = rv[m - 1];
                    }
                    rc[k] = col;
                    rv[k] = 0.0;
                    rv[k] = rv[k] + va;
                    used[row]++;
                }
            }
        }
        size = size * ratio;
    }

    /* Compaction of the filled slots (cg.cu:1763-1784). */
    long long out = 0;
    rowstr[0] = 0;
    for (int j = 0; j < n; j++) {
        if (out + used[j] > cap) {
            free(scol); free(sval); free(slot); free(used);
            free(arow); free(acol); free(aelt);
            return ORC_ECAP;
        }
        for (int k = 0; k < used[j]; k++) {
            colidx[out] = scol[slot[j] + k];
            a[out] = sval[slot[j] + k];
            out++;
        }
        rowstr[j + 1] = (int)out;
    }
    *nnz_out = out;
    free(scol); free(sval); free(slot); free(used);
    free(arow); free(acol); free(aelt);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* FNV-1a-64 over the CSR: rowstr[0..n], then for each entry its column
 * and the 8 bytes of its value read as a u64.  Ints are widened to u64. */
uint64_t orc_csr_hash(int n, const int *rowstr, const int *colidx, const double *a)
{
    uint64_t h = 0xcbf29ce484222325ULL;
    const uint64_t prime = 0x100000001b3ULL;
    for (int j = 0; j <= n; j++) {
        h ^= (uint64_t)(int64_t)rowstr[j];
        h *= prime;
    }
    for (int k = 0; k < rowstr[n]; k++) {
        uint64_t bits;
        memcpy(&bits, &a[k], 8);
        h ^= (uint64_t)(int64_t)colidx[k];
        h *= prime;
        h ^= bits;
        h *= prime;
    }
    return h;
}

/* ------------------------------------------------------------------ */
/* y = A x over the CSR, each row summed left to right (cg.cu:691-697). */
void orc_spmv(int n, const int *rowstr, const int *colidx, const double *a,
              const double *x, double *y)
{
    for (int j = 0; j < n; j++) {
        double sum = 0.0;
        for (int k = rowstr[j]; k < rowstr[j + 1]; k++)
            sum = sum + a[k] * x[colidx[k]];
        y[j] = sum;
    }
}

/* conj_grad (cg.cu:653-801): `cgitmax` CG iterations on A z = x from
 * z = 0 (the reference fixes cgitmax = 25), then rnorm = ||x - A z||.
 * On return r holds A z, p and q the last search direction and A p.
 * Vectors hold at least n+1 entries; entry n is initialised as the
 * reference does (cg.cu:670-675) but never enters a dot product.       */
void orc_conj_grad(int n, const int *rowstr, const int *colidx, const double *a,
                   const double *x, double *z, double *p, double *q, double *r,
                   int cgitmax, double *rnorm)
{
    double rho = 0.0;
    for (int j = 0; j < n + 1; j++) {
        q[j] = 0.0;
        z[j] = 0.0;
        r[j] = x[j];
        p[j] = r[j];
    }
    for (int j = 0; j < n; j++)
        rho = rho + r[j] * r[j];
    for (int it = 1; it <= cgitmax; it++) {
        orc_spmv(n, rowstr, colidx, a, p, q);
        double d = 0.0;
        for (int j = 0; j < n; j++)
            d = d + p[j] * q[j];
        double alpha = rho / d;
        double rho0 = rho;
        rho = 0.0;
        for (int j = 0; j < n; j++) {
            z[j] = z[j] + alpha * p[j];
            r[j] = r[j] - alpha * q[j];
        }
        for (int j = 0; j < n; j++)
            rho = rho + r[j] * r[j];
        double beta = rho / rho0;
        for (int j = 0; j < n; j++)
            p[j] = r[j] + beta * p[j];
    }
    orc_spmv(n, rowstr, colidx, a, z, r);
    double sum = 0.0;
    for (int j = 0; j < n; j++) {
        double d = x[j] - r[j];
        sum = sum + d * d;
    }
    *rnorm = sqrt(sum);
}

/* The same conj_grad with every row/vector loop split across OpenMP
 * threads (reductions in OpenMP's order, so results agree with the
 * serial form to rounding, not bitwise).                              */
static void orc_conj_grad_omp(int n, const int *rowstr, const int *colidx,
                              const double *a, const double *x, double *z,
                              double *p, double *q, double *r, int cgitmax,
                              double *rnorm)
{
    double rho = 0.0;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n + 1; j++) {
        q[j] = 0.0;
        z[j] = 0.0;
        r[j] = x[j];
        p[j] = x[j];
    }
#pragma omp parallel for schedule(static) reduction(+ : rho)
    for (int j = 0; j < n; j++)
        rho += r[j] * r[j];
    for (int it = 1; it <= cgitmax; it++) {
        double d = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : d)
        for (int j = 0; j < n; j++) {
            double sum = 0.0;
            for (int k = rowstr[j]; k < rowstr[j + 1]; k++)
                sum = sum + a[k] * p[colidx[k]];
            q[j] = sum;
            d += p[j] * sum;
        }
        double alpha = rho / d;
        double rho0 = rho;
        rho = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rho)
        for (int j = 0; j < n; j++) {
            z[j] = z[j] + alpha * p[j];
            r[j] = r[j] - alpha * q[j];
            rho += r[j] * r[j];
        }
        double beta = rho / rho0;
#pragma omp parallel for schedule(static)
        for (int j = 0; j < n; j++)
            p[j] = r[j] + beta * p[j];
    }
    double sum = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : sum)
    for (int j = 0; j < n; j++) {
        double s = 0.0;
        for (int k = rowstr[j]; k < rowstr[j + 1]; k++)
            s = s + a[k] * z[colidx[k]];
        r[j] = s;
        double d = x[j] - s;
        sum += d * d;
    }
    *rnorm = sqrt(sum);
}

static double orc_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* The inverse power iteration (cg.cu:485-520): x = 1, then per outer
 * step z = conj_grad(x), zeta = shift + 1/(x.z), x = z/||z||.  Writes
 * per-step zeta and rnorm; `threads` <= 1 runs the serial conj_grad,
 * otherwise the OpenMP one on that many threads.  Returns the wall
 * seconds of the outer loop through *seconds (may be NULL).  x_out
 * (may be NULL) receives the final x (n entries).                      */
int orc_power_iterate(int n, const int *rowstr, const int *colidx, const double *a,
                      double shift, int niter, int cgitmax, int threads,
                      double *zeta_trace, double *rnorm_trace, double *x_out,
                      double *seconds)
{
    double *buf = (double *)malloc(sizeof(double) * 5 * ((size_t)n + 2));
    if (!buf)
        return ORC_ENOMEM;
    double *x = buf, *z = x + n + 2, *p = z + n + 2, *q = p + n + 2, *r = q + n + 2;
    for (int j = 0; j < n + 1; j++)
        x[j] = 1.0;
#ifdef _OPENMP
    if (threads > 1)
        omp_set_num_threads(threads);
#endif
    double t0 = orc_now();
    for (int it = 0; it < niter; it++) {
        double rnorm;
        if (threads > 1)
            orc_conj_grad_omp(n, rowstr, colidx, a, x, z, p, q, r, cgitmax, &rnorm);
        else
            orc_conj_grad(n, rowstr, colidx, a, x, z, p, q, r, cgitmax, &rnorm);
        double t1 = 0.0, t2 = 0.0;
        for (int j = 0; j < n; j++) {
            t1 = t1 + x[j] * z[j];
            t2 = t2 + z[j] * z[j];
        }
        t2 = 1.0 / sqrt(t2);
        double zeta = shift + 1.0 / t1;
        for (int j = 0; j < n; j++)
            x[j] = t2 * z[j];
        if (zeta_trace)
            zeta_trace[it] = zeta;
        if (rnorm_trace)
            rnorm_trace[it] = rnorm;
    }
    if (seconds)
        *seconds = orc_now() - t0;
    if (x_out)
        memcpy(x_out, x, sizeof(double) * (size_t)n);
    free(buf);
    return ORC_OK;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

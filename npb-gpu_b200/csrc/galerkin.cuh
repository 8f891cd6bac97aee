// galerkin.cuh -- the small dense part of the Galerkin start on previous
// power-iteration iterates, shared by the single-system and batched solvers.
//
// The iterates x_j of the inverse power iteration span a Krylov space of A
// (x_{j+1} is A^-1 x_j scaled), and A x_j is the previous step's end-of-
// solve product A z scaled, so the Galerkin solution of A z = x on the last
// v iterates costs dot products only: with V = [x_k, ..., x_{k-v+1}] and
// W = A V, solve (V^T A V) y = V^T x and start from z0 = V y, A z0 = W y.
#pragma once

#include <cuda_runtime.h>

namespace cgb {

// At most kMaxRecycle previous iterates; the Gram values x_a . A x_b
// (a <= b, packed by b) followed by the right-hand sides x_a . x.
constexpr int kMaxRecycle = 4;
constexpr int kGramPairs = kMaxRecycle * (kMaxRecycle + 1) / 2;
constexpr int kGramValues = kGramPairs + kMaxRecycle;

__device__ __forceinline__ int gram_index(int a, int b)  // a <= b < v, packed by b
{
    return b * (b + 1) / 2 + a;
}

// Coefficients y from the Gram totals g[] (pairs at gram_index, right-hand
// sides at kGramPairs + b); one thread.  Cholesky of N = -V^T A V (SPD for
// negative definite A); a direction whose pivot falls below tau N_00 is left
// out, tau raised until the combination stays within 100x of its A-norm (so
// W y is accurate to ~1e-14 of x).  Returns the number of directions kept.
static __device__ __noinline__ int galerkin_solve(const double *g, int v, double *y)
{
    constexpr int R = kMaxRecycle;
    // every loop has the fixed trip count R and predicates on v, so the
    // small arrays stay in registers; a left-out direction has zero L, u, y
    double N[R][R], c[R];
#pragma unroll
    for (int b = 0; b < R; b++) {
#pragma unroll
        for (int a = 0; a <= b; a++) {
            const double e = (b < v) ? -g[gram_index(a, b)] : 0.0;
            N[a][b] = e;
            N[b][a] = e;
        }
        c[b] = (b < v) ? g[kGramPairs + b] : 0.0;
    }
    if (!(N[0][0] > 0.0)) {
#pragma unroll
        for (int a = 0; a < R; a++)
            if (a < v) y[a] = 0.0;
        return 0;
    }
    const double taus[4] = {1e-12, 1e-10, 1e-8, 1e-6};
    double yy[R];
    int kept = 1;
    for (int t = 0; t < 5; t++) {
        // t == 4: the first direction alone
        const double tau = t < 4 ? taus[t] * N[0][0] : 1e300;
        double L[R][R], u[R];
        bool keep[R];
        kept = 0;
#pragma unroll
        for (int i = 0; i < R; i++) {
            double d = N[i][i];
#pragma unroll
            for (int k = 0; k < i; k++) d -= L[i][k] * L[i][k];
            keep[i] = (i < v) && ((i == 0) || d > tau);
            kept += keep[i] ? 1 : 0;
            const double lii = keep[i] ? sqrt(d) : 1.0;
            L[i][i] = keep[i] ? lii : 0.0;
#pragma unroll
            for (int j = i + 1; j < R; j++) {
                double e = N[j][i];
#pragma unroll
                for (int k = 0; k < i; k++) e -= L[j][k] * L[i][k];
                L[j][i] = keep[i] ? e / lii : 0.0;
            }
#pragma unroll
            for (int j = 0; j < i; j++) L[j][i] = 0.0;
        }
        // N y = -c on the kept directions
#pragma unroll
        for (int i = 0; i < R; i++) {
            double e = -c[i];
#pragma unroll
            for (int k = 0; k < i; k++) e -= L[i][k] * u[k];
            u[i] = keep[i] ? e / L[i][i] : 0.0;
        }
#pragma unroll
        for (int i = R - 1; i >= 0; i--) {
            double e = u[i];
#pragma unroll
            for (int j = i + 1; j < R; j++) e -= L[j][i] * yy[j];
            yy[i] = keep[i] ? e / L[i][i] : 0.0;
        }
        // growth of the combination in the A-norm: sum |y_a| ||x_a||_A
        // against ||z0||_A; accept when the cancellation is mild
        double num = 0.0, zA = 0.0;
#pragma unroll
        for (int a = 0; a < R; a++) {
            num += (a < v) ? fabs(yy[a]) * sqrt(N[a][a]) : 0.0;
#pragma unroll
            for (int b = 0; b < R; b++) zA += yy[a] * N[a][b] * yy[b];
        }
        if (t == 4 || (zA > 0.0 && num <= 100.0 * sqrt(zA) && isfinite(num))) break;
    }
#pragma unroll
    for (int a = 0; a < R; a++)
        if (a < v) y[a] = yy[a];
    return kept;
}

}  // namespace cgb

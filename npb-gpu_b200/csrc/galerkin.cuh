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
    double N[kMaxRecycle][kMaxRecycle], c[kMaxRecycle];
    for (int b = 0; b < v; b++) {
        for (int a = 0; a <= b; a++) N[a][b] = N[b][a] = -g[gram_index(a, b)];
        c[b] = g[kGramPairs + b];
    }
    if (!(N[0][0] > 0.0)) {
        for (int a = 0; a < v; a++) y[a] = 0.0;
        return 0;
    }
    const double taus[4] = {1e-12, 1e-10, 1e-8, 1e-6};
    for (int t = 0; t < 5; t++) {
        // t == 4: the first direction alone
        const double tau = t < 4 ? taus[t] * N[0][0] : 1e300;
        double L[kMaxRecycle][kMaxRecycle], u[kMaxRecycle];
        bool keep[kMaxRecycle];
        int kept = 0;
        for (int i = 0; i < v; i++) {
            double d = N[i][i];
            for (int k = 0; k < i; k++)
                if (keep[k]) d -= L[i][k] * L[i][k];
            keep[i] = (i == 0) || d > tau;
            if (!keep[i]) continue;
            kept++;
            L[i][i] = sqrt(d);
            for (int j = i + 1; j < v; j++) {
                double e = N[j][i];
                for (int k = 0; k < i; k++)
                    if (keep[k]) e -= L[j][k] * L[i][k];
                L[j][i] = e / L[i][i];
            }
        }
        // N y = -c on the kept directions
        for (int i = 0; i < v; i++) {
            if (!keep[i]) { u[i] = 0.0; continue; }
            double e = -c[i];
            for (int k = 0; k < i; k++)
                if (keep[k]) e -= L[i][k] * u[k];
            u[i] = e / L[i][i];
        }
        for (int i = v - 1; i >= 0; i--) {
            if (!keep[i]) { y[i] = 0.0; continue; }
            double e = u[i];
            for (int j = i + 1; j < v; j++)
                if (keep[j]) e -= L[j][i] * y[j];
            y[i] = e / L[i][i];
        }
        // growth of the combination in the A-norm: sum |y_a| ||x_a||_A
        // against ||z0||_A; accept when the cancellation is mild
        double num = 0.0, zA = 0.0;
        for (int a = 0; a < v; a++) {
            num += fabs(y[a]) * sqrt(N[a][a]);
            for (int b = 0; b < v; b++) zA += y[a] * N[a][b] * y[b];
        }
        if (t == 4 || (zA > 0.0 && num <= 100.0 * sqrt(zA) && isfinite(num))) return kept;
    }
    return 1;
}

}  // namespace cgb

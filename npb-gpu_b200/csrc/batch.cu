// batch.cu -- many independent CG inverse power iterations of uneven order
// in one persistent launch.
//
// Each CTA takes systems from a device work queue (an atomic ticket over the
// systems sorted by stored entries, largest first) and runs a system's whole
// power iteration (GMAP/NPB-GPU CUDA/CG/cg.cu:485-520 with conj_grad,
// cg.cu:653-801) alone, so every synchronisation is a CTA barrier.  The
// search vector p lives only in shared memory (FP64, up to kBatchMaxN rows),
// so the SpMV's gathers are shared-memory loads; x, z, r, q stay in global
// memory, coalesced per CTA.
//
// Modes (per launch):
//   fixed  the reference algorithm: cgitmax FP64 CG steps from z = 0;
//   mixed  FP32 matrix values times FP32-rounded p with FP32 row sums, FP64
//          dots and updates, true-residual replacement with the FP64 matrix
//          and restart (as the single-system mixed solver), stopped at
//          ||r|| <= tol ||x||.  A system whose iteration shows p.Ap >= 0
//          (the NPB matrices are negative definite; small orders with large
//          nonzer are not), a non-finite residual, or no convergence within
//          cgitmax is solved again from the start with the fixed FP64
//          algorithm at the reference's 25 steps (cg.cu's cgitmax), so its
//          zeta is the reference algorithm's; its status says so.  (On an
//          indefinite system an eigenvalue of A near zero can make zeta
//          sensitive beyond what a 1e-12 residual pins down, so agreement
//          with the reference needs the reference's own iteration there.)
//   learned  the mixed mode preconditioned by M = F^T F per system (F lower
//          triangular with a positive diagonal, cgb_batch_set_preconditioner:
//          the learned factor G diag(-A)^-1/2), CG on -A; the factor's
//          off-diagonal values are BF16 with 16-bit columns, its diagonal
//          FP32 (applied to FP64 vectors); both factor products gather from
//          a shared-memory copy of the vector.  An outer step whose
//          preconditioned iteration stalls (|r|^2 not halved in four steps,
//          or r.y <= 0) continues as plain CG; a system showing p.Ap >= 0 is
//          re-solved with the FP64 reference algorithm, as in the mixed mode.
// Lanes per row are a per-system choice (the autotuner's, by row length).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include <cuda_bf16.h>

#include "cgb_internal.h"
#include "device_common.cuh"
#include "galerkin.cuh"

namespace cgb {
namespace batch {

constexpr int kBatchMaxN = 27000;  // rows of the largest system (shared p: 8 bytes a row)
constexpr int kReferenceCgitmax = 25;  // cg.cu's cgitmax: the FP64 re-solve of a mixed failure
constexpr int kMaxTeam = 8;            // CTAs that may share one system
constexpr int kTeamValues = 16;        // values one team reduction can carry
constexpr int kSyncStride = 32;        // words between barrier counters (128-byte lines)
constexpr long long kTeamWaitNs = 2000000000LL;  // limit of one team-barrier wait
static_assert(kTeamValues >= kGramValues, "team reductions must carry the Gram values");

struct SysDesc {
    int n;
    int lanes;           // lanes per row (2, 4, 8, 16, 32)
    int team;            // CTAs that solve the system together (1, 2, 4 or 8)
    int flanes;          // lanes per row of the preconditioner's factor products
    long long row_off;   // into rowstr_all (n+1 entries)
    long long nnz_off;   // into colidx_all / a_all
    long long vec_off;   // into the vector arrays (n+8 entries)
    long long f_row_off; // into the factor row pointers (F and F^T: n+1 entries each)
    long long f_off;     // into the factor entries (F and F^T: the same count)
    double shift;
};

// Batch modes (the launch's kernel).
constexpr int kModeFixed = 0;
constexpr int kModeMixed = 1;
constexpr int kModeLearned = 2;

struct BatchArgs {
    int nsys;
    const SysDesc *__restrict__ sys;
    const int *__restrict__ rowstr;
    const int *__restrict__ colidx;
    const double *__restrict__ a;
    const float *__restrict__ a32;
    double *x, *z, *r, *q;
    unsigned *queue;
    int mode;            // 0 fixed, 1 mixed (the launch's kernel)
    int niter, cgitmax, refresh_every;
    double tol;
    double *zeta, *rnorm;
    int *iters, *status;  // status: 0 = done; 1 = mixed iteration gave up (solved again in FP64)
    // mixed mode: Galerkin start on the last `recycle` iterates; slot j of
    // system s at hx/hw + j * hstride + vec_off
    double *hx, *hw;
    long long hstride;
    int recycle;
    // teams: the search vector's exchange copy (vec_off layout), per system
    // a barrier's 64-bit arrival count (2 * kSyncStride words a system, one
    // 256-byte line) and 2 x kMaxTeam x kTeamValues reduction slots
    double *pg;
    unsigned *team_sync;
    double *team_part;
    int *dev_status;     // kDevOk, or kDevTimeout once a team wait ran out
    // learned mode: the factor F (lower, rows of F) and F^T (rows of F^T),
    // BF16 values and 16-bit columns; the preconditioned residual y (FP64)
    // and two FP32 exchange vectors (r and F r) in the vec_off layout, and
    // per system the outer steps that fell back to plain CG
    const int *fptr, *ftptr;
    const unsigned short *fcol, *ftcol;
    const __nv_bfloat16 *fval, *ftval;
    const float *fdiag;  // the factor's diagonal (FP32, at f_row_off), kept out of the CSR
    double *y;
    float *rg, *tg;
    int *fallbacks;
};

// This CTA's part of a system: rows [lo, hi) of `size` members (balanced by
// stored entries), and the team's barrier and reduction slots.  `par`
// alternates the slot set between consecutive reductions: a member can be
// at most one reduction ahead of the slowest, so it never overwrites slots
// that one still reads.
struct Team {
    int id, member, size, lo, hi, par;
};

// The team's barrier words and reduction slots (computed where used: kept in
// registers across the CG loop they would crowd it).
struct TeamMem {
    unsigned long long *arrivals;  // the team barrier's count (zeroed every launch)
    double *part;
    int *status;  // the launch's device status word
};

__device__ __forceinline__ TeamMem team_mem(const BatchArgs &B, int id)
{
    TeamMem M;
    M.arrivals = reinterpret_cast<unsigned long long *>(B.team_sync + size_t(id) * (2 * kSyncStride));
    M.part = B.team_part + size_t(id) * (2 * kMaxTeam * kTeamValues);
    M.status = B.dev_status;
    return M;
}

// First row whose rowstr entry is >= target (rowstr ascending, n+1 entries).
__device__ __forceinline__ int first_row_at(const int *rowstr, int n, long long target)
{
    int a = 0, b = n;
    while (a < b) {
        const int m = (a + b) >> 1;
        if (rowstr[m] < target) a = m + 1;
        else b = m;
    }
    return a;
}

__device__ __forceinline__ Team make_team(const BatchArgs &B, int id, const SysDesc &S, int member)
{
    Team T;
    T.id = id;
    T.member = member;
    T.size = S.team;
    T.par = 0;
    if (T.size == 1) {
        T.lo = 0;
        T.hi = S.n;
    } else {
        const int *rowstr = B.rowstr + S.row_off;
        const long long nnz = rowstr[S.n];
        T.lo = member == 0 ? 0 : first_row_at(rowstr, S.n, nnz * member / T.size);
        T.hi = member == T.size - 1 ? S.n : first_row_at(rowstr, S.n, nnz * (member + 1) / T.size);
    }
    return T;
}

// CTA sums of nq (<= kGramValues) per-thread values, in a fixed order, into
// out[] (shared, every thread); four values a round keep the static shared
// memory small beside the up to 216 KB of p.
__device__ __forceinline__ void cta_sum_multi(const double *vals, int nq, double *out)
{
    constexpr int kRound = 4;
    __shared__ double red[32][kRound];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int q0 = 0; q0 < kGramValues; q0 += kRound) {
        if (q0 < nq) {
#pragma unroll
            for (int k = 0; k < kRound; k++) {
                if (q0 + k < nq && q0 + k < kGramValues) {
                    const double v = warp_sum(vals[q0 + k < kGramValues ? q0 + k : 0]);
                    if (l == 0) red[w][k] = v;
                }
            }
            __syncthreads();
            if (threadIdx.x < kRound && q0 + int(threadIdx.x) < nq) {
                double t = 0.0;
                for (int i = 0; i < int(blockDim.x >> 5); i++) t += red[i][threadIdx.x];
                out[q0 + threadIdx.x] = t;
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ double cta_sum(double v, double *red)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < int(blockDim.x >> 5); i++) s += red[i];
    return s;  // every thread, same order
}

__device__ __forceinline__ bool team_barrier(const TeamMem &M, const Team &T)
{
    return counted_barrier(M.arrivals, unsigned(T.size), M.status, kTeamWaitNs);
}

// Team sum of one value per thread: the CTA sum, then (teams) the members'
// sums added in member order by every member, so all members hold the same
// bits and take the same branches.  The barrier inside also publishes every
// global write the members made before it.  False: a team wait failed.
__device__ __forceinline__ bool team_sum(const BatchArgs &B, Team &T, double v, double *red,
                                         double &out)
{
    const double s = cta_sum(v, red);
    if (T.size == 1) {
        out = s;
        return true;
    }
    const TeamMem M = team_mem(B, T.id);
    double *slot = M.part + T.par * (kMaxTeam * kTeamValues);
    if (threadIdx.x == 0) slot[T.member * kTeamValues] = s;
    T.par ^= 1;
    if (!team_barrier(M, T)) return false;
    double t = 0.0;
    for (int m = 0; m < T.size; m++) t += __ldcg(slot + m * kTeamValues);
    out = t;
    return true;
}

// team_sum of nq values a thread, into out[] (shared).
__device__ __forceinline__ bool team_sum_multi(const TeamMem &M, Team &T, const double *vals,
                                               int nq, double *out)
{
    cta_sum_multi(vals, nq, out);
    if (T.size == 1) return true;
    double *slot = M.part + T.par * (kMaxTeam * kTeamValues);
    if (int(threadIdx.x) < nq) slot[T.member * kTeamValues + threadIdx.x] = out[threadIdx.x];
    T.par ^= 1;
    if (!team_barrier(M, T)) return false;
    if (int(threadIdx.x) < nq) {
        double t = 0.0;
        for (int m = 0; m < T.size; m++) t += __ldcg(slot + m * kTeamValues + threadIdx.x);
        out[threadIdx.x] = t;
    }
    __syncthreads();
    return true;
}

// After a team barrier that followed the members' writes of their rows of
// p to pg: the other members' rows into this CTA's shared copy.
__device__ __forceinline__ void team_gather_p(const Team &T, const double *pg, double *p, int n)
{
    if (T.size == 1) return;
    for (int j = threadIdx.x; j < T.lo; j += blockDim.x) p[j] = __ldcg(pg + j);
    for (int j = T.hi + threadIdx.x; j < n; j += blockDim.x) p[j] = __ldcg(pg + j);
    __syncthreads();
}

// q[j] = (A v)[j] for rows [lo, hi) of the system with S.lanes lanes per
// row; v in shared memory (FP64) or, v_gl, global memory (v_gl_shared: a
// team's vector, read through L2, since other members' rows may have been
// written since this SM last cached them); products in FP64 or (F32) in FP32 with FP32 row sums; returns this
// thread's share of sum_j dv[j] q[j] (dv: shared p or null).  The lane count
// is a run-time value: one instance of the solver serves every system (an
// instance per lane count inlined under one switch needed 128 registers a
// thread and spilled; one needs about 84).
template <typename T>
struct NoDeduce {
    using type = T;
};

template <bool F32, int kU, typename VS = double>
__device__ __forceinline__ double sys_spmv(const BatchArgs &B, const SysDesc &S, int lo, int hi,
                                           const typename NoDeduce<VS>::type *v_sh,
                                           const double *v_gl, double *q,
                                           const double *dv_sh, bool v_gl_shared = false)
{
    const int *rowstr = B.rowstr + S.row_off;
    const int *colidx = B.colidx + S.nnz_off;
    const double *a = B.a + S.nnz_off;
    const float *a32 = B.a32 ? B.a32 + S.nnz_off : nullptr;
    const int LPR = S.lanes;
    const int lane = threadIdx.x & (LPR - 1), grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    double dacc = 0.0;
    for (int row = lo + grp; row < hi; row += ngrp) {
        const int k0 = rowstr[row], k1 = rowstr[row + 1];
        double s64 = 0.0;
        float s32 = 0.f;
        for (int k = k0 + lane; k < k1; k += kU * LPR) {
            int c[kU];
            double av[kU];
            float af[kU];
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const int kk = k + u * LPR;
                if (kk < k1) {
                    c[u] = __ldcs(colidx + kk);
                    if (F32) af[u] = __ldcs(a32 + kk);
                    else av[u] = __ldcs(a + kk);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; u++) {
                if (k + u * LPR < k1) {
                    const double pv = v_sh ? double(v_sh[c[u]])
                                           : (v_gl_shared ? __ldcg(v_gl + c[u]) : v_gl[c[u]]);
                    if (F32) s32 = fmaf(af[u], float(pv), s32);
                    else s64 = fma(av[u], pv, s64);
                }
            }
        }
        double s;
        if (F32) s = double(group_sum_f_rt(s32, mask, LPR));
        else s = group_sum_rt(s64, mask, LPR);
        if (lane == 0) {
            q[row] = s;
            if (dv_sh) dacc = fma(dv_sh[row], s, dacc);
        }
    }
    return dacc;
}

struct GalerkinIn {
    const double *hx, *hw;
    long long hstride, vec_off;
    const double *x;
    double *z, *r, *pg, *p;
    Team T;
    TeamMem M;
    int outer, m, v;
};

struct GalerkinOut {
    double acc, xx;  // this thread's share of r.r; x_k.x_k
    int par, ok;     // the team's next slot parity; 0 when a team wait failed
};

// Galerkin start of a mixed solve on x_k .. x_{k-v+1} (v >= 1) for this
// CTA's rows: z0 = V y, r = x - W y (A z0 = W y), p = r; the Gram values are
// team sums, so every member solves the same small system.
static __device__ __forceinline__ GalerkinOut galerkin_body(GalerkinIn in)
{
    __shared__ double g_sh[kTeamValues];
    __shared__ double y_sh[kMaxRecycle];
    const int lo = in.T.lo, hi = in.T.hi, m = in.m, v = in.v, outer = in.outer;
    const bool team = in.T.size > 1;
    GalerkinOut out{0.0, 0.0, in.T.par, 0};
    long long off[kMaxRecycle];
#pragma unroll
    for (int a = 0; a < kMaxRecycle; a++) off[a] = ((outer - a) % m + m) % m * in.hstride + in.vec_off;
    const int npairs = v * (v + 1) / 2;
    double vals[kGramValues];
#pragma unroll
    for (int q = 0; q < kGramValues; q++) vals[q] = 0.0;
    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        const double xv = in.x[j];
#pragma unroll
        for (int b = 0; b < kMaxRecycle; b++) {
            if (b < v) {
                const double xb = in.hx[off[b] + j], wb = in.hw[off[b] + j];
#pragma unroll
                for (int a = 0; a <= b; a++)
                    vals[gram_index(a, b)] =
                        fma(a == b ? xb : in.hx[off[a] + j], wb, vals[gram_index(a, b)]);
                vals[kGramPairs + b] = fma(xb, xv, vals[kGramPairs + b]);
            }
        }
    }
    double packed[kGramValues];
#pragma unroll
    for (int q = 0; q < kGramValues; q++) packed[q] = 0.0;
#pragma unroll
    for (int q = 0; q < kGramPairs; q++)
        if (q < npairs) packed[q] = vals[q];
#pragma unroll
    for (int b = 0; b < kMaxRecycle; b++)
        if (b < v) packed[npairs + b] = vals[kGramPairs + b];
    Team T = in.T;
    if (!team_sum_multi(in.M, T, packed, npairs + v, g_sh)) return out;
    out.par = T.par;
    if (threadIdx.x == 0) {
        double g[kGramValues], y[kMaxRecycle];
        for (int q = 0; q < kGramValues; q++) g[q] = 0.0;
        for (int q = 0; q < npairs; q++) g[q] = g_sh[q];
        for (int b = 0; b < v; b++) g[kGramPairs + b] = g_sh[npairs + b];
        galerkin_solve(g, v, y);
        for (int a = 0; a < kMaxRecycle; a++) y_sh[a] = a < v ? y[a] : 0.0;
    }
    __syncthreads();
    out.xx = g_sh[npairs];  // x_k . x_k
    double acc = 0.0;
    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        double z0 = 0.0, az = 0.0;
#pragma unroll
        for (int a = 0; a < kMaxRecycle; a++) {
            if (a < v) {
                z0 = fma(y_sh[a], in.hx[off[a] + j], z0);
                az = fma(y_sh[a], in.hw[off[a] + j], az);
            }
        }
        const double rv = in.x[j] - az;
        in.z[j] = z0;
        in.r[j] = rv;
        if (in.p) {  // (the learned mode sets its own start vectors)
            in.p[j] = rv;
            if (team) in.pg[j] = rv;
        }
        acc = fma(rv, rv, acc);
    }
    out.acc = acc;
    out.ok = 1;
    return out;
}

// Out of line for the kernels with teams: it runs once an outer step, and
// inlined there its arrays crowd the CG loop's registers.
static __device__ __noinline__ GalerkinOut batch_galerkin(GalerkinIn in)
{
    return galerkin_body(in);
}

constexpr int kSolveOk = 0;
constexpr int kSolveGaveUp = 1;   // mixed: p.Ap >= 0, a non-finite residual, or no convergence
constexpr int kSolveAborted = 2;  // a team wait failed (dev_status says why)

// One system's power iteration on this CTA's rows [T.lo, T.hi) (all rows
// without a team).  Every CTA keeps the whole search vector in shared
// memory; a team's members exchange their rows of it through pg after each
// update.  Every branch depends on team sums only, so the members run the
// same sequence of barriers.  cgitmax: the fixed mode's exact count, the
// mixed mode's cap.
template <bool mixed, int kU, bool kTeams>
__device__ int solve_system(const BatchArgs &B, const SysDesc &S, Team &T, int cgitmax, double *p,
                            double *red, int *iters_out, double *zeta_out, double *rnorm_out)
{
    if (!kTeams) {  // a kernel without teams: the team code folds away
        T.size = 1;
        T.lo = 0;
        T.hi = S.n;
    }
    const int n = S.n, lo = T.lo, hi = T.hi;
    const bool team = kTeams && T.size > 1;
    double *x = B.x + S.vec_off, *z = B.z + S.vec_off, *r = B.r + S.vec_off, *q = B.q + S.vec_off;
    double *pg = B.pg + S.vec_off;
    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) x[j] = 1.0;
    __syncthreads();
    int total = 0;
    double zeta = 0.0, rnorm = 0.0;
    for (int outer = 0; outer < B.niter; outer++) {
        double acc = 0.0;
        const int m = B.recycle;
        const int v = (mixed && m > 0) ? min(outer, m) : 0;
        double xx = 0.0;
        if (v > 0) {
            GalerkinIn in{B.hx, B.hw, B.hstride, S.vec_off, x, z, r, pg, p, T, team_mem(B, T.id),
                          outer, m, v};
            const GalerkinOut g = kTeams ? batch_galerkin(in) : galerkin_body(in);
            if (!g.ok) return kSolveAborted;
            T.par = g.par;
            acc = g.acc;
            xx = g.xx;
        } else {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double xv = x[j];
                z[j] = 0.0;
                r[j] = xv;
                p[j] = xv;
                if (team) pg[j] = xv;
                acc = fma(xv, xv, acc);
            }
        }
        double rho;
        if (!team_sum(B, T, acc, red, rho)) return kSolveAborted;  // barrier: p complete
        team_gather_p(T, pg, p, n);
        if (v == 0) xx = rho;
        const double stop2 = B.tol * B.tol * xx;
        double rho_cycle = rho;
        int it = 0, since = 0;
        bool fresh = true;
        for (;;) {
            if (!mixed) {
                if (it >= cgitmax) break;
            } else {
                bool refresh = false;
                if (rho <= stop2) {
                    if (fresh) break;
                    refresh = true;
                } else if (!fresh && (since >= B.refresh_every || rho <= 1e-12 * rho_cycle)) {
                    refresh = true;
                }
                if (!refresh && it >= cgitmax) return kSolveGaveUp;  // not converged
                if (refresh) {
                    // r = x - A z (FP64 matrix; every member's z rows were
                    // published by the last team sum), restart p = r
                    sys_spmv<false, kU>(B, S, lo, hi, nullptr, z, q, nullptr, team);
                    __syncthreads();
                    acc = 0.0;
                    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                        const double rv = x[j] - q[j];
                        r[j] = rv;
                        p[j] = rv;
                        if (team) pg[j] = rv;
                        acc = fma(rv, rv, acc);
                    }
                    if (!team_sum(B, T, acc, red, rho)) return kSolveAborted;
                    team_gather_p(T, pg, p, n);
                    rho_cycle = rho;
                    since = 0;
                    fresh = true;
                    continue;
                }
            }
            const double dpart = mixed ? sys_spmv<true, kU>(B, S, lo, hi, p, nullptr, q, p)
                                       : sys_spmv<false, kU>(B, S, lo, hi, p, nullptr, q, p);
            double d;
            if (!team_sum(B, T, dpart, red, d)) return kSolveAborted;  // barrier: q complete
            if (mixed && !(d < 0.0)) return kSolveGaveUp;  // not negative definite (or NaN)
            const double alpha = rho / d;
            const double rho0 = rho;
            acc = 0.0;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                z[j] = fma(alpha, p[j], z[j]);
                const double rv = fma(-alpha, q[j], r[j]);
                r[j] = rv;
                acc = fma(rv, rv, acc);
            }
            if (!team_sum(B, T, acc, red, rho)) return kSolveAborted;
            if (mixed && !(rho < INFINITY)) return kSolveGaveUp;  // non-finite residual
            const double beta = rho / rho0;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double pv = fma(beta, p[j], r[j]);
                p[j] = pv;
                if (team) pg[j] = pv;
            }
            if (team) {
                if (!team_barrier(team_mem(B, T.id), T)) return kSolveAborted;
                team_gather_p(T, pg, p, n);
            } else {
                __syncthreads();
            }
            it++;
            since++;
            fresh = false;
        }
        total += it;
        // q = A z (FP64): a product, or from the true residual r = x - A z
        // the mixed iteration just accepted; rnorm = ||x - A z||, x.z, z.z
        if (mixed && fresh) {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) q[j] = x[j] - r[j];
        } else {
            sys_spmv<false, kU>(B, S, lo, hi, nullptr, z, q, nullptr, team);
        }
        __syncthreads();
        double res = 0.0, xz = 0.0, zz = 0.0;
        for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
            const double xv = x[j], zv = z[j], dv = xv - q[j];
            res = fma(dv, dv, res);
            xz = fma(xv, zv, xz);
            zz = fma(zv, zv, zz);
        }
        double t0, t1, t2;
        if (!team_sum(B, T, res, red, t0) || !team_sum(B, T, xz, red, t1) ||
            !team_sum(B, T, zz, red, t2))
            return kSolveAborted;
        rnorm = sqrt(t0);
        zeta = S.shift + 1.0 / t1;
        const double norm = 1.0 / sqrt(t2);
        if (mixed && m > 0) {
            // the next iterate and A times it into the ring
            const long long slot = (outer + 1) % m * B.hstride + S.vec_off;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double xn = norm * z[j];
                B.hx[slot + j] = xn;
                B.hw[slot + j] = norm * q[j];
                x[j] = xn;
            }
        } else {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) x[j] = norm * z[j];
        }
        __syncthreads();
    }
    *iters_out = total;
    *zeta_out = zeta;
    *rnorm_out = rnorm;
    return kSolveOk;
}

// One factor product for rows [lo, hi): out[row] = sum_k val[k] v[col[k]] +
// diag[row] dvec[row] -- the off-diagonal entries (BF16 values widened to
// FP32, 16-bit columns, v an FP32 vector in shared memory, FP32 row sums)
// and the diagonal (FP32) times an FP64 vector -- with `lanes` lanes a row,
// written as FP32 (out32) and/or FP64 (out64); returns this thread's share
// of sum dot[row] out[row] (dot may be null).
template <int kU>
__device__ __forceinline__ double sys_fprod(const int *ptr, const unsigned short *col,
                                            const __nv_bfloat16 *val, int lanes, int lo, int hi,
                                            const float *v, const float *diag, const double *dvec,
                                            float *out32, double *out64, const double *dot)
{
    const int LPR = lanes;
    const int lane = threadIdx.x & (LPR - 1), grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    double dacc = 0.0;
    for (int row = lo + grp; row < hi; row += ngrp) {
        const int k0 = ptr[row], k1 = ptr[row + 1];
        float s = 0.f;
        for (int k = k0 + lane; k < k1; k += kU * LPR) {
            unsigned short c[kU];
            __nv_bfloat16 w[kU];
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const int kk = k + u * LPR;
                if (kk < k1) {
                    c[u] = __ldcs(col + kk);
                    w[u] = __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short *>(val) + kk));
                }
            }
#pragma unroll
            for (int u = 0; u < kU; u++)
                if (k + u * LPR < k1) s = fmaf(__bfloat162float(w[u]), v[c[u]], s);
        }
        s = group_sum_f_rt(s, mask, LPR);
        if (lane == 0) {
            const double t = fma(double(diag[row]), dvec[row], double(s));
            if (out32) out32[row] = float(t);
            if (out64) out64[row] = t;
            if (dot) dacc = fma(dot[row], t, dacc);
        }
    }
    return dacc;
}

// Team copy of an FP32 vector held in shared memory: this CTA wrote its rows
// [lo, hi) to both v_sh and the global copy g; after a team barrier the
// other members' rows come from g.
__device__ __forceinline__ void team_gather_f(const Team &T, const float *g, float *v_sh, int n)
{
    if (T.size == 1) return;
    for (int j = threadIdx.x; j < T.lo; j += blockDim.x) v_sh[j] = __ldcg(g + j);
    for (int j = T.hi + threadIdx.x; j < n; j += blockDim.x) v_sh[j] = __ldcg(g + j);
    __syncthreads();
}

// The learned mode's view of one system: its vectors and factor arrays.
struct PcgSys {
    double *x, *z, *r, *q, *pg, *y;
    float *rg, *tg, *p32, *v32;
    const float *fdiag;
    const int *fptr, *ftptr;
    const unsigned short *fcol, *ftcol;
    const __nv_bfloat16 *fval, *ftval;
};

// y = M r' = F^T (F r') (use) or y = r' (plain CG), and rho = r'.y (a team
// sum).  On entry v32 holds r' in FP32 for every row; on return it holds
// F r' (use).  False: a team wait failed.
template <int kU>
__device__ __forceinline__ bool pcg_apply(const BatchArgs &B, const SysDesc &S, Team &T,
                                          const PcgSys &V, bool use, double *red, double &rho)
{
    const int n = S.n, lo = T.lo, hi = T.hi;
    const bool team = T.size > 1;
    double dacc = 0.0;
    if (use) {
        // t = F r' (own rows) to the global copy, and in FP64 to q
        sys_fprod<kU>(V.fptr, V.fcol, V.fval, S.flanes, lo, hi, V.v32, V.fdiag, V.r, V.tg, V.q,
                      nullptr);
        // every row of t into v32, once every thread (and member) is done with r'
        if (team) {
            if (!team_barrier(team_mem(B, T.id), T)) return false;
            for (int j = threadIdx.x; j < n; j += blockDim.x) V.v32[j] = __ldcg(V.tg + j);
        } else {
            __syncthreads();
            for (int j = threadIdx.x; j < n; j += blockDim.x) V.v32[j] = V.tg[j];
        }
        __syncthreads();
        // y = F^T t (own rows), with the r'.y share
        dacc = sys_fprod<kU>(V.ftptr, V.ftcol, V.ftval, S.flanes, lo, hi, V.v32, V.fdiag, V.q,
                             nullptr, V.y, V.r);
    } else {
        for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
            const double rv = V.r[j];
            V.y[j] = rv;
            dacc = fma(rv, rv, dacc);
        }
    }
    return team_sum(B, T, dacc, red, rho);
}

// After this CTA wrote its rows of p to pg (FP64) and p32: the whole p32
// (a team barrier and the other members' rows from pg; or a CTA barrier).
template <bool kTeams>
__device__ __forceinline__ bool pcg_publish_p(const BatchArgs &B, const Team &T, const PcgSys &V,
                                              int n)
{
    if (kTeams && T.size > 1) {
        if (!team_barrier(team_mem(B, T.id), T)) return false;
        for (int j = threadIdx.x; j < T.lo; j += blockDim.x) V.p32[j] = float(__ldcg(V.pg + j));
        for (int j = T.hi + threadIdx.x; j < n; j += blockDim.x) V.p32[j] = float(__ldcg(V.pg + j));
    }
    __syncthreads();
    return true;
}

// One system's power iteration in the learned mode: preconditioned CG on
// A' = -A with b' = -x (the same solution z), M = F^T F, FP32 products
// (A32 and the factors) inside FP64 refinement with the mixed mode's
// true-residual replacement and restart, stopped at a true residual
// ||x - A z|| <= tol ||x||.  Shared memory holds p and the factor
// products' vector in FP32; the FP64 search vector is pg.  An outer step
// whose preconditioned iteration stalls continues as plain CG
// (*fallbacks_out counts those steps); p.A'p <= 0 (A not negative
// definite), a non-finite residual or no convergence gives up, and the
// caller re-solves with the FP64 reference algorithm.
template <int kU, bool kTeams>
__device__ int solve_system_pcg(const BatchArgs &B, const SysDesc &S, Team &T, int cgitmax,
                                double *smem, double *red, int *iters_out, double *zeta_out,
                                double *rnorm_out, int *fallbacks_out)
{
    if (!kTeams) {
        T.size = 1;
        T.lo = 0;
        T.hi = S.n;
    }
    const int n = S.n, lo = T.lo, hi = T.hi;
    const bool team = kTeams && T.size > 1;
    PcgSys V;
    V.x = B.x + S.vec_off;
    V.z = B.z + S.vec_off;
    V.r = B.r + S.vec_off;
    V.q = B.q + S.vec_off;
    V.pg = B.pg + S.vec_off;
    V.y = B.y + S.vec_off;
    V.rg = B.rg + S.vec_off;
    V.tg = B.tg + S.vec_off;
    V.p32 = reinterpret_cast<float *>(smem);
    V.v32 = V.p32 + ((n + 8 + 3) & ~3);
    V.fdiag = B.fdiag + S.f_row_off;
    V.fptr = B.fptr + S.f_row_off;
    V.ftptr = B.ftptr + S.f_row_off;
    V.fcol = B.fcol + S.f_off;
    V.ftcol = B.ftcol + S.f_off;
    V.fval = B.fval + S.f_off;
    V.ftval = B.ftval + S.f_off;
    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) V.x[j] = 1.0;
    __syncthreads();
    int total = 0, fallbacks = 0;
    double zeta = 0.0, rnorm = 0.0;
    for (int outer = 0; outer < B.niter; outer++) {
        double acc = 0.0, xx = 0.0;
        const int m = B.recycle;
        const int v = m > 0 ? min(outer, m) : 0;
        if (v > 0) {
            // Galerkin start: z0, r = x - A z0 (no p written)
            GalerkinIn in{B.hx, B.hw, B.hstride, S.vec_off, V.x, V.z, V.r, V.pg, nullptr, T,
                          team_mem(B, T.id), outer, m, v};
            const GalerkinOut g = kTeams ? batch_galerkin(in) : galerkin_body(in);
            if (!g.ok) return kSolveAborted;
            T.par = g.par;
            xx = g.xx;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double rv = -V.r[j];  // r' = A z0 - x
                V.r[j] = rv;
                V.v32[j] = float(rv);
                if (team) V.rg[j] = float(rv);
                acc = fma(rv, rv, acc);
            }
        } else {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double xv = V.x[j];
                V.z[j] = 0.0;
                V.r[j] = -xv;
                V.v32[j] = float(-xv);
                if (team) V.rg[j] = float(-xv);
                acc = fma(xv, xv, acc);
            }
        }
        double rr;
        if (!team_sum(B, T, acc, red, rr)) return kSolveAborted;  // barrier: r' published
        team_gather_f(T, V.rg, V.v32, n);
        if (v == 0) xx = rr;
        const double stop2 = B.tol * B.tol * xx;
        double rr_cycle = rr;
        double hist[4] = {rr, rr, rr, rr};  // |r'|^2 of the last four steps
        bool use = true;
        double rho = 0.0;
        if (!pcg_apply<kU>(B, S, T, V, use, red, rho)) return kSolveAborted;
        if (!(rho > 0.0)) {
            use = false;
            if (!pcg_apply<kU>(B, S, T, V, false, red, rho)) return kSolveAborted;
        }
        for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
            const double pv = V.y[j];
            V.pg[j] = pv;
            V.p32[j] = float(pv);
        }
        if (!pcg_publish_p<kTeams>(B, T, V, n)) return kSolveAborted;
        int it = 0, since = 0;
        bool fresh = true;
        for (;;) {
            bool refresh = false;
            if (rr <= stop2) {
                if (fresh) break;
                refresh = true;
            } else if (!fresh && (since >= B.refresh_every || rr <= 1e-12 * rr_cycle)) {
                refresh = true;
            }
            if (!refresh && it >= cgitmax) return kSolveGaveUp;  // not converged
            bool restart = refresh;
            if (refresh) {
                // r' = A z - x with the FP64 matrix (z published by the last team sum)
                sys_spmv<false, kU>(B, S, lo, hi, nullptr, V.z, V.q, nullptr, team);
                __syncthreads();
                acc = 0.0;
                for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                    const double rv = V.q[j] - V.x[j];
                    V.r[j] = rv;
                    V.v32[j] = float(rv);
                    if (team) V.rg[j] = float(rv);
                    acc = fma(rv, rv, acc);
                }
                if (!team_sum(B, T, acc, red, rr)) return kSolveAborted;
                team_gather_f(T, V.rg, V.v32, n);
                rr_cycle = rr;
                hist[0] = hist[1] = hist[2] = hist[3] = rr;
                since = 0;
                fresh = true;
                if (rr <= stop2) break;
            } else {
                // q = A32 p32 (FP32 products); p.A'p = -p.q
                const double dpart = sys_spmv<true, kU, float>(B, S, lo, hi, V.p32, nullptr, V.q, V.pg);
                double d;
                if (!team_sum(B, T, dpart, red, d)) return kSolveAborted;
                const double pAp = -d;
                if (!(pAp > 0.0)) return kSolveGaveUp;  // not negative definite (or NaN)
                const double alpha = rho / pAp;
                acc = 0.0;
                for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                    V.z[j] = fma(alpha, V.pg[j], V.z[j]);
                    const double rv = fma(alpha, V.q[j], V.r[j]);  // r' -= alpha A'p
                    V.r[j] = rv;
                    V.v32[j] = float(rv);
                    if (team) V.rg[j] = float(rv);
                    acc = fma(rv, rv, acc);
                }
                if (!team_sum(B, T, acc, red, rr)) return kSolveAborted;
                if (!(rr < INFINITY)) return kSolveGaveUp;  // non-finite residual
                team_gather_f(T, V.rg, V.v32, n);
                it++;
                since++;
                fresh = false;
                // stall: no halving of |r'|^2 over four steps
                if (use && since >= 4 && rr > 0.25 * hist[0]) {
                    use = false;
                    restart = true;
                }
                hist[0] = hist[1];
                hist[1] = hist[2];
                hist[2] = hist[3];
                hist[3] = rr;
            }
            double rho_new = 0.0;
            if (!pcg_apply<kU>(B, S, T, V, use, red, rho_new)) return kSolveAborted;
            if (use && !(rho_new > 0.0)) {
                use = false;
                restart = true;
                if (!pcg_apply<kU>(B, S, T, V, false, red, rho_new)) return kSolveAborted;
            }
            const double beta = restart ? 0.0 : rho_new / rho;
            rho = rho_new;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double pv = fma(beta, V.pg[j], V.y[j]);
                V.pg[j] = pv;
                V.p32[j] = float(pv);
            }
            if (!pcg_publish_p<kTeams>(B, T, V, n)) return kSolveAborted;
        }
        total += it;
        if (!use) fallbacks++;
        // q = A z: from the true residual r' = A z - x just accepted, else a product
        if (fresh) {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) V.q[j] = V.x[j] + V.r[j];
        } else {
            sys_spmv<false, kU>(B, S, lo, hi, nullptr, V.z, V.q, nullptr, team);
        }
        __syncthreads();
        double res = 0.0, xz = 0.0, zz = 0.0;
        for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
            const double xv = V.x[j], zv = V.z[j], dv = xv - V.q[j];
            res = fma(dv, dv, res);
            xz = fma(xv, zv, xz);
            zz = fma(zv, zv, zz);
        }
        double t0, t1, t2;
        if (!team_sum(B, T, res, red, t0) || !team_sum(B, T, xz, red, t1) ||
            !team_sum(B, T, zz, red, t2))
            return kSolveAborted;
        rnorm = sqrt(t0);
        zeta = S.shift + 1.0 / t1;
        const double norm = 1.0 / sqrt(t2);
        if (m > 0) {
            const long long slot = (outer + 1) % m * B.hstride + S.vec_off;
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
                const double xn = norm * V.z[j];
                B.hx[slot + j] = xn;
                B.hw[slot + j] = norm * V.q[j];
                V.x[j] = xn;
            }
        } else {
            for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) V.x[j] = norm * V.z[j];
        }
        __syncthreads();
    }
    *iters_out = total;
    *zeta_out = zeta;
    *rnorm_out = rnorm;
    *fallbacks_out = fallbacks;
    return kSolveOk;
}

// This CTA's share (member `member` of the system's team) of one system.  A
// mixed or learned solve that gives up (an indefinite system shows
// p.Ap >= 0 within the first iterations) is redone at once by the same team
// with the reference algorithm (FP64, exactly the reference's 25 CG
// iterations an outer step) and marked status 1; its outputs are that
// solve's alone.  A learned solve in which some outer step fell back to
// plain CG is marked status 2.  False: a team wait failed and the CTA must
// stop.
template <int kMode, int kU, bool kTeams>
__device__ bool run_system(const BatchArgs &B, int id, int member, const SysDesc &S, double *p,
                           double *red)
{
    Team T = make_team(B, id, S, member);
    int iters = 0, fallbacks = 0;
    double zeta = 0.0, rnorm = 0.0;
    int rc;
    if constexpr (kMode == kModeLearned)
        rc = solve_system_pcg<kU, kTeams>(B, S, T, B.cgitmax, p, red, &iters, &zeta, &rnorm,
                                          &fallbacks);
    else
        rc = solve_system<kMode == kModeMixed, kU, kTeams>(B, S, T, B.cgitmax, p, red, &iters,
                                                           &zeta, &rnorm);
    const bool gave_up = kMode != kModeFixed && rc == kSolveGaveUp;
    if (gave_up) {
        __syncthreads();
        fallbacks = 0;
        rc = solve_system<false, kU, kTeams>(B, S, T, kReferenceCgitmax, p, red, &iters, &zeta,
                                             &rnorm);
    }
    if (rc == kSolveAborted) return false;
    if (threadIdx.x == 0 && member == 0) {
        B.zeta[id] = zeta;
        B.rnorm[id] = rnorm;
        B.iters[id] = iters;
        B.status[id] = gave_up ? 1 : (fallbacks > 0 ? 2 : 0);
        if (B.fallbacks) B.fallbacks[id] = fallbacks;
    }
    return true;
}

// Persistent over a cooperative (co-resident) grid: CTAs take the next work
// slot of `list` (count entries; slot = system * kMaxTeam + member, a team's
// slots adjacent, systems largest first) from the queue until it is empty.
// A member waits for its team only on slots already handed out or the next
// ones to be, so every team forms.  kUnroll: entries a lane loads before it
// uses the first (the loads in flight per SM are threads x kUnroll).
// kTeams: compiled with the team exchanges (a launch whose systems all run
// alone takes the instance without them, which needs fewer registers).
template <int kMode, int kMaxThreads, int kUnroll, bool kTeams>
__global__ void __launch_bounds__(kMaxThreads, 1) batch_kernel(BatchArgs B, const int *list, int count)
{
    extern __shared__ __align__(16) double p_sh[];
    __shared__ double red[32];
    __shared__ int s_next;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_next = ld_relaxed_i32(B.dev_status) != kDevOk ? count : int(atomicAdd(B.queue, 1u));
        __syncthreads();
        const int k = s_next;
        if (k >= count) break;
        const int slot = list[k];
        const int id = slot / kMaxTeam;
        const SysDesc S = B.sys[id];
        if (!run_system<kMode, kUnroll, kTeams>(B, id, slot % kMaxTeam, S, p_sh, red)) break;
    }
}

static __global__ void to_fp32_batch(const double *__restrict__ in, float *__restrict__ out,
                                     long long count)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = float(in[i]);
}

}  // namespace batch
}  // namespace cgb

using namespace cgb;
using namespace cgb::batch;

#define BT_TRY(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(CGB_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                         \
    } while (0)

struct cgb_batch {
    int device = 0;
    int sms = 148;
    int nsys = 0;
    int max_n = 0;
    long long total_nnz = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<SysDesc> desc;
    std::vector<double> mean_len;
    std::vector<long long> nnz;   // stored entries per system
    std::vector<int> order;       // systems, largest first
    std::vector<int> slots;       // work list of the last launch (system * kMaxTeam + member)
    SysDesc *d_sys = nullptr;
    int *d_slots = nullptr;
    int *d_rowstr = nullptr, *d_colidx = nullptr;
    double *d_a = nullptr;
    float *d_a32 = nullptr;
    double *d_x = nullptr, *d_z = nullptr, *d_r = nullptr, *d_q = nullptr, *d_pg = nullptr;
    unsigned *d_queue = nullptr;
    unsigned *d_team_sync = nullptr;
    double *d_team_part = nullptr;
    int *d_dev_status = nullptr;
    double *d_zeta = nullptr, *d_rnorm = nullptr;
    int *d_iters = nullptr, *d_status = nullptr;
    double *d_hx = nullptr, *d_hw = nullptr;  // Galerkin-start ring, kMaxRecycle x vec_total each
    long long vec_total = 0;
    // learned mode: per system the factor F (lower) and F^T as CSR with BF16
    // value bits and 16-bit columns (host copies until the next learned
    // solve packs them), and the device arrays they are packed into
    std::vector<std::vector<int>> h_fptr, h_ftptr;
    std::vector<std::vector<unsigned short>> h_fcol, h_ftcol, h_fval, h_ftval;
    std::vector<std::vector<float>> h_fdiag;
    std::vector<double> fmean;     // factor entries per row
    bool prec_dirty = false;
    int *d_fptr = nullptr, *d_ftptr = nullptr;
    float *d_fdiag = nullptr;
    unsigned short *d_fcol = nullptr, *d_ftcol = nullptr, *d_fval = nullptr, *d_ftval = nullptr;
    double *d_y = nullptr;
    float *d_rg = nullptr, *d_tg = nullptr;
    int *d_fallbacks = nullptr;
    int block = 512;
    int unroll = 4;  // 512-thread shape: 4 or 8 entries a lane in flight (1024 threads: 4)
    // lane policy: lanes = 32 if mean >= t2, 16 if >= t1, 8 if >= t0, else 4
    double t0 = 16.0, t1 = 40.0, t2 = 96.0;
    // team policy: a system gets 2, 4 or 8 CTAs while its work per CTA is
    // above team_frac x (the batch's work / the grid's CTAs); 0 = no teams
    double team_frac = 0.5;
    int resident = 0;  // CTAs of the last launch's grid (team sizes depend on it)
};

namespace {

template <typename T>
cudaError_t balloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

template <typename T>
void bfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

void batch_release(cgb_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    bfree(b->d_sys); bfree(b->d_slots); bfree(b->d_rowstr); bfree(b->d_colidx); bfree(b->d_a);
    bfree(b->d_a32); bfree(b->d_x); bfree(b->d_z); bfree(b->d_r); bfree(b->d_q); bfree(b->d_pg);
    bfree(b->d_queue); bfree(b->d_team_sync); bfree(b->d_team_part); bfree(b->d_dev_status);
    bfree(b->d_zeta); bfree(b->d_rnorm); bfree(b->d_iters); bfree(b->d_status);
    bfree(b->d_hx); bfree(b->d_hw);
    bfree(b->d_fptr); bfree(b->d_ftptr); bfree(b->d_fcol); bfree(b->d_ftcol); bfree(b->d_fval);
    bfree(b->d_ftval); bfree(b->d_fdiag); bfree(b->d_y); bfree(b->d_rg); bfree(b->d_tg); bfree(b->d_fallbacks);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int lanes_by_policy(const cgb_batch *b, double mean)
{
    if (mean >= b->t2) return 32;
    if (mean >= b->t1) return 16;
    if (mean >= b->t0) return 8;
    return 4;
}

// Lanes per row and team size of every system for a grid of `grid` CTAs,
// and the work list (largest systems first, a team's slots adjacent);
// uploaded on the batch's stream.  The work of a system is counted as its
// SpMV bytes (12 a stored entry, 8 a row for p and q).
int apply_policy(cgb_batch *b, int grid)
{
    b->resident = grid;
    std::vector<double> work(b->nsys);
    double total = 0.0;
    for (int i = 0; i < b->nsys; i++) {
        work[i] = 12.0 * double(b->nnz[i]) + 16.0 * b->desc[i].n;
        total += work[i];
    }
    const double per_cta = total / std::max(grid, 1);
    b->slots.clear();
    for (int i : b->order) {
        SysDesc &d = b->desc[i];
        d.lanes = lanes_by_policy(b, b->mean_len[i]);
        d.flanes = b->fmean.empty() ? 4 : lanes_by_policy(b, b->fmean[i]);
        int t = 1;
        if (b->team_frac > 0.0)
            while (t < kMaxTeam && 2 * t <= grid && work[i] / t > b->team_frac * per_cta) t *= 2;
        d.team = t;
        for (int m = 0; m < t; m++) b->slots.push_back(i * kMaxTeam + m);
    }
    BT_TRY(cudaMemcpyAsync(b->d_sys, b->desc.data(), sizeof(SysDesc) * b->nsys,
                           cudaMemcpyHostToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->d_slots, b->slots.data(), sizeof(int) * b->slots.size(),
                           cudaMemcpyHostToDevice, b->stream));
    return CGB_OK;
}

// One cooperative launch (every CTA resident: team members wait for each
// other) of the kernel for the block shape: 512 threads may use 128
// registers a thread, 1024 threads 64.
using BatchKernel = void (*)(BatchArgs, const int *, int);

template <int kMode, bool kTeams>
BatchKernel pick_kernel(const cgb_batch *b)
{
    return b->block > 512 ? batch_kernel<kMode, 1024, 4, kTeams>
                          : (b->unroll > 4 ? batch_kernel<kMode, 512, 8, kTeams>
                                           : batch_kernel<kMode, 512, 4, kTeams>);
}

template <int kMode>
int launch_all(cgb_batch *b, const BatchArgs &A0)
{
    // p (FP64), or in the learned mode p and the factor products' vector in
    // FP32 (the second starting at a 16-byte boundary)
    const size_t smem = sizeof(double) * size_t(b->max_n + 10);
    // residency does not depend on the instance (same shape, one CTA an SM
    // at most by the launch bounds); the policy then says whether any
    // system gets a team
    BatchKernel k = pick_kernel<kMode, true>(b);
    BT_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    BT_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, b->block, smem));
    if (per_sm < 1) return set_error(CGB_ERR_STATE, "batch kernel cannot be resident");
    const int resident = per_sm * b->sms;
    int st = apply_policy(b, resident);
    if (st) return st;
    if (b->slots.size() == size_t(b->nsys)) {  // no teams
        k = pick_kernel<kMode, false>(b);
        BT_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int per = 0;
        BT_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, b->block, smem));
        if (per < per_sm) return set_error(CGB_ERR_STATE, "batch kernel cannot be resident");
    }
    const int count = int(b->slots.size());
    const int grid = std::min(resident, count);
    BT_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned), b->stream));
    BT_TRY(cudaMemsetAsync(b->d_dev_status, 0, sizeof(int), b->stream));
    BT_TRY(cudaMemsetAsync(b->d_team_sync, 0, sizeof(unsigned) * 2 * kSyncStride * b->nsys, b->stream));
    BatchArgs A = A0;
    const int *list = b->d_slots;
    void *args[] = {&A, &list, const_cast<int *>(&count)};
    BT_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(k), dim3(grid), dim3(b->block),
                                       args, smem, b->stream));
    return CGB_OK;
}

// Round-to-nearest-even FP32 -> BF16 bits (NaN kept quiet).
unsigned short bf16_bits(float f)
{
    unsigned u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return static_cast<unsigned short>((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return static_cast<unsigned short>(u >> 16);
}

// Packs every system's factor into the device arrays (after
// cgb_batch_set_preconditioner changed one) and allocates the learned
// mode's vectors.  Every system must have a factor.
int pack_factors(cgb_batch *b)
{
    if (!b->prec_dirty && b->d_fptr) return CGB_OK;
    long long rows = 0, ents = 0;
    for (int i = 0; i < b->nsys; i++) {
        if (b->h_fptr[i].empty())
            return set_error(CGB_ERR_STATE,
                             "batch: learned mode needs a preconditioner for every system (system %d has none)", i);
        rows += b->desc[i].n + 1;
        ents += b->h_fptr[i].back();
    }
    bfree(b->d_fptr); bfree(b->d_ftptr); bfree(b->d_fcol); bfree(b->d_ftcol);
    bfree(b->d_fval); bfree(b->d_ftval); bfree(b->d_fdiag);
    if (balloc(&b->d_fptr, rows) || balloc(&b->d_ftptr, rows) || balloc(&b->d_fdiag, rows) ||
        balloc(&b->d_fcol, ents + 64) ||
        balloc(&b->d_ftcol, ents + 64) || balloc(&b->d_fval, ents + 64) ||
        balloc(&b->d_ftval, ents + 64) ||
        (!b->d_y && (balloc(&b->d_y, b->vec_total) || balloc(&b->d_rg, b->vec_total) ||
                     balloc(&b->d_tg, b->vec_total) || balloc(&b->d_fallbacks, b->nsys))))
        return set_error(CGB_ERR_NOMEM, "batch: factor allocation failed");
    b->fmean.assign(b->nsys, 0.0);
    long long ro = 0, eo = 0;
    for (int i = 0; i < b->nsys; i++) {
        SysDesc &d = b->desc[i];
        const long long ne = b->h_fptr[i].back();
        d.f_row_off = ro;
        d.f_off = eo;
        b->fmean[i] = double(ne) / d.n;  // off-diagonal entries a row
        const size_t nr = size_t(d.n) + 1;
        BT_TRY(cudaMemcpyAsync(b->d_fptr + ro, b->h_fptr[i].data(), sizeof(int) * nr, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_ftptr + ro, b->h_ftptr[i].data(), sizeof(int) * nr, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_fdiag + ro, b->h_fdiag[i].data(), sizeof(float) * d.n, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_fcol + eo, b->h_fcol[i].data(), 2 * ne, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_ftcol + eo, b->h_ftcol[i].data(), 2 * ne, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_fval + eo, b->h_fval[i].data(), 2 * ne, cudaMemcpyHostToDevice, b->stream));
        BT_TRY(cudaMemcpyAsync(b->d_ftval + eo, b->h_ftval[i].data(), 2 * ne, cudaMemcpyHostToDevice, b->stream));
        ro += (long long)nr;
        eo += ne;
    }
    BT_TRY(cudaStreamSynchronize(b->stream));  // the host copies may change after this
    b->prec_dirty = false;
    return CGB_OK;
}

// One launch over all systems (mixed: a system whose mixed solve gives up
// is solved again in FP64 by the same CTAs and marked status 1).
int launch(cgb_batch *b, const cgb_batch_params &P, double *ms)
{
    BatchArgs A{};
    A.nsys = b->nsys;
    A.sys = b->d_sys;
    A.rowstr = b->d_rowstr;
    A.colidx = b->d_colidx;
    A.a = b->d_a;
    A.a32 = b->d_a32;
    A.x = b->d_x;
    A.z = b->d_z;
    A.r = b->d_r;
    A.q = b->d_q;
    A.pg = b->d_pg;
    A.queue = b->d_queue;
    A.team_sync = b->d_team_sync;
    A.team_part = b->d_team_part;
    A.dev_status = b->d_dev_status;
    A.mode = P.mode == CGB_MODE_MIXED ? kModeMixed
             : P.mode == CGB_MODE_MIXED_LEARNED ? kModeLearned : kModeFixed;
    A.fallbacks = b->d_fallbacks;  // (allocated by the first learned solve)
    if (A.mode == kModeLearned) {
        const int st = pack_factors(b);
        if (st) return st;
        A.fptr = b->d_fptr;
        A.ftptr = b->d_ftptr;
        A.fdiag = b->d_fdiag;
        A.fcol = b->d_fcol;
        A.ftcol = b->d_ftcol;
        A.fval = reinterpret_cast<const __nv_bfloat16 *>(b->d_fval);
        A.ftval = reinterpret_cast<const __nv_bfloat16 *>(b->d_ftval);
        A.y = b->d_y;
        A.rg = b->d_rg;
        A.tg = b->d_tg;
        A.fallbacks = b->d_fallbacks;
    }
    A.niter = P.niter;
    A.cgitmax = P.cgitmax;
    A.refresh_every = P.refresh_every > 0 ? P.refresh_every : 10;
    A.tol = P.tol;
    A.zeta = b->d_zeta;
    A.rnorm = b->d_rnorm;
    A.iters = b->d_iters;
    A.status = b->d_status;
    A.hx = b->d_hx;
    A.hw = b->d_hw;
    A.hstride = b->vec_total;
    A.recycle = P.recycle;
    BT_TRY(cudaEventRecord(b->ev0, b->stream));
    const int st = A.mode == kModeLearned ? launch_all<kModeLearned>(b, A)
                   : A.mode == kModeMixed ? launch_all<kModeMixed>(b, A)
                                          : launch_all<kModeFixed>(b, A);
    if (st) return st;
    BT_TRY(cudaEventRecord(b->ev1, b->stream));
    BT_TRY(cudaStreamSynchronize(b->stream));
    int dev = 0;
    BT_TRY(cudaMemcpy(&dev, b->d_dev_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (dev != kDevOk)
        return set_error(CGB_ERR_TIMEOUT, "batch: a team wait ran past %lld ns (device status %d)",
                         kTeamWaitNs, dev);
    float f = 0.f;
    BT_TRY(cudaEventElapsedTime(&f, b->ev0, b->ev1));
    if (ms) *ms = f;
    return CGB_OK;
}

}  // namespace

extern "C" {

void cgb_default_batch_params(cgb_batch_params *p)
{
    if (!p) return;
    p->niter = 15;
    p->mode = CGB_MODE_FP64;
    p->cgitmax = 25;
    p->tol = 1e-12;
    p->refresh_every = 10;
    p->recycle = 4;
}

int cgb_batch_create(int device, int nsys, const int *n, const int *const *rowstr,
                     const int *const *colidx, const double *const *a, const double *shift,
                     cgb_batch **out)
{
    if (!out || nsys < 1 || !n || !rowstr || !colidx || !a || !shift)
        return set_error(CGB_ERR_INVALID, "batch: null argument or no systems");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "no CUDA device %d", device);
    cudaDeviceProp prop;
    BT_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return set_error(CGB_ERR_NO_DEVICE, "device %d is not sm_100", device);
    long long rows_total = 0, nnz_total = 0, vec_total = 0;
    int max_n = 0;
    for (int s = 0; s < nsys; s++) {
        if (n[s] < 1 || n[s] > kBatchMaxN)
            return set_error(CGB_ERR_CAPACITY, "batch: system %d has n = %d (1..%d)", s, n[s],
                             kBatchMaxN);
        if (!rowstr[s] || !colidx[s] || !a[s] || rowstr[s][0] != 0)
            return set_error(CGB_ERR_BAD_MATRIX, "batch: system %d has a bad CSR", s);
        for (int j = 0; j < n[s]; j++)
            if (rowstr[s][j + 1] < rowstr[s][j])
                return set_error(CGB_ERR_BAD_MATRIX, "batch: system %d rowstr decreases", s);
        for (int k = 0; k < rowstr[s][n[s]]; k++)
            if (colidx[s][k] < 0 || colidx[s][k] >= n[s] || !std::isfinite(a[s][k]))
                return set_error(CGB_ERR_BAD_MATRIX, "batch: system %d entry %d invalid", s, k);
        rows_total += n[s] + 1;
        nnz_total += rowstr[s][n[s]];
        vec_total += n[s] + 8;
        max_n = std::max(max_n, n[s]);
    }
    BT_TRY(cudaSetDevice(device));
    cgb_batch *b = new (std::nothrow) cgb_batch;
    if (!b) return set_error(CGB_ERR_NOMEM, "batch allocation failed");
    b->device = device;
    b->sms = prop.multiProcessorCount;
    b->nsys = nsys;
    b->max_n = max_n;
    b->total_nnz = nnz_total;
    b->vec_total = vec_total;
    b->desc.resize(nsys);
    b->h_fptr.resize(nsys);
    b->h_fdiag.resize(nsys);
    b->h_ftptr.resize(nsys);
    b->h_fcol.resize(nsys);
    b->h_ftcol.resize(nsys);
    b->h_fval.resize(nsys);
    b->h_ftval.resize(nsys);
    b->mean_len.resize(nsys);
    b->nnz.resize(nsys);
    long long ro = 0, no = 0, vo = 0;
    for (int s = 0; s < nsys; s++) {
        SysDesc &d = b->desc[s];
        d.n = n[s];
        d.row_off = ro;
        d.nnz_off = no;
        d.vec_off = vo;
        d.shift = shift[s];
        d.lanes = 32;
        d.flanes = 4;
        d.team = 1;
        d.f_row_off = d.f_off = 0;
        b->nnz[s] = rowstr[s][n[s]];
        b->mean_len[s] = double(rowstr[s][n[s]]) / n[s];
        ro += n[s] + 1;
        no += rowstr[s][n[s]];
        vo += n[s] + 8;
    }
    std::vector<int> &order = b->order;
    order.resize(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) {
        return rowstr[i][n[i]] > rowstr[j][n[j]];
    });
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess &&
              !balloc(&b->d_sys, nsys) && !balloc(&b->d_slots, size_t(nsys) * kMaxTeam) &&
              !balloc(&b->d_rowstr, rows_total) && !balloc(&b->d_colidx, nnz_total + 64) &&
              !balloc(&b->d_a, nnz_total + 64) && !balloc(&b->d_a32, nnz_total + 64) &&
              !balloc(&b->d_x, vec_total) && !balloc(&b->d_z, vec_total) &&
              !balloc(&b->d_r, vec_total) && !balloc(&b->d_q, vec_total) &&
              !balloc(&b->d_pg, vec_total) && !balloc(&b->d_queue, 1) &&
              !balloc(&b->d_team_sync, size_t(nsys) * 2 * kSyncStride) &&
              !balloc(&b->d_team_part, size_t(nsys) * 2 * kMaxTeam * kTeamValues) &&
              !balloc(&b->d_dev_status, 1) && !balloc(&b->d_zeta, nsys) && !balloc(&b->d_rnorm, nsys) &&
              !balloc(&b->d_iters, nsys) && !balloc(&b->d_status, nsys) &&
              !balloc(&b->d_hx, kMaxRecycle * vec_total) &&
              !balloc(&b->d_hw, kMaxRecycle * vec_total);
    if (!ok) {
        batch_release(b);
        return set_error(CGB_ERR_NOMEM, "batch device allocation failed");
    }
    for (int s = 0; s < nsys; s++) {
        const SysDesc &d = b->desc[s];
        const long long nz = rowstr[s][n[s]];
        // on the batch's stream, so the FP32 conversion below runs after them
        if (cudaMemcpyAsync(b->d_rowstr + d.row_off, rowstr[s], sizeof(int) * (n[s] + 1),
                            cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
            cudaMemcpyAsync(b->d_colidx + d.nnz_off, colidx[s], sizeof(int) * nz,
                            cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
            cudaMemcpyAsync(b->d_a + d.nnz_off, a[s], sizeof(double) * nz, cudaMemcpyHostToDevice,
                            b->stream) != cudaSuccess) {
            batch_release(b);
            return set_error(CGB_ERR_CUDA, "batch upload failed");
        }
    }
    to_fp32_batch<<<4 * b->sms, 256, 0, b->stream>>>(b->d_a, b->d_a32, nnz_total);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
        batch_release(b);
        return set_error(CGB_ERR_CUDA, "batch set-up failed");
    }
    *out = b;
    return CGB_OK;
}

int cgb_batch_destroy(cgb_batch *b)
{
    batch_release(b);
    return CGB_OK;
}

int cgb_batch_solve(cgb_batch *b, const cgb_batch_params *params, double *zeta, double *rnorm,
                    int *iters, int *status, double *device_ms)
{
    if (!b || !params) return set_error(CGB_ERR_INVALID, "batch: null argument");
    const cgb_batch_params P = *params;
    if (P.niter < 1 || P.cgitmax < 1 ||
        (P.mode != CGB_MODE_FP64 && P.mode != CGB_MODE_MIXED && P.mode != CGB_MODE_MIXED_LEARNED) ||
        (P.mode != CGB_MODE_FP64 && !(P.tol > 0.0)) || P.recycle < 0 || P.recycle > kMaxRecycle)
        return set_error(CGB_ERR_INVALID,
                         "batch: niter, cgitmax >= 1; mode FP64, MIXED or MIXED_LEARNED (tol > 0); "
                         "recycle 0..%d",
                         kMaxRecycle);
    BT_TRY(cudaSetDevice(b->device));
    double ms = 0.0;
    int st = launch(b, P, &ms);
    if (st) return st;
    if (zeta) BT_TRY(cudaMemcpy(zeta, b->d_zeta, sizeof(double) * b->nsys, cudaMemcpyDeviceToHost));
    if (rnorm) BT_TRY(cudaMemcpy(rnorm, b->d_rnorm, sizeof(double) * b->nsys, cudaMemcpyDeviceToHost));
    if (iters) BT_TRY(cudaMemcpy(iters, b->d_iters, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost));
    if (status) BT_TRY(cudaMemcpy(status, b->d_status, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost));
    if (device_ms) *device_ms = ms;
    return CGB_OK;
}

// Autotuner: times the batch (mode and sizes of `params`) for each block
// shape {512 threads with 4 or 8 entries a lane in flight, 1024 threads
// with 4} and each lane policy (row-length thresholds for 4/8/16/32
// lanes per row), then for the best of those each team policy (no teams,
// team_frac 0.25, 0.5, 1), keeps the fastest and reports it.
int cgb_batch_tune(cgb_batch *b, const cgb_batch_params *params, int *block_out, double *t0_out,
                   double *t1_out, double *t2_out, double *best_ms)
{
    if (!b || !params) return set_error(CGB_ERR_INVALID, "batch: null argument");
    BT_TRY(cudaSetDevice(b->device));
    struct Cand {
        int block, unroll;
        double t0, t1, t2;
        double team_frac;
    };
    const Cand shapes[] = {{512, 4, 16, 40, 96, 0.5},  {512, 4, 8, 24, 64, 0.5},
                           {512, 4, 24, 64, 160, 0.5}, {512, 8, 16, 40, 96, 0.5},
                           {512, 8, 8, 24, 64, 0.5},   {512, 8, 24, 64, 160, 0.5},
                           {1024, 4, 16, 40, 96, 0.5}, {1024, 4, 8, 24, 64, 0.5},
                           {512, 4, 1e9, 1e9, 0, 0.5}};
    double best = 1e30;
    Cand bc = shapes[0];
    auto trial = [&](const Cand &c) -> int {
        b->block = c.block;
        b->unroll = c.unroll;
        b->t0 = c.t0;
        b->t1 = c.t1;
        b->t2 = c.t2;
        b->team_frac = c.team_frac;
        double ms = 0.0;
        const int st = launch(b, *params, &ms);
        if (st) return st;
        if (ms < best) {
            best = ms;
            bc = c;
        }
        return CGB_OK;
    };
    for (const Cand &c : shapes) {
        const int st = trial(c);
        if (st) return st;
    }
    const Cand shape = bc;
    for (double f : {0.0, 0.25, 1.0}) {
        Cand c = shape;
        c.team_frac = f;
        const int st = trial(c);
        if (st) return st;
    }
    b->block = bc.block;
    b->unroll = bc.unroll;
    b->t0 = bc.t0;
    b->t1 = bc.t1;
    b->t2 = bc.t2;
    b->team_frac = bc.team_frac;
    if (block_out) *block_out = bc.block;
    if (t0_out) *t0_out = bc.t0;
    if (t1_out) *t1_out = bc.t1;
    if (t2_out) *t2_out = bc.t2;
    if (best_ms) *best_ms = best;
    return CGB_OK;
}

int cgb_batch_policy(cgb_batch *b, int *unroll, double *team_frac, int *teams)
{
    if (!b) return set_error(CGB_ERR_INVALID, "batch: null argument");
    if (unroll) *unroll = b->block > 512 ? 4 : b->unroll;
    if (team_frac) *team_frac = b->team_frac;
    if (teams) {
        // the current policy's teams (tune may have tried another last)
        if (b->resident > 0) {
            const int st = apply_policy(b, b->resident);
            if (st) return st;
        }
        int t = 0;
        for (const SysDesc &d : b->desc) t += d.team > 1;
        *teams = t;
    }
    return CGB_OK;
}

int cgb_batch_set_preconditioner(cgb_batch *b, int sys, const int *fptr, const int *fcol,
                                 const double *fval)
{
    if (!b || !fptr || !fcol || !fval) return set_error(CGB_ERR_INVALID, "batch: null argument");
    if (sys < 0 || sys >= b->nsys) return set_error(CGB_ERR_INVALID, "batch: no system %d", sys);
    const int n = b->desc[sys].n;
    if (fptr[0] != 0) return set_error(CGB_ERR_BAD_MATRIX, "factor: fptr[0] != 0");
    for (int i = 0; i < n; i++) {
        if (fptr[i + 1] < fptr[i]) return set_error(CGB_ERR_BAD_MATRIX, "factor: fptr decreases at %d", i);
        bool diag = false;
        for (int k = fptr[i]; k < fptr[i + 1]; k++) {
            if (fcol[k] < 0 || fcol[k] > i)
                return set_error(CGB_ERR_BAD_MATRIX, "factor: entry (%d, %d) not in the lower triangle", i, fcol[k]);
            if (!std::isfinite(fval[k])) return set_error(CGB_ERR_NUMERIC, "factor: non-finite value in row %d", i);
            if (fcol[k] == i) {
                if (!(fval[k] > 0.0)) return set_error(CGB_ERR_NUMERIC, "factor: diagonal of row %d not positive", i);
                diag = true;
            }
        }
        if (!diag) return set_error(CGB_ERR_BAD_MATRIX, "factor: row %d has no diagonal", i);
    }
    // rows in ascending column order, repeated columns summed; the diagonal
    // (FP32) apart, the rest to BF16 (rounding the diagonal, ~1, to BF16
    // would perturb M about as much as the off-diagonal part corrects)
    std::vector<int> optr(n + 1, 0), ocol;
    std::vector<float> oval, dg(n, 0.f);
    std::vector<std::pair<int, double>> row;
    ocol.reserve(size_t(fptr[n]));
    oval.reserve(size_t(fptr[n]));
    for (int i = 0; i < n; i++) {
        bool ascending = true;  // the common case (the learned factor's rows): no sort
        for (int k = fptr[i] + 1; k < fptr[i + 1]; k++) ascending &= fcol[k] > fcol[k - 1];
        if (ascending) {
            for (int k = fptr[i]; k < fptr[i + 1]; k++) {
                ocol.push_back(fcol[k]);
                oval.push_back(float(fval[k]));
            }
            dg[i] = oval.back();
            ocol.pop_back();
            oval.pop_back();
            optr[i + 1] = int(ocol.size());
            continue;
        }
        row.clear();
        for (int k = fptr[i]; k < fptr[i + 1]; k++) row.emplace_back(fcol[k], fval[k]);
        std::stable_sort(row.begin(), row.end(), [](const std::pair<int, double> &x,
                                                    const std::pair<int, double> &y) {
            return x.first < y.first;
        });
        for (size_t k = 0; k < row.size(); k++) {
            if (k > 0 && row[k].first == row[k - 1].first) {
                row[k].second += row[k - 1].second;
                ocol.pop_back();
                oval.pop_back();
            }
            ocol.push_back(row[k].first);
            oval.push_back(float(row[k].second));
        }
        dg[i] = oval.back();  // the diagonal: the last of the ascending columns <= i
        ocol.pop_back();
        oval.pop_back();
        optr[i + 1] = int(ocol.size());
    }
    const int nf = optr[n];
    std::vector<int> tptr(n + 1, 0);
    for (int k = 0; k < nf; k++) tptr[ocol[k] + 1]++;
    for (int i = 0; i < n; i++) tptr[i + 1] += tptr[i];
    std::vector<unsigned short> tcol(nf), tval(nf), fc(nf), fv(nf);
    std::vector<int> cur(tptr.begin(), tptr.end() - 1);
    for (int i = 0; i < n; i++)
        for (int k = optr[i]; k < optr[i + 1]; k++) {
            const unsigned short bits = bf16_bits(oval[k]);
            fc[k] = static_cast<unsigned short>(ocol[k]);
            fv[k] = bits;
            const int at = cur[ocol[k]]++;
            tcol[at] = static_cast<unsigned short>(i);
            tval[at] = bits;
        }
    b->h_fdiag[sys] = std::move(dg);
    b->h_fptr[sys] = std::move(optr);
    b->h_ftptr[sys] = std::move(tptr);
    b->h_fcol[sys] = std::move(fc);
    b->h_fval[sys] = std::move(fv);
    b->h_ftcol[sys] = std::move(tcol);
    b->h_ftval[sys] = std::move(tval);
    b->prec_dirty = true;
    return CGB_OK;
}

int cgb_batch_fallbacks(cgb_batch *b, int *fallbacks)
{
    if (!b || !fallbacks) return set_error(CGB_ERR_INVALID, "batch: null argument");
    if (!b->d_fallbacks) {
        std::fill(fallbacks, fallbacks + b->nsys, 0);
        return CGB_OK;
    }
    BT_TRY(cudaSetDevice(b->device));
    BT_TRY(cudaMemcpy(fallbacks, b->d_fallbacks, sizeof(int) * b->nsys, cudaMemcpyDeviceToHost));
    return CGB_OK;
}

int cgb_batch_set_team_frac(cgb_batch *b, double team_frac)
{
    if (!b || !(team_frac >= 0.0) || team_frac > 1e6)
        return set_error(CGB_ERR_INVALID, "batch: team_frac must be in [0, 1e6]");
    b->team_frac = team_frac;
    return CGB_OK;
}

}  // extern "C"

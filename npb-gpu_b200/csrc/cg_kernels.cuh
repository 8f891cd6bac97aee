// cg_kernels.cuh -- the FP64 CG kernels of libcgb (sm_100a).
//
// One cooperative, persistent kernel runs a whole outer step of the inverse
// power iteration (GMAP/NPB-GPU CUDA/CG/cg.cu:500-520): the conj_grad
// iterations (cg.cu:653-801), the explicit residual ||x - A z||, and the
// zeta / normalisation update (cg.cu:508-519).  The reference spreads the
// same work over 157 launches and 54 blocking device-to-host copies per
// outer step (kernels one..eleven, cg.cu:848-1265); here the reductions
// finish on the device and every phase boundary is a bounded grid barrier.
//
// Work split: CTA c owns rows [row_split[c], row_split[c+1]), chosen on the
// host so every CTA holds about the same number of stored entries.  A CTA
// computes the SpMV rows it owns and all vector updates of those rows, so
// only the gathers of p (or z) cross CTA boundaries.  Reductions: each CTA
// writes one partial per quantity; after the barrier every CTA sums the
// partials in the same fixed order, so all CTAs take identical control
// decisions and results are run-to-run deterministic.
#pragma once

#include "device_common.cuh"

namespace cgb {

// Partial-sum slots (each holds `gpad` doubles, one per CTA).
enum Slot { kSlotRho = 0, kSlotD = 1, kSlotXX = 2, kSlotRes = 3, kSlotXZ = 4, kSlotZZ = 5,
            kSlotCount = 6 };

// Per-step trace record written by CTA 0.
struct StepTrace {
    double zeta;
    double rnorm;
    double inner;  // inner iterations taken (as double for a flat record)
    double rho;    // final recursive residual norm squared
};

struct OuterArgs {
    int n;
    const int *__restrict__ rowstr;
    const int *__restrict__ colidx;
    const double *__restrict__ a;
    double *x, *z, *p, *q, *r;
    const int *__restrict__ row_split;  // gridDim.x + 1 entries
    double *part;                       // kSlotCount * gpad
    int gpad;
    GridBarrier gb;
    double shift;
    int cgitmax;     // fixed mode: exact count; tolerance mode: cap
    int fixed;       // 1: reference semantics (no tolerance test, z0 = 0)
    double tol;      // tolerance mode: stop when ||r|| <= tol * ||x||
    int warm;        // tolerance mode: z0 = x / (zeta_prev - shift) when step > 0
    int step;        // outer step index (trace slot)
    int finish;      // 1: zeta + x update (power iteration); 0: conj_grad only
    StepTrace *trace;
};

// Streams rows [row0,row1) of the CSR times `v` into `out` with LPR lanes per
// row; each lane covers two consecutive entries per chunk (16-byte value and
// 8-byte index loads from an even start, masked to the row), four chunks in
// flight per trip.  Returns, in the group leader lanes, sum_row dotv[row]*out[row]
// (0 elsewhere; dotv may be null).  a/colidx are padded past nnz so the
// aligned-down and rounded-up vector loads stay inside the allocation.
template <int LPR>
__device__ __forceinline__ double spmv_rows_fp64(const int *__restrict__ rowstr,
                                                 const int *__restrict__ colidx,
                                                 const double *__restrict__ a, const double *v,
                                                 double *out, int row0, int row1,
                                                 const double *dotv)
{
    constexpr int kStep = 2 * LPR;
    constexpr int kUnroll = 4;
    const int lane = threadIdx.x % LPR;
    const int grp = threadIdx.x / LPR;
    const int ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    double dacc = 0.0;
    for (int row = row0 + grp; row < row1; row += ngrp) {
        const int k0 = __ldg(rowstr + row);
        const int k1 = __ldg(rowstr + row + 1);
        double s = 0.0;
        for (int k = (k0 & ~1) + 2 * lane; k < k1; k += kUnroll * kStep) {
            double2 av[kUnroll];
            int2 cv[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    av[u] = ld_stream(reinterpret_cast<const double2 *>(a + kk));
                    cv[u] = ld_stream(reinterpret_cast<const int2 *>(colidx + kk));
                }
            }
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    if (kk >= k0) s = fma(av[u].x, v[cv[u].x], s);
                    if (kk + 1 < k1) s = fma(av[u].y, v[cv[u].y], s);
                }
            }
        }
        s = group_sum<LPR>(s, mask);
        if (lane == 0) {
            out[row] = s;
            if (dotv) dacc = fma(dotv[row], s, dacc);
        }
    }
    return dacc;
}

// Writes this CTA's share of a reduction into slot `slot`.
__device__ __forceinline__ void put_partial(const OuterArgs &A, int slot, double v, double *scratch)
{
    const double s = block_sum(v, scratch);
    if (threadIdx.x == 0) A.part[slot * A.gpad + blockIdx.x] = s;
}

__device__ __forceinline__ double get_total(const OuterArgs &A, int slot, double *bcast)
{
    return all_partials(A.part + slot * A.gpad, gridDim.x, bcast);
}

// Leaves the kernel when a barrier failed (time-out or another CTA's failure).
#define CGB_BARRIER_OR_RETURN(A) \
    do {                         \
        if (!grid_barrier((A).gb)) return; \
    } while (0)

template <int LPR>
__global__ void __launch_bounds__(512, 2) outer_step_fp64(OuterArgs A)
{
    __shared__ double scratch[32];
    __shared__ double bcast[8];
    const int row0 = A.row_split[blockIdx.x];
    const int row1 = A.row_split[blockIdx.x + 1];
    // the reference initialises n+1 vector entries (cg.cu:670-675); the
    // last CTA also owns entry n, which never enters a dot product
    const int vend = (blockIdx.x == gridDim.x - 1) ? row1 + 1 : row1;

    // ---- start of conj_grad: z0, r0 = x - A z0, p0 = r0, rho0 = r0.r0
    double zeta_prev = 0.0;
    const bool warm = (!A.fixed) && A.warm && A.step > 0;
    if (warm) zeta_prev = A.trace[A.step - 1].zeta;
    double acc = 0.0, accx = 0.0;
    if (!warm) {
        for (int j = row0 + threadIdx.x; j < vend; j += blockDim.x) {
            const double xv = A.x[j];
            A.q[j] = 0.0;
            A.z[j] = 0.0;
            A.r[j] = xv;
            A.p[j] = xv;
            if (j < A.n) acc = fma(xv, xv, acc);
        }
        put_partial(A, kSlotRho, acc, scratch);
    } else {
        const double mu = 1.0 / (zeta_prev - A.shift);
        for (int j = row0 + threadIdx.x; j < vend; j += blockDim.x) {
            const double xv = A.x[j];
            A.q[j] = 0.0;
            A.z[j] = (j < A.n) ? mu * xv : 0.0;
        }
        CGB_BARRIER_OR_RETURN(A);
        // r = x - A z0 (own rows); the SpMV writes A z0 into r first
        spmv_rows_fp64<LPR>(A.rowstr, A.colidx, A.a, A.z, A.r, row0, row1, nullptr);
        __syncthreads();
        for (int j = row0 + threadIdx.x; j < vend; j += blockDim.x) {
            const double xv = A.x[j];
            const double rv = (j < A.n) ? xv - A.r[j] : xv;
            A.r[j] = rv;
            A.p[j] = rv;
            if (j < A.n) {
                acc = fma(rv, rv, acc);
                accx = fma(xv, xv, accx);
            }
        }
        put_partial(A, kSlotRho, acc, scratch);
        put_partial(A, kSlotXX, accx, scratch);
    }
    CGB_BARRIER_OR_RETURN(A);
    double rho = get_total(A, kSlotRho, &bcast[0]);
    const double xx = warm ? get_total(A, kSlotXX, &bcast[1]) : rho;
    const double stop2 = A.tol * A.tol * xx;

    // ---- CG iterations (cg.cu:678-768)
    int it = 0;
    for (; it < A.cgitmax; it++) {
        if (!A.fixed && rho <= stop2) break;
        // q = A p, d = p.q
        acc = spmv_rows_fp64<LPR>(A.rowstr, A.colidx, A.a, A.p, A.q, row0, row1, A.p);
        put_partial(A, kSlotD, acc, scratch);
        CGB_BARRIER_OR_RETURN(A);
        const double d = get_total(A, kSlotD, &bcast[2]);
        const double alpha = rho / d;
        const double rho0 = rho;
        // z += alpha p, r -= alpha q, rho = r.r
        acc = 0.0;
        for (int j = row0 + threadIdx.x; j < row1; j += blockDim.x) {
            A.z[j] = fma(alpha, A.p[j], A.z[j]);
            const double rv = fma(-alpha, A.q[j], A.r[j]);
            A.r[j] = rv;
            acc = fma(rv, rv, acc);
        }
        put_partial(A, kSlotRho, acc, scratch);
        CGB_BARRIER_OR_RETURN(A);
        rho = get_total(A, kSlotRho, &bcast[3]);
        const double beta = rho / rho0;
        // p = r + beta p
        for (int j = row0 + threadIdx.x; j < row1; j += blockDim.x)
            A.p[j] = fma(beta, A.p[j], A.r[j]);
        CGB_BARRIER_OR_RETURN(A);
    }

    // ---- rnorm = ||x - A z|| (cg.cu:777-800), x.z and z.z (cg.cu:508-511)
    spmv_rows_fp64<LPR>(A.rowstr, A.colidx, A.a, A.z, A.r, row0, row1, nullptr);
    __syncthreads();
    double res = 0.0, xz = 0.0, zz = 0.0;
    for (int j = row0 + threadIdx.x; j < row1; j += blockDim.x) {
        const double xv = A.x[j], zv = A.z[j];
        const double dv = xv - A.r[j];
        res = fma(dv, dv, res);
        xz = fma(xv, zv, xz);
        zz = fma(zv, zv, zz);
    }
    put_partial(A, kSlotRes, res, scratch);
    put_partial(A, kSlotXZ, xz, scratch);
    put_partial(A, kSlotZZ, zz, scratch);
    CGB_BARRIER_OR_RETURN(A);
    const double sum = get_total(A, kSlotRes, &bcast[4]);
    const double t1 = get_total(A, kSlotXZ, &bcast[5]);
    const double t2 = get_total(A, kSlotZZ, &bcast[6]);
    const double rnorm = sqrt(sum);
    const double zeta = A.shift + 1.0 / t1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.trace[A.step].zeta = zeta;
        A.trace[A.step].rnorm = rnorm;
        A.trace[A.step].inner = double(it);
        A.trace[A.step].rho = rho;
        if (!isfinite(zeta) || !isfinite(rnorm)) raise_status(A.gb.status, kDevNonFinite);
    }
    if (A.finish) {
        const double norm = 1.0 / sqrt(t2);
        for (int j = row0 + threadIdx.x; j < row1; j += blockDim.x) A.x[j] = norm * A.z[j];
    }
}

// x = 1 over n+1 entries (cg.cu:485-488).
__global__ void fill_ones(double *x, int count)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        x[j] = 1.0;
}

// Standalone q = A p with the p.q reduction fused (the work of reference
// kernels three and four, cg.cu:937-1004): per-CTA partials, the last CTA to
// finish (ticket counter) sums them in a fixed order into *dot.
struct SpmvArgs {
    int n;
    const int *__restrict__ rowstr;
    const int *__restrict__ colidx;
    const double *__restrict__ a;
    const double *p;
    double *q;
    const int *__restrict__ row_split;
    double *part;
    unsigned *ticket;
    double *dot;
};

template <int LPR>
__global__ void __launch_bounds__(512, 2) spmv_dot_fp64(SpmvArgs S)
{
    __shared__ double scratch[32];
    __shared__ bool last;
    const int row0 = S.row_split[blockIdx.x];
    const int row1 = S.row_split[blockIdx.x + 1];
    double acc = spmv_rows_fp64<LPR>(S.rowstr, S.colidx, S.a, S.p, S.q, row0, row1, S.p);
    const double s = block_sum(acc, scratch);
    if (threadIdx.x == 0) {
        S.part[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(S.ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        if (threadIdx.x < 32) {
            double t = 0.0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) t += __ldcg(S.part + i);
            t = warp_sum(t);
            if (threadIdx.x == 0) {
                *S.dot = t;
                *S.ticket = 0u;
            }
        }
    }
}

// Self-test of the bounded wait: CTA 1 never arrives, so CTA 0's barrier
// wait runs into its limit and records kDevTimeout.
__global__ void barrier_timeout_probe(GridBarrier gb)
{
    if (blockIdx.x == 1) return;
    (void)grid_barrier(gb);
}

}  // namespace cgb

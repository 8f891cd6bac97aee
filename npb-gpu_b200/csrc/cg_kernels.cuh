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
//
// Two SpMV policies share the CG body:
//   RowSpmv<LPR>        LPR lanes per row, the gathered vector read through
//                       L1/L2 (any CSR);
//   TiledSpmv<LPR, R>   the gathered vector staged through shared memory in
//                       column blocks of W entries by TMA bulk copies
//                       (cp.async.bulk + mbarrier, double-buffered), each
//                       row's entries of block b streamed from the segment
//                       [seg[b][j], seg[b+1][j]) of the unchanged CSR
//                       (columns sorted within rows), partial row sums kept
//                       in shared memory.  Gathers become shared-memory
//                       loads instead of random 32-byte L2 sector reads.
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

// Column tiling of the CSR for TiledSpmv.
struct Tiling {
    const int *__restrict__ seg;  // (nblk + 1) x seg_stride entry offsets
    int seg_stride;               // >= n
    int nblk;                     // number of column blocks
    int width;                    // columns per block (entries of the staged vector)
    int max_rows;                 // capacity of the shared row accumulator
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
    Tiling tile;
    double shift;
    int cgitmax;     // fixed mode: exact count; tolerance mode: cap
    int fixed;       // 1: reference semantics (no tolerance test, z0 = 0)
    double tol;      // tolerance mode: stop when ||r|| <= tol * ||x||
    int warm;        // tolerance mode: z0 = x / (zeta_prev - shift) when step > 0
    int step;        // outer step index (trace slot)
    int finish;      // 1: zeta + x update (power iteration); 0: conj_grad only
    StepTrace *trace;
};

// ------------------------------------------------------------ row policy
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

template <int LPR>
struct RowSpmv {
    static constexpr int kThreads = 512;
    static constexpr int kMinBlocks = 2;
    int row0, row1;
    __device__ void setup(const OuterArgs &, int r0, int r1)
    {
        row0 = r0;
        row1 = r1;
    }
    // out[own rows] = (A v)[own rows]; returns this thread's share of dotv.out.
    // `ok` is cleared when a wait failed (never, for this policy).
    __device__ __forceinline__ double apply(const OuterArgs &A, const double *v, double *out,
                                            const double *dotv, bool &ok)
    {
        ok = true;
        return spmv_rows_fp64<LPR>(A.rowstr, A.colidx, A.a, v, out, row0, row1, dotv);
    }
};

// ---------------------------------------------------------- tiled policy
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Orders earlier generic-proxy accesses before later async-proxy (TMA) ones.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

// 1-D bulk copy global -> shared completing on `bar` (one elected thread).
// src, dst 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes,
                                          uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of `bar`; false after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if ((long long)(global_ns() - t0) > limit_ns) return false;
    return true;
}

// Dynamic shared memory of TiledSpmv: two staging buffers of `width`
// doubles, the row accumulator, two mbarriers.
__host__ __device__ inline size_t tiled_smem_bytes(int width, int max_rows)
{
    return size_t(2) * width * sizeof(double) + size_t(max_rows) * sizeof(double) + 64;
}

template <int LPR, int R>
struct TiledSpmv {
    static constexpr int kThreads = 1024;
    static constexpr int kMinBlocks = 1;
    static constexpr int kChunks = 2;  // chunks of 2*LPR entries in flight per row
    int row0, row1;
    double *buf;      // 2 x width
    double *acc;      // max_rows
    uint64_t *bars;   // 2
    unsigned parity;  // bit i: next phase parity of buffer i

    __device__ void setup(const OuterArgs &A, int r0, int r1)
    {
        extern __shared__ __align__(128) unsigned char tiled_smem[];
        row0 = r0;
        row1 = r1;
        buf = reinterpret_cast<double *>(tiled_smem);
        acc = buf + 2 * size_t(A.tile.width);
        bars = reinterpret_cast<uint64_t *>(acc + A.tile.max_rows);
        parity = 0;
        if (threadIdx.x == 0) {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
        }
        __syncthreads();
    }

    __device__ __forceinline__ void issue(const OuterArgs &A, const double *v, int b, int slot)
    {
        const int w = A.tile.width;
        const int cols = min(w, A.n - b * w);
        const unsigned bytes = (unsigned(cols) * 8u + 15u) & ~15u;
        bulk_load(buf + size_t(slot) * w, v + size_t(b) * w, bytes, &bars[slot]);
    }

    __device__ __forceinline__ double apply(const OuterArgs &A, const double *v, double *out,
                                            const double *dotv, bool &ok)
    {
        const Tiling &T = A.tile;
        const int lane = threadIdx.x % LPR;
        const int grp = threadIdx.x / LPR;
        const int ngrp = blockDim.x / LPR;
        const unsigned mask =
            LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
        const int nrows = row1 - row0;
        for (int i = threadIdx.x; i < nrows; i += blockDim.x) acc[i] = 0.0;
        if (threadIdx.x == 0) {
            fence_proxy_async();  // v was written by generic stores before the grid barrier
            issue(A, v, 0, 0);
            if (T.nblk > 1) issue(A, v, 1, 1);
        }
        __syncthreads();
        bool failed = false;
        for (int b = 0; b < T.nblk; b++) {
            const int slot = b & 1;
            if (!mbar_wait(&bars[slot], (parity >> slot) & 1u, A.gb.limit_ns)) failed = true;
            parity ^= 1u << slot;
            if (!failed) {
                const double *pv = buf + size_t(slot) * T.width - size_t(b) * T.width;
                const int *sb = T.seg + size_t(b) * T.seg_stride;
                const int *se = sb + T.seg_stride;
                for (int j0 = row0 + grp; j0 < row1; j0 += R * ngrp) {
                    int k0[R], k1[R];
                    double s[R];
                    int span = 0;
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        const int j = j0 + r * ngrp;
                        k0[r] = (j < row1) ? __ldg(sb + j) : 0;
                        k1[r] = (j < row1) ? __ldg(se + j) : 0;
                        s[r] = 0.0;
                        span = max(span, k1[r] - (k0[r] & ~1));
                    }
                    for (int off = 2 * lane; off < span; off += 2 * LPR * kChunks) {
                        double2 av[R][kChunks];
                        int2 cv[R][kChunks];
#pragma unroll
                        for (int r = 0; r < R; r++)
#pragma unroll
                            for (int c = 0; c < kChunks; c++) {
                                const int kk = (k0[r] & ~1) + off + c * 2 * LPR;
                                if (kk < k1[r]) {
                                    av[r][c] = ld_stream(reinterpret_cast<const double2 *>(A.a + kk));
                                    cv[r][c] = ld_stream(reinterpret_cast<const int2 *>(A.colidx + kk));
                                }
                            }
#pragma unroll
                        for (int r = 0; r < R; r++)
#pragma unroll
                            for (int c = 0; c < kChunks; c++) {
                                const int kk = (k0[r] & ~1) + off + c * 2 * LPR;
                                if (kk < k1[r]) {
                                    if (kk >= k0[r]) s[r] = fma(av[r][c].x, pv[cv[r][c].x], s[r]);
                                    if (kk + 1 < k1[r]) s[r] = fma(av[r][c].y, pv[cv[r][c].y], s[r]);
                                }
                            }
                    }
#pragma unroll
                    for (int r = 0; r < R; r++) {
                        const double t = group_sum<LPR>(s[r], mask);
                        const int j = j0 + r * ngrp;
                        if (lane == 0 && j < row1) acc[j - row0] += t;
                    }
                }
            }
            // everyone is done with this slot; refill it with block b+2
            if (__syncthreads_or(failed)) {
                ok = false;
                if (threadIdx.x == 0) raise_status(A.gb.status, kDevTimeout);
                // let the copies already issued (blocks b and b+1) land before
                // the CTA leaves; a completed phase returns at once
                (void)mbar_wait(&bars[slot], ((parity >> slot) & 1u) ^ 1u, A.gb.limit_ns);
                if (b + 1 < T.nblk)
                    (void)mbar_wait(&bars[slot ^ 1], (parity >> (slot ^ 1)) & 1u, A.gb.limit_ns);
                return 0.0;
            }
            if (threadIdx.x == 0 && b + 2 < T.nblk) {
                fence_proxy_async();  // generic reads of the slot before the async refill
                issue(A, v, b + 2, slot);
            }
        }
        double dacc = 0.0;
        for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
            const double t = acc[i];
            out[row0 + i] = t;
            if (dotv) dacc = fma(dotv[row0 + i], t, dacc);
        }
        ok = true;
        return dacc;
    }
};

// ------------------------------------------------------------- CG body
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
#define CGB_SPMV_OR_RETURN(ok) \
    do {                       \
        if (!(ok)) return;     \
    } while (0)

template <class Spmv>
__device__ __forceinline__ void outer_step_body(const OuterArgs &A)
{
    __shared__ double scratch[32];
    __shared__ double bcast[8];
    const int row0 = A.row_split[blockIdx.x];
    const int row1 = A.row_split[blockIdx.x + 1];
    Spmv sp;
    sp.setup(A, row0, row1);
    bool ok = true;
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
        sp.apply(A, A.z, A.r, nullptr, ok);
        CGB_SPMV_OR_RETURN(ok);
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
        acc = sp.apply(A, A.p, A.q, A.p, ok);
        CGB_SPMV_OR_RETURN(ok);
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
    sp.apply(A, A.z, A.r, nullptr, ok);
    CGB_SPMV_OR_RETURN(ok);
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

template <int LPR>
__global__ void __launch_bounds__(512, 2) outer_step_fp64(OuterArgs A)
{
    outer_step_body<RowSpmv<LPR>>(A);
}

template <int LPR, int R>
__global__ void __launch_bounds__(1024, 1) outer_step_fp64_tiled(OuterArgs A)
{
    outer_step_body<TiledSpmv<LPR, R>>(A);
}

// x = 1 over n+1 entries (cg.cu:485-488).
static __global__ void fill_ones(double *x, int count)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        x[j] = 1.0;
}

// Standalone q = A p with the p.q reduction fused (the work of reference
// kernels three and four, cg.cu:937-1004): per-CTA partials, the last CTA to
// finish (ticket counter) sums them in a fixed order into *dot.
struct SpmvArgs {
    OuterArgs A;      // matrix, vectors p/q, row split, tiling
    unsigned *ticket;
    double *dot;
};

template <class Spmv>
__device__ __forceinline__ void spmv_dot_body(const SpmvArgs &S)
{
    __shared__ double scratch[32];
    __shared__ bool last;
    const OuterArgs &A = S.A;
    Spmv sp;
    sp.setup(A, A.row_split[blockIdx.x], A.row_split[blockIdx.x + 1]);
    bool ok = true;
    double acc = sp.apply(A, A.p, A.q, A.p, ok);
    if (!ok) return;
    const double s = block_sum(acc, scratch);
    if (threadIdx.x == 0) {
        A.part[blockIdx.x] = s;
        __threadfence();
        last = (atomicAdd(S.ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        __threadfence();
        if (threadIdx.x < 32) {
            double t = 0.0;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) t += __ldcg(A.part + i);
            t = warp_sum(t);
            if (threadIdx.x == 0) {
                *S.dot = t;
                *S.ticket = 0u;
            }
        }
    }
}

template <int LPR>
__global__ void __launch_bounds__(512, 2) spmv_dot_fp64(SpmvArgs S)
{
    spmv_dot_body<RowSpmv<LPR>>(S);
}

template <int LPR, int R>
__global__ void __launch_bounds__(1024, 1) spmv_dot_fp64_tiled(SpmvArgs S)
{
    spmv_dot_body<TiledSpmv<LPR, R>>(S);
}

// Segment table of the column tiling: seg[b*stride + j] = first entry of row
// j whose column is >= b*width (b < nblk), seg[nblk*stride + j] = end of row
// j; *unsorted is set when some row's columns do not ascend.
static __global__ void build_segments(const int *__restrict__ rowstr, const int *__restrict__ colidx,
                               int n, int nblk, int width, int *seg, int stride, int *unsorted)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int k0 = rowstr[j], k1 = rowstr[j + 1];
        int bad = 0;
        for (int k = k0 + 1; k < k1; k++) bad |= (colidx[k] <= colidx[k - 1]);
        if (bad) atomicOr(unsorted, 1);
        for (int b = 0; b < nblk; b++) {
            const int lo_col = b * width;
            int lo = k0, hi = k1;  // first k with colidx[k] >= lo_col
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (colidx[mid] < lo_col) lo = mid + 1;
                else hi = mid;
            }
            seg[size_t(b) * stride + j] = lo;
        }
        seg[size_t(nblk) * stride + j] = k1;
    }
}

// Self-test of the bounded wait: CTA 1 never arrives, so CTA 0's barrier
// wait runs into its limit and records kDevTimeout.
static __global__ void barrier_timeout_probe(GridBarrier gb)
{
    if (blockIdx.x == 1) return;
    (void)grid_barrier(gb);
}

}  // namespace cgb

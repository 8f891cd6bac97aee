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
// Lanes per row are a per-system choice (the autotuner's, by row length).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "cgb_internal.h"
#include "device_common.cuh"
#include "galerkin.cuh"

namespace cgb {
namespace batch {

constexpr int kBatchMaxN = 27000;  // rows of the largest system (shared p: 8 bytes a row)
constexpr int kReferenceCgitmax = 25;  // cg.cu's cgitmax: the FP64 re-solve of a mixed failure

struct SysDesc {
    int n;
    int lanes;           // lanes per row (2, 4, 8, 16, 32)
    long long row_off;   // into rowstr_all (n+1 entries)
    long long nnz_off;   // into colidx_all / a_all
    long long vec_off;   // into the vector arrays (n+8 entries)
    double shift;
};

struct BatchArgs {
    int nsys;
    const SysDesc *__restrict__ sys;
    const int *__restrict__ order;      // systems, largest first
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
};

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

// q[j] = (A v)[j] for all rows of the system with LPR lanes per row; v in
// shared memory (FP64), products in FP64 or (F32) in FP32 with FP32 row sums;
// returns this thread's share of sum_j dv[j] q[j] (dv: shared p or null).
template <int LPR, bool F32>
__device__ __forceinline__ double sys_spmv(const BatchArgs &B, const SysDesc &S, const double *v_sh,
                                           const double *v_gl, double *q, const double *dv_sh)
{
    const int *rowstr = B.rowstr + S.row_off;
    const int *colidx = B.colidx + S.nnz_off;
    const double *a = B.a + S.nnz_off;
    const float *a32 = B.a32 ? B.a32 + S.nnz_off : nullptr;
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    double dacc = 0.0;
    for (int row = grp; row < S.n; row += ngrp) {
        const int k0 = rowstr[row], k1 = rowstr[row + 1];
        double s64 = 0.0;
        float s32 = 0.f;
        for (int k = k0 + lane; k < k1; k += 4 * LPR) {
            int c[4];
            double av[4];
            float af[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int kk = k + u * LPR;
                if (kk < k1) {
                    c[u] = __ldcs(colidx + kk);
                    if (F32) af[u] = __ldcs(a32 + kk);
                    else av[u] = __ldcs(a + kk);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (k + u * LPR < k1) {
                    const double pv = v_sh ? v_sh[c[u]] : v_gl[c[u]];
                    if (F32) s32 = fmaf(af[u], float(pv), s32);
                    else s64 = fma(av[u], pv, s64);
                }
            }
        }
        double s;
        if (F32) s = double(group_sum_f<LPR>(s32, mask));
        else s = group_sum<LPR>(s64, mask);
        if (lane == 0) {
            q[row] = s;
            if (dv_sh) dacc = fma(dv_sh[row], s, dacc);
        }
    }
    return dacc;
}

// One system's power iteration.  Returns false when the mixed iteration met
// p.Ap >= 0, a non-finite residual, or did not converge (the caller then
// runs the fixed mode).
template <int LPR, bool mixed>
__device__ bool solve_system(const BatchArgs &B, const SysDesc &S, double *p, double *red,
                             int *iters_out, double *zeta_out, double *rnorm_out)
{
    const int n = S.n;
    double *x = B.x + S.vec_off, *z = B.z + S.vec_off, *r = B.r + S.vec_off, *q = B.q + S.vec_off;
    for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = 1.0;
    __syncthreads();
    int total = 0;
    double zeta = 0.0, rnorm = 0.0;
    for (int outer = 0; outer < B.niter; outer++) {
        double acc = 0.0;
        const int m = B.recycle;
        const int v = (mixed && m > 0) ? min(outer, m) : 0;
        double xx = 0.0;
        if (v > 0) {
            // Galerkin start on x_k .. x_{k-v+1}: z0 = V y, A z0 = W y
            __shared__ double g_sh[kGramValues];
            __shared__ double y_sh[kMaxRecycle];
            long long off[kMaxRecycle];
#pragma unroll
            for (int a = 0; a < kMaxRecycle; a++)
                off[a] = ((outer - a) % m + m) % m * B.hstride + S.vec_off;
            const int npairs = v * (v + 1) / 2;
            double vals[kGramValues];
#pragma unroll
            for (int q = 0; q < kGramValues; q++) vals[q] = 0.0;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const double xv = x[j];
#pragma unroll
                for (int b = 0; b < kMaxRecycle; b++) {
                    if (b < v) {
                        const double xb = B.hx[off[b] + j], wb = B.hw[off[b] + j];
#pragma unroll
                        for (int a = 0; a <= b; a++)
                            vals[gram_index(a, b)] = fma(a == b ? xb : B.hx[off[a] + j], wb,
                                                         vals[gram_index(a, b)]);
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
            cta_sum_multi(packed, npairs + v, g_sh);
            if (threadIdx.x == 0) {
                double g[kGramValues], y[kMaxRecycle];
                for (int q = 0; q < kGramValues; q++) g[q] = 0.0;
                for (int q = 0; q < npairs; q++) g[q] = g_sh[q];
                for (int b = 0; b < v; b++) g[kGramPairs + b] = g_sh[npairs + b];
                galerkin_solve(g, v, y);
                for (int a = 0; a < kMaxRecycle; a++) y_sh[a] = a < v ? y[a] : 0.0;
            }
            __syncthreads();
            xx = g_sh[npairs];  // x_k . x_k
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                double z0 = 0.0, az = 0.0;
#pragma unroll
                for (int a = 0; a < kMaxRecycle; a++) {
                    if (a < v) {
                        z0 = fma(y_sh[a], B.hx[off[a] + j], z0);
                        az = fma(y_sh[a], B.hw[off[a] + j], az);
                    }
                }
                const double rv = x[j] - az;
                z[j] = z0;
                r[j] = rv;
                p[j] = rv;
                acc = fma(rv, rv, acc);
            }
        } else {
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const double xv = x[j];
                z[j] = 0.0;
                r[j] = xv;
                p[j] = xv;
                acc = fma(xv, xv, acc);
            }
        }
        double rho = cta_sum(acc, red);  // includes a barrier: p complete
        if (v == 0) xx = rho;
        const double stop2 = B.tol * B.tol * xx;
        double rho_cycle = rho;
        int it = 0, since = 0;
        bool fresh = true;
        for (;;) {
            if (!mixed) {
                if (it >= B.cgitmax) break;
            } else {
                bool refresh = false;
                if (rho <= stop2) {
                    if (fresh) break;
                    refresh = true;
                } else if (!fresh && (since >= B.refresh_every || rho <= 1e-12 * rho_cycle)) {
                    refresh = true;
                }
                if (!refresh && it >= B.cgitmax) return false;  // not converged: fall back
                if (refresh) {
                    // r = x - A z (FP64 matrix, z from global memory), restart p = r
                    sys_spmv<LPR, false>(B, S, nullptr, z, q, nullptr);
                    __syncthreads();
                    acc = 0.0;
                    for (int j = threadIdx.x; j < n; j += blockDim.x) {
                        const double rv = x[j] - q[j];
                        r[j] = rv;
                        p[j] = rv;
                        acc = fma(rv, rv, acc);
                    }
                    rho = cta_sum(acc, red);
                    rho_cycle = rho;
                    since = 0;
                    fresh = true;
                    continue;
                }
            }
            const double dpart = mixed ? sys_spmv<LPR, true>(B, S, p, nullptr, q, p)
                                       : sys_spmv<LPR, false>(B, S, p, nullptr, q, p);
            const double d = cta_sum(dpart, red);  // barrier: q complete
            if (mixed && !(d < 0.0)) return false;  // not negative definite (or NaN): fall back
            const double alpha = rho / d;
            const double rho0 = rho;
            acc = 0.0;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                z[j] = fma(alpha, p[j], z[j]);
                const double rv = fma(-alpha, q[j], r[j]);
                r[j] = rv;
                acc = fma(rv, rv, acc);
            }
            rho = cta_sum(acc, red);
            if (mixed && !(rho < INFINITY)) return false;  // non-finite residual: fall back
            const double beta = rho / rho0;
            for (int j = threadIdx.x; j < n; j += blockDim.x) p[j] = fma(beta, p[j], r[j]);
            __syncthreads();
            it++;
            since++;
            fresh = false;
        }
        total += it;
        // q = A z (FP64): a product, or from the true residual r = x - A z
        // the mixed iteration just accepted; rnorm = ||x - A z||, x.z, z.z
        if (mixed && fresh) {
            for (int j = threadIdx.x; j < n; j += blockDim.x) q[j] = x[j] - r[j];
        } else {
            sys_spmv<LPR, false>(B, S, nullptr, z, q, nullptr);
        }
        __syncthreads();
        double res = 0.0, xz = 0.0, zz = 0.0;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double xv = x[j], zv = z[j], dv = xv - q[j];
            res = fma(dv, dv, res);
            xz = fma(xv, zv, xz);
            zz = fma(zv, zv, zz);
        }
        rnorm = sqrt(cta_sum(res, red));
        const double t1 = cta_sum(xz, red);
        const double t2 = cta_sum(zz, red);
        zeta = S.shift + 1.0 / t1;
        const double norm = 1.0 / sqrt(t2);
        if (mixed && m > 0) {
            // the next iterate and A times it into the ring
            const long long slot = (outer + 1) % m * B.hstride + S.vec_off;
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                const double xn = norm * z[j];
                B.hx[slot + j] = xn;
                B.hw[slot + j] = norm * q[j];
                x[j] = xn;
            }
        } else {
            for (int j = threadIdx.x; j < n; j += blockDim.x) x[j] = norm * z[j];
        }
        __syncthreads();
    }
    *iters_out = total;
    *zeta_out = zeta;
    *rnorm_out = rnorm;
    return true;
}

// One system; status 1 marks a mixed solve that must be redone in FP64
// (the host launches the FP64 kernel on those systems next).
template <int LPR, bool mixed>
__device__ void run_system(const BatchArgs &B, int id, double *p, double *red)
{
    const SysDesc S = B.sys[id];
    int iters = 0;
    double zeta = 0.0, rnorm = 0.0;
    const bool ok = solve_system<LPR, mixed>(B, S, p, red, &iters, &zeta, &rnorm);
    if (threadIdx.x == 0) {
        B.zeta[id] = zeta;
        B.rnorm[id] = rnorm;
        B.iters[id] = iters;
        B.status[id] = ok ? 0 : 1;
    }
}

// Persistent: CTAs take the next system of `list` (count entries) from the
// work queue until it is empty.
template <bool mixed, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads, 1) batch_kernel(BatchArgs B, const int *list, int count)
{
    extern __shared__ __align__(16) double p_sh[];
    __shared__ double red[32];
    __shared__ int s_next;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_next = int(atomicAdd(B.queue, 1u));
        __syncthreads();
        const int k = s_next;
        if (k >= count) break;
        const int id = list[k];
        switch (B.sys[id].lanes) {
        case 2: run_system<2, mixed>(B, id, p_sh, red); break;
        case 4: run_system<4, mixed>(B, id, p_sh, red); break;
        case 8: run_system<8, mixed>(B, id, p_sh, red); break;
        case 16: run_system<16, mixed>(B, id, p_sh, red); break;
        default: run_system<32, mixed>(B, id, p_sh, red); break;
        }
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
    SysDesc *d_sys = nullptr;
    int *d_order = nullptr;
    int *d_rowstr = nullptr, *d_colidx = nullptr;
    double *d_a = nullptr;
    float *d_a32 = nullptr;
    double *d_x = nullptr, *d_z = nullptr, *d_r = nullptr, *d_q = nullptr;
    unsigned *d_queue = nullptr;
    double *d_zeta = nullptr, *d_rnorm = nullptr;
    int *d_iters = nullptr, *d_status = nullptr;
    int *d_redo = nullptr;
    double *d_hx = nullptr, *d_hw = nullptr;  // Galerkin-start ring, kMaxRecycle x vec_total each
    long long vec_total = 0;
    int block = 512;
    // lane policy: lanes = 32 if mean >= t2, 16 if >= t1, 8 if >= t0, else 4
    double t0 = 16.0, t1 = 40.0, t2 = 96.0;
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
    bfree(b->d_sys); bfree(b->d_order); bfree(b->d_rowstr); bfree(b->d_colidx); bfree(b->d_a);
    bfree(b->d_a32); bfree(b->d_x); bfree(b->d_z); bfree(b->d_r); bfree(b->d_q);
    bfree(b->d_queue); bfree(b->d_zeta); bfree(b->d_rnorm); bfree(b->d_iters); bfree(b->d_status); bfree(b->d_redo);
    bfree(b->d_hx); bfree(b->d_hw);
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

int apply_lanes(cgb_batch *b)
{
    for (int i = 0; i < b->nsys; i++) b->desc[i].lanes = lanes_by_policy(b, b->mean_len[i]);
    BT_TRY(cudaMemcpy(b->d_sys, b->desc.data(), sizeof(SysDesc) * b->nsys, cudaMemcpyHostToDevice));
    return CGB_OK;
}

// The kernel for a block shape: 512 threads may use 128 registers a thread,
// 1024 threads 64.
template <bool mixed>
int launch_list(cgb_batch *b, const BatchArgs &A, const int *d_list, int count)
{
    if (count == 0) return CGB_OK;
    void (*k)(BatchArgs, const int *, int) =
        b->block > 512 ? batch_kernel<mixed, 1024> : batch_kernel<mixed, 512>;
    const size_t smem = sizeof(double) * size_t(b->max_n + 8);
    BT_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    BT_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, b->block, smem));
    if (per_sm < 1) return set_error(CGB_ERR_STATE, "batch kernel cannot be resident");
    const int grid = std::min(per_sm * b->sms, count);
    BT_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned), b->stream));
    k<<<grid, b->block, smem, b->stream>>>(A, d_list, count);
    BT_TRY(cudaGetLastError());
    return CGB_OK;
}

// Mixed: all systems in FP32-SpMV refinement, then the ones marked status 1
// again in FP64 (status stays 1 for them).  FP64: all systems once.
int launch(cgb_batch *b, const cgb_batch_params &P, double *ms)
{
    BatchArgs A{};
    A.nsys = b->nsys;
    A.sys = b->d_sys;
    A.order = b->d_order;
    A.rowstr = b->d_rowstr;
    A.colidx = b->d_colidx;
    A.a = b->d_a;
    A.a32 = b->d_a32;
    A.x = b->d_x;
    A.z = b->d_z;
    A.r = b->d_r;
    A.q = b->d_q;
    A.queue = b->d_queue;
    A.mode = P.mode == CGB_MODE_MIXED ? 1 : 0;
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
    int st;
    if (A.mode == 1) {
        st = launch_list<true>(b, A, b->d_order, b->nsys);
        if (st) return st;
        std::vector<int> status(b->nsys), order(b->nsys);
        BT_TRY(cudaMemcpyAsync(status.data(), b->d_status, sizeof(int) * b->nsys,
                               cudaMemcpyDeviceToHost, b->stream));
        BT_TRY(cudaMemcpyAsync(order.data(), b->d_order, sizeof(int) * b->nsys,
                               cudaMemcpyDeviceToHost, b->stream));
        BT_TRY(cudaStreamSynchronize(b->stream));
        std::vector<int> redo;
        for (int k = 0; k < b->nsys; k++)
            if (status[order[k]] != 0) redo.push_back(order[k]);
        if (!redo.empty()) {
            BT_TRY(cudaMemcpyAsync(b->d_redo, redo.data(), sizeof(int) * redo.size(),
                                   cudaMemcpyHostToDevice, b->stream));
            A.mode = 0;
            A.cgitmax = kReferenceCgitmax;
            A.recycle = 0;
            st = launch_list<false>(b, A, b->d_redo, int(redo.size()));
            if (st) return st;
            // the FP64 pass wrote status 0 for these systems; mark them re-solved
            BT_TRY(cudaStreamSynchronize(b->stream));
            std::vector<int> ones(redo.size(), 1);
            for (size_t i = 0; i < redo.size(); i++)
                BT_TRY(cudaMemcpyAsync(b->d_status + redo[i], &ones[i], sizeof(int),
                                       cudaMemcpyHostToDevice, b->stream));
        }
    } else {
        st = launch_list<false>(b, A, b->d_order, b->nsys);
        if (st) return st;
    }
    BT_TRY(cudaEventRecord(b->ev1, b->stream));
    BT_TRY(cudaStreamSynchronize(b->stream));
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
    b->mean_len.resize(nsys);
    long long ro = 0, no = 0, vo = 0;
    for (int s = 0; s < nsys; s++) {
        SysDesc &d = b->desc[s];
        d.n = n[s];
        d.row_off = ro;
        d.nnz_off = no;
        d.vec_off = vo;
        d.shift = shift[s];
        d.lanes = 32;
        b->mean_len[s] = double(rowstr[s][n[s]]) / n[s];
        ro += n[s] + 1;
        no += rowstr[s][n[s]];
        vo += n[s] + 8;
    }
    std::vector<int> order(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) {
        return rowstr[i][n[i]] > rowstr[j][n[j]];
    });
    bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess &&
              !balloc(&b->d_sys, nsys) && !balloc(&b->d_order, nsys) &&
              !balloc(&b->d_rowstr, rows_total) && !balloc(&b->d_colidx, nnz_total + 64) &&
              !balloc(&b->d_a, nnz_total + 64) && !balloc(&b->d_a32, nnz_total + 64) &&
              !balloc(&b->d_x, vec_total) && !balloc(&b->d_z, vec_total) &&
              !balloc(&b->d_r, vec_total) && !balloc(&b->d_q, vec_total) &&
              !balloc(&b->d_queue, 1) && !balloc(&b->d_zeta, nsys) && !balloc(&b->d_rnorm, nsys) &&
              !balloc(&b->d_iters, nsys) && !balloc(&b->d_status, nsys) &&
              !balloc(&b->d_redo, nsys) && !balloc(&b->d_hx, kMaxRecycle * vec_total) &&
              !balloc(&b->d_hw, kMaxRecycle * vec_total);
    if (!ok) {
        batch_release(b);
        return set_error(CGB_ERR_NOMEM, "batch device allocation failed");
    }
    for (int s = 0; s < nsys; s++) {
        const SysDesc &d = b->desc[s];
        const long long nz = rowstr[s][n[s]];
        if (cudaMemcpy(b->d_rowstr + d.row_off, rowstr[s], sizeof(int) * (n[s] + 1),
                       cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(b->d_colidx + d.nnz_off, colidx[s], sizeof(int) * nz,
                       cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(b->d_a + d.nnz_off, a[s], sizeof(double) * nz, cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            batch_release(b);
            return set_error(CGB_ERR_CUDA, "batch upload failed");
        }
    }
    to_fp32_batch<<<4 * b->sms, 256, 0, b->stream>>>(b->d_a, b->d_a32, nnz_total);
    if (cudaMemcpy(b->d_order, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess || apply_lanes(b) != CGB_OK) {
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
    if (P.niter < 1 || P.cgitmax < 1 || (P.mode != CGB_MODE_FP64 && P.mode != CGB_MODE_MIXED) ||
        (P.mode == CGB_MODE_MIXED && !(P.tol > 0.0)) || P.recycle < 0 || P.recycle > kMaxRecycle)
        return set_error(CGB_ERR_INVALID,
                         "batch: niter, cgitmax >= 1; mode FP64 or MIXED (tol > 0); recycle 0..%d",
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
// shape {512, 1024} and each lane policy (row-length thresholds for 4/8/16/32
// lanes per row), keeps the fastest and reports it.
int cgb_batch_tune(cgb_batch *b, const cgb_batch_params *params, int *block_out, double *t0_out,
                   double *t1_out, double *t2_out, double *best_ms)
{
    if (!b || !params) return set_error(CGB_ERR_INVALID, "batch: null argument");
    BT_TRY(cudaSetDevice(b->device));
    struct Cand {
        int block;
        double t0, t1, t2;
    };
    const Cand cands[] = {{512, 16, 40, 96},  {512, 8, 24, 64},   {512, 24, 64, 160},
                          {1024, 16, 40, 96}, {1024, 8, 24, 64},  {512, 1e9, 1e9, 0}};
    double best = 1e30;
    Cand bc = cands[0];
    for (const Cand &c : cands) {
        b->block = c.block;
        b->t0 = c.t0;
        b->t1 = c.t1;
        b->t2 = c.t2;
        int st = apply_lanes(b);
        if (st) return st;
        double ms = 0.0;
        st = launch(b, *params, &ms);
        if (st) return st;
        if (ms < best) {
            best = ms;
            bc = c;
        }
    }
    b->block = bc.block;
    b->t0 = bc.t0;
    b->t1 = bc.t1;
    b->t2 = bc.t2;
    int st = apply_lanes(b);
    if (st) return st;
    if (block_out) *block_out = bc.block;
    if (t0_out) *t0_out = bc.t0;
    if (t1_out) *t1_out = bc.t1;
    if (t2_out) *t2_out = bc.t2;
    if (best_ms) *best_ms = best;
    return CGB_OK;
}

}  // extern "C"

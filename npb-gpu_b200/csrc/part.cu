// part.cu -- one system's inverse power iteration with its rows split over
// several GPUs (ranks): the NPB classes D and E, whose matrices a single
// GPU's persistent kernel also runs but whose work divides across GPUs.
//
// Rank r of `world` owns the rows [r m, min((r+1) m, n)), m = ceil(n/world),
// as CSR with global column indices.  The reference algorithm (conj_grad,
// cg.cu:653-801, fixed cgitmax FP64 steps) runs with the same recurrence;
// per CG iteration the only exchanges are one all-gather of the search
// vector p (each rank gathers its rows' columns from the whole vector) and
// two all-reduces of one scalar (p.q, r.r).  Every scalar stays on the
// device: a rank's kernels write their local partial sum, the collective
// turns it into the global one, the next kernel reads it -- so a solve is
// one stream of kernels and collectives with no host round trip.
//
// Collectives: NCCL, loaded on demand (dlopen, so libcgb has no link-time
// NCCL dependency) and driven by an ncclUniqueId the caller distributes; or,
// for k ranks of one process on one device, by device copies and a summing
// kernel (cgb_part_group_power_iterate) -- the same kernels and the same
// partitioned data flow, which is how this path is tested on one GPU.
//
// Sums: a row is summed by LPR lanes of a group in a fixed order; a rank's
// partial dot products are summed in a fixed order (per-CTA partials, the
// last CTA adds them); across ranks the collective adds the ranks' values.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>  // types only: the functions are looked up at run time

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "cgb_internal.h"
#include "spmv_policies.cuh"

namespace cgb {
namespace part {

constexpr int kBlock = 256;
constexpr int kMaxGrid = 1024;

// Device scalars of a rank (doubles): local partials and the global sums.
enum Scalar {
    kRhoA = 0, kRhoB = 1,  // rho, two slots: iteration it reads slot it % 2 and writes the other
    kLocD = 2, kGlobD = 3,  // p.q
    kLocR = 4,              // r.r (local; the global goes to the next rho slot)
    kLocRes = 5, kLocXZ = 6, kLocZZ = 7,   // ||x - A z||^2, x.z, z.z (local)
    kGlobRes = 8, kGlobXZ = 9, kGlobZZ = 10,
    kScalars = 16
};

// ----------------------------------------------------------------- NCCL
struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*all_gather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    const char *(*error_string)(ncclResult_t) = nullptr;
    ncclResult_t (*comm_abort)(ncclComm_t) = nullptr;
    ncclResult_t (*async_error)(ncclComm_t, ncclResult_t *) = nullptr;
    bool ok = false;
};

NcclApi g_nccl;
std::once_flag g_nccl_once;

const NcclApi *nccl()
{
    std::call_once(g_nccl_once, [] {
        // The NCCL to use: the one CGB_NCCL_LIBRARY names; else one already
        // in the process (a framework's, e.g. torch's); else the system's.
        // A process holds one libnccl.so.2 (later users bind to the loaded
        // one by its soname), so the first to load it picks it for all.
        void *h = nullptr;
        const char *path = std::getenv("CGB_NCCL_LIBRARY");
        if (path && *path) h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        NcclApi a;
        a.get_unique_id = reinterpret_cast<decltype(a.get_unique_id)>(dlsym(h, "ncclGetUniqueId"));
        a.comm_init_rank = reinterpret_cast<decltype(a.comm_init_rank)>(dlsym(h, "ncclCommInitRank"));
        a.comm_destroy = reinterpret_cast<decltype(a.comm_destroy)>(dlsym(h, "ncclCommDestroy"));
        a.all_reduce = reinterpret_cast<decltype(a.all_reduce)>(dlsym(h, "ncclAllReduce"));
        a.all_gather = reinterpret_cast<decltype(a.all_gather)>(dlsym(h, "ncclAllGather"));
        a.error_string = reinterpret_cast<decltype(a.error_string)>(dlsym(h, "ncclGetErrorString"));
        a.comm_abort = reinterpret_cast<decltype(a.comm_abort)>(dlsym(h, "ncclCommAbort"));
        a.async_error = reinterpret_cast<decltype(a.async_error)>(dlsym(h, "ncclCommGetAsyncError"));
        a.ok = a.get_unique_id && a.comm_init_rank && a.comm_destroy && a.all_reduce &&
               a.all_gather && a.error_string && a.comm_abort && a.async_error;
        g_nccl = a;
    });
    return g_nccl.ok ? &g_nccl : nullptr;
}

// -------------------------------------------------------------- kernels
// This CTA's rows of the rank's n_own: a contiguous range.
__device__ __forceinline__ void cta_rows(int n_own, int &r0, int &r1)
{
    const int per = (n_own + gridDim.x - 1) / gridDim.x;
    r0 = min(n_own, int(blockIdx.x) * per);
    r1 = min(n_own, r0 + per);
}

// Sums of `nv` per-thread values over the grid into out[0..nv): per-CTA sums
// (fixed shuffle order) in part[v * gridDim.x + cta], then the last CTA to
// finish (a ticket) adds them in CTA order.
__device__ __forceinline__ void grid_sums(const double *v, int nv, double *part, unsigned *ticket,
                                          double *out)
{
    __shared__ double red[32];
    __shared__ bool last;
    for (int k = 0; k < nv; k++) {
        const double s = block_sum(v[k], red);
        if (threadIdx.x == 0) part[k * gridDim.x + blockIdx.x] = s;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < 32) {
        for (int k = 0; k < nv; k++) {
            double t = 0.0;
            for (int i = threadIdx.x; i < int(gridDim.x); i += 32) t += __ldcg(part + k * gridDim.x + i);
            t = warp_sum(t);
            if (threadIdx.x == 0) out[k] = t;
        }
        if (threadIdx.x == 0) *ticket = 0u;
    }
}

struct PartArgs {
    int n_own;
    const double *x;
    double *z, *r, *q;
    double *pown;        // this rank's rows of the gathered vector (pfull + rank m)
    double *sc;          // kScalars device scalars
    double *part;        // 3 * kMaxGrid per-CTA partials
    unsigned *ticket;    // [0]: the reductions' ticket, [1]: outer steps done
    double *trace;       // (zeta, rnorm) per outer step
    int trace_cap;       // outer steps the trace holds
};

// z = 0, r = x, p = x for the own rows; local x.x into the rho slot `slot`
// (the collective makes it global in place).
__global__ void __launch_bounds__(kBlock) k_start(PartArgs P, int slot)
{
    int r0, r1;
    cta_rows(P.n_own, r0, r1);
    double acc = 0.0;
    for (int j = r0 + threadIdx.x; j < r1; j += blockDim.x) {
        const double xv = P.x[j];
        P.z[j] = 0.0;
        P.r[j] = xv;
        P.pown[j] = xv;
        acc = fma(xv, xv, acc);
    }
    grid_sums(&acc, 1, P.part, P.ticket, P.sc + slot);
}

// q = A p for the own rows (p gathered whole); local p.q (kLocD) unless
// `dot` is 0.
// L2 hints: the matrix stream is read once a product (evict_first, not
// kept in L1); the gathered vector -- up to 72 MB at class E, within the
// 126 MB L2 -- is read ~nnz/n times a product (evict_last).
__device__ __forceinline__ uint64_t policy_first()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, %1;" : "=l"(pol) : "f"(1.f));
    return pol;
}

__device__ __forceinline__ uint64_t policy_last()
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, %1;" : "=l"(pol) : "f"(1.f));
    return pol;
}

__device__ __forceinline__ int2 ld_cols2(const int *p, uint64_t pol)
{
    int2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
        : "=r"(v.x), "=r"(v.y)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ int ld_col1(const int *p, uint64_t pol)
{
    int v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ double ld_val1(const double *p, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ double ld_gather(const double *p, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

// q = A p over this CTA's rows [r0, r1): LPR lanes a row, two entries a lane
// a load (pair loads from even entries; the last entry of the block alone),
// four loads in flight, lanes summed by a fixed xor tree.  Returns this
// thread's share of dotv . q.
template <int LPR>
__device__ __forceinline__ double part_rows(const MatrixView &M, const double *__restrict__ v,
                                            double *out, int r0, int r1, const double *dotv)
{
    constexpr int kStep = 2 * LPR, kUnroll = 4;
    const uint64_t first = policy_first(), last = policy_last();
    const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR, ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    const long long end = M.csr_entries;
    double dacc = 0.0;
    for (int row = r0 + grp; row < r1; row += ngrp) {
        const int k0 = __ldg(M.rowstr + row), k1 = __ldg(M.rowstr + row + 1);
        double s = 0.0;
        for (int k = (k0 & ~1) + 2 * lane; k < k1; k += kUnroll * kStep) {
            double2 av[kUnroll];
            int2 cv[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    if (kk + 1 < end) {
                        av[u] = ld_stream(reinterpret_cast<const double2 *>(M.a + kk), first);
                        cv[u] = ld_cols2(M.colidx + kk, first);
                    } else {
                        av[u] = make_double2(ld_val1(M.a + kk, first), 0.0);
                        cv[u] = make_int2(ld_col1(M.colidx + kk, first), 0);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    if (kk >= k0) s = fma(av[u].x, ld_gather(v + cv[u].x, last), s);
                    if (kk + 1 < k1) s = fma(av[u].y, ld_gather(v + cv[u].y, last), s);
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
__global__ void __launch_bounds__(kBlock) k_spmv(PartArgs P, MatrixView M, const double *pfull,
                                                 double *out, int dot)
{
    int r0, r1;
    cta_rows(P.n_own, r0, r1);
    double acc = part_rows<LPR>(M, pfull, out, r0, r1, dot ? P.pown : nullptr);
    if (dot) grid_sums(&acc, 1, P.part, P.ticket, P.sc + kLocD);
}

// alpha = rho / (p.q); z += alpha p; r -= alpha q; local r.r (kLocR).
__global__ void __launch_bounds__(kBlock) k_update(PartArgs P, int slot)
{
    const double alpha = P.sc[slot] / P.sc[kGlobD];
    int r0, r1;
    cta_rows(P.n_own, r0, r1);
    double acc = 0.0;
    for (int j = r0 + threadIdx.x; j < r1; j += blockDim.x) {
        P.z[j] = fma(alpha, P.pown[j], P.z[j]);
        const double rv = fma(-alpha, P.q[j], P.r[j]);
        P.r[j] = rv;
        acc = fma(rv, rv, acc);
    }
    grid_sums(&acc, 1, P.part, P.ticket, P.sc + kLocR);
}

// beta = rho' / rho; p = r + beta p for the own rows.
__global__ void __launch_bounds__(kBlock) k_pupdate(PartArgs P, int slot, int slot_new)
{
    const double beta = P.sc[slot_new] / P.sc[slot];
    int r0, r1;
    cta_rows(P.n_own, r0, r1);
    for (int j = r0 + threadIdx.x; j < r1; j += blockDim.x) P.pown[j] = fma(beta, P.pown[j], P.r[j]);
}

// local ||x - A z||^2, x.z, z.z (q = A z) into kLocRes..kLocZZ.
__global__ void __launch_bounds__(kBlock) k_final(PartArgs P)
{
    int r0, r1;
    cta_rows(P.n_own, r0, r1);
    double v[3] = {0.0, 0.0, 0.0};
    for (int j = r0 + threadIdx.x; j < r1; j += blockDim.x) {
        const double xv = P.x[j], zv = P.z[j], d = xv - P.q[j];
        v[0] = fma(d, d, v[0]);
        v[1] = fma(xv, zv, v[1]);
        v[2] = fma(zv, zv, v[2]);
    }
    grid_sums(v, 3, P.part, P.ticket, P.sc + kLocRes);
}

// zeta and rnorm of this outer step into the trace (at the count of steps
// done, which it advances), then x = z / ||z||.  The step's kernels are one
// graph, replayed per outer step: the count is the only thing that differs.
__global__ void __launch_bounds__(kBlock) k_finish(PartArgs P, double shift)
{
    const double zeta = shift + 1.0 / P.sc[kGlobXZ];
    const double norm = 1.0 / sqrt(P.sc[kGlobZZ]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned step = P.ticket[1];
        if (step < unsigned(P.trace_cap)) {
            P.trace[2 * step] = zeta;
            P.trace[2 * step + 1] = sqrt(P.sc[kGlobRes]);
        }
        P.ticket[1] = step + 1;
    }
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < P.n_own; j += gridDim.x * blockDim.x)
        const_cast<double *>(P.x)[j] = norm * P.z[j];
}

// Group mode: out[s][dst] = sum over the k ranks of their scalar `src`
// (ranks added in rank order), for `count` consecutive scalars.
__global__ void k_group_sum(double *const *scalars, int k, int src, int dst, int count)
{
    const int c = threadIdx.x;
    if (c >= count) return;
    double t = 0.0;
    for (int s = 0; s < k; s++) t += scalars[s][src + c];
    for (int s = 0; s < k; s++) scalars[s][dst + c] = t;
}

__global__ void k_fill_ones(double *x, int count)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        x[j] = 1.0;
}

}  // namespace part
}  // namespace cgb

using namespace cgb;
using namespace cgb::part;

struct cgb_part {
    int device = 0, n = 0, world = 1, rank = 0, m = 0, row0 = 0, n_own = 0, lpr = 8, grid = 1;
    long long nnz = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int *d_rowstr = nullptr, *d_colidx = nullptr;
    double *d_a = nullptr;
    double *d_x = nullptr, *d_z = nullptr, *d_r = nullptr, *d_q = nullptr;
    double *d_pfull = nullptr;  // world * m entries
    double *d_sc = nullptr, *d_part = nullptr, *d_trace = nullptr;
    unsigned *d_ticket = nullptr;
    int trace_cap = 0;
    ncclComm_t comm = nullptr;
    bool warmed = false;   // the communicator's first collectives made
    bool aborted = false;  // the communicator was aborted (a peer failed or a wait ran out)
    double wait_limit_s = 600.0;
};

namespace {

#define PART_TRY(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(CGB_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                         \
    } while (0)

template <typename T>
cudaError_t palloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

template <typename T>
void pfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

void part_release(cgb_part *p)
{
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->comm && nccl()) nccl()->comm_destroy(p->comm);
    pfree(p->d_rowstr); pfree(p->d_colidx); pfree(p->d_a); pfree(p->d_x); pfree(p->d_z);
    pfree(p->d_r); pfree(p->d_q); pfree(p->d_pfull); pfree(p->d_sc); pfree(p->d_part);
    pfree(p->d_trace); pfree(p->d_ticket);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

int rows_of(int n, int world, int rank, int *m, int *row0, int *n_own)
{
    if (n < 1 || world < 1 || rank < 0 || rank >= world)
        return set_error(CGB_ERR_INVALID, "part: n >= 1 and 0 <= rank < world required");
    const int mm = int((static_cast<long long>(n) + world - 1) / world);
    const int r0 = int(std::min<long long>(n, static_cast<long long>(rank) * mm));
    *m = mm;
    *row0 = r0;
    *n_own = std::min(n, r0 + mm) - r0;
    return CGB_OK;
}

PartArgs args_of(cgb_part *p)
{
    PartArgs P;
    P.n_own = p->n_own;
    P.x = p->d_x;
    P.z = p->d_z;
    P.r = p->d_r;
    P.q = p->d_q;
    P.pown = p->d_pfull + static_cast<size_t>(p->rank) * p->m;
    P.sc = p->d_sc;
    P.part = p->d_part;
    P.ticket = p->d_ticket;
    P.trace = p->d_trace;
    P.trace_cap = p->trace_cap;
    return P;
}

MatrixView view_of(cgb_part *p)
{
    MatrixView M{};
    M.rowstr = p->d_rowstr;
    M.colidx = p->d_colidx;
    M.a = p->d_a;
    M.csr_entries = p->nnz;  // unpadded: the last entry is loaded alone
    M.ncols = p->n;
    return M;
}

cudaError_t launch_spmv(cgb_part *p, const double *v, double *out, int dot, cudaStream_t s)
{
    const PartArgs P = args_of(p);
    const MatrixView M = view_of(p);
    switch (p->lpr) {
    case 2: k_spmv<2><<<p->grid, kBlock, 0, s>>>(P, M, v, out, dot); break;
    case 4: k_spmv<4><<<p->grid, kBlock, 0, s>>>(P, M, v, out, dot); break;
    case 8: k_spmv<8><<<p->grid, kBlock, 0, s>>>(P, M, v, out, dot); break;
    case 16: k_spmv<16><<<p->grid, kBlock, 0, s>>>(P, M, v, out, dot); break;
    default: k_spmv<32><<<p->grid, kBlock, 0, s>>>(P, M, v, out, dot); break;
    }
    return cudaGetLastError();
}

// The collectives a solve needs, for one rank (NCCL) or for k ranks of
// one process on one device (device copies and k_group_sum).
struct Collectives {
    cgb_part *const *parts;
    int k;                 // ranks driven by this call (1 with NCCL)
    cudaStream_t stream;   // the stream every rank's work goes on (group mode)
    double *const *d_scalars = nullptr;  // group mode: the k ranks' scalar arrays (device)

    int allreduce(int src, int dst, int count)
    {
        if (parts[0]->comm) {
            cgb_part *p = parts[0];
            const ncclResult_t r = nccl()->all_reduce(p->d_sc + src, p->d_sc + dst, count, ncclFloat64,
                                                      ncclSum, p->comm, p->stream);
            if (r != ncclSuccess)
                return set_error(CGB_ERR_CUDA, "ncclAllReduce: %s", nccl()->error_string(r));
            return CGB_OK;
        }
        k_group_sum<<<1, 32, 0, stream>>>(d_scalars, k, src, dst, count);
        PART_TRY(cudaGetLastError());
        return CGB_OK;
    }

    // every rank's own block of `buf_of(rank)` into every rank's pfull
    int allgather(bool from_z)
    {
        if (parts[0]->comm) {
            cgb_part *p = parts[0];
            const double *send = from_z ? p->d_z : p->d_pfull + static_cast<size_t>(p->rank) * p->m;
            const ncclResult_t r = nccl()->all_gather(send, p->d_pfull, p->m, ncclFloat64, p->comm,
                                                      p->stream);
            if (r != ncclSuccess)
                return set_error(CGB_ERR_CUDA, "ncclAllGather: %s", nccl()->error_string(r));
            return CGB_OK;
        }
        for (int s = 0; s < k; s++) {
            const cgb_part *src = parts[s];
            const double *own = from_z ? src->d_z : src->d_pfull + static_cast<size_t>(src->rank) * src->m;
            for (int d = 0; d < k; d++) {
                if (d == s && !from_z) continue;
                PART_TRY(cudaMemcpyAsync(parts[d]->d_pfull + static_cast<size_t>(src->rank) * src->m, own,
                                         sizeof(double) * src->m, cudaMemcpyDeviceToDevice, stream));
            }
        }
        return CGB_OK;
    }
};

// One outer step of the power iteration over the ranks `parts` (k of them,
// one each with NCCL): the reference's outer-loop body (cg.cu:485-520)
// with the reference algorithm's conj_grad split by rows.  Enqueued on
// `stream` (captured into the solve's graph).
int enqueue_step(cgb_part *const *parts, int k, Collectives &C, double shift, int cgitmax,
                 cudaStream_t stream)
{
    auto each = [&](auto &&fn) -> int {
        for (int i = 0; i < k; i++) {
            fn(parts[i], args_of(parts[i]));
            PART_TRY(cudaGetLastError());
        }
        return CGB_OK;
    };
    int st = each([&](cgb_part *p, const PartArgs &P) {
        k_start<<<p->grid, kBlock, 0, stream>>>(P, kRhoA);
    });
    if (st) return st;
    if ((st = C.allreduce(kRhoA, kRhoA, 1)) || (st = C.allgather(false))) return st;
    for (int it = 0; it < cgitmax; it++) {
        const int slot = (it & 1) ? kRhoB : kRhoA, slot_new = (it & 1) ? kRhoA : kRhoB;
        for (int i = 0; i < k; i++) {
            cgb_part *p = parts[i];
            PART_TRY(launch_spmv(p, p->d_pfull, p->d_q, 1, stream));
        }
        if ((st = C.allreduce(kLocD, kGlobD, 1))) return st;
        st = each([&](cgb_part *p, const PartArgs &P) {
            k_update<<<p->grid, kBlock, 0, stream>>>(P, slot);
        });
        if (st) return st;
        if ((st = C.allreduce(kLocR, slot_new, 1))) return st;
        st = each([&](cgb_part *p, const PartArgs &P) {
            k_pupdate<<<p->grid, kBlock, 0, stream>>>(P, slot, slot_new);
        });
        if (st) return st;
        if ((st = C.allgather(false))) return st;
    }
    // ||x - A z||, x.z, z.z (cg.cu:777-800, :508-511) on the gathered z
    if ((st = C.allgather(true))) return st;
    for (int i = 0; i < k; i++) {
        cgb_part *p = parts[i];
        PART_TRY(launch_spmv(p, p->d_pfull, p->d_q, 0, stream));
    }
    st = each([&](cgb_part *p, const PartArgs &P) { k_final<<<p->grid, kBlock, 0, stream>>>(P); });
    if (st) return st;
    if ((st = C.allreduce(kLocRes, kGlobRes, 3))) return st;
    return each([&](cgb_part *p, const PartArgs &P) {
        k_finish<<<p->grid, kBlock, 0, stream>>>(P, shift);
    });
}

// Waits for `stream`.  With a communicator the wait is a poll that also
// watches NCCL's asynchronous error state and the part's time limit: a
// failed or silent peer makes this rank abort its communicator (its NCCL
// kernels then return) instead of waiting for ever.  The part cannot make
// collectives afterwards.
int wait_stream(cgb_part *p, cudaStream_t stream)
{
    if (!p || !p->comm) {
        PART_TRY(cudaStreamSynchronize(stream));
        return CGB_OK;
    }
    const NcclApi *api = nccl();
    const auto t0 = std::chrono::steady_clock::now();
    auto seconds = [&] {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    for (;;) {
        const cudaError_t e = cudaStreamQuery(stream);
        if (e == cudaSuccess) return CGB_OK;
        if (e != cudaErrorNotReady)
            return set_error(CGB_ERR_CUDA, "part: the solve failed: %s", cudaGetErrorString(e));
        ncclResult_t ar = ncclSuccess;
        api->async_error(p->comm, &ar);
        const bool expired = seconds() > p->wait_limit_s;
        if ((ar != ncclSuccess && ar != ncclInProgress) || expired) {
            api->comm_abort(p->comm);
            p->comm = nullptr;
            p->aborted = true;
            // the aborted communicator's kernels return; give them a bounded while
            const auto t1 = std::chrono::steady_clock::now();
            while (cudaStreamQuery(stream) == cudaErrorNotReady &&
                   std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count() < 10.0)
                std::this_thread::sleep_for(std::chrono::microseconds(200));
            return expired ? set_error(CGB_ERR_TIMEOUT, "part: rank %d waited %.0f s for its peers; "
                                       "communicator aborted", p->rank, p->wait_limit_s)
                           : set_error(CGB_ERR_CUDA, "part: NCCL reported %s; communicator aborted",
                                       api->error_string(ar));
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// x = 1 and the step count 0 on every rank, then the outer step captured
// once as a graph and launched niter times between ev0 and ev1.
int run_solve(cgb_part *const *parts, int k, Collectives &C, int niter, double shift, int cgitmax,
              cudaStream_t stream, cudaEvent_t ev0, cudaEvent_t ev1)
{
    cgb_part *const watch = parts[0]->comm ? parts[0] : nullptr;
    for (int i = 0; i < k; i++) {
        cgb_part *p = parts[i];
        k_fill_ones<<<p->grid, kBlock, 0, stream>>>(p->d_x, p->m);
        PART_TRY(cudaGetLastError());
        PART_TRY(cudaMemsetAsync(p->d_ticket + 1, 0, sizeof(unsigned), stream));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    PART_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_step(parts, k, C, shift, cgitmax, stream);
    const cudaError_t ec = cudaStreamEndCapture(stream, &graph);
    if (!st && ec != cudaSuccess)
        st = set_error(CGB_ERR_CUDA, "part: capture failed: %s", cudaGetErrorString(ec));
    if (!st && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        st = set_error(CGB_ERR_CUDA, "part: graph instantiation failed");
    cudaError_t e = cudaSuccess;
    if (!st) {
        e = cudaEventRecord(ev0, stream);
        for (int step = 0; step < niter && e == cudaSuccess; step++) e = cudaGraphLaunch(exec, stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev1, stream);
        if (e != cudaSuccess) st = set_error(CGB_ERR_CUDA, "part: the solve failed: %s", cudaGetErrorString(e));
        else st = wait_stream(watch, stream);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    return st;
}

int ensure_trace(cgb_part *p, int niter)
{
    if (niter <= p->trace_cap) return CGB_OK;
    pfree(p->d_trace);
    if (palloc(&p->d_trace, 2 * size_t(niter))) return set_error(CGB_ERR_NOMEM, "part: trace allocation failed");
    p->trace_cap = niter;
    return CGB_OK;
}

// A part without its matrix: device checks, stream, events and vectors.
int part_shell(int device, int n, int world, int rank, cgb_part **out)
{
    int m = 0, r0 = 0, own = 0;
    int st = rows_of(n, world, rank, &m, &r0, &own);
    if (st) return st;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "part: no CUDA device %d", device);
    int major = 0, sms = 0;
    PART_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    PART_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (major != 10) return set_error(CGB_ERR_NO_DEVICE, "part: device %d is not sm_100", device);
    PART_TRY(cudaSetDevice(device));
    cgb_part *p = new (std::nothrow) cgb_part;
    if (!p) return set_error(CGB_ERR_NOMEM, "part allocation failed");
    p->device = device;
    p->n = n;
    p->world = world;
    p->rank = rank;
    p->m = m;
    p->row0 = r0;
    p->n_own = own;
    p->grid = std::max(1, std::min({4 * sms, kMaxGrid, (own + 63) / 64}));
    const size_t vm = static_cast<size_t>(m);
    const bool ok = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaEventCreate(&p->ev0) == cudaSuccess && cudaEventCreate(&p->ev1) == cudaSuccess &&
                    !palloc(&p->d_x, vm) && !palloc(&p->d_z, vm) && !palloc(&p->d_r, vm) &&
                    !palloc(&p->d_q, vm) && !palloc(&p->d_pfull, vm * size_t(world)) &&
                    !palloc(&p->d_sc, kScalars) && !palloc(&p->d_part, 3 * size_t(kMaxGrid)) &&
                    !palloc(&p->d_ticket, 2);
    const cudaStream_t s = p->stream;
    const bool zeroed = ok && cudaMemsetAsync(p->d_pfull, 0, sizeof(double) * vm * world, s) == cudaSuccess &&
                        cudaMemsetAsync(p->d_z, 0, sizeof(double) * vm, s) == cudaSuccess &&
                        cudaMemsetAsync(p->d_sc, 0, sizeof(double) * kScalars, s) == cudaSuccess &&
                        cudaMemsetAsync(p->d_ticket, 0, 2 * sizeof(unsigned), s) == cudaSuccess &&
                        cudaStreamSynchronize(s) == cudaSuccess;
    if (!zeroed) {
        part_release(p);
        return set_error(ok ? CGB_ERR_CUDA : CGB_ERR_NOMEM, "part: device set-up failed");
    }
    *out = p;
    return CGB_OK;
}

// Lanes per row from the mean row length, then the communicator (a
// collective call when nccl_id is given).  Releases the part on failure.
int part_finish(cgb_part *p, const void *nccl_id)
{
    const double mean = double(p->nnz) / p->n_own;
    p->lpr = mean >= 96 ? 32 : mean >= 40 ? 16 : mean >= 16 ? 8 : mean >= 6 ? 4 : 2;
    if (!nccl_id) return CGB_OK;
    const int st = cgb_part_join(p, nccl_id);
    if (st) part_release(p);
    return st;
}

int read_traces(cgb_part *p, int niter, double *zeta, double *rnorm)
{
    std::vector<double> t(2 * size_t(niter));
    PART_TRY(cudaMemcpy(t.data(), p->d_trace, sizeof(double) * t.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < niter; i++) {
        if (zeta) zeta[i] = t[2 * i];
        if (rnorm) rnorm[i] = t[2 * i + 1];
        if (!std::isfinite(t[2 * i]) || !std::isfinite(t[2 * i + 1]))
            return set_error(CGB_ERR_NUMERIC, "part: non-finite zeta or residual at step %d", i);
    }
    return CGB_OK;
}

}  // namespace

extern "C" {

int cgb_part_rows(int n, int world, int rank, int *row0, int *row1)
{
    int m = 0, r0 = 0, own = 0;
    const int st = rows_of(n, world, rank, &m, &r0, &own);
    if (st) return st;
    if (row0) *row0 = r0;
    if (row1) *row1 = r0 + own;
    return CGB_OK;
}

int cgb_nccl_unique_id(void *id_out)
{
    if (!id_out) return set_error(CGB_ERR_INVALID, "part: null id buffer");
    const NcclApi *api = nccl();
    if (!api) return set_error(CGB_ERR_STATE, "part: libnccl.so.2 not found");
    ncclUniqueId id;
    const ncclResult_t r = api->get_unique_id(&id);
    if (r != ncclSuccess) return set_error(CGB_ERR_CUDA, "ncclGetUniqueId: %s", api->error_string(r));
    std::memcpy(id_out, &id, sizeof(id));
    return CGB_OK;
}

int cgb_part_create(int device, int n, int world, int rank, const int *rowstr, const int *colidx,
                    const double *a, const void *nccl_id, cgb_part **out)
{
    if (!out || !rowstr || !colidx || !a) return set_error(CGB_ERR_INVALID, "part: null argument");
    *out = nullptr;
    int m = 0, r0 = 0, own = 0;
    int st = rows_of(n, world, rank, &m, &r0, &own);
    if (st) return st;
    if (own < 1) return set_error(CGB_ERR_INVALID, "part: rank %d of %d owns no rows of n = %d", rank, world, n);
    if (rowstr[0] != 0) return set_error(CGB_ERR_BAD_MATRIX, "part: rowstr[0] != 0");
    for (int i = 0; i < own; i++)
        if (rowstr[i + 1] < rowstr[i]) return set_error(CGB_ERR_BAD_MATRIX, "part: rowstr decreases at %d", i);
    const long long nnz = rowstr[own];
    for (long long k = 0; k < nnz; k++)
        if (colidx[k] < 0 || colidx[k] >= n || !std::isfinite(a[k]))
            return set_error(CGB_ERR_BAD_MATRIX, "part: entry %lld invalid", k);
    cgb_part *p = nullptr;
    if ((st = part_shell(device, n, world, rank, &p))) return st;
    p->nnz = nnz;
    const cudaStream_t s = p->stream;
    bool copied = !palloc(&p->d_rowstr, size_t(own) + 1) && !palloc(&p->d_colidx, size_t(nnz)) &&
                  !palloc(&p->d_a, size_t(nnz));
    if (!copied) {
        part_release(p);
        return set_error(CGB_ERR_NOMEM, "part: device allocation of the CSR failed");
    }
    copied =
        cudaMemcpyAsync(p->d_rowstr, rowstr, sizeof(int) * (own + 1), cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(p->d_colidx, colidx, sizeof(int) * nnz, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaMemcpyAsync(p->d_a, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess;
    if (!copied) {
        part_release(p);
        return set_error(CGB_ERR_CUDA, "part: upload failed");
    }
    if ((st = part_finish(p, nccl_id))) return st;
    *out = p;
    return CGB_OK;
}

int cgb_part_create_generated(int device, int n, int nonzer, double rcond, double shift, double seed,
                              int world, int rank, const void *nccl_id, cgb_part **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "part: null argument");
    *out = nullptr;
    int m = 0, r0 = 0, own = 0;
    int st = rows_of(n, world, rank, &m, &r0, &own);
    if (st) return st;
    if (own < 1) return set_error(CGB_ERR_INVALID, "part: rank %d of %d owns no rows of n = %d", rank, world, n);
    cgb_part *p = nullptr;
    if ((st = part_shell(device, n, world, rank, &p))) return st;
    DeviceCsr csr;
    if ((st = makea_on_device(device, n, nonzer, rcond, shift, seed, &csr, r0, r0 + own))) {
        for (void *q : {(void *)csr.rowstr, (void *)csr.colidx, (void *)csr.a})
            if (q) cudaFree(q);
        part_release(p);
        return st;
    }
    p->d_rowstr = csr.rowstr;
    p->d_colidx = csr.colidx;
    p->d_a = csr.a;
    p->nnz = csr.nnz;
    if ((st = part_finish(p, nccl_id))) return st;
    *out = p;
    return CGB_OK;
}

int cgb_part_join(cgb_part *p, const void *nccl_id)
{
    if (!p || !nccl_id) return set_error(CGB_ERR_INVALID, "part: null part or id");
    if (p->comm || p->aborted) return set_error(CGB_ERR_STATE, "part: already joined a communicator");
    PART_TRY(cudaSetDevice(p->device));
    const NcclApi *api = nccl();
    if (!api) return set_error(CGB_ERR_STATE, "part: libnccl.so.2 not found");
    ncclUniqueId id;
    std::memcpy(&id, nccl_id, sizeof(id));
    const ncclResult_t r = api->comm_init_rank(&p->comm, p->world, id, p->rank);
    if (r != ncclSuccess) {
        p->comm = nullptr;
        return set_error(CGB_ERR_CUDA, "ncclCommInitRank: %s", api->error_string(r));
    }
    return CGB_OK;
}

int cgb_part_set_wait_limit(cgb_part *p, double seconds)
{
    if (!p || !(seconds > 0.0)) return set_error(CGB_ERR_INVALID, "part: a positive limit required");
    p->wait_limit_s = seconds;
    return CGB_OK;
}

int cgb_part_info(const cgb_part *p, int *row0, int *row1, long long *nnz)
{
    if (!p) return set_error(CGB_ERR_INVALID, "part: null part");
    if (row0) *row0 = p->row0;
    if (row1) *row1 = p->row0 + p->n_own;
    if (nnz) *nnz = p->nnz;
    return CGB_OK;
}

int cgb_part_destroy(cgb_part *p)
{
    part_release(p);
    return CGB_OK;
}

int cgb_part_power_iterate(cgb_part *p, int niter, double shift, int cgitmax, double *zeta_trace,
                           double *rnorm_trace, double *device_ms)
{
    if (!p || niter < 1 || cgitmax < 1 || !std::isfinite(shift))
        return set_error(CGB_ERR_INVALID, "part: niter, cgitmax >= 1 and a finite shift required");
    if (p->aborted) return set_error(CGB_ERR_STATE, "part: its communicator was aborted");
    if (!p->comm && p->world > 1)
        return set_error(CGB_ERR_STATE, "part: a rank of world %d needs a communicator (an NCCL id "
                         "at create, or cgb_part_join)", p->world);
    PART_TRY(cudaSetDevice(p->device));
    int st = ensure_trace(p, niter);
    if (st) return st;
    cgb_part *const parts[1] = {p};
    if (!p->comm) {
        // world 1 without NCCL: the group path with one rank
        return cgb_part_group_power_iterate(const_cast<cgb_part **>(parts), 1, niter, shift, cgitmax,
                                            zeta_trace, rnorm_trace, device_ms);
    }
    Collectives C{parts, 1, p->stream};
    if (!p->warmed) {
        // NCCL sets up its connections on a communicator's first collectives:
        // make them outside the capture (their results are overwritten)
        if ((st = C.allreduce(kLocD, kGlobD, 1)) || (st = C.allgather(false)) ||
            (st = wait_stream(p, p->stream)))
            return st;
        p->warmed = true;
    }
    st = run_solve(parts, 1, C, niter, shift, cgitmax, p->stream, p->ev0, p->ev1);
    if (st) return st;
    float ms = 0.f;
    PART_TRY(cudaEventElapsedTime(&ms, p->ev0, p->ev1));
    if (device_ms) *device_ms = ms;
    return read_traces(p, niter, zeta_trace, rnorm_trace);
}

int cgb_part_group_power_iterate(cgb_part **parts, int k, int niter, double shift, int cgitmax,
                                 double *zeta_trace, double *rnorm_trace, double *device_ms)
{
    if (!parts || k < 1 || niter < 1 || cgitmax < 1 || !std::isfinite(shift))
        return set_error(CGB_ERR_INVALID, "part group: k, niter, cgitmax >= 1 and a finite shift");
    const int world = parts[0]->world, n = parts[0]->n, device = parts[0]->device;
    if (k != world) return set_error(CGB_ERR_INVALID, "part group: %d ranks given for world %d", k, world);
    for (int i = 0; i < k; i++) {
        if (!parts[i] || parts[i]->rank != i || parts[i]->world != world || parts[i]->n != n ||
            parts[i]->device != device)
            return set_error(CGB_ERR_INVALID, "part group: rank %d is not rank %d of this world on this device", i, i);
        if (parts[i]->comm && k > 1)
            return set_error(CGB_ERR_STATE, "part group: rank %d has an NCCL communicator", i);
    }
    PART_TRY(cudaSetDevice(device));
    for (int i = 0; i < k; i++) {
        const int st = ensure_trace(parts[i], niter);
        if (st) return st;
    }
    // every rank's work on rank 0's stream, in rank order
    const cudaStream_t s = parts[0]->stream;
    double **d_scalars = nullptr;
    std::vector<double *> h_scalars(k);
    for (int i = 0; i < k; i++) h_scalars[i] = parts[i]->d_sc;
    if (palloc(&d_scalars, size_t(k))) return set_error(CGB_ERR_NOMEM, "part group: allocation failed");
    cudaError_t e = cudaMemcpyAsync(d_scalars, h_scalars.data(), sizeof(double *) * k,
                                    cudaMemcpyHostToDevice, s);
    int st = e == cudaSuccess ? CGB_OK : set_error(CGB_ERR_CUDA, "part group: %s", cudaGetErrorString(e));
    if (!st) {
        Collectives C{parts, k, s, d_scalars};
        st = run_solve(parts, k, C, niter, shift, cgitmax, s, parts[0]->ev0, parts[0]->ev1);
    }
    cudaStreamSynchronize(s);
    pfree(d_scalars);
    if (st) return st;
    float ms = 0.f;
    PART_TRY(cudaEventElapsedTime(&ms, parts[0]->ev0, parts[0]->ev1));
    if (device_ms) *device_ms = ms;
    return read_traces(parts[0], niter, zeta_trace, rnorm_trace);
}

}  // extern "C"

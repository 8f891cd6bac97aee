// session.cu -- the C ABI of libcgb: device set-up, the conj_grad-compatible
// call, the CUDA-graph power iteration and diagnostics.
//
// Reference call surface being replaced (GMAP/NPB-GPU CUDA/CG/cg.cu):
//   setup_gpu   :1390-1603  device pick, allocation, H2D upload
//   conj_grad   :653-801    (CPU) / conj_grad_gpu :803-846 (GPU)
//   outer loop  :491-522    timed inverse power iteration
//   release_gpu :1370-1388
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "cg_kernels.cuh"
#include "cgb_internal.h"

namespace cgb {

static thread_local char g_last_error[512] = "";

int set_error(int status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

#define CUDA_TRY(call)                                                                  \
    do {                                                                                \
        cudaError_t err_ = (call);                                                      \
        if (err_ != cudaSuccess)                                                        \
            return set_error(CGB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,              \
                             cudaGetErrorString(err_), __FILE__, __LINE__);             \
    } while (0)

namespace {

constexpr int kPad = 64;              // entries of padding after a / colidx
constexpr long long kDefaultWaitNs = 2000000000LL;

template <typename T>
cudaError_t dev_alloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

using OuterKernel = void (*)(OuterArgs);
using SpmvKernel = void (*)(SpmvArgs);

constexpr int kKindRow = 1;
constexpr int kKindTiled = 2;
constexpr int kTileWidth = 12288;          // doubles per staged column block (96 KB)
constexpr size_t kSmemLimit = 227 * 1024;  // opt-in shared memory per CTA on sm_100

// A launch configuration of the persistent kernels.
struct Plan {
    int kind = 0;        // kKindRow / kKindTiled
    int lpr = 32;        // lanes per row
    int rows = 1;        // rows in flight per lane group (tiled)
    OuterKernel outer = nullptr;
    SpmvKernel spmv = nullptr;
    int block = 512;
    int grid = 0;
    size_t smem = 0;
    int max_rows = 0;    // tiled: row accumulator capacity
};

bool kernels_for(int kind, int lpr, int rows, OuterKernel *outer, SpmvKernel *spmv)
{
    if (kind == kKindRow) {
        switch (lpr) {
        case 2: *outer = outer_step_fp64<2>; *spmv = spmv_dot_fp64<2>; return true;
        case 4: *outer = outer_step_fp64<4>; *spmv = spmv_dot_fp64<4>; return true;
        case 8: *outer = outer_step_fp64<8>; *spmv = spmv_dot_fp64<8>; return true;
        case 16: *outer = outer_step_fp64<16>; *spmv = spmv_dot_fp64<16>; return true;
        case 32: *outer = outer_step_fp64<32>; *spmv = spmv_dot_fp64<32>; return true;
        default: return false;
        }
    }
    if (kind == kKindTiled) {
        if (lpr == 4 && rows == 2) { *outer = outer_step_fp64_tiled<4, 2>; *spmv = spmv_dot_fp64_tiled<4, 2>; return true; }
        if (lpr == 8 && rows == 1) { *outer = outer_step_fp64_tiled<8, 1>; *spmv = spmv_dot_fp64_tiled<8, 1>; return true; }
        if (lpr == 8 && rows == 2) { *outer = outer_step_fp64_tiled<8, 2>; *spmv = spmv_dot_fp64_tiled<8, 2>; return true; }
        if (lpr == 16 && rows == 1) { *outer = outer_step_fp64_tiled<16, 1>; *spmv = spmv_dot_fp64_tiled<16, 1>; return true; }
        return false;
    }
    return false;
}

// Lanes per row from the mean row length: enough lanes that each covers a
// few 2-entry chunks, at most a warp.
int lanes_for_mean(double mean_len)
{
    if (mean_len >= 96.0) return 32;
    if (mean_len >= 40.0) return 16;
    if (mean_len >= 16.0) return 8;
    if (mean_len >= 6.0) return 4;
    return 2;
}

int check_device(int device, cudaDeviceProp *prop)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return set_error(CGB_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "device %d out of range (count %d)", device, count);
    CUDA_TRY(cudaGetDeviceProperties(prop, device));
    if (prop->major != 10)
        return set_error(CGB_ERR_NO_DEVICE,
                         "device %d is sm_%d%d; this library is built for sm_100a only", device,
                         prop->major, prop->minor);
    if (!prop->cooperativeLaunch)
        return set_error(CGB_ERR_NO_DEVICE, "device %d lacks cooperative launch", device);
    return CGB_OK;
}

int validate_csr(int n, const int *rowstr, const int *colidx, const double *a)
{
    if (n < 1 || !rowstr || !colidx || !a)
        return set_error(CGB_ERR_INVALID, "CSR: n must be >= 1 and arrays non-null");
    if (rowstr[0] != 0) return set_error(CGB_ERR_BAD_MATRIX, "CSR: rowstr[0] = %d, want 0", rowstr[0]);
    for (int j = 0; j < n; j++)
        if (rowstr[j + 1] < rowstr[j])
            return set_error(CGB_ERR_BAD_MATRIX, "CSR: rowstr decreases at row %d", j);
    const long long nnz = rowstr[n];
    for (long long k = 0; k < nnz; k++) {
        if (colidx[k] < 0 || colidx[k] >= n)
            return set_error(CGB_ERR_BAD_MATRIX, "CSR: colidx[%lld] = %d outside [0, %d)", k,
                             colidx[k], n);
        if (!std::isfinite(a[k]))
            return set_error(CGB_ERR_NUMERIC, "CSR: a[%lld] is not finite", k);
    }
    return CGB_OK;
}

}  // namespace
}  // namespace cgb

using namespace cgb;

struct cgb_session {
    int device = 0;
    int n = 0;
    long long nnz = 0;
    long long nnz_cap = 0;
    cgb_options opts{};
    cudaDeviceProp prop{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    int *d_rowstr = nullptr;
    int *d_colidx = nullptr;
    double *d_a = nullptr;
    double *d_vec = nullptr;  // x, z, p, q, r: vstride doubles each
    size_t vstride = 0;
    double *d_part = nullptr;
    int gpad = 0;
    unsigned *d_sync = nullptr;  // [0] count, [32] gen, [64] ticket (128-byte lines)
    int *d_status = nullptr;
    int *d_split = nullptr;
    StepTrace *d_trace = nullptr;
    int trace_cap = 0;
    double *d_dot = nullptr;

    Plan plan;
    int *d_seg = nullptr;        // tiled: (nblk+1) x seg_stride segment offsets
    int seg_stride = 0;
    int nblk = 0;
    bool sorted = false;         // columns ascending within every row
    int *d_flag = nullptr;       // device scratch flag (unsorted rows)
    std::vector<int> h_rowstr_copy;

    const int *h_rowstr = nullptr;
    const int *h_colidx = nullptr;
    const double *h_a = nullptr;

    // graph of the last power iteration shape
    cudaGraphExec_t graph = nullptr;
    int g_niter = -1, g_cgitmax = -1, g_fixed = -1, g_warm = -1;
    double g_shift = 0.0, g_tol = -1.0;

    double *x() { return d_vec; }
    double *z() { return d_vec + vstride; }
    double *p() { return d_vec + 2 * vstride; }
    double *q() { return d_vec + 3 * vstride; }
    double *r() { return d_vec + 4 * vstride; }
    unsigned *count() { return d_sync; }
    unsigned *gen() { return d_sync + 32; }
    unsigned *ticket() { return d_sync + 64; }
};

namespace cgb {
namespace {

void drop_graph(cgb_session *s)
{
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->g_niter = -1;
}

void release(cgb_session *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    drop_graph(s);
    cudaFree(s->d_rowstr);
    cudaFree(s->d_colidx);
    cudaFree(s->d_a);
    cudaFree(s->d_vec);
    cudaFree(s->d_part);
    cudaFree(s->d_sync);
    cudaFree(s->d_status);
    cudaFree(s->d_split);
    cudaFree(s->d_trace);
    cudaFree(s->d_dot);
    cudaFree(s->d_seg);
    cudaFree(s->d_flag);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// Row split with balanced (stored entries + a per-row allowance for the
// vector updates) per CTA.
void make_split(int n, const int *rowstr, int grid, std::vector<int> &split)
{
    split.assign(grid + 1, n);
    const double per_row = 8.0;
    const double total = double(rowstr[n]) + per_row * n;
    int j = 0;
    split[0] = 0;
    for (int c = 1; c < grid; c++) {
        const double target = total * c / grid;
        while (j < n && double(rowstr[j]) + per_row * j < target) j++;
        split[c] = j;
    }
    split[grid] = n;
}

OuterArgs outer_args(cgb_session *s)
{
    OuterArgs A{};
    A.n = s->n;
    A.rowstr = s->d_rowstr;
    A.colidx = s->d_colidx;
    A.a = s->d_a;
    A.x = s->x();
    A.z = s->z();
    A.p = s->p();
    A.q = s->q();
    A.r = s->r();
    A.row_split = s->d_split;
    A.part = s->d_part;
    A.gpad = s->gpad;
    A.gb.count = s->count();
    A.gb.gen = s->gen();
    A.gb.status = s->d_status;
    A.gb.limit_ns = s->opts.wait_limit_ns > 0 ? s->opts.wait_limit_ns : kDefaultWaitNs;
    A.tile.seg = s->d_seg;
    A.tile.seg_stride = s->seg_stride;
    A.tile.nblk = s->nblk;
    A.tile.width = kTileWidth;
    A.tile.max_rows = s->plan.max_rows;
    A.trace = s->d_trace;
    return A;
}

cudaError_t launch_outer(cgb_session *s, const OuterArgs &A)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(s->plan.grid);
    cfg.blockDim = dim3(s->plan.block);
    cfg.dynamicSmemBytes = s->plan.smem;
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, s->plan.outer, A);
}

// Segment table of the column tiling, built on the device from the uploaded
// CSR (build_segments); also reports whether every row has ascending
// columns, which the tiled kernels need.
int build_tiling(cgb_session *s)
{
    const int n = s->n;
    s->nblk = (n + kTileWidth - 1) / kTileWidth;
    s->seg_stride = (n + 31) & ~31;
    const size_t count = size_t(s->nblk + 1) * s->seg_stride;
    cudaFree(s->d_seg);
    s->d_seg = nullptr;
    if (dev_alloc(&s->d_seg, count) != cudaSuccess)
        return set_error(CGB_ERR_NOMEM, "segment table allocation failed");
    CUDA_TRY(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream));
    build_segments<<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(
        s->d_rowstr, s->d_colidx, n, s->nblk, kTileWidth, s->d_seg, s->seg_stride, s->d_flag);
    CUDA_TRY(cudaGetLastError());
    int unsorted = 0;
    CUDA_TRY(cudaMemcpyAsync(&unsorted, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->sorted = (unsorted == 0);
    if (!s->sorted) {
        cudaFree(s->d_seg);
        s->d_seg = nullptr;
        s->nblk = 0;
    }
    return CGB_OK;
}

// Fills `pl` for (kind, lpr, rows): kernels, occupancy-sized cooperative grid,
// shared memory.  Returns false when the configuration cannot run here.
bool make_plan(cgb_session *s, int kind, int lpr, int rows, Plan *pl)
{
    Plan P;
    P.kind = kind;
    P.lpr = lpr;
    P.rows = rows;
    if (!kernels_for(kind, lpr, rows, &P.outer, &P.spmv)) return false;
    if (kind == kKindRow) {
        P.block = s->opts.block_threads ? s->opts.block_threads : 512;
        P.smem = 0;
        // almost nothing lives in shared memory: give L1 the room
        if (cudaFuncSetAttribute(P.outer, cudaFuncAttributePreferredSharedMemoryCarveout, 0) ||
            cudaFuncSetAttribute(P.spmv, cudaFuncAttributePreferredSharedMemoryCarveout, 0))
            return false;
    } else {
        if (!s->sorted || s->d_seg == nullptr) return false;
        P.block = 1024;
        // rows per CTA with one CTA per SM, balanced as make_split does
        const int grid = std::min(s->prop.multiProcessorCount, s->n);
        std::vector<int> split;
        make_split(s->n, s->h_rowstr_copy.data(), grid, split);
        int mr = 0;
        for (int c = 0; c < grid; c++) mr = std::max(mr, split[c + 1] - split[c]);
        P.max_rows = (mr + 31) & ~31;
        P.smem = tiled_smem_bytes(kTileWidth, P.max_rows);
        if (P.smem > kSmemLimit) return false;
        if (cudaFuncSetAttribute(P.outer, cudaFuncAttributeMaxDynamicSharedMemorySize, int(P.smem)) ||
            cudaFuncSetAttribute(P.spmv, cudaFuncAttributeMaxDynamicSharedMemorySize, int(P.smem)))
            return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, P.outer, P.block, P.smem) != cudaSuccess ||
        per_sm < 1)
        return false;
    per_sm = std::min(per_sm, kind == kKindTiled ? 1 : 4);
    P.grid = std::max(1, std::min(per_sm * s->prop.multiProcessorCount, s->n));
    if (P.grid > s->gpad) return false;
    *pl = P;
    return true;
}

// Makes `pl` the session's plan: uploads its row split.
int apply_plan(cgb_session *s, const Plan &pl)
{
    std::vector<int> split;
    make_split(s->n, s->h_rowstr_copy.data(), pl.grid, split);
    CUDA_TRY(cudaMemcpy(s->d_split, split.data(), sizeof(int) * (pl.grid + 1), cudaMemcpyHostToDevice));
    s->plan = pl;
    drop_graph(s);
    return CGB_OK;
}

SpmvArgs spmv_args(cgb_session *s)
{
    SpmvArgs S{};
    S.A = outer_args(s);
    S.ticket = s->ticket();
    S.dot = s->d_dot;
    return S;
}

// Mean device ms of `reps` standalone SpMV launches under the current plan.
int time_plan_spmv(cgb_session *s, int reps, double *ms_out)
{
    SpmvArgs S = spmv_args(s);
    const Plan &P = s->plan;
    fill_ones<<<s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->p(), s->n + 1);
    for (int i = 0; i < 2; i++) P.spmv<<<P.grid, P.block, P.smem, s->stream>>>(S);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
    for (int i = 0; i < reps; i++) P.spmv<<<P.grid, P.block, P.smem, s->stream>>>(S);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_out = double(ms) / reps;
    int st = 0;
    CUDA_TRY(cudaMemcpy(&st, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != kDevOk) {
        CUDA_TRY(cudaMemset(s->d_status, 0, sizeof(int)));
        return set_error(CGB_ERR_TIMEOUT, "SpMV wait failed (status %d)", st);
    }
    return CGB_OK;
}

// Picks the plan: the one the options force, else the fastest standalone
// SpMV among the candidates (the session's autotuner).
int choose_plan(cgb_session *s)
{
    const cgb_options &o = s->opts;
    const double mean = double(s->nnz) / double(s->n);
    std::vector<Plan> cands;
    auto add = [&](int kind, int lpr, int rows) {
        Plan p;
        if (make_plan(s, kind, lpr, rows, &p)) cands.push_back(p);
    };
    const int want_kind = o.spmv_kernel;
    if (want_kind == 0 || want_kind == kKindRow) {
        if (o.lanes_per_row > 0) add(kKindRow, o.lanes_per_row, 1);
        else {
            const int l = lanes_for_mean(mean);
            add(kKindRow, l, 1);
            if (want_kind == 0 && l > 2) add(kKindRow, l / 2, 1);
        }
    }
    if ((want_kind == 0 || want_kind == kKindTiled) && s->sorted && s->n >= 2 * kTileWidth) {
        if (o.lanes_per_row > 0) {
            add(kKindTiled, o.lanes_per_row, o.rows_in_flight > 0 ? o.rows_in_flight : 1);
        } else {
            add(kKindTiled, 4, 2);
            add(kKindTiled, 8, 2);
            add(kKindTiled, 8, 1);
            add(kKindTiled, 16, 1);
        }
    }
    if (cands.empty()) return set_error(CGB_ERR_INVALID, "no kernel configuration fits these options");
    if (cands.size() == 1) return apply_plan(s, cands[0]);
    double best = 1e30;
    int bi = 0;
    for (size_t i = 0; i < cands.size(); i++) {
        int st = apply_plan(s, cands[i]);
        if (st) return st;
        double ms = 0.0;
        st = time_plan_spmv(s, 10, &ms);
        if (st) return st;
        if (ms < best) {
            best = ms;
            bi = int(i);
        }
    }
    return apply_plan(s, cands[bi]);
}

int upload_matrix(cgb_session *s, const int *rowstr, const int *colidx, const double *a)
{
    const long long nnz = rowstr[s->n];
    if (nnz > s->nnz_cap) {
        cudaFree(s->d_colidx);
        cudaFree(s->d_a);
        s->d_colidx = nullptr;
        s->d_a = nullptr;
        if (dev_alloc(&s->d_colidx, nnz + kPad) != cudaSuccess ||
            dev_alloc(&s->d_a, nnz + kPad) != cudaSuccess)
            return set_error(CGB_ERR_NOMEM, "device allocation of %lld entries failed", nnz);
        s->nnz_cap = nnz;
    }
    s->nnz = nnz;
    CUDA_TRY(cudaMemcpyAsync(s->d_rowstr, rowstr, sizeof(int) * (s->n + 1), cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_colidx, colidx, sizeof(int) * nnz, cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_a, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_colidx + nnz, 0, sizeof(int) * kPad, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_a + nnz, 0, sizeof(double) * kPad, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->h_rowstr = rowstr;
    s->h_colidx = colidx;
    s->h_a = a;
    // same row pointers as before (e.g. the same matrix uploaded again): the
    // row split and tuned plan still hold; only the segment table is rebuilt
    const bool same_rows = s->plan.outer != nullptr &&
                           s->h_rowstr_copy.size() == size_t(s->n) + 1 &&
                           std::equal(rowstr, rowstr + s->n + 1, s->h_rowstr_copy.begin());
    s->h_rowstr_copy.assign(rowstr, rowstr + s->n + 1);
    const bool was_tiled = s->plan.kind == kKindTiled;
    s->sorted = false;
    cudaFree(s->d_seg);
    s->d_seg = nullptr;
    s->nblk = 0;
    if (s->n >= 2 * kTileWidth) {
        int st = build_tiling(s);
        if (st) return st;
    }
    if (same_rows && (!was_tiled || s->sorted)) {
        drop_graph(s);
        return CGB_OK;
    }
    s->plan = Plan();
    return choose_plan(s);
}

int ensure_trace(cgb_session *s, int niter)
{
    if (niter <= s->trace_cap) return CGB_OK;
    cudaFree(s->d_trace);
    s->d_trace = nullptr;
    if (dev_alloc(&s->d_trace, size_t(niter)) != cudaSuccess)
        return set_error(CGB_ERR_NOMEM, "trace allocation failed");
    s->trace_cap = niter;
    drop_graph(s);
    return CGB_OK;
}

// Reads the device status word after a synchronised launch; on failure
// resets the barrier words so the session stays usable.
int collect_status(cgb_session *s)
{
    int st = 0;
    CUDA_TRY(cudaMemcpy(&st, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st == kDevOk) return CGB_OK;
    CUDA_TRY(cudaMemset(s->d_sync, 0, sizeof(unsigned) * 96));
    CUDA_TRY(cudaMemset(s->d_status, 0, sizeof(int)));
    if (st == kDevTimeout)
        return set_error(CGB_ERR_TIMEOUT, "a grid barrier wait hit its %lld ns limit",
                         (long long)(s->opts.wait_limit_ns > 0 ? s->opts.wait_limit_ns : kDefaultWaitNs));
    if (st == kDevNonFinite) return set_error(CGB_ERR_NUMERIC, "non-finite zeta or residual");
    return set_error(CGB_ERR_CUDA, "device status %d", st);
}

// Enqueues one power iteration (x = 1, then niter outer-step kernels) on the
// session stream.
cudaError_t enqueue_power(cgb_session *s, const cgb_solve_params &P)
{
    cudaError_t e = cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream);
    if (e != cudaSuccess) return e;
    fill_ones<<<std::max(1, std::min(s->prop.multiProcessorCount, (s->n + 1 + 255) / 256)), 256, 0,
                s->stream>>>(s->x(), s->n + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    OuterArgs A = outer_args(s);
    A.shift = P.shift;
    A.cgitmax = P.cgitmax;
    A.fixed = (P.mode == CGB_MODE_FP64) ? 1 : 0;
    A.tol = P.tol;
    A.warm = P.warm_start;
    A.finish = 1;
    for (int it = 0; it < P.niter; it++) {
        A.step = it;
        e = launch_outer(s, A);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int check_params(const cgb_solve_params &P)
{
    if (P.niter < 1) return set_error(CGB_ERR_INVALID, "niter must be >= 1");
    if (P.cgitmax < 0) return set_error(CGB_ERR_INVALID, "cgitmax must be >= 0");
    if (!std::isfinite(P.shift)) return set_error(CGB_ERR_INVALID, "shift must be finite");
    if (P.mode != CGB_MODE_FP64 && P.mode != CGB_MODE_FP64_TOL)
        return set_error(CGB_ERR_INVALID, "mode %d is not available in this build", P.mode);
    if (P.mode != CGB_MODE_FP64 && !(P.tol > 0.0))
        return set_error(CGB_ERR_INVALID, "tolerance modes need tol > 0");
    return CGB_OK;
}

}  // namespace
}  // namespace cgb

// ======================================================================= ABI
extern "C" {

const char *cgb_status_string(int status)
{
    switch (status) {
    case CGB_OK: return "ok";
    case CGB_ERR_INVALID: return "invalid argument";
    case CGB_ERR_NOMEM: return "out of memory";
    case CGB_ERR_CAPACITY: return "output capacity too small";
    case CGB_ERR_CUDA: return "CUDA error";
    case CGB_ERR_TIMEOUT: return "device wait timed out";
    case CGB_ERR_NO_DEVICE: return "no usable sm_100 device";
    case CGB_ERR_STATE: return "invalid state";
    case CGB_ERR_NUMERIC: return "non-finite value";
    case CGB_ERR_BAD_MATRIX: return "malformed CSR matrix";
    default: return "unknown status";
    }
}

const char *cgb_last_error(void) { return cgb::g_last_error; }

int cgb_version(void) { return 10000 * 0 + 100 * 1 + 0; }

long long cgb_nz_bound(int n, int nonzer)
{
    if (n < 1 || nonzer < 0) return 0;
    return (long long)n * (nonzer + 1) * (nonzer + 1);
}

int cgb_makea(int n, int nonzer, double rcond, double shift, double seed, int *rowstr,
              int *colidx, double *a, long long nz_capacity, long long *nnz_out)
{
    return cgb::makea(n, nonzer, rcond, shift, seed, rowstr, colidx, a, nz_capacity, nnz_out);
}

void cgb_default_options(cgb_options *o)
{
    if (!o) return;
    o->device = 0;
    o->lanes_per_row = 0;
    o->block_threads = 0;
    o->wait_limit_ns = 0;
    o->use_graph = 1;
    o->keep_fp32_copy = 1;
    o->spmv_kernel = 0;
    o->rows_in_flight = 0;
}

void cgb_default_solve_params(cgb_solve_params *p)
{
    if (!p) return;
    p->niter = 15;
    p->shift = 10.0;
    p->mode = CGB_MODE_FP64;
    p->cgitmax = 25;
    p->tol = 1e-12;
    p->refresh_every = 10;
    p->warm_start = 0;
}

int cgb_device_info(int device, int *sm_count, int *cc_major, int *cc_minor,
                    long long *global_mem_bytes)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return set_error(CGB_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= count) return set_error(CGB_ERR_NO_DEVICE, "bad device %d", device);
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (cc_major) *cc_major = prop.major;
    if (cc_minor) *cc_minor = prop.minor;
    if (global_mem_bytes) *global_mem_bytes = (long long)prop.totalGlobalMem;
    return CGB_OK;
}

int cgb_create(int n, const int *rowstr, const int *colidx, const double *a,
               const cgb_options *opts, cgb_session **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "out is null");
    *out = nullptr;
    int st = validate_csr(n, rowstr, colidx, a);
    if (st) return st;
    cgb_options o;
    cgb_default_options(&o);
    if (opts) o = *opts;
    if (o.lanes_per_row != 0 && o.lanes_per_row != 2 && o.lanes_per_row != 4 &&
        o.lanes_per_row != 8 && o.lanes_per_row != 16 && o.lanes_per_row != 32)
        return set_error(CGB_ERR_INVALID, "lanes_per_row must be 0, 2, 4, 8, 16 or 32");
    if (o.block_threads != 0 && o.block_threads != 256 && o.block_threads != 512)
        return set_error(CGB_ERR_INVALID, "block_threads must be 0, 256 or 512");
    if (o.spmv_kernel < 0 || o.spmv_kernel > 2)
        return set_error(CGB_ERR_INVALID, "spmv_kernel must be 0 (auto), 1 (row) or 2 (tiled)");
    if (o.rows_in_flight < 0 || o.rows_in_flight > 2)
        return set_error(CGB_ERR_INVALID, "rows_in_flight must be 0, 1 or 2");
    cudaDeviceProp prop;
    st = check_device(o.device, &prop);
    if (st) return st;
    CUDA_TRY(cudaSetDevice(o.device));

    cgb_session *s = new (std::nothrow) cgb_session;
    if (!s) return set_error(CGB_ERR_NOMEM, "session allocation failed");
    s->device = o.device;
    s->n = n;
    s->opts = o;
    s->prop = prop;
    s->vstride = (size_t(n) + 2 + 31) & ~size_t(31);
    s->gpad = 4 * prop.multiProcessorCount;
#define CREATE_TRY(call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            int rc_ = set_error(e_ == cudaErrorMemoryAllocation ? CGB_ERR_NOMEM : CGB_ERR_CUDA, \
                                "%s: %s", #call, cudaGetErrorString(e_));                 \
            release(s);                                                                   \
            return rc_;                                                                   \
        }                                                                                 \
    } while (0)
    CREATE_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CREATE_TRY(cudaEventCreate(&s->ev0));
    CREATE_TRY(cudaEventCreate(&s->ev1));
    CREATE_TRY(dev_alloc(&s->d_rowstr, size_t(n) + 1));
    CREATE_TRY(dev_alloc(&s->d_vec, 5 * s->vstride));
    CREATE_TRY(cudaMemset(s->d_vec, 0, sizeof(double) * 5 * s->vstride));
    CREATE_TRY(dev_alloc(&s->d_part, size_t(kSlotCount) * s->gpad));
    CREATE_TRY(dev_alloc(&s->d_sync, 96));
    CREATE_TRY(cudaMemset(s->d_sync, 0, sizeof(unsigned) * 96));
    CREATE_TRY(dev_alloc(&s->d_status, 1));
    CREATE_TRY(cudaMemset(s->d_status, 0, sizeof(int)));
    CREATE_TRY(dev_alloc(&s->d_split, size_t(s->gpad) + 1));
    CREATE_TRY(dev_alloc(&s->d_dot, 1));
    CREATE_TRY(dev_alloc(&s->d_flag, 1));
#undef CREATE_TRY
    st = ensure_trace(s, 128);
    if (st == CGB_OK) st = upload_matrix(s, rowstr, colidx, a);
    if (st != CGB_OK) {
        release(s);
        return st;
    }
    *out = s;
    return CGB_OK;
}

int cgb_upload(cgb_session *s, const int *rowstr, const int *colidx, const double *a)
{
    if (!s) return set_error(CGB_ERR_INVALID, "session is null");
    int st = validate_csr(s->n, rowstr, colidx, a);
    if (st) return st;
    CUDA_TRY(cudaSetDevice(s->device));
    return upload_matrix(s, rowstr, colidx, a);
}

int cgb_destroy(cgb_session *s)
{
    release(s);
    return CGB_OK;
}

int cgb_conj_grad(cgb_session *s, const int *colidx, const int *rowstr, const double *x,
                  double *z, const double *a, double *p, double *q, double *r, double *rnorm)
{
    if (!s || !x || !z || !p || !q || !r || !rnorm)
        return set_error(CGB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->device));
    if (colidx != s->h_colidx || rowstr != s->h_rowstr || a != s->h_a) {
        int st = cgb_upload(s, rowstr, colidx, a);
        if (st) return st;
    }
    const size_t bytes = sizeof(double) * (size_t(s->n) + 1);
    CUDA_TRY(cudaMemcpyAsync(s->x(), x, bytes, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    OuterArgs A = outer_args(s);
    A.shift = 0.0;
    A.cgitmax = 25;  // cgitmax of the reference (cg.cu:666)
    A.fixed = 1;
    A.tol = 0.0;
    A.warm = 0;
    A.step = 0;
    A.finish = 0;
    CUDA_TRY(launch_outer(s, A));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    int st = collect_status(s);
    if (st) return st;
    CUDA_TRY(cudaMemcpy(z, s->z(), bytes, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(p, s->p(), bytes, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(q, s->q(), bytes, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(r, s->r(), bytes, cudaMemcpyDeviceToHost));
    StepTrace t;
    CUDA_TRY(cudaMemcpy(&t, s->d_trace, sizeof(t), cudaMemcpyDeviceToHost));
    *rnorm = t.rnorm;
    return CGB_OK;
}

int cgb_power_iterate(cgb_session *s, const cgb_solve_params *params, double *zeta_trace,
                      double *rnorm_trace, int *iters_trace, double *x_out,
                      cgb_solve_result *res)
{
    if (!s || !params) return set_error(CGB_ERR_INVALID, "null session or params");
    const cgb_solve_params P = *params;
    int st = check_params(P);
    if (st) return st;
    CUDA_TRY(cudaSetDevice(s->device));
    st = ensure_trace(s, P.niter);
    if (st) return st;
    const int fixed = P.mode == CGB_MODE_FP64 ? 1 : 0;
    if (s->opts.use_graph) {
        const bool same = s->graph && s->g_niter == P.niter && s->g_cgitmax == P.cgitmax &&
                          s->g_fixed == fixed && s->g_warm == P.warm_start &&
                          s->g_shift == P.shift && s->g_tol == P.tol;
        if (!same) {
            drop_graph(s);
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue_power(s, P);
            cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
            if (e != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return set_error(CGB_ERR_CUDA, "graph capture failed: %s",
                                 cudaGetErrorString(e != cudaSuccess ? e : e2));
            }
            e = cudaGraphInstantiate(&s->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                s->graph = nullptr;
                return set_error(CGB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
            }
            s->g_niter = P.niter;
            s->g_cgitmax = P.cgitmax;
            s->g_fixed = fixed;
            s->g_warm = P.warm_start;
            s->g_shift = P.shift;
            s->g_tol = P.tol;
        }
        CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
        CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
        CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    } else {
        CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
        CUDA_TRY(enqueue_power(s, P));
        CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    st = collect_status(s);
    if (st) return st;
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    std::vector<StepTrace> tr(P.niter);
    CUDA_TRY(cudaMemcpy(tr.data(), s->d_trace, sizeof(StepTrace) * P.niter, cudaMemcpyDeviceToHost));
    int total_inner = 0;
    for (int i = 0; i < P.niter; i++) {
        if (zeta_trace) zeta_trace[i] = tr[i].zeta;
        if (rnorm_trace) rnorm_trace[i] = tr[i].rnorm;
        if (iters_trace) iters_trace[i] = int(tr[i].inner);
        total_inner += int(tr[i].inner);
    }
    if (x_out) CUDA_TRY(cudaMemcpy(x_out, s->x(), sizeof(double) * s->n, cudaMemcpyDeviceToHost));
    if (res) {
        res->zeta = tr[P.niter - 1].zeta;
        res->rnorm = tr[P.niter - 1].rnorm;
        res->device_ms = ms;
        res->total_inner = total_inner;
        res->fallbacks = 0;
    }
    return CGB_OK;
}

int cgb_time_spmv(cgb_session *s, int reps, int fp32, double *ms_per_launch)
{
    if (!s || reps < 1 || !ms_per_launch) return set_error(CGB_ERR_INVALID, "bad arguments");
    if (fp32) return set_error(CGB_ERR_INVALID, "FP32 SpMV is not available in this build");
    CUDA_TRY(cudaSetDevice(s->device));
    return time_plan_spmv(s, reps, ms_per_launch);
}

int cgb_plan_info(cgb_session *s, int *kind, int *lanes_per_row, int *rows_in_flight, int *grid,
                  int *block, long long *smem_bytes)
{
    if (!s) return set_error(CGB_ERR_INVALID, "session is null");
    if (kind) *kind = s->plan.kind;
    if (lanes_per_row) *lanes_per_row = s->plan.lpr;
    if (rows_in_flight) *rows_in_flight = s->plan.rows;
    if (grid) *grid = s->plan.grid;
    if (block) *block = s->plan.block;
    if (smem_bytes) *smem_bytes = (long long)s->plan.smem;
    return CGB_OK;
}

int cgb_time_outer_steps(cgb_session *s, int niter, double shift, double *kernel_ms,
                         double *graph_gap_ms)
{
    if (!s || niter < 1 || !kernel_ms || !graph_gap_ms)
        return set_error(CGB_ERR_INVALID, "bad arguments");
    CUDA_TRY(cudaSetDevice(s->device));
    int st = ensure_trace(s, niter);
    if (st) return st;
    std::vector<cudaEvent_t> ev(niter + 1);
    for (auto &e : ev) CUDA_TRY(cudaEventCreate(&e));
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    fill_ones<<<s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->x(), s->n + 1);
    OuterArgs A = outer_args(s);
    A.shift = shift;
    A.cgitmax = 25;
    A.fixed = 1;
    A.finish = 1;
    for (int it = 0; it < niter; it++) {
        CUDA_TRY(cudaEventRecord(ev[it], s->stream));
        A.step = it;
        CUDA_TRY(launch_outer(s, A));
    }
    CUDA_TRY(cudaEventRecord(ev[niter], s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    double total = 0.0;
    for (int it = 0; it < niter; it++) {
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, ev[it], ev[it + 1]));
        total += ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    st = collect_status(s);
    if (st) return st;
    *kernel_ms = total / niter;
    // the graph's per-step cost beyond one kernel: time a graph of niter steps
    cgb_solve_params P;
    cgb_default_solve_params(&P);
    P.niter = niter;
    P.shift = shift;
    cgb_solve_result res;
    st = cgb_power_iterate(s, &P, nullptr, nullptr, nullptr, nullptr, &res);
    if (st) return st;
    *graph_gap_ms = res.device_ms / niter - *kernel_ms;
    return CGB_OK;
}

int cgb_selftest_wait_timeout(cgb_session *s, long long limit_ns, int *device_status)
{
    if (!s || !device_status || limit_ns <= 0 || limit_ns > 10000000000LL)
        return set_error(CGB_ERR_INVALID, "limit_ns must be in (0, 1e10]");
    CUDA_TRY(cudaSetDevice(s->device));
    GridBarrier gb;
    gb.count = s->count();
    gb.gen = s->gen();
    gb.status = s->d_status;
    gb.limit_ns = limit_ns;
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    barrier_timeout_probe<<<2, 32, 0, s->stream>>>(gb);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(cudaMemcpy(device_status, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    return collect_status(s);
}

int cgb_host_alloc(void **ptr, long long bytes)
{
    if (!ptr || bytes <= 0) return set_error(CGB_ERR_INVALID, "bad arguments");
    CUDA_TRY(cudaHostAlloc(ptr, size_t(bytes), cudaHostAllocDefault));
    return CGB_OK;
}

int cgb_host_free(void *ptr)
{
    if (ptr) CUDA_TRY(cudaFreeHost(ptr));
    return CGB_OK;
}

}  // extern "C"

// session.cu -- the C ABI of libcgb: device set-up, the conj_grad-compatible
// call, the CUDA-graph power iteration, the SpMV autotuner and diagnostics.
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
#include <thread>
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

constexpr int kPad = 64;                   // entries of padding after matrix arrays
constexpr long long kDefaultWaitNs = 2000000000LL;
constexpr size_t kSmemLimit = 227 * 1024;  // opt-in shared memory per CTA on sm_100
constexpr int kKindRow = 1;
constexpr int kKindSliced = 2;
constexpr int kKindSlicedPrefetch = 3;  // option and report only: sliced plan with prefetch = 1

template <typename T>
cudaError_t dev_alloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

// Grow-only buffer: keeps *p when it already holds `count` elements, so a
// re-upload of the same structure allocates nothing.
template <typename T>
cudaError_t dev_reserve(T **p, size_t *cap, size_t count)
{
    if (*p && *cap >= count) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
    if (e == cudaSuccess) *cap = count;
    return e;
}

template <typename T>
void dev_free(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

using OuterKernel = void (*)(OuterArgs);
using SpmvKernel = void (*)(SpmvArgs);

// A launch configuration of the persistent kernels.
struct Plan {
    int kind = 0;  // kKindRow / kKindSliced
    int lpr = 0;   // row policy: lanes per row
    OuterKernel fp64 = nullptr;
    OuterKernel mixed = nullptr;
    OuterKernel pcg = nullptr;
    SpmvKernel spmv = nullptr;    // standalone SpMV (FP64; the row kernels also FP32 by flag)
    SpmvKernel spmv32 = nullptr;  // standalone FP32 SpMV
    int block = 512;        // FP64 outer step and standalone SpMV
    int block_mixed = 512;  // mixed outer step
    int block_pcg = 512;    // preconditioned outer step
    int prefetch = 0;       // sliced: L2 prefetch of the next block's slices
    double l2_keep = 0.0;   // sliced: bytes of the matrix stream kept in L2 across products
    int grid = 0;
    size_t smem = 0;
};

bool row_kernels(int lpr, Plan *P)
{
    switch (lpr) {
    case 2: P->fp64 = outer_step_fp64<2>; P->mixed = outer_step_mixed<2>; P->pcg = outer_step_pcg<2>; P->spmv = P->spmv32 = spmv_dot_row<2>; return true;
    case 4: P->fp64 = outer_step_fp64<4>; P->mixed = outer_step_mixed<4>; P->pcg = outer_step_pcg<4>; P->spmv = P->spmv32 = spmv_dot_row<4>; return true;
    case 8: P->fp64 = outer_step_fp64<8>; P->mixed = outer_step_mixed<8>; P->pcg = outer_step_pcg<8>; P->spmv = P->spmv32 = spmv_dot_row<8>; return true;
    case 16: P->fp64 = outer_step_fp64<16>; P->mixed = outer_step_mixed<16>; P->pcg = outer_step_pcg<16>; P->spmv = P->spmv32 = spmv_dot_row<16>; return true;
    case 32: P->fp64 = outer_step_fp64<32>; P->mixed = outer_step_mixed<32>; P->pcg = outer_step_pcg<32>; P->spmv = P->spmv32 = spmv_dot_row<32>; return true;
    default: return false;
    }
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

// Pointers and row pointers (rowstr[0] = 0, never decreasing).
int validate_rowstr(int n, const int *rowstr, const int *colidx, const double *a)
{
    if (n < 1 || !rowstr || !colidx || !a)
        return set_error(CGB_ERR_INVALID, "CSR: n must be >= 1 and arrays non-null");
    if (rowstr[0] != 0) return set_error(CGB_ERR_BAD_MATRIX, "CSR: rowstr[0] = %d, want 0", rowstr[0]);
    for (int j = 0; j < n; j++)
        if (rowstr[j + 1] < rowstr[j])
            return set_error(CGB_ERR_BAD_MATRIX, "CSR: rowstr decreases at row %d", j);
    return CGB_OK;
}

// Entries: columns in [0, n), finite values.
int validate_entries(int n, const int *rowstr, const int *colidx, const double *a)
{
    const long long nnz = rowstr[n];
    // entries checked in parallel chunks; the first bad entry (lowest index)
    // is reported, as a serial scan would
    const long long kChunk = 1 << 20;
    const long long nchunks = (nnz + kChunk - 1) / kChunk;
    std::vector<long long> first_bad(size_t(std::max<long long>(nchunks, 1)), -1);
    auto scan = [&](long long c0, long long c1) {
        for (long long c = c0; c < c1; c++) {
            const long long e = std::min(nnz, (c + 1) * kChunk);
            for (long long k = c * kChunk; k < e; k++)
                if (colidx[k] < 0 || colidx[k] >= n || !std::isfinite(a[k])) {
                    first_bad[size_t(c)] = k;
                    break;
                }
        }
    };
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const long long nt = std::min<long long>(hw, nchunks);
    if (nt <= 1) {
        scan(0, nchunks);
    } else {
        std::vector<std::thread> pool;
        for (long long t = 1; t < nt; t++)
            pool.emplace_back(scan, nchunks * t / nt, nchunks * (t + 1) / nt);
        scan(0, nchunks / nt);
        for (auto &th : pool) th.join();
    }
    for (long long c = 0; c < nchunks; c++) {
        const long long k = first_bad[size_t(c)];
        if (k < 0) continue;
        if (colidx[k] < 0 || colidx[k] >= n)
            return set_error(CGB_ERR_BAD_MATRIX, "CSR: colidx[%lld] = %d outside [0, %d)", k,
                             colidx[k], n);
        return set_error(CGB_ERR_NUMERIC, "CSR: a[%lld] is not finite", k);
    }
    return CGB_OK;
}

int validate_csr(int n, const int *rowstr, const int *colidx, const double *a)
{
    const int st = validate_rowstr(n, rowstr, colidx, a);
    return st ? st : validate_entries(n, rowstr, colidx, a);
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

    // CSR (reference layout) and its FP32 values
    int *d_rowstr = nullptr;
    int *d_colidx = nullptr;
    double *d_a = nullptr;
    // staging copy of a re-uploaded CSR: the host validates the entries while
    // it crosses to the device, and only a valid matrix replaces the session's
    int *d_rowstr_in = nullptr, *d_colidx_in = nullptr;
    double *d_a_in = nullptr;
    size_t cap_rowstr_in = 0, cap_colidx_in = 0, cap_a_in = 0;
    float *d_a32 = nullptr;
    // vectors: x, z, p, q, r (vstride doubles each) and p32
    double *d_vec = nullptr;
    float *d_p32 = nullptr;
    float *d_r32 = nullptr;
    __nv_bfloat16 *d_r16 = nullptr, *d_t16 = nullptr;  // the sliced factor products' vectors
    double *d_y = nullptr;
    double *d_hx = nullptr, *d_hw = nullptr;  // Galerkin-start ring: kMaxRecycle vectors each
    size_t vstride = 0;
    // preconditioner factor F (lower, CSR) and F^T, FP32 values
    int *d_f_ptr = nullptr, *d_f_col = nullptr, *d_ft_ptr = nullptr, *d_ft_col = nullptr;
    float *d_f_val = nullptr, *d_ft_val = nullptr;
    bool has_prec = false;
    long long prec_nnz = 0;  // entries of the preconditioner factor
    // reductions, barrier, status, trace
    double *d_part = nullptr;
    int gpad = 0;
    unsigned *d_sync = nullptr;  // [0] count, [32] gen, [64] ticket (128-byte lines)
    int *d_status = nullptr;
    int *d_flag = nullptr;
    int *d_split = nullptr;
    StepTrace *d_trace = nullptr;
    int trace_cap = 0;
    double *d_dot = nullptr;

    // sliced layout (built for the sliced plan's row split)
    int *d_seg = nullptr;
    int seg_stride = 0;
    int nblk = 0;
    bool sorted = false;
    bool l2_marked = false;  // a solve ran with an L2 keep fraction (lines at evict_last)
    int sliced_grid = 0;   // grid the layout was built for (0: none)
    int sliced_max_rows = 0;
    int sliced_nacc = 2;           // row accumulators (4 when they fit: FP32 pipeline depth)
    int prec_panels = 1;           // row panels of the factor copies' interleaved rows
    int *d_chunk_slice = nullptr;  // shared by A, F and F^T (same row split)
    size_t cap_chunk = 0, cap_seg = 0;  // allocated elements of d_chunk_slice, d_seg
    cgb::SliceSet sa;              // A: FP64 values (+ FP32 copy)
    cgb::SliceSet sf, sft;         // F and F^T: FP32 values
    int layout_gen = 0;            // bumped by every build of A's slices
    int prec_gen = -1;             // layout_gen sf / sft were built for

    Plan plan;
    std::vector<int> h_rowstr_copy;
    const int *h_rowstr = nullptr;
    const int *h_colidx = nullptr;
    const double *h_a = nullptr;

    // graph of the last power iteration shape
    cudaGraphExec_t graph = nullptr;
    cgb_solve_params g_params{};
    std::vector<unsigned char> g_sig;  // GraphSig bytes of the captured iteration
    bool g_valid = false;

    double *x() { return d_vec; }
    double *z() { return d_vec + vstride; }
    double *p() { return d_vec + 2 * vstride; }
    double *q() { return d_vec + 3 * vstride; }
    double *r() { return d_vec + 4 * vstride; }
    // the grid barrier's 64-bit arrival count (its own 128-byte line)
    unsigned long long *arrivals() { return reinterpret_cast<unsigned long long *>(d_sync); }
    unsigned *ticket() { return d_sync + 64; }
};

namespace cgb {
namespace {

void drop_graph(cgb_session *s)
{
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->g_valid = false;
}

void free_set(SliceSet &t)
{
    dev_free(t.srow);
    dev_free(t.width);
    dev_free(t.off);
    dev_free(t.sval);
    dev_free(t.sval32);
    dev_free(t.sval16);
    dev_free(t.scol);
    dev_free(t.chunk_slice);
    t = SliceSet();
}

void free_prec_slices(cgb_session *s)
{
    free_set(s->sf);
    free_set(s->sft);
    s->prec_gen = -1;
}

void free_sliced(cgb_session *s)
{
    dev_free(s->d_chunk_slice);
    s->cap_chunk = 0;
    free_set(s->sa);
    free_prec_slices(s);
    s->sliced_grid = 0;
}

// Marks A's sliced copy stale without freeing its buffers (a rebuild of
// the same size reuses them).
void invalidate_sliced(cgb_session *s)
{
    free_prec_slices(s);
    s->sliced_grid = 0;
}

// Enqueues the demotion of the sliced copy's L2 lines to normal priority.
void demote_matrix_lines(cgb_session *s)
{
    const SliceSet &t = s->sa;
    const std::pair<const void *, size_t> spans[3] = {
        {t.sval, size_t(t.entries) * sizeof(double)},
        {t.sval32, size_t(t.entries) * sizeof(float)},
        {t.scol, size_t(t.entries) * sizeof(unsigned short)}};
    for (const auto &sp : spans)
        if (sp.first && sp.second)
            l2_demote<<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(
                static_cast<const char *>(sp.first), sp.second);
}

void release(cgb_session *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    drop_graph(s);
    if (s->l2_marked) {
        demote_matrix_lines(s);  // lines kept at evict_last go back to normal priority
        cudaStreamSynchronize(s->stream);
    }
    free_sliced(s);
    dev_free(s->d_rowstr);
    dev_free(s->d_colidx);
    dev_free(s->d_a);
    dev_free(s->d_a32);
    dev_free(s->d_rowstr_in);
    dev_free(s->d_colidx_in);
    dev_free(s->d_a_in);
    dev_free(s->d_vec);
    dev_free(s->d_p32);
    dev_free(s->d_r32);
    dev_free(s->d_r16);
    dev_free(s->d_t16);
    dev_free(s->d_y);
    dev_free(s->d_hx);
    dev_free(s->d_hw);
    dev_free(s->d_f_ptr);
    dev_free(s->d_f_col);
    dev_free(s->d_f_val);
    dev_free(s->d_ft_ptr);
    dev_free(s->d_ft_col);
    dev_free(s->d_ft_val);
    dev_free(s->d_part);
    dev_free(s->d_sync);
    dev_free(s->d_status);
    dev_free(s->d_flag);
    dev_free(s->d_split);
    dev_free(s->d_trace);
    dev_free(s->d_dot);
    dev_free(s->d_seg);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// Points the sliced members of M at slice set t (A's column blocks; A's
// row split unless t is interleaved).
void set_slices(cgb_session *s, const SliceSet &t, MatrixView *M)
{
    M->sval = t.sval;
    M->sval32 = t.sval32;
    M->sval16 = t.sval16;
    M->scol = t.scol;
    M->srow = t.srow;
    M->slice_off = t.off;
    M->slice_width = t.width;
    M->chunk_slice = t.chunk_slice ? t.chunk_slice : s->d_chunk_slice;
    M->nblk = t.blocks ? t.blocks : s->nblk;
    M->width = t.block_cols ? t.block_cols : kSliceWidth;
    M->max_rows = s->sliced_max_rows;
    M->nacc = s->sliced_nacc;
    M->interleaved = t.interleaved;
    M->panels = t.panels;
    M->slice_entries = t.entries + kPad;
    M->ncols = s->n;
}

// Keep fractions of the sliced streams for a solve whose products are FP64
// (fp32 = 0) or FP32 (fp32 = 1): the plan's L2 budget over the stream's
// bytes (values + 16-bit columns); the other stream is not kept.
void set_keep(const cgb_session *s, MatrixView *M, int fp32)
{
    M->keep64 = M->keep32 = M->keep16 = 0.f;
    if (s->plan.kind != kKindSliced || s->plan.l2_keep <= 0.0 || s->sa.entries <= 0) return;
    const double bytes = double(s->sa.entries) * (fp32 ? 6.0 : 10.0);
    const float f = float(std::min(1.0, s->plan.l2_keep / bytes));
    if (fp32) M->keep32 = f;
    else M->keep64 = f;
}

MatrixView matrix_view(cgb_session *s)
{
    MatrixView M{};
    M.rowstr = s->d_rowstr;
    M.colidx = s->d_colidx;
    M.a = s->d_a;
    M.a32 = s->d_a32;
    M.csr_entries = s->nnz + kPad;
    M.ncols = s->n;
    set_slices(s, s->sa, &M);
    set_keep(s, &M, 0);
    return M;
}

OuterArgs outer_args(cgb_session *s)
{
    OuterArgs A{};
    A.n = s->n;
    A.M = matrix_view(s);
    A.x = s->x();
    A.z = s->z();
    A.p = s->p();
    A.q = s->q();
    A.r = s->r();
    A.p32 = s->d_p32;
    A.r32 = s->d_r32;
    A.r16 = s->d_r16;
    A.t16 = s->d_t16;
    A.y = s->d_y;
    A.F.rowstr = s->d_f_ptr;
    A.F.colidx = s->d_f_col;
    A.F.a32 = s->d_f_val;
    A.FT.rowstr = s->d_ft_ptr;
    A.FT.colidx = s->d_ft_col;
    A.FT.a32 = s->d_ft_val;
    A.F.csr_entries = A.FT.csr_entries = s->prec_nnz + kPad;
    A.F.ncols = A.FT.ncols = s->n;
    if (s->prec_gen == s->layout_gen && s->prec_gen >= 0) {
        set_slices(s, s->sf, &A.F);
        set_slices(s, s->sft, &A.FT);
    }
    A.row_split = s->d_split;
    A.part = s->d_part;
    A.gpad = s->gpad;
    A.gb.arrivals = s->arrivals();
    A.gb.status = s->d_status;
    A.gb.limit_ns = s->opts.wait_limit_ns > 0 ? s->opts.wait_limit_ns : kDefaultWaitNs;
    A.refresh_every = 10;
    A.trace = s->d_trace;
    A.hx = s->d_hx;
    A.hw = s->d_hw;
    A.hstride = s->vstride;
    A.recycle = 0;
    return A;
}

cudaError_t launch_outer(cgb_session *s, OuterKernel k, const OuterArgs &A)
{
    if (A.M.keep64 > 0.f || A.M.keep32 > 0.f || A.M.keep16 > 0.f) s->l2_marked = true;
    const Plan &P = s->plan;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(P.grid);
    cfg.blockDim = dim3(k == P.mixed ? P.block_mixed : k == P.pcg ? P.block_pcg : P.block);
    cfg.dynamicSmemBytes = s->plan.smem;
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, A);
}

// Segment table of the column blocking, built on the device; also finds
// whether every row has ascending columns (the sliced layout needs it).
int build_segments_table(cgb_session *s)
{
    const int n = s->n;
    s->nblk = (n + kSliceWidth - 1) / kSliceWidth;
    s->seg_stride = (n + 31) & ~31;
    const size_t count = size_t(s->nblk + 1) * s->seg_stride;
    if (dev_reserve(&s->d_seg, &s->cap_seg, count) != cudaSuccess)
        return set_error(CGB_ERR_NOMEM, "segment table allocation failed");
    CUDA_TRY(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream));
    build_segments<<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(
        s->d_rowstr, s->d_colidx, n, s->nblk, kSliceWidth, s->d_seg, s->seg_stride, s->d_flag);
    CUDA_TRY(cudaGetLastError());
    int unsorted = 0;
    CUDA_TRY(cudaMemcpyAsync(&unsorted, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->sorted = (unsorted == 0);
    if (!s->sorted) s->nblk = 0;
    return CGB_OK;
}

// Chunk table of a sliced copy: first slice of each (CTA c, block b), 32
// rows a slice; rows per CTA from `rows_of(c)`.  Returns the slice count.
template <typename RowsOf>
int chunk_table(int grid, int panels, int nblk, RowsOf rows_of, std::vector<int> &chunk_slice)
{
    const size_t chunks = size_t(grid) * panels * nblk;
    chunk_slice.assign(chunks + 1, 0);
    int total = 0;
    for (int c = 0; c < grid; c++) {
        const int rows = rows_of(c);
        for (int k = 0; k < panels; k++) {
            const int prow = panel_begin(rows, k + 1, panels) - panel_begin(rows, k, panels);
            for (int b = 0; b < nblk; b++) {
                chunk_slice[(size_t(c) * panels + k) * nblk + b] = total;
                total += (prow + 31) / 32;
            }
        }
    }
    chunk_slice[chunks] = total;
    return total;
}

// Steps 1-3 of a sliced copy of one matrix over `grid` CTAs: row order per
// slice, slice offsets, then values (FP64 and/or FP32) and local columns.
// `seg` is the matrix's segment table; rows are the CTAs' ranges of d_split
// or, with `interleave`, every grid-th row.  t->chunk_slice must be set.
template <typename ST>
int fill_set(cgb_session *s, int grid, bool interleave, const int *seg, const int *d_colidx,
             const ST *vals, int total, bool want64, bool want32, bool want16, SliceSet *t)
{
    const int nblk = t->blocks ? t->blocks : s->nblk;
    const int bcols = t->block_cols ? t->block_cols : kSliceWidth;
    const int nchunks = grid * t->panels * nblk;
    const int ig = interleave ? grid : 0;
    t->interleaved = interleave ? 1 : 0;
    if (dev_reserve(&t->srow, &t->cap_srow, size_t(total) * 32) ||
        dev_reserve(&t->width, &t->cap_width, size_t(total)) ||
        dev_reserve(&t->off, &t->cap_off, size_t(total) + 1))
        return set_error(CGB_ERR_NOMEM, "sliced layout: metadata allocation failed");
    slice_sort_rows<<<nchunks, 256, 0, s->stream>>>(seg, s->seg_stride, nblk, s->d_split, ig,
                                                   t->panels, s->n, t->chunk_slice, t->srow,
                                                   t->width);
    CUDA_TRY(cudaGetLastError());
    slice_offsets<<<1, 1024, 0, s->stream>>>(t->width, total, t->off);
    CUDA_TRY(cudaGetLastError());
    unsigned entries = 0;
    CUDA_TRY(cudaMemcpyAsync(&entries, t->off + total, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    t->entries = entries;
    if ((want64 && dev_reserve(&t->sval, &t->cap_sval, size_t(entries) + kPad)) ||
        dev_reserve(&t->scol, &t->cap_scol, size_t(entries) + kPad) ||
        (want32 && dev_reserve(&t->sval32, &t->cap_sval32, size_t(entries) + kPad)) ||
        (want16 && dev_reserve(&t->sval16, &t->cap_sval16, size_t(entries) + kPad)))
        return set_error(CGB_ERR_NOMEM, "sliced layout: %u entries do not fit", entries);
    slice_fill<ST><<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(
        seg, s->seg_stride, nblk, bcols, s->d_split, ig, t->panels, s->n, t->chunk_slice, nchunks,
        d_colidx, vals, t->srow, t->width, t->off, total, t->sval, t->sval32, t->sval16, t->scol);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return CGB_OK;
}

// The sliced copy of the matrix for a row split over `grid` CTAs (one per SM).
int build_sliced(cgb_session *s, int grid)
{
    invalidate_sliced(s);
    std::vector<int> split;
    make_split(s->n, s->h_rowstr_copy.data(), grid, split);
    // dynamic shared memory must fit beside the kernels' static arrays
    size_t static_smem = 0;
    for (const void *k : {(const void *)outer_step_fp64_sliced, (const void *)outer_step_mixed_sliced,
                          (const void *)outer_step_pcg_sliced, (const void *)spmv_dot_sliced,
                          (const void *)spmv_dot_sliced32, (const void *)outer_step_fp64_sliced_pf,
                          (const void *)outer_step_mixed_sliced_pf, (const void *)spmv_dot_sliced_pf,
                          (const void *)spmv_dot_sliced32_pf, (const void *)outer_step_fp64_sliced_pn,
                          (const void *)outer_step_mixed_sliced_pn, (const void *)outer_step_pcg_sliced_pn,
                          (const void *)spmv_dot_sliced_pn, (const void *)spmv_dot_sliced32_pn}) {
        cudaFuncAttributes fa;
        CUDA_TRY(cudaFuncGetAttributes(&fa, k));
        static_smem = std::max(static_smem, size_t(fa.sharedSizeBytes));
    }
    const size_t room = kSmemLimit - std::min(kSmemLimit, static_smem);
    // rows two accumulators can hold beside the staging (a multiple of 32,
    // below the 16-bit local-row marker)
    const size_t fixed = sliced_smem_bytes(0, 2);
    int cap = room > fixed ? int(std::min<size_t>((room - fixed) / (2 * sizeof(double)), 0xffe0) & ~size_t(31))
                           : 0;
    if (cap < 32) return set_error(CGB_ERR_STATE, "sliced layout: no shared memory for accumulators");
    if (s->opts.panel_rows > 0) cap = std::min(cap, std::max(32, s->opts.panel_rows & ~31));
    // accumulators: the largest row range, or the interleaved share of the
    // preconditioner's copies; a CTA whose rows exceed them walks its rows
    // in row panels (every column block once per panel)
    int rows_a = 0;
    for (int c = 0; c < grid; c++) rows_a = std::max(rows_a, split[c + 1] - split[c]);
    const int rows_f = interleaved_rows(s->n, 0, grid);
    const int pa = std::max(1, (rows_a + cap - 1) / cap), pf = std::max(1, (rows_f + cap - 1) / cap);
    const int max_rows = std::max((rows_a + pa - 1) / pa, (rows_f + pf - 1) / pf);
    s->sliced_max_rows = (max_rows + 31) & ~31;
    s->sliced_nacc = sliced_smem_bytes(s->sliced_max_rows, kMaxSlots) <= room ? kMaxSlots : 2;
    s->prec_panels = pf;
    s->sa.panels = pa;
    std::vector<int> chunk_slice;
    const int total = chunk_table(grid, pa, s->nblk, [&](int c) { return split[c + 1] - split[c]; },
                                  chunk_slice);
    if (dev_reserve(&s->d_chunk_slice, &s->cap_chunk, chunk_slice.size()))
        return set_error(CGB_ERR_NOMEM, "sliced layout: metadata allocation failed");
    CUDA_TRY(cudaMemcpyAsync(s->d_split, split.data(), sizeof(int) * (grid + 1), cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_chunk_slice, chunk_slice.data(), sizeof(int) * chunk_slice.size(),
                             cudaMemcpyHostToDevice, s->stream));
    s->sa.chunk_slice = nullptr;  // the session's table
    const int st = [&] {
        SliceSet &t = s->sa;
        t.chunk_slice = s->d_chunk_slice;
        const int r = fill_set<double>(s, grid, false, s->d_seg, s->d_colidx, s->d_a, total, true,
                                       s->opts.keep_fp32_copy != 0, false, &t);
        t.chunk_slice = nullptr;
        return r;
    }();
    if (st) return st;
    s->sliced_grid = grid;
    s->layout_gen++;
    return CGB_OK;
}

// Sliced copies of F and F^T (BF16 values) with interleaved row ownership, built on
// first use by the preconditioned solver after each change of F or of A's
// layout.  F^T rows ascend by construction; F rows are sorted by the setter.
int ensure_prec_slices(cgb_session *s)
{
    if (s->plan.kind != kKindSliced || !s->has_prec) return CGB_OK;
    if (s->prec_gen == s->layout_gen) return CGB_OK;
    free_prec_slices(s);
    const int n = s->n, grid = s->sliced_grid;
    // wider column blocks than A's: F and F^T hold half of A's entries a
    // row, so fewer, fuller blocks keep the per-block latency down
    const int bcols = kFactorBlockCols, blocks = (n + bcols - 1) / bcols;
    std::vector<int> chunk_slice;
    const int panels = s->prec_panels;
    const int total = chunk_table(grid, panels, blocks, [&](int c) { return interleaved_rows(n, c, grid); },
                                  chunk_slice);
    const size_t count = size_t(blocks + 1) * s->seg_stride;
    int *seg = nullptr;
    if (dev_alloc(&seg, count) != cudaSuccess)
        return set_error(CGB_ERR_NOMEM, "factor segment table allocation failed");
    int st = CGB_OK;
    const int *ptrs[2] = {s->d_f_ptr, s->d_ft_ptr};
    const int *cols[2] = {s->d_f_col, s->d_ft_col};
    const float *vals[2] = {s->d_f_val, s->d_ft_val};
    SliceSet *sets[2] = {&s->sf, &s->sft};
    for (int m = 0; m < 2 && st == CGB_OK; m++) {
        sets[m]->block_cols = bcols;
        sets[m]->blocks = blocks;
        sets[m]->panels = panels;
        cudaError_t e = dev_alloc(&sets[m]->chunk_slice, chunk_slice.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sets[m]->chunk_slice, chunk_slice.data(), sizeof(int) * chunk_slice.size(),
                                cudaMemcpyHostToDevice, s->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->stream);
        if (e == cudaSuccess) {
            build_segments<<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(
                ptrs[m], cols[m], n, blocks, bcols, seg, s->seg_stride, s->d_flag);
            e = cudaGetLastError();
        }
        int unsorted = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&unsorted, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = set_error(CGB_ERR_CUDA, "factor slices: %s", cudaGetErrorString(e));
        else if (unsorted) st = set_error(CGB_ERR_STATE, "factor rows not in ascending column order");
        else st = fill_set<float>(s, grid, true, seg, cols[m], vals[m], total, false, false, true,
                                  sets[m]);
    }
    dev_free(seg);
    if (st) {
        free_prec_slices(s);
        return st;
    }
    s->prec_gen = s->layout_gen;
    drop_graph(s);
    return CGB_OK;
}

// Fills `pl` for (kind, lpr): kernels, occupancy-sized cooperative grid,
// shared memory.  Returns false when the configuration cannot run here.
bool make_plan(cgb_session *s, int kind, int lpr, Plan *pl, int prefetch = 0, int grid_cap = 0)
{
    Plan P;
    P.kind = kind;
    P.lpr = lpr;
    P.prefetch = kind == kKindSliced ? prefetch : 0;
    if (kind == kKindRow) {
        if (!row_kernels(lpr, &P)) return false;
        P.block = s->opts.block_threads ? s->opts.block_threads : 512;
        P.block_mixed = P.block_pcg = P.block;
        P.smem = 0;
        // almost nothing lives in shared memory: give L1 the room
        for (OuterKernel k : {P.fp64, P.mixed, P.pcg})
            if (cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 0)) return false;
        if (cudaFuncSetAttribute(P.spmv, cudaFuncAttributePreferredSharedMemoryCarveout, 0)) return false;
    } else if (kind == kKindSliced) {
        // 32-bit slice offsets: keep the padded copy well below 2^32 entries
        if (!s->sorted || s->d_seg == nullptr || s->n < 2 * kSliceWidth || s->nnz > (1LL << 30))
            return false;
        const int grid = std::min(s->prop.multiProcessorCount, s->n);
        if (s->sliced_grid != grid && build_sliced(s, grid) != CGB_OK) return false;
        // more rows a CTA than the accumulators hold: the row-panel
        // instances (which have no L2-prefetch form)
        const bool pa = s->sa.panels > 1, pp = pa || s->prec_panels > 1;
        if (pa && prefetch) return false;
        P.fp64 = pa ? outer_step_fp64_sliced_pn : prefetch ? outer_step_fp64_sliced_pf : outer_step_fp64_sliced;
        P.mixed = pa ? outer_step_mixed_sliced_pn
                     : prefetch ? outer_step_mixed_sliced_pf : outer_step_mixed_sliced;
        P.pcg = pp ? outer_step_pcg_sliced_pn : outer_step_pcg_sliced;
        P.spmv = pa ? spmv_dot_sliced_pn : prefetch ? spmv_dot_sliced_pf : spmv_dot_sliced;
        P.spmv32 = pa ? spmv_dot_sliced32_pn : prefetch ? spmv_dot_sliced32_pf : spmv_dot_sliced32;
        P.block = kSlicedBlock;
        P.block_mixed = kSlicedMixedBlock;
        P.block_pcg = kSlicedPcgBlock;
        P.smem = sliced_smem_bytes(s->sliced_max_rows, s->sliced_nacc);
        for (OuterKernel k : {P.fp64, P.mixed, P.pcg})
            if (raise_smem_limit(reinterpret_cast<const void *>(k), P.smem)) return false;
        for (SpmvKernel k : {P.spmv, P.spmv32})
            if (raise_smem_limit(reinterpret_cast<const void *>(k), P.smem)) return false;
    } else {
        return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, P.fp64, P.block, P.smem) != cudaSuccess ||
        per_sm < 1)
        return false;
    const std::pair<OuterKernel, int> others[2] = {{P.mixed, P.block_mixed}, {P.pcg, P.block_pcg}};
    for (const auto &kb : others) {
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kb.first, kb.second, P.smem) !=
                cudaSuccess ||
            per < 1)
            return false;
        per_sm = std::min(per_sm, per);
    }
    per_sm = std::min(per_sm, kind == kKindSliced ? 1 : 4);
    P.grid = std::max(1, std::min(per_sm * s->prop.multiProcessorCount, s->n));
    if (grid_cap > 0) P.grid = std::min(P.grid, grid_cap);
    if (P.grid > s->gpad) return false;
    *pl = P;
    return true;
}

// Makes `pl` the session's plan: uploads its row split.
int apply_plan(cgb_session *s, const Plan &pl)
{
    std::vector<int> split;
    make_split(s->n, s->h_rowstr_copy.data(), pl.grid, split);
    CUDA_TRY(cudaMemcpyAsync(s->d_split, split.data(), sizeof(int) * (pl.grid + 1),
                             cudaMemcpyHostToDevice, s->stream));
    // the barrier's arrival count must be a multiple of the new grid size
    CUDA_TRY(cudaMemsetAsync(s->d_sync, 0, sizeof(unsigned long long), s->stream));
    s->plan = pl;
    drop_graph(s);
    return CGB_OK;
}

SpmvArgs spmv_args(cgb_session *s, int fp32)
{
    SpmvArgs S{};
    S.A = outer_args(s);
    S.ticket = s->ticket();
    S.dot = s->d_dot;
    S.fp32 = fp32;
    return S;
}

// Mean device ms of `reps` standalone SpMV launches under the current plan.
int time_plan_spmv(cgb_session *s, int reps, int fp32, double *ms_out)
{
    if (fp32 && !s->d_a32) return set_error(CGB_ERR_STATE, "no FP32 copy (keep_fp32_copy = 0)");
    SpmvArgs S = spmv_args(s, fp32);
    set_keep(s, &S.A.M, fp32);
    if (S.A.M.keep64 > 0.f || S.A.M.keep32 > 0.f) s->l2_marked = true;
    const Plan &P = s->plan;
    fill_ones<<<s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->p(), s->n + 1);
    if (fp32) {
        to_fp32<<<s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->p(), s->d_p32, s->n + 1);
    }
    const SpmvKernel k = fp32 ? P.spmv32 : P.spmv;
    for (int i = 0; i < 2; i++) k<<<P.grid, P.block, P.smem, s->stream>>>(S);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
    for (int i = 0; i < reps; i++) k<<<P.grid, P.block, P.smem, s->stream>>>(S);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_out = double(ms) / reps;
    int st = 0;
    CUDA_TRY(cudaMemcpy(&st, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != kDevOk) {
        CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
        return set_error(CGB_ERR_TIMEOUT, "SpMV wait failed (status %d)", st);
    }
    return CGB_OK;
}

int ensure_trace(cgb_session *s, int niter);

// Device ms of one FP64 outer step (25 CG iterations and the residual
// product, from x = 1) under the current plan: one warm-up step, then the
// mean of two.  The iterates' values do not matter here; a non-finite
// status (a matrix the power iteration cannot use) is cleared, a timed-out
// wait is an error.
int time_plan_outer(cgb_session *s, double *ms_out)
{
    constexpr int kSteps = 3;
    int st = ensure_trace(s, kSteps);
    if (st) return st;
    // each candidate starts from neutral L2 priorities: lines the previous
    // one kept at evict_last would otherwise flatter its timing
    if (s->plan.kind == kKindSliced) demote_matrix_lines(s);
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    fill_ones<<<s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->x(), s->n + 1);
    OuterArgs A = outer_args(s);
    A.shift = 0.0;
    A.cgitmax = 25;
    A.fixed = 1;
    A.finish = 1;
    for (int it = 0; it < kSteps; it++) {
        if (it == 1) CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
        A.step = it;
        CUDA_TRY(launch_outer(s, s->plan.fp64, A));
    }
    CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_out = double(ms) / (kSteps - 1);
    int dst = 0;
    CUDA_TRY(cudaMemcpy(&dst, s->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (dst == kDevOk) return CGB_OK;
    CUDA_TRY(cudaMemsetAsync(s->d_sync, 0, sizeof(unsigned) * 96, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    if (dst == kDevNonFinite) return CGB_OK;
    return set_error(dst == kDevTimeout ? CGB_ERR_TIMEOUT : CGB_ERR_CUDA,
                     "outer step failed while timing the plan (device status %d)", dst);
}

// Below this order the autotuner also tries the row plan on 16, 32 and 64
// CTAs.
constexpr int kSmallGridRows = 40000;

// Picks the plan: the one the options force, else the candidate with the
// fastest FP64 outer step (the session's autotuner; the outer step, not a
// standalone product, because the candidates' order can differ between the
// two by a few per cent).
int choose_plan(cgb_session *s)
{
    const cgb_options &o = s->opts;
    const double mean = double(s->nnz) / double(s->n);
    std::vector<Plan> cands;
    auto add = [&](int kind, int lpr, int prefetch) {
        Plan p;
        if (make_plan(s, kind, lpr, &p, prefetch)) cands.push_back(p);
    };
    const int want = o.spmv_kernel;
    if (want == 0 || want == kKindRow) {
        if (o.lanes_per_row > 0) add(kKindRow, o.lanes_per_row, 0);
        else {
            const int l = lanes_for_mean(mean);
            add(kKindRow, l, 0);
            if (want == 0 && l > 2) add(kKindRow, l / 2, 0);
            // a small matrix on every SM is mostly grid barriers (class S:
            // 1400 rows, about 5 a CTA on 296 CTAs): also a few CTAs, each
            // with many rows, whose barriers cost less than the parallelism
            // they give up
            if (want == 0 && s->n < kSmallGridRows)
                for (int cap : {16, 32, 64}) {
                    Plan p;
                    if (make_plan(s, kKindRow, l, &p, 0, cap) && p.grid == cap) cands.push_back(p);
                }
        }
    }
    if (want == 0 || want == kKindSliced || want == kKindSlicedPrefetch) {
        // the sliced plan with and without the L2 prefetch of each warp's
        // next-block slices (latency-bound short chunks gain, streaming ones lose)
        // each instance with the matrix stream kept in L2 for the budgets
        // below (the fraction of lines at evict_last is budget / stream)
        for (int pf = 0; pf < 2; pf++) {
            if ((pf == 1 && want == kKindSliced) || (pf == 0 && want == kKindSlicedPrefetch)) continue;
            for (double keep : {0.0, 48e6, 64e6}) {
                const size_t before = cands.size();
                add(kKindSliced, 0, pf);
                if (cands.size() > before) cands.back().l2_keep = keep;
            }
        }
    }
    if (cands.empty()) return set_error(CGB_ERR_INVALID, "no kernel configuration fits these options");
    if (cands.size() == 1) return apply_plan(s, cands[0]);
    // alternating rounds, best time per candidate: the prefetch pair differs
    // by a few per cent, about what the clock drifts over one round
    std::vector<double> best(cands.size(), 1e30);
    for (int round = 0; round < 3; round++) {
        const double lead = *std::min_element(best.begin(), best.end());
        for (size_t i = 0; i < cands.size(); i++) {
            if (best[i] > 1.1 * lead) continue;  // clearly behind after the first round
            int st = apply_plan(s, cands[i]);
            if (st) return st;
            double ms = 0.0;
            st = time_plan_outer(s, &ms);
            if (st) return st;
            best[i] = std::min(best[i], ms);
        }
    }
    size_t bi = 0;
    for (size_t i = 1; i < cands.size(); i++)
        if (best[i] < best[bi]) bi = i;
    return apply_plan(s, cands[bi]);
}

// from_staging: the CSR is already on the device in the staging buffers
// (cgb_upload); otherwise it is copied from the host arrays.
int upload_matrix(cgb_session *s, const int *rowstr, const int *colidx, const double *a,
                  bool from_staging = false)
{
    const long long nnz = rowstr[s->n];
    if (nnz > s->nnz_cap) {
        dev_free(s->d_colidx);
        dev_free(s->d_a);
        dev_free(s->d_a32);
        if (dev_alloc(&s->d_colidx, nnz + kPad) != cudaSuccess ||
            dev_alloc(&s->d_a, nnz + kPad) != cudaSuccess ||
            (s->opts.keep_fp32_copy && dev_alloc(&s->d_a32, nnz + kPad) != cudaSuccess))
            return set_error(CGB_ERR_NOMEM, "device allocation of %lld entries failed", nnz);
        s->nnz_cap = nnz;
    }
    s->nnz = nnz;
    const cudaMemcpyKind kind = from_staging ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CUDA_TRY(cudaMemcpyAsync(s->d_rowstr, from_staging ? s->d_rowstr_in : rowstr,
                             sizeof(int) * (s->n + 1), kind, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_colidx, from_staging ? s->d_colidx_in : colidx, sizeof(int) * nnz,
                             kind, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_a, from_staging ? s->d_a_in : a, sizeof(double) * nnz, kind,
                             s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_colidx + nnz, 0, sizeof(int) * kPad, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_a + nnz, 0, sizeof(double) * kPad, s->stream));
    if (s->d_a32) {
        to_fp32<<<4 * s->prop.multiProcessorCount, 256, 0, s->stream>>>(s->d_a, s->d_a32, nnz + kPad);
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->h_rowstr = rowstr;
    s->h_colidx = colidx;
    s->h_a = a;
    // same row pointers as before (e.g. the same matrix uploaded again): the
    // row split and tuned plan still hold; the column tables are rebuilt
    const bool same_rows = s->plan.fp64 != nullptr &&
                           s->h_rowstr_copy.size() == size_t(s->n) + 1 &&
                           std::equal(rowstr, rowstr + s->n + 1, s->h_rowstr_copy.begin());
    s->h_rowstr_copy.assign(rowstr, rowstr + s->n + 1);
    const int kept_kind = s->plan.kind;
    const int kept_grid = s->sliced_grid;
    invalidate_sliced(s);
    s->sorted = false;
    s->nblk = 0;
    if (s->n >= 2 * kSliceWidth) {
        int st = build_segments_table(s);
        if (st) return st;
    }
    if (same_rows && (kept_kind == kKindRow || (s->sorted && build_sliced(s, kept_grid) == CGB_OK))) {
        // the captured graph stays if every launch argument is unchanged
        // (buffers reused in place); cgb_power_iterate compares them
        return CGB_OK;
    }
    s->plan = Plan();
    return choose_plan(s);
}

int ensure_trace(cgb_session *s, int niter)
{
    if (niter <= s->trace_cap) return CGB_OK;
    dev_free(s->d_trace);
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
    CUDA_TRY(cudaMemsetAsync(s->d_sync, 0, sizeof(unsigned) * 96, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    if (st == kDevTimeout)
        return set_error(CGB_ERR_TIMEOUT, "a device wait hit its %lld ns limit",
                         (long long)(s->opts.wait_limit_ns > 0 ? s->opts.wait_limit_ns : kDefaultWaitNs));
    if (st == kDevNonFinite) return set_error(CGB_ERR_NUMERIC, "non-finite zeta or residual");
    return set_error(CGB_ERR_CUDA, "device status %d", st);
}

bool is_mixed(int mode) { return mode == CGB_MODE_MIXED || mode == CGB_MODE_MIXED_LEARNED; }

// Enqueues one power iteration (x = 1, then niter outer-step kernels) on the
// session stream.
// Arguments of every outer-step launch of a power iteration (`step` apart).
OuterArgs power_args(cgb_session *s, const cgb_solve_params &P)
{
    OuterArgs A = outer_args(s);
    A.shift = P.shift;
    A.cgitmax = P.cgitmax;
    A.fixed = (P.mode == CGB_MODE_FP64) ? 1 : 0;
    A.tol = P.tol;
    A.refresh_every = P.refresh_every > 0 ? P.refresh_every : 10;
    A.finish = 1;
    A.recycle = P.mode == CGB_MODE_FP64 ? 0 : P.recycle;
    // the stream that dominates the mode is the one kept in L2 (none in the
    // preconditioned mode: there it measured slower, 63.4 vs 62.0 ms at C)
    if (P.mode == CGB_MODE_MIXED_LEARNED) A.M.keep64 = A.M.keep32 = A.M.keep16 = 0.f;
    else set_keep(s, &A.M, is_mixed(P.mode) ? 1 : 0);
    return A;
}

OuterKernel power_kernel(const cgb_session *s, const cgb_solve_params &P)
{
    return P.mode == CGB_MODE_MIXED_LEARNED ? s->plan.pcg
           : P.mode == CGB_MODE_MIXED       ? s->plan.mixed
                                            : s->plan.fp64;
}

// What a captured power iteration depends on besides its parameters: the
// launch arguments and shapes.  Compared bytewise (built zero-filled), so a
// re-upload that keeps every buffer and the plan keeps the graph.
struct GraphSig {
    OuterArgs A;
    OuterKernel k;
    int grid, block, block_mixed, block_pcg;
    size_t smem;
};

void graph_sig(cgb_session *s, const cgb_solve_params &P, GraphSig *g)
{
    std::memset(g, 0, sizeof(*g));
    const OuterArgs A = power_args(s, P);
    std::memcpy(&g->A, &A, sizeof(A));
    g->k = power_kernel(s, P);
    g->grid = s->plan.grid;
    g->block = s->plan.block;
    g->block_mixed = s->plan.block_mixed;
    g->block_pcg = s->plan.block_pcg;
    g->smem = s->plan.smem;
}

cudaError_t enqueue_power(cgb_session *s, const cgb_solve_params &P)
{
    cudaError_t e = cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream);
    if (e != cudaSuccess) return e;
    fill_ones<<<std::max(1, std::min(s->prop.multiProcessorCount, (s->n + 1 + 255) / 256)), 256, 0,
                s->stream>>>(s->x(), s->n + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    OuterArgs A = power_args(s, P);
    const OuterKernel k = power_kernel(s, P);
    // the sliced preconditioned kernel reads F / F^T slices (ensure_prec_slices)
    if (P.mode == CGB_MODE_MIXED_LEARNED && s->plan.kind == kKindSliced && A.F.srow == nullptr)
        return cudaErrorInvalidValue;
    for (int it = 0; it < P.niter; it++) {
        A.step = it;
        e = launch_outer(s, k, A);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int check_params(cgb_session *s, const cgb_solve_params &P)
{
    if (P.niter < 1) return set_error(CGB_ERR_INVALID, "niter must be >= 1");
    if (P.cgitmax < 0) return set_error(CGB_ERR_INVALID, "cgitmax must be >= 0");
    if (!std::isfinite(P.shift)) return set_error(CGB_ERR_INVALID, "shift must be finite");
    if (P.mode < CGB_MODE_FP64 || P.mode > CGB_MODE_MIXED_LEARNED)
        return set_error(CGB_ERR_INVALID, "unknown mode %d", P.mode);
    if (P.mode == CGB_MODE_MIXED_LEARNED && !s->has_prec)
        return set_error(CGB_ERR_STATE, "preconditioned mode needs cgb_set_preconditioner first");
    if (P.mode != CGB_MODE_FP64 && !(P.tol > 0.0))
        return set_error(CGB_ERR_INVALID, "tolerance modes need tol > 0");
    if (P.recycle < 0 || P.recycle > kMaxRecycle)
        return set_error(CGB_ERR_INVALID, "recycle must be 0..%d", kMaxRecycle);
    if (is_mixed(P.mode) && !s->d_a32)
        return set_error(CGB_ERR_STATE, "mixed mode needs the FP32 copy (keep_fp32_copy = 1)");
    return CGB_OK;
}

// What one more kernel costs a solve's graph beyond its own work: graphs
// of `niter` and of 1 launch of an empty kernel with the FP64 outer step's
// shape (grid, block, dynamic shared memory, cooperative), each timed with
// events around the graph launch; the difference over niter - 1 launches
// is the launch, dispatch and teardown cost of one outer step.  Best of
// five alternating trials (ms per launch).
int time_launch_overhead(cgb_session *s, int niter, double *ms_out)
{
    const Plan &P = s->plan;
    CUDA_TRY(cudaFuncSetAttribute(launch_probe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(P.smem)));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(P.grid);
    cfg.blockDim = dim3(P.block);
    cfg.dynamicSmemBytes = P.smem;
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaGraphExec_t ex[2] = {nullptr, nullptr};
    const int counts[2] = {std::max(niter, 2), 1};
    int st = CGB_OK;
    for (int g = 0; g < 2 && st == CGB_OK; g++) {
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
        for (int i = 0; i < counts[g] && e == cudaSuccess; i++) e = cudaLaunchKernelEx(&cfg, launch_probe, i);
        cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
        if (e == cudaSuccess && e2 == cudaSuccess) e = cudaGraphInstantiate(&ex[g], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess || e2 != cudaSuccess)
            st = set_error(CGB_ERR_CUDA, "launch-overhead graph: %s",
                           cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    double best[2] = {1e30, 1e30};
    for (int trial = 0; trial < 6 && st == CGB_OK; trial++) {
        for (int g = 0; g < 2; g++) {
            float ms = 0.f;
            if (cudaEventRecord(s->ev0, s->stream) != cudaSuccess ||
                cudaGraphLaunch(ex[g], s->stream) != cudaSuccess ||
                cudaEventRecord(s->ev1, s->stream) != cudaSuccess ||
                cudaStreamSynchronize(s->stream) != cudaSuccess ||
                cudaEventElapsedTime(&ms, s->ev0, s->ev1) != cudaSuccess) {
                st = set_error(CGB_ERR_CUDA, "launch-overhead timing failed");
                break;
            }
            if (trial > 0) best[g] = std::min(best[g], double(ms));  // trial 0 warms up
        }
    }
    for (auto &x : ex)
        if (x) cudaGraphExecDestroy(x);
    if (st) return st;
    *ms_out = std::max(0.0, (best[0] - best[1]) / (counts[0] - 1));
    return CGB_OK;
}

bool same_params(const cgb_solve_params &a, const cgb_solve_params &b)
{
    return a.niter == b.niter && a.shift == b.shift && a.mode == b.mode && a.cgitmax == b.cgitmax &&
           a.tol == b.tol && a.refresh_every == b.refresh_every && a.recycle == b.recycle;
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

int cgb_version(void) { return 10000 * 0 + 100 * 2 + 0; }

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
    o->panel_rows = 0;
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
    p->recycle = 4;
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

}  // extern "C"

namespace {

// A session without its matrix: options checked, device buffers allocated.
int create_shell(int n, const cgb_options *opts, cgb_session **out)
{
    int st = CGB_OK;
    cgb_options o;
    cgb_default_options(&o);
    if (opts) o = *opts;
    if (o.lanes_per_row != 0 && o.lanes_per_row != 2 && o.lanes_per_row != 4 &&
        o.lanes_per_row != 8 && o.lanes_per_row != 16 && o.lanes_per_row != 32)
        return set_error(CGB_ERR_INVALID, "lanes_per_row must be 0, 2, 4, 8, 16 or 32");
    if (o.block_threads != 0 && o.block_threads != 256 && o.block_threads != 512)
        return set_error(CGB_ERR_INVALID, "block_threads must be 0, 256 or 512");
    if (o.spmv_kernel < 0 || o.spmv_kernel > 3)
        return set_error(CGB_ERR_INVALID,
                         "spmv_kernel must be 0 (auto), 1 (row), 2 (sliced) or 3 (sliced, L2 prefetch)");
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
    s->vstride = (size_t(n) + 8 + 31) & ~size_t(31);
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
    CREATE_TRY(cudaMemsetAsync(s->d_vec, 0, sizeof(double) * 5 * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_p32, s->vstride));
    CREATE_TRY(cudaMemsetAsync(s->d_p32, 0, sizeof(float) * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_r32, s->vstride));
    CREATE_TRY(cudaMemsetAsync(s->d_r32, 0, sizeof(float) * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_r16, s->vstride));
    CREATE_TRY(cudaMemsetAsync(s->d_r16, 0, 2 * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_t16, s->vstride));
    CREATE_TRY(cudaMemsetAsync(s->d_t16, 0, 2 * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_y, s->vstride));
    CREATE_TRY(cudaMemsetAsync(s->d_y, 0, sizeof(double) * s->vstride, s->stream));
    CREATE_TRY(dev_alloc(&s->d_hx, kMaxRecycle * s->vstride));
    CREATE_TRY(dev_alloc(&s->d_hw, kMaxRecycle * s->vstride));
    CREATE_TRY(dev_alloc(&s->d_part, size_t(kSlotCount) * s->gpad));
    CREATE_TRY(dev_alloc(&s->d_sync, 96));
    CREATE_TRY(cudaMemsetAsync(s->d_sync, 0, sizeof(unsigned) * 96, s->stream));
    CREATE_TRY(dev_alloc(&s->d_status, 1));
    CREATE_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    CREATE_TRY(dev_alloc(&s->d_flag, 1));
    CREATE_TRY(dev_alloc(&s->d_split, size_t(s->gpad) + 1));
    CREATE_TRY(dev_alloc(&s->d_dot, 1));
#undef CREATE_TRY
    st = ensure_trace(s, 128);
    if (st != CGB_OK) {
        release(s);
        return st;
    }
    *out = s;
    return CGB_OK;
}

}  // namespace

extern "C" {

int cgb_create(int n, const int *rowstr, const int *colidx, const double *a,
               const cgb_options *opts, cgb_session **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "out is null");
    *out = nullptr;
    int st = validate_csr(n, rowstr, colidx, a);
    if (st) return st;
    cgb_session *s = nullptr;
    st = create_shell(n, opts, &s);
    if (st) return st;
    st = upload_matrix(s, rowstr, colidx, a);
    if (st != CGB_OK) {
        release(s);
        return st;
    }
    *out = s;
    return CGB_OK;
}

int cgb_create_generated(int n, int nonzer, double rcond, double shift, double seed,
                         const cgb_options *opts, cgb_session **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "out is null");
    *out = nullptr;
    cgb_session *s = nullptr;
    int st = create_shell(n, opts, &s);
    if (st) return st;
    DeviceCsr csr;
    st = makea_on_device(s->device, n, nonzer, rcond, shift, seed, &csr);
    if (st == CGB_OK) {
        // the generated arrays become the staging copy the upload reads
        dev_free(s->d_rowstr_in);
        dev_free(s->d_colidx_in);
        dev_free(s->d_a_in);
        s->d_rowstr_in = csr.rowstr;
        s->d_colidx_in = csr.colidx;
        s->d_a_in = csr.a;
        s->cap_rowstr_in = size_t(n) + 1;
        s->cap_colidx_in = s->cap_a_in = size_t(csr.nnz);
        csr.rowstr = csr.colidx = nullptr;
        csr.a = nullptr;
        st = cudaSetDevice(s->device) == cudaSuccess
                 ? upload_matrix(s, csr.h_rowstr.data(), nullptr, nullptr, true)
                 : set_error(CGB_ERR_CUDA, "cudaSetDevice failed");
        // no host arrays behind this matrix: any host CSR passed later uploads
        s->h_rowstr = nullptr;
        s->h_colidx = nullptr;
        s->h_a = nullptr;
    }
    for (void *p : {(void *)csr.rowstr, (void *)csr.colidx, (void *)csr.a})
        if (p) cudaFree(p);
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
    int st = validate_rowstr(s->n, rowstr, colidx, a);
    if (st) return st;
    CUDA_TRY(cudaSetDevice(s->device));
    // the copy to the staging buffers runs while the host checks the
    // entries; the session's matrix changes only when they are valid
    const size_t n1 = size_t(s->n) + 1, nnz = size_t(rowstr[s->n]);
    if (dev_reserve(&s->d_rowstr_in, &s->cap_rowstr_in, n1) != cudaSuccess ||
        dev_reserve(&s->d_colidx_in, &s->cap_colidx_in, nnz) != cudaSuccess ||
        dev_reserve(&s->d_a_in, &s->cap_a_in, nnz) != cudaSuccess)
        return set_error(CGB_ERR_NOMEM, "staging allocation of %zu entries failed", nnz);
    CUDA_TRY(cudaMemcpyAsync(s->d_rowstr_in, rowstr, sizeof(int) * n1, cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_colidx_in, colidx, sizeof(int) * nnz, cudaMemcpyHostToDevice,
                             s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_a_in, a, sizeof(double) * nnz, cudaMemcpyHostToDevice, s->stream));
    st = validate_entries(s->n, rowstr, colidx, a);
    // the copies read the caller's arrays: done before returning either way
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (st) return st;
    return upload_matrix(s, rowstr, colidx, a, true);
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
    A.step = 0;
    A.finish = 0;
    CUDA_TRY(launch_outer(s, s->plan.fp64, A));
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

int cgb_matrix_changed(cgb_session *s)
{
    if (!s) return set_error(CGB_ERR_INVALID, "session is null");
    // no host array compares equal now: the next cgb_conj_grad uploads
    s->h_rowstr = nullptr;
    s->h_colidx = nullptr;
    s->h_a = nullptr;
    return CGB_OK;
}

int cgb_power_iterate(cgb_session *s, const cgb_solve_params *params, double *zeta_trace,
                      double *rnorm_trace, int *iters_trace, double *x_out,
                      cgb_solve_result *res)
{
    if (!s || !params) return set_error(CGB_ERR_INVALID, "null session or params");
    const cgb_solve_params P = *params;
    int st = check_params(s, P);
    if (st) return st;
    CUDA_TRY(cudaSetDevice(s->device));
    st = ensure_trace(s, P.niter);
    if (st) return st;
    if (P.mode == CGB_MODE_MIXED_LEARNED) {
        st = ensure_prec_slices(s);
        if (st) return st;
    }
    if (s->opts.use_graph) {
        GraphSig sig;
        graph_sig(s, P, &sig);
        const unsigned char *sb = reinterpret_cast<const unsigned char *>(&sig);
        const bool same_sig = s->g_sig.size() == sizeof(sig) &&
                              std::memcmp(s->g_sig.data(), sb, sizeof(sig)) == 0;
        if (!(s->g_valid && same_params(s->g_params, P) && same_sig)) {
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
            s->g_params = P;
            s->g_sig.assign(sb, sb + sizeof(sig));
            s->g_valid = true;
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
    int total_inner = 0, refreshes = 0, fallbacks = 0;
    for (int i = 0; i < P.niter; i++) {
        if (P.mode == CGB_MODE_MIXED_LEARNED) fallbacks += int(tr[i].spare[0]);
        if (zeta_trace) zeta_trace[i] = tr[i].zeta;
        if (rnorm_trace) rnorm_trace[i] = tr[i].rnorm;
        if (iters_trace) iters_trace[i] = int(tr[i].inner);
        total_inner += int(tr[i].inner);
        refreshes += int(tr[i].refresh);
    }
    if (x_out) CUDA_TRY(cudaMemcpy(x_out, s->x(), sizeof(double) * s->n, cudaMemcpyDeviceToHost));
    if (res) {
        res->zeta = tr[P.niter - 1].zeta;
        res->rnorm = tr[P.niter - 1].rnorm;
        res->device_ms = ms;
        res->total_inner = total_inner;
        res->fallbacks = fallbacks;
        res->refreshes = refreshes;
    }
    return CGB_OK;
}

int cgb_set_preconditioner(cgb_session *s, const int *fptr, const int *fcol, const double *fval)
{
    if (!s || !fptr || !fcol || !fval) return set_error(CGB_ERR_INVALID, "null argument");
    const int n = s->n;
    if (fptr[0] != 0) return set_error(CGB_ERR_BAD_MATRIX, "factor: fptr[0] != 0");
    for (int i = 0; i < n; i++) {
        if (fptr[i + 1] < fptr[i]) return set_error(CGB_ERR_BAD_MATRIX, "factor: fptr decreases at %d", i);
        bool diag = false;
        for (int k = fptr[i]; k < fptr[i + 1]; k++) {
            if (fcol[k] < 0 || fcol[k] > i)
                return set_error(CGB_ERR_BAD_MATRIX, "factor: entry (%d, %d) not in the lower triangle", i, fcol[k]);
            if (!std::isfinite(fval[k])) return set_error(CGB_ERR_NUMERIC, "factor: non-finite value in row %d", i);
            if (fcol[k] == i) {
                if (!(fval[k] > 0.0))
                    return set_error(CGB_ERR_NUMERIC, "factor: diagonal of row %d not positive", i);
                diag = true;
            }
        }
        if (!diag) return set_error(CGB_ERR_BAD_MATRIX, "factor: row %d has no diagonal", i);
    }
    // F with each row in ascending column order, repeated columns summed
    // (the sliced products need ascending rows); values rounded to FP32
    std::vector<int> optr(n + 1, 0), ocol;
    std::vector<float> val32;
    ocol.reserve(size_t(fptr[n]));
    val32.reserve(size_t(fptr[n]));
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < n; i++) {
        bool ascending = true;  // the common case (the learned factor's rows): no sort
        for (int k = fptr[i] + 1; k < fptr[i + 1]; k++) ascending &= fcol[k] > fcol[k - 1];
        if (ascending) {
            for (int k = fptr[i]; k < fptr[i + 1]; k++) {
                ocol.push_back(fcol[k]);
                val32.push_back(float(fval[k]));
            }
            optr[i + 1] = int(ocol.size());
            continue;
        }
        row.clear();
        for (int k = fptr[i]; k < fptr[i + 1]; k++) row.emplace_back(fcol[k], fval[k]);
        std::stable_sort(row.begin(), row.end(),
                         [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                             return a.first < b.first;
                         });
        for (size_t k = 0; k < row.size(); k++) {
            if (k > 0 && row[k].first == row[k - 1].first) {
                row[k].second += row[k - 1].second;
                ocol.pop_back();
                val32.pop_back();
            }
            ocol.push_back(row[k].first);
            val32.push_back(float(row[k].second));
        }
        optr[i + 1] = int(ocol.size());
    }
    const long long nf = optr[n];
    s->prec_nnz = nf;
    // transpose (rows of F^T = columns of F), rows in ascending order
    std::vector<int> tptr(n + 1, 0), tcol(nf);
    std::vector<float> tval(nf);
    for (long long k = 0; k < nf; k++) tptr[ocol[k] + 1]++;
    for (int i = 0; i < n; i++) tptr[i + 1] += tptr[i];
    std::vector<int> cur(tptr.begin(), tptr.end() - 1);
    for (int i = 0; i < n; i++)
        for (int k = optr[i]; k < optr[i + 1]; k++) {
            const int at = cur[ocol[k]]++;
            tcol[at] = i;
            tval[at] = val32[k];
        }
    CUDA_TRY(cudaSetDevice(s->device));
    free_prec_slices(s);
    dev_free(s->d_f_ptr); dev_free(s->d_f_col); dev_free(s->d_f_val);
    dev_free(s->d_ft_ptr); dev_free(s->d_ft_col); dev_free(s->d_ft_val);
    s->has_prec = false;
    if (dev_alloc(&s->d_f_ptr, size_t(n) + 1) || dev_alloc(&s->d_f_col, size_t(nf) + kPad) ||
        dev_alloc(&s->d_f_val, size_t(nf) + kPad) || dev_alloc(&s->d_ft_ptr, size_t(n) + 1) ||
        dev_alloc(&s->d_ft_col, size_t(nf) + kPad) || dev_alloc(&s->d_ft_val, size_t(nf) + kPad))
        return set_error(CGB_ERR_NOMEM, "factor allocation failed");
    CUDA_TRY(cudaMemsetAsync(s->d_f_col, 0, sizeof(int) * (nf + kPad), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_f_val, 0, sizeof(float) * (nf + kPad), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_ft_col, 0, sizeof(int) * (nf + kPad), s->stream));
    CUDA_TRY(cudaMemsetAsync(s->d_ft_val, 0, sizeof(float) * (nf + kPad), s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_f_ptr, optr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_f_col, ocol.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_f_val, val32.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_ft_ptr, tptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_ft_col, tcol.data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->d_ft_val, tval.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, s->stream));
    s->has_prec = true;
    drop_graph(s);
    return CGB_OK;
}

int cgb_time_spmv(cgb_session *s, int reps, int fp32, double *ms_per_launch)
{
    if (!s || reps < 1 || !ms_per_launch) return set_error(CGB_ERR_INVALID, "bad arguments");
    CUDA_TRY(cudaSetDevice(s->device));
    return time_plan_spmv(s, reps, fp32 ? 1 : 0, ms_per_launch);
}

int cgb_plan_info(cgb_session *s, int *kind, int *lanes_per_row, int *grid, int *block,
                  long long *smem_bytes, long long *layout_entries)
{
    if (!s) return set_error(CGB_ERR_INVALID, "session is null");
    if (kind) *kind = s->plan.kind == kKindSliced && s->plan.prefetch ? kKindSlicedPrefetch : s->plan.kind;
    if (lanes_per_row) *lanes_per_row = s->plan.lpr;
    if (grid) *grid = s->plan.grid;
    if (block) *block = s->plan.block;
    if (smem_bytes) *smem_bytes = (long long)s->plan.smem;
    if (layout_entries) *layout_entries = s->plan.kind == kKindSliced ? s->sa.entries : s->nnz;
    return CGB_OK;
}

int cgb_check_status(int *word)
{
    if (!word) return set_error(CGB_ERR_INVALID, "word is null");
#ifdef CGB_CHECKED
    int zero = 0;
    CUDA_TRY(cudaMemcpyFromSymbol(word, g_check_word, sizeof(int)));
    CUDA_TRY(cudaMemcpyToSymbol(g_check_word, &zero, sizeof(int)));
#else
    *word = -1;
#endif
    return CGB_OK;
}

int cgb_plan_l2_keep(cgb_session *s, double *bytes)
{
    if (!s || !bytes) return set_error(CGB_ERR_INVALID, "bad arguments");
    *bytes = s->plan.kind == kKindSliced ? s->plan.l2_keep : 0.0;
    return CGB_OK;
}

int cgb_plan_panels(cgb_session *s, int *panels, int *prec_panels)
{
    if (!s || !panels || !prec_panels) return set_error(CGB_ERR_INVALID, "bad arguments");
    const bool sliced = s->plan.kind == kKindSliced;
    *panels = sliced ? s->sa.panels : 0;
    *prec_panels = sliced ? s->prec_panels : 0;
    return CGB_OK;
}

int cgb_set_l2_keep(cgb_session *s, double bytes)
{
    if (!s || !(bytes >= 0.0) || bytes > 1e12) return set_error(CGB_ERR_INVALID, "bytes must be in [0, 1e12]");
    s->plan.l2_keep = bytes;
    drop_graph(s);
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
        CUDA_TRY(launch_outer(s, s->plan.fp64, A));
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
    st = time_launch_overhead(s, niter, graph_gap_ms);
    return st;
}

int cgb_time_barrier(cgb_session *s, int iters, double *us_per_barrier)
{
    if (!s || iters < 1 || iters > 10000000 || !us_per_barrier)
        return set_error(CGB_ERR_INVALID, "bad arguments");
    CUDA_TRY(cudaSetDevice(s->device));
    GridBarrier gb;
    gb.arrivals = s->arrivals();
    gb.status = s->d_status;
    gb.limit_ns = s->opts.wait_limit_ns > 0 ? s->opts.wait_limit_ns : kDefaultWaitNs;
    CUDA_TRY(cudaMemsetAsync(s->d_status, 0, sizeof(int), s->stream));
    // the plan's grid (its count stays a multiple of it) with the FP64
    // outer step's block size
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(s->plan.grid);
    cfg.blockDim = dim3(s->plan.block);
    cfg.stream = s->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, barrier_loop, gb, 16));  // warm-up
    CUDA_TRY(cudaEventRecord(s->ev0, s->stream));
    CUDA_TRY(cudaLaunchKernelEx(&cfg, barrier_loop, gb, iters));
    CUDA_TRY(cudaEventRecord(s->ev1, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *us_per_barrier = 1e3 * double(ms) / iters;
    return collect_status(s);
}

int cgb_selftest_wait_timeout(cgb_session *s, long long limit_ns, int *device_status)
{
    if (!s || !device_status || limit_ns <= 0 || limit_ns > 10000000000LL)
        return set_error(CGB_ERR_INVALID, "limit_ns must be in (0, 1e10]");
    CUDA_TRY(cudaSetDevice(s->device));
    GridBarrier gb;
    gb.arrivals = s->arrivals();
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

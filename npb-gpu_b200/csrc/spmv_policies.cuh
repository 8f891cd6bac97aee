// spmv_policies.cuh -- the two SpMV policies of the persistent CG kernels.
//
// Both compute out[j] = (A v)[j] for the rows [row0, row1) the CTA owns and
// return this thread's share of dotv . out (FP64).  They are generic in the
// value type VT: double for the FP64 solver (the reference's precision,
// cg.cu:691-697), float for the FP32 SpMV of the mixed-precision solver
// (matrix values and gathered vector in FP32, FP32 accumulation per row).
//
//   RowSpmv<LPR>   CSR as the reference stores it; LPR lanes per row, each
//                  lane two consecutive entries per chunk (one 16/8-byte load
//                  of values, one 8-byte load of indices, from an even start,
//                  masked to the row; single loads for a last entry that
//                  ends the arrays), four chunks in flight; the gathered
//                  vector is read through L1/L2.
//   SlicedSpmv     a sliced copy of the matrix built on the device (built by
//                  cg_kernels.cuh): per CTA and per column block of W columns,
//                  the CTA's rows sorted by length and packed 32 to a slice,
//                  stored column-major by step pairs (entry k of the slice's
//                  lane i at offset + 64 (k/2) + 2 i + k%2, widths rounded up
//                  to even) with 16-bit local columns, so a lane reads two
//                  steps per load: one 16/8-byte value pair and one 4-byte
//                  column pair.  The block
//                  of v is staged in shared memory by TMA bulk copies
//                  (cp.async.bulk + mbarrier) into a 2-slot ring; warps walk
//                  the blocks independently and the last warp done with a
//                  block refills its slot with block b+2, so no CTA-wide
//                  barrier sits between blocks.  Gathers are shared-memory
//                  loads; each row accumulates in registers, then into one of
//                  two shared accumulators (by block parity: blocks b and b+1
//                  may run at once, b+2 only after all of b), summed at the
//                  end -- deterministic.  The preconditioner's factor copies
//                  gather a BF16 vector (FP32 row sums), so a staged block
//                  spans twice the columns.
#pragma once

#include <cuda_bf16.h>

#include "device_common.cuh"

namespace cgb {

template <typename VT>
struct Pair;
template <>
struct Pair<double> {
    using T = double2;
};
template <>
struct Pair<float> {
    using T = float2;
};
template <>
struct Pair<__nv_bfloat16> {
    using T = __nv_bfloat162;
};

// Stored value -> arithmetic type (BF16 values widen exactly to FP32).
__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }

// L2 policy of a matrix stream: a `keep` fraction of its lines (chosen by
// the hardware from their addresses, so the same lines every product) at
// priority evict_last, the others evict_first.
__device__ __forceinline__ uint64_t l2_stream_policy(float keep)
{
    uint64_t pol;
    if (keep > 0.f)
        asm("createpolicy.fractional.L2::evict_last.L2::evict_first.b64 %0, %1;"
            : "=l"(pol)
            : "f"(fminf(keep, 1.f)));
    else
        asm("createpolicy.fractional.L2::evict_first.b64 %0, %1;" : "=l"(pol) : "f"(1.f));
    return pol;
}

// Read-only loads of the matrix stream under an L2 policy (not kept in L1).
__device__ __forceinline__ double2 ld_stream(const double2 *p, uint64_t pol)
{
    double2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
        : "=d"(v.x), "=d"(v.y)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float2 ld_stream(const float2 *p, uint64_t pol)
{
    float2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
        : "=f"(v.x), "=f"(v.y)
        : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ unsigned ld_stream_u32(const void *p, uint64_t pol)
{
    unsigned v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ __nv_bfloat162 ld_stream(const __nv_bfloat162 *p, uint64_t pol)
{
    const unsigned u = ld_stream_u32(p, pol);
    __nv_bfloat162 v;
    v.x = __ushort_as_bfloat16(static_cast<unsigned short>(u & 0xffffu));
    v.y = __ushort_as_bfloat16(static_cast<unsigned short>(u >> 16));
    return v;
}

__device__ __forceinline__ ushort2 ld_stream(const ushort2 *p, uint64_t pol)
{
    const unsigned u = ld_stream_u32(p, pol);
    return make_ushort2(static_cast<unsigned short>(u & 0xffffu), static_cast<unsigned short>(u >> 16));
}

__device__ __forceinline__ double fma_vt(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fma_vt(float a, float b, float c) { return fmaf(a, b, c); }

// Row-sum type of a gathered vector type: FP64 and FP32 sum in their own
// precision, a BF16 vector (the factor products) in FP32.
template <typename VT>
struct SumType {
    using T = VT;
};
template <>
struct SumType<__nv_bfloat16> {
    using T = float;
};

template <int W, typename VT>
__device__ __forceinline__ VT group_sum_vt(VT v, unsigned mask)
{
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
    return v;
}

// Device arrays of one sliced copy (host-side bookkeeping; any pointer may
// be null when that precision is not kept).
struct SliceSet {
    unsigned short *srow = nullptr;   // local row per (slice, lane)
    int *width = nullptr;             // steps per slice (even)
    unsigned *off = nullptr;          // first entry per slice, + total
    double *sval = nullptr;           // FP64 values
    float *sval32 = nullptr;          // FP32 values
    __nv_bfloat16 *sval16 = nullptr;  // BF16 values
    unsigned short *scol = nullptr;   // local columns
    int *chunk_slice = nullptr;       // own chunk table (null: the session's)
    int interleaved = 0;              // rows owned round-robin by the CTAs
    int panels = 1;                   // pieces a CTA's rows are walked in
    int block_cols = 0, blocks = 0;   // columns per block, blocks (0: the session's)
    long long entries = 0;            // padded entries
    // allocated capacities (elements): a rebuild reuses buffers that fit
    size_t cap_srow = 0, cap_width = 0, cap_off = 0, cap_sval = 0, cap_sval32 = 0,
           cap_sval16 = 0, cap_scol = 0;
};

// Matrix in both layouts, both precisions (unused members may be null).
struct MatrixView {
    const int *__restrict__ rowstr;
    const int *__restrict__ colidx;
    const double *__restrict__ a;      // FP64 values (CSR order)
    const float *__restrict__ a32;     // FP32 values (CSR order), mixed mode
    // sliced layout
    const double *__restrict__ sval;   // FP64 values, slice order
    const float *__restrict__ sval32;  // FP32 values, slice order
    const __nv_bfloat16 *__restrict__ sval16;  // BF16 values, slice order (factor copies)
    const unsigned short *__restrict__ scol;  // column - b*W
    const unsigned short *__restrict__ srow;  // local row per (slice, lane); 0xffff = none
    const unsigned *__restrict__ slice_off;   // first entry of each slice
    const int *__restrict__ slice_width;      // steps of each slice
    const int *__restrict__ chunk_slice;      // ((c*panels + k)*nblk + b) -> first slice
    int nblk;                                 // column blocks
    int width;                                // columns per block
    int max_rows;                             // shared accumulator capacity
    int interleaved;                          // 0: CTA c owns its contiguous row range;
                                              // 1: CTA c owns rows c, c + G, c + 2G, ...
    int nacc;                                 // accumulators in shared memory (2 or 4)
    int panels;                               // a CTA's rows are walked in this many
                                              // consecutive pieces (row panels), each
                                              // over every column block: 1 unless the
                                              // rows exceed the accumulators
    // bounds of the checked build: CSR entries and sliced entries (each with
    // the padding after them), columns of the gathered vector
    long long csr_entries, slice_entries;
    int ncols;
    // sliced walk: fraction of the stream's 128-byte lines (FP64, FP32, BF16
    // values with their columns) loaded with L2 priority evict_last -- kept
    // in L2 from one product to the next -- the rest evict_first; 0 = all
    // evict_first (a pure stream)
    float keep64, keep32, keep16;
};

// Rows of CTA `c` of `grid` under interleaved ownership.
__host__ __device__ inline int interleaved_rows(int n, int c, int grid)
{
    return c < n ? (n - c + grid - 1) / grid : 0;
}

// First of a CTA's `rows` rows (local index) in row panel k of `panels`.
__host__ __device__ inline int panel_begin(int rows, int k, int panels)
{
    return int((long long)rows * k / panels);
}

template <typename VT>
__device__ __forceinline__ const VT *csr_values(const MatrixView &M);
template <>
__device__ __forceinline__ const double *csr_values<double>(const MatrixView &M) { return M.a; }
template <>
__device__ __forceinline__ const float *csr_values<float>(const MatrixView &M) { return M.a32; }
template <typename VT>
__device__ __forceinline__ const VT *slice_values(const MatrixView &M);
template <>
__device__ __forceinline__ const double *slice_values<double>(const MatrixView &M) { return M.sval; }
template <>
__device__ __forceinline__ const float *slice_values<float>(const MatrixView &M) { return M.sval32; }
template <>
__device__ __forceinline__ const __nv_bfloat16 *slice_values<__nv_bfloat16>(const MatrixView &M)
{
    return M.sval16;
}

// ------------------------------------------------------------ row policy
template <int LPR, typename VT>
__device__ __forceinline__ double spmv_rows(const MatrixView &M, const VT *v, double *out, int row0,
                                            int row1, const double *dotv)
{
    using P2 = typename Pair<VT>::T;
    constexpr int kStep = 2 * LPR;
    constexpr int kUnroll = 4;
    const VT *__restrict__ a = csr_values<VT>(M);
    const int lane = threadIdx.x % LPR;
    const int grp = threadIdx.x / LPR;
    const int ngrp = blockDim.x / LPR;
    const unsigned mask =
        LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << ((threadIdx.x & 31) & ~(LPR - 1)));
    double dacc = 0.0;
    for (int row = row0 + grp; row < row1; row += ngrp) {
        const int k0 = __ldg(M.rowstr + row);
        const int k1 = __ldg(M.rowstr + row + 1);
        VT s = VT(0);
        for (int k = (k0 & ~1) + 2 * lane; k < k1; k += kUnroll * kStep) {
            P2 av[kUnroll];
            int2 cv[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    if (kk + 1 < M.csr_entries) {
                        av[u] = __ldcs(reinterpret_cast<const P2 *>(a + kk));
                        cv[u] = __ldcs(reinterpret_cast<const int2 *>(M.colidx + kk));
                    } else if (CGB_IN_RANGE(kk, M.csr_entries, kCheckStream)) {
                        // the last entry of an unpadded CSR (the caller's
                        // arrays of cgb_conj_grad_noalloc): no pair load
                        // past its end
                        av[u].x = __ldcs(a + kk);
                        av[u].y = VT(0);
                        cv[u] = make_int2(__ldcs(M.colidx + kk), 0);
                    } else {
                        av[u].x = av[u].y = VT(0);
                        cv[u] = make_int2(0, 0);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kUnroll; u++) {
                const int kk = k + u * kStep;
                if (kk < k1) {
                    if (kk >= k0 && CGB_IN_RANGE(cv[u].x, M.ncols, kCheckGather))
                        s = fma_vt(av[u].x, v[cv[u].x], s);
                    if (kk + 1 < k1 && CGB_IN_RANGE(cv[u].y, M.ncols, kCheckGather))
                        s = fma_vt(av[u].y, v[cv[u].y], s);
                }
            }
        }
        s = group_sum_vt<LPR>(s, mask);
        if (lane == 0) {
            const double t = double(s);
            out[row] = t;
            if (dotv) dacc = fma(dotv[row], t, dacc);
        }
    }
    return dacc;
}

template <int LPR>
struct RowSpmv {
    static constexpr bool kSliced = false;
    int row0, row1;
    __device__ void setup(const MatrixView &, int r0, int r1)
    {
        row0 = r0;
        row1 = r1;
    }
    template <typename VT>
    __device__ __forceinline__ double apply(const MatrixView &M, const VT *v, double *out,
                                            const double *dotv, int, long long, int *, bool &ok)
    {
        ok = true;
        return spmv_rows<LPR, VT>(M, v, out, row0, row1, dotv);
    }
};

// ---------------------------------------------------------- sliced policy

// Staging and dynamic shared memory of the sliced policy: 192 KB of vector
// staging (2 slots of 12288 doubles, or up to 4 slots of 12288 floats) and
// one accumulator of max_rows doubles per slot in use.
constexpr int kSliceWidth = 12288;  // columns per block
constexpr int kFactorBlockCols = 49152;  // columns per block of the preconditioner's copies
                                         // (a BF16 vector: 96 KB a block)
constexpr size_t kStagingBytes = 2 * size_t(12288) * 8;
constexpr int kMaxSlots = 4;
__host__ __device__ inline size_t sliced_smem_bytes(int max_rows, int nacc)
{
    return 128 + kStagingBytes + size_t(nacc) * size_t(max_rows) * sizeof(double);
}

// L2 prefetch of one slice (all lanes' entries: per step pair 64 values and
// 64 columns, contiguous), spread over the warp's lanes; prefetches do not
// wait, so a warp pulls its next block's slices toward L2 while it works.
template <typename ST>
__device__ __forceinline__ void prefetch_slice_l2(const ST *vals, const unsigned short *scol,
                                                  unsigned base, int wp, int lane)
{
    constexpr int kVLines = int((64 * sizeof(ST) + 127) / 128);  // 128-byte lines of values a pair
    const int lines = wp * (kVLines + 1);
    for (int L = lane; L < lines; L += 32) {
        const int m = L / (kVLines + 1), k = L % (kVLines + 1);
        const char *ptr = k < kVLines
                              ? reinterpret_cast<const char *>(vals + base + 64u * unsigned(m)) + 128 * k
                              : reinterpret_cast<const char *>(scol + base + 64u * unsigned(m));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
    }
}

// kU64 / kU32 / kU16: step pairs in flight per lane for FP64 / FP32 / BF16
// values (more for kernels with fewer, register-richer threads; BF16 by
// default twice the FP32 count).
//
// Pipeline: a block of the vector is staged by one bulk copy into a slot
// (S slots: 2 for an FP64 vector, M.nacc for an FP32 one); warps walk the
// blocks independently and the last warp done with block b refills its slot
// with block b + S, so warps may spread over S consecutive blocks and each
// slot has its own row accumulator (summed in a fixed order at the end).
// With an FP32 vector a warp reads its first slice's metadata of a block
// before waiting for the block's copy, and the next slice's metadata while
// it works on the current one.
// kPanels: walk the CTA's rows in M.panels row panels (instances for
// matrices whose rows per CTA exceed the accumulators); without it one walk
// over the CTA's rows, and the per-panel bookkeeping compiles away.
template <int kU64, int kU32, bool kOutline = false, bool kL2Prefetch = true, bool kPanels = false,
          int kU16 = 2 * kU32>
struct SlicedSpmvT {
    static constexpr bool kSliced = true;
    // Dynamic shared memory: the control words first (fixed offsets), then
    // the staging, then the accumulators; every address is a constant offset
    // from the array, so the policy keeps only three registers of state.
    static constexpr size_t kCtrlBytes = 128;
    int row0, row1;
    unsigned parity;         // bit i: next phase parity of slot i

    __device__ static unsigned char *smem()
    {
        extern __shared__ __align__(128) unsigned char sliced_smem[];
        return sliced_smem;
    }
    __device__ static uint64_t *bars() { return reinterpret_cast<uint64_t *>(smem()); }  // kMaxSlots
    __device__ static int *cnt() { return reinterpret_cast<int *>(smem() + 8 * kMaxSlots); }
    __device__ static int *abort_flag() { return cnt() + kMaxSlots; }
    __device__ static unsigned char *buf() { return smem() + kCtrlBytes; }
    __device__ static double *acc() { return reinterpret_cast<double *>(smem() + kCtrlBytes + kStagingBytes); }

    __device__ void setup(const MatrixView &, int r0, int r1)
    {
        row0 = r0;
        row1 = r1;
        parity = 0;
        if (threadIdx.x == 0) {
            for (int i = 0; i < kMaxSlots; i++) {
                mbar_init(&bars()[i], 1);
                cnt()[i] = 0;
            }
            *abort_flag() = 0;
        }
        __syncthreads();
    }

    template <typename VT>
    __device__ __forceinline__ void issue(const MatrixView &M, const VT *v, int n, int b, int slot)
    {
        const int cols = min(M.width, n - b * M.width);
        const unsigned bytes = (unsigned(cols) * unsigned(sizeof(VT)) + 15u) & ~15u;
        bulk_load(buf() + size_t(slot) * M.width * sizeof(VT), v + size_t(b) * M.width, bytes,
                  &bars()[slot]);
    }

    // kOutline: the SpMV is a called function with its own register budget
    // (for kernels whose solver state would otherwise crowd the SpMV loop).
    // VT: the gathered vector and the row sums; ST: the stored values
    // (VT, or BF16 under an FP32 vector).
    template <typename VT, typename ST = VT>
    __device__ __forceinline__ double apply(const MatrixView &M, const VT *v, double *out,
                                            const double *dotv, int n, long long limit_ns,
                                            int *status, bool &ok)
    {
        if constexpr (kOutline)
            return apply_outlined<VT, ST>(M, v, out, dotv, n, limit_ns, status, ok);
        else return apply_body<VT, ST>(M, v, out, dotv, n, limit_ns, status, ok);
    }

    template <typename VT, typename ST>
    __device__ __noinline__ double apply_outlined(const MatrixView &M, const VT *v, double *out,
                                                  const double *dotv, int n, long long limit_ns,
                                                  int *status, bool &ok)
    {
        return apply_body<VT, ST>(M, v, out, dotv, n, limit_ns, status, ok);
    }

    template <typename VT, typename ST>
    __device__ __forceinline__ double apply_body(const MatrixView &M, const VT *v, double *out,
                                                 const double *dotv, int n, long long limit_ns,
                                                 int *status, bool &ok)
    {
        using P2 = typename Pair<ST>::T;
        constexpr int kU = sizeof(ST) == 8 ? kU64 : sizeof(ST) == 4 ? kU32 : kU16;
        const ST *__restrict__ vals = slice_values<ST>(M);
        const uint64_t pol =
            l2_stream_policy(sizeof(ST) == 8 ? M.keep64 : sizeof(ST) == 4 ? M.keep32 : M.keep16);
        // slots in use: as many blocks of the vector as the staging holds,
        // at most one accumulator each
        const int S = min(M.nacc, int(kStagingBytes / (size_t(M.width) * sizeof(VT))));
        const size_t slot_bytes = size_t(M.width) * sizeof(VT);
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        const int nwarps = blockDim.x >> 5;
        // output rows: the CTA's range, or (interleaved copy) every grid-th row
        double *const acc = SlicedSpmvT::acc();
        uint64_t *const bars = SlicedSpmvT::bars();
        int *const cnt = SlicedSpmvT::cnt();
        int *const abort = abort_flag();
        double dacc = 0.0;
        // row panel pk: local rows [i0, i0 + nrows) of the CTA, a walk over
        // every column block of its own chunks (one panel unless the CTA's
        // rows exceed the accumulators)
        const int panels = kPanels ? M.panels : 1;
        for (int pk = 0; pk < panels; pk++) {
            const int chunk0 = (int(blockIdx.x) * panels + pk) * M.nblk;
            if (pk > 0) __syncthreads();  // the previous panel's sums are read out
            for (int i = threadIdx.x; i < S * M.max_rows; i += blockDim.x) acc[i] = 0.0;
            if (threadIdx.x == 0) {
                fence_proxy_async();  // v was written by generic stores before the grid barrier
                for (int b = 0; b < S && b < M.nblk; b++) issue(M, v, n, b, b);
            }
            // this warp's slices of block b toward L2 (one block ahead of use)
            // (only in the kL2Prefetch instances: it pays where the walk is
            // latency-bound -- short column-block chunks -- and costs where it
            // streams, so the plan's autotuner picks the instance)
            auto prefetch_block = [&](int b) {
                if (!kL2Prefetch || b >= M.nblk) return;
                const int t0 = __ldg(M.chunk_slice + chunk0 + b);
                const int t1 = __ldg(M.chunk_slice + chunk0 + b + 1);
                for (int t = t0 + (warp + (b * 7) % nwarps) % nwarps; t < t1; t += nwarps)
                    prefetch_slice_l2(vals, M.scol, __ldg(M.slice_off + t), __ldg(M.slice_width + t) >> 1,
                                      lane);
            };
            prefetch_block(0);
            __syncthreads();
            bool failed = false;
            for (int b = 0; b < M.nblk && !failed; b++) {
                const int slot = b % S;
                const int s0 = __ldg(M.chunk_slice + chunk0 + b);  // this matrix's blocks
                const int s1 = __ldg(M.chunk_slice + chunk0 + b + 1);
                prefetch_block(b + 1);
                // rotate the warp -> slice assignment from block to block so the
                // widest slices do not always land on the same warps
                const int rot = (b * 7) % nwarps;
                // one slice: lane `lane` of slice entries at off, wp step pairs
                auto run_slice = [&](unsigned off, int wp, unsigned short row, const VT *pv,
                                     double *accb) {
                    using AT = typename SumType<VT>::T;
                    AT sum = AT(0);
                    for (int m = 0; m < wp; m += kU) {
                        P2 av[kU];
                        ushort2 cv[kU];
    #pragma unroll
                        for (int u = 0; u < kU; u++) {
                            if (m + u < wp) {
                                const unsigned e = off + 64u * unsigned(m + u);
                                if (CGB_IN_RANGE(e + 1, M.slice_entries, kCheckStream)) {
                                    av[u] = ld_stream(reinterpret_cast<const P2 *>(vals + e), pol);
                                    cv[u] = ld_stream(reinterpret_cast<const ushort2 *>(M.scol + e), pol);
                                } else {
                                    av[u].x = av[u].y = ST(0.f);
                                    cv[u] = make_ushort2(0, 0);
                                }
                            }
                        }
    #pragma unroll
                        for (int u = 0; u < kU; u++) {
                            if (m + u < wp) {
                                if (CGB_IN_RANGE(cv[u].x, M.width, kCheckGather))
                                    sum = fma_vt(AT(widen(av[u].x)), AT(widen(pv[cv[u].x])), sum);
                                if (CGB_IN_RANGE(cv[u].y, M.width, kCheckGather))
                                    sum = fma_vt(AT(widen(av[u].y)), AT(widen(pv[cv[u].y])), sum);
                            }
                        }
                    }
                    if (row != 0xffffu && CGB_IN_RANGE(row, M.max_rows, kCheckRow)) accb[row] += double(sum);
                };
                const VT *pv = reinterpret_cast<const VT *>(buf() + size_t(slot) * slot_bytes);
                double *accb = acc + size_t(slot) * M.max_rows;
                if constexpr (sizeof(VT) == 8) {
                    // FP64 vector: long slices, the plain walk measures fastest
                    if (!mbar_wait(&bars[slot], (parity >> slot) & 1u, limit_ns, abort)) {
                        failed = true;
                        *abort = 1;
                        break;
                    }
                    parity ^= 1u << slot;
                    for (int s = s0 + (warp + rot) % nwarps; s < s1; s += nwarps)
                        run_slice(__ldg(M.slice_off + s) + 2u * lane, __ldg(M.slice_width + s) >> 1,
                                  __ldg(M.srow + size_t(s) * 32 + lane), pv, accb);
                } else {
                    // FP32 vector: the first slice's metadata before the wait,
                    // the next slice's while the current one streams
                    int s = s0 + (warp + rot) % nwarps;
                    unsigned off = 0;
                    int wp = 0;
                    unsigned short row = 0xffffu;
                    if (s < s1) {
                        off = __ldg(M.slice_off + s) + 2u * lane;
                        wp = __ldg(M.slice_width + s) >> 1;
                        row = __ldg(M.srow + size_t(s) * 32 + lane);
                    }
                    if (!mbar_wait(&bars[slot], (parity >> slot) & 1u, limit_ns, abort)) {
                        failed = true;
                        *abort = 1;
                        break;
                    }
                    parity ^= 1u << slot;
                    while (s < s1) {
                        const int sn = s + nwarps;
                        unsigned offn = 0;
                        int wpn = 0;
                        unsigned short rown = 0xffffu;
                        if (sn < s1) {
                            offn = __ldg(M.slice_off + sn) + 2u * lane;
                            wpn = __ldg(M.slice_width + sn) >> 1;
                            rown = __ldg(M.srow + size_t(sn) * 32 + lane);
                        }
                        run_slice(off, wp, row, pv, accb);
                        s = sn;
                        off = offn;
                        wp = wpn;
                        row = rown;
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    if (atomicAdd(&cnt[slot], 1) == nwarps - 1) {
                        cnt[slot] = 0;
                        if (b + S < M.nblk) {
                            fence_proxy_async();  // all warps' reads of the slot before the refill
                            issue(M, v, n, b + S, slot);
                        }
                    }
                }
            }
            if (__syncthreads_or(failed)) {
                ok = false;
                if (threadIdx.x == 0) {
                    raise_status(status, kDevTimeout);
                    // let issued copies land before the CTA leaves (a completed
                    // phase returns at once)
                    for (int i = 0; i < S; i++) (void)mbar_wait(&bars[i], (parity >> i) & 1u, limit_ns, nullptr);
                }
                __syncthreads();
                return 0.0;
            }
            const int own = M.interleaved ? interleaved_rows(n, blockIdx.x, gridDim.x) : row1 - row0;
            const int stride = M.interleaved ? int(gridDim.x) : 1;
            const int i0 = panel_begin(own, pk, panels);
            const int nrows = panel_begin(own, pk + 1, panels) - i0;
            const int base = (M.interleaved ? int(blockIdx.x) : row0) + i0 * stride;
            for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
                double t = acc[i];
                for (int k = 1; k < S; k++) t += acc[size_t(k) * M.max_rows + i];
                const int row = base + i * stride;
                out[row] = t;
                if (dotv) dacc = fma(dotv[row], t, dacc);
            }
        }
        // with one panel, row i's sum is written by thread i % blockDim, the
        // thread that reads it next in the callers' row loops; panels shift
        // that mapping, so the CTA synchronizes before any of its threads
        // reads an output row
        if constexpr (kPanels) __syncthreads();
        ok = true;
        return dacc;
    }
};

// Per kernel (pair counts and block shapes measured on B200): the FP64
// outer step and the standalone SpMVs (768 threads, 80 registers), the
// mixed outer step (768), the preconditioned one (512, 128 registers).
using SlicedSpmv = SlicedSpmvT<6, 6, false, false>;
using SlicedSpmvPf = SlicedSpmvT<6, 6, false, true>;
using SlicedSpmvMixed = SlicedSpmvT<4, 6, false, false>;
using SlicedSpmvMixedPf = SlicedSpmvT<4, 6, false, true>;
using SlicedSpmvPcg = SlicedSpmvT<4, 10, false, false, false, 8>;
// row-panel instances (no L2 prefetch)
using SlicedSpmvPanels = SlicedSpmvT<6, 6, false, false, true>;
using SlicedSpmvMixedPanels = SlicedSpmvT<4, 6, false, false, true>;
using SlicedSpmvPcgPanels = SlicedSpmvT<4, 6, false, false, true>;

}  // namespace cgb

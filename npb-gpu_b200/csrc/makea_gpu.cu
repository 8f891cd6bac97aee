// makea_gpu.cu -- the NPB CG matrix assembled on the GPU, bit-identical to
// the reference's makea() + sparse() (GMAP/NPB-GPU CUDA/CG/cg.cu:1303-1368,
// :1611-1785) and to the host generator in makea.cpp.
//
// The n sparse vectors (one LCG stream with rejection sampling, inherently
// sequential and cheap) are drawn on the host; the assembly -- n * (nonzer+1)^2
// outer-product contributions, 38 M at class C -- runs on the device:
//   1. per row, the vectors that touch it (an incidence transpose with
//      atomic slots, then each row's short list sorted by vector index);
//   2. per row, its contributions in generation order (vector i, then entry
//      u of that vector), values formed with the reference's rounding:
//      val[u] * (scale_i * val[s]), and on the diagonal of vector i's own row
//      + rcond then - shift, each a separately rounded operation;
//   3. per row, a sort by (column, generation index) in shared memory and a
//      left-to-right sum of each column's contributions starting from 0.0 --
//      the order in which the reference's insertion loop meets them;
//   4. row lengths -> rowstr (host scan), compaction, copy out.
// Explicit __dmul_rn / __dadd_rn keep every product and sum separately
// rounded (no contraction into fused multiply-adds).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cgb_internal.h"

namespace cgb {
namespace gen {

constexpr int kFoldThreads = 256;
constexpr int kMaxRowContrib = 2048;  // contributions of one row held in shared memory
constexpr int kGroupsPerThread = kMaxRowContrib / kFoldThreads;

// 1a. per row: vectors touching it, and its contribution count
__global__ void row_counts(const int *__restrict__ count, const int *__restrict__ pos, int n,
                           int width, int *nvec, unsigned long long *ncontrib)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = count[i];
        for (int s = 0; s < c; s++) {
            const int row = pos[size_t(i) * width + s];
            atomicAdd(&nvec[row], 1);
            atomicAdd(&ncontrib[row], (unsigned long long)c);
        }
    }
}

// 1b. per row: the (vector, entry) keys i * 32 + s, unordered
__global__ void fill_lists(const int *__restrict__ count, const int *__restrict__ pos, int n,
                           int width, const long long *__restrict__ voff, int *cursor,
                           unsigned *list)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = count[i];
        for (int s = 0; s < c; s++) {
            const int row = pos[size_t(i) * width + s];
            const int at = atomicAdd(&cursor[row], 1);
            list[voff[row] + at] = unsigned(i) * 32u + unsigned(s);
        }
    }
}

// 1c. each row's list by vector index (lists are short: insertion sort)
__global__ void sort_lists(const long long *__restrict__ voff, int n, unsigned *list)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        unsigned *l = list + voff[row];
        const int len = int(voff[row + 1] - voff[row]);
        for (int a = 1; a < len; a++) {
            const unsigned key = l[a];
            int b = a - 1;
            while (b >= 0 && l[b] > key) {
                l[b + 1] = l[b];
                b--;
            }
            l[b + 1] = key;
        }
    }
}

// 2. one warp per row: contributions in generation order
__global__ void contributions(const int *__restrict__ count, const int *__restrict__ pos,
                              const double *__restrict__ val, const double *__restrict__ scale,
                              int n, int width, double rcond, double shift,
                              const long long *__restrict__ voff, const unsigned *__restrict__ list,
                              const long long *__restrict__ coff, int *ccol, double *cval)
{
    const int lane = threadIdx.x & 31;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n;
         row += (gridDim.x * blockDim.x) >> 5) {
        long long at = coff[row];
        for (long long k = voff[row]; k < voff[row + 1]; k++) {
            const unsigned key = list[k];
            const int i = int(key >> 5), s = int(key & 31u);
            const int c = count[i];
            const size_t base = size_t(i) * width;
            const double sc = __dmul_rn(scale[i], val[base + s]);
            for (int u = lane; u < c; u += 32) {
                const int col = pos[base + u];
                double va = __dmul_rn(val[base + u], sc);
                if (col == row && row == i) {
                    va = __dadd_rn(va, rcond);
                    va = __dsub_rn(va, shift);
                }
                ccol[at + u] = col;
                cval[at + u] = va;
            }
            at += c;
        }
    }
}

// 3. one CTA per row: sort by (column, generation index), fold each column
// left to right from 0.0; unique entries overwrite the row's contribution
// slots, their count into ucount[row].  A row longer than kMaxRowContrib
// sets *overflow and is left alone.
__global__ void __launch_bounds__(kFoldThreads) fold_rows(const long long *__restrict__ coff, int n,
                                                          int *ccol, double *cval, int *ucount,
                                                          int *overflow)
{
    __shared__ unsigned long long key[kMaxRowContrib];
    __shared__ int start_rank[kMaxRowContrib];
    __shared__ int warp_tot[kFoldThreads / 32];
    for (int row = blockIdx.x; row < n; row += gridDim.x) {
        const long long base = coff[row];
        const int len = int(coff[row + 1] - base);
        if (len > kMaxRowContrib) {
            if (threadIdx.x == 0) {
                atomicExch(overflow, 1);
                ucount[row] = 0;
            }
            continue;
        }
        int pow2 = 1;
        while (pow2 < len) pow2 <<= 1;
        for (int t = threadIdx.x; t < pow2; t += blockDim.x)
            key[t] = t < len ? (uint64_t(uint32_t(ccol[base + t])) << 32) | uint32_t(t)
                             : ~0ull;
        __syncthreads();
        // bitonic sort, ascending
        for (int k = 2; k <= pow2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = threadIdx.x; t < pow2; t += blockDim.x) {
                    const int o = t ^ j;
                    if (o > t) {
                        const bool up = (t & k) == 0;
                        const unsigned long long x = key[t], y = key[o];
                        if ((x > y) == up) {
                            key[t] = y;
                            key[o] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        // group starts and their ranks (block-wide exclusive scan of flags)
        const int per = (len + blockDim.x - 1) / blockDim.x;
        const int t0 = threadIdx.x * per, t1 = min(len, t0 + per);
        int mine = 0;
        for (int t = t0; t < t1; t++)
            mine += (t == 0 || (key[t] >> 32) != (key[t - 1] >> 32)) ? 1 : 0;
        // scan of `mine` over threads
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) warp_tot[w] = incl;
        __syncthreads();
        int before = 0;
        for (int q = 0; q < w; q++) before += warp_tot[q];
        int rank = before + incl - mine;
        for (int t = t0; t < t1; t++) {
            const bool st = (t == 0 || (key[t] >> 32) != (key[t - 1] >> 32));
            start_rank[t] = st ? rank : -1;
            rank += st ? 1 : 0;
        }
        int total = 0;
        for (int q = 0; q < int(blockDim.x >> 5); q++) total += warp_tot[q];
        __syncthreads();
        // each group start sums its group in generation order; results are
        // staged in registers, then written after everyone has read cval
        double gsum[kGroupsPerThread];
        int gcol[kGroupsPerThread], grank[kGroupsPerThread], ng = 0;
        for (int t = threadIdx.x; t < len; t += blockDim.x) {
            if (start_rank[t] < 0) continue;
            const int col = int(key[t] >> 32);
            double sum = 0.0;
            for (int e = t; e < len && int(key[e] >> 32) == col; e++)
                sum = __dadd_rn(sum, cval[base + int(key[e] & 0xffffffffu)]);
            // t advances by blockDim.x from threadIdx.x < len <= kMaxRowContrib,
            // so a thread meets at most kGroupsPerThread starts
            gsum[ng] = sum;
            gcol[ng] = col;
            grank[ng] = start_rank[t];
            ng++;
        }
        __syncthreads();
        for (int g = 0; g < ng; g++) {
            ccol[base + grank[g]] = gcol[g];
            cval[base + grank[g]] = gsum[g];
        }
        if (threadIdx.x == 0) ucount[row] = total;
        __syncthreads();
    }
}

// 4. compaction into the final CSR
__global__ void compact(const long long *__restrict__ coff, const int *__restrict__ rowstr, int n,
                        const int *__restrict__ ccol, const double *__restrict__ cval, int *colidx,
                        double *a)
{
    const int lane = threadIdx.x & 31;
    for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n;
         row += (gridDim.x * blockDim.x) >> 5) {
        const long long src = coff[row];
        const int dst = rowstr[row], len = rowstr[row + 1] - rowstr[row];
        for (int t = lane; t < len; t += 32) {
            colidx[dst + t] = ccol[src + t];
            a[dst + t] = cval[src + t];
        }
    }
}

template <typename T>
cudaError_t galloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

struct DeviceBuffers {
    int *count = nullptr, *pos = nullptr, *nvec = nullptr, *cursor = nullptr, *ccol = nullptr;
    int *ucount = nullptr, *rowstr = nullptr, *colidx = nullptr, *flag = nullptr;
    double *val = nullptr, *scale = nullptr, *cval = nullptr, *a = nullptr;
    unsigned long long *ncontrib = nullptr;
    long long *voff = nullptr, *coff = nullptr;
    unsigned *list = nullptr;
    ~DeviceBuffers()
    {
        for (void *p : {(void *)count, (void *)pos, (void *)nvec, (void *)cursor, (void *)ccol,
                        (void *)ucount, (void *)rowstr, (void *)colidx, (void *)flag, (void *)val,
                        (void *)scale, (void *)cval, (void *)a, (void *)ncontrib, (void *)voff,
                        (void *)coff, (void *)list})
            if (p) cudaFree(p);
    }
};

}  // namespace gen
}  // namespace cgb

using namespace cgb;
using namespace cgb::gen;

#define GEN_TRY(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(e_ == cudaErrorMemoryAllocation ? CGB_ERR_NOMEM : CGB_ERR_CUDA, \
                             "makea_device: %s: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

extern "C" int cgb_makea_device(int device, int n, int nonzer, double rcond, double shift,
                                double seed, int *rowstr, int *colidx, double *a,
                                long long nz_capacity, long long *nnz_out)
{
    if (!rowstr || !nnz_out) return set_error(CGB_ERR_INVALID, "makea_device: null outputs");
    if (!(rcond > 0.0) || !std::isfinite(shift))
        return set_error(CGB_ERR_INVALID, "makea_device: rcond must be > 0 and shift finite");
    if (nonzer + 1 > 32) return set_error(CGB_ERR_INVALID, "makea_device: nonzer must be <= 31");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return set_error(CGB_ERR_NO_DEVICE, "makea_device: no CUDA device %d", device);
    GenVectors v;
    int st = draw_generator_vectors(n, nonzer, rcond, seed, v);
    if (st) return st;
    GEN_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    GEN_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return set_error(CGB_ERR_NO_DEVICE, "makea_device: device %d is not sm_100", device);
    const int w = v.width, sms = prop.multiProcessorCount;
    DeviceBuffers d;
    GEN_TRY(galloc(&d.count, n));
    GEN_TRY(galloc(&d.pos, size_t(n) * w));
    GEN_TRY(galloc(&d.val, size_t(n) * w));
    GEN_TRY(galloc(&d.scale, n));
    GEN_TRY(galloc(&d.nvec, n));
    GEN_TRY(galloc(&d.ncontrib, n));
    GEN_TRY(cudaMemcpy(d.count, v.count.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemcpy(d.pos, v.pos.data(), sizeof(int) * size_t(n) * w, cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemcpy(d.val, v.val.data(), sizeof(double) * size_t(n) * w, cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemcpy(d.scale, v.scale.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemset(d.nvec, 0, sizeof(int) * n));
    GEN_TRY(cudaMemset(d.ncontrib, 0, sizeof(unsigned long long) * n));
    const int grid = 8 * sms;
    row_counts<<<grid, 256>>>(d.count, d.pos, n, w, d.nvec, d.ncontrib);
    GEN_TRY(cudaGetLastError());
    // offsets (host scans of n counts)
    std::vector<int> nvec(n);
    std::vector<unsigned long long> ncon(n);
    GEN_TRY(cudaMemcpy(nvec.data(), d.nvec, sizeof(int) * n, cudaMemcpyDeviceToHost));
    GEN_TRY(cudaMemcpy(ncon.data(), d.ncontrib, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost));
    std::vector<long long> voff(size_t(n) + 1, 0), coff(size_t(n) + 1, 0);
    for (int j = 0; j < n; j++) {
        voff[j + 1] = voff[j] + nvec[j];
        coff[j + 1] = coff[j] + (long long)ncon[j];
    }
    const long long nlist = voff[n], ncon_total = coff[n];
    GEN_TRY(galloc(&d.voff, size_t(n) + 1));
    GEN_TRY(galloc(&d.coff, size_t(n) + 1));
    GEN_TRY(galloc(&d.cursor, n));
    GEN_TRY(galloc(&d.list, size_t(nlist)));
    GEN_TRY(galloc(&d.ccol, size_t(ncon_total)));
    GEN_TRY(galloc(&d.cval, size_t(ncon_total)));
    GEN_TRY(galloc(&d.ucount, n));
    GEN_TRY(galloc(&d.flag, 1));
    GEN_TRY(cudaMemcpy(d.voff, voff.data(), sizeof(long long) * (size_t(n) + 1), cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemcpy(d.coff, coff.data(), sizeof(long long) * (size_t(n) + 1), cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemset(d.cursor, 0, sizeof(int) * n));
    GEN_TRY(cudaMemset(d.flag, 0, sizeof(int)));
    fill_lists<<<grid, 256>>>(d.count, d.pos, n, w, d.voff, d.cursor, d.list);
    sort_lists<<<grid, 256>>>(d.voff, n, d.list);
    contributions<<<grid, 256>>>(d.count, d.pos, d.val, d.scale, n, w, rcond, shift, d.voff, d.list,
                                 d.coff, d.ccol, d.cval);
    fold_rows<<<std::min(n, 16 * sms), kFoldThreads>>>(d.coff, n, d.ccol, d.cval, d.ucount, d.flag);
    GEN_TRY(cudaGetLastError());
    int flag = 0;
    GEN_TRY(cudaMemcpy(&flag, d.flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return set_error(CGB_ERR_CAPACITY, "makea_device: a row exceeds the fold capacity");
    std::vector<int> ucount(n);
    GEN_TRY(cudaMemcpy(ucount.data(), d.ucount, sizeof(int) * n, cudaMemcpyDeviceToHost));
    long long nnz = 0;
    for (int j = 0; j < n; j++) nnz += ucount[j];
    *nnz_out = nnz;
    if (nnz > nz_capacity)
        return set_error(CGB_ERR_CAPACITY, "makea_device: nz_capacity %lld < nnz %lld", nz_capacity, nnz);
    if (nnz > 0x7fffffffLL)
        return set_error(CGB_ERR_CAPACITY, "makea_device: nnz %lld overflows int32 rowstr", nnz);
    if (!colidx || !a) return set_error(CGB_ERR_INVALID, "makea_device: null colidx/a");
    rowstr[0] = 0;
    for (int j = 0; j < n; j++) rowstr[j + 1] = rowstr[j] + ucount[j];
    GEN_TRY(galloc(&d.rowstr, size_t(n) + 1));
    GEN_TRY(galloc(&d.colidx, size_t(nnz)));
    GEN_TRY(galloc(&d.a, size_t(nnz)));
    GEN_TRY(cudaMemcpy(d.rowstr, rowstr, sizeof(int) * (size_t(n) + 1), cudaMemcpyHostToDevice));
    compact<<<grid, 256>>>(d.coff, d.rowstr, n, d.ccol, d.cval, d.colidx, d.a);
    GEN_TRY(cudaGetLastError());
    GEN_TRY(cudaMemcpy(colidx, d.colidx, sizeof(int) * size_t(nnz), cudaMemcpyDeviceToHost));
    GEN_TRY(cudaMemcpy(a, d.a, sizeof(double) * size_t(nnz), cudaMemcpyDeviceToHost));
    return CGB_OK;
}

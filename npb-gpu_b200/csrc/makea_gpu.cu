// makea_gpu.cu -- the NPB CG matrix assembled on the GPU, bit-identical to
// the reference's makea() + sparse() (GMAP/NPB-GPU CUDA/CG/cg.cu:1303-1368,
// :1611-1785) and to the host generator in makea.cpp.
//
// The n sparse vectors (one LCG stream with rejection sampling) are drawn
// on the device in parallel (pair_ends ... draw_vectors below: a vector's
// length in draws depends only on where it starts, so every start is parsed
// at once and the chain from the first draw follows by jump pointers); the
// geometric weights, a running product rounded at every step, are the one
// O(n) loop left on the host.  The assembly -- n * (nonzer+1)^2
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

// ---------------------------------------------------------------- vectors
// The n sparse vectors (sprnvc + vecset, cg.cu:1798-1857) from one LCG
// stream.  Draw k of the stream is x_k * 2^-46, x_k = seed * 5^13^k mod 2^46
// (c_randdp.cpp:84-114 in integer form); main() throws draw 1 away
// (cg.cu:406-408), so the vectors consume pairs (value, where) = draws
// (2 + 2m, 3 + 2m), m = 0, 1, ...  A candidate position is
// int(pow2 * where) + 1 = (x >> (46 - log2 pow2)) + 1 (pow2 a power of two,
// so the product is exact); it is rejected when > n or already drawn for
// this vector.  How many pairs a vector consumes depends only on the pair
// it starts at, which makes the draw parallel:
//   1. pair_ends:   for every pair m < D, the pair after a vector starting at
//                   m (D when it would run past the buffer);
//   2. jump_double: ten rounds of J(m) <- J(J(m)): 1024 vectors ahead;
//   3. chain_heads: one thread walks the 1024-vector jumps from pair 0, then
//      chain_starts: a thread per 1024 vectors walks the single steps -> the
//                   first pair of every vector;
//   4. draw_vectors: vector i parsed again from its first pair, vecset's 0.5
//                   at position i added -- the host draw's layout.
constexpr uint64_t kMask46 = (uint64_t(1) << 46) - 1;
constexpr uint64_t kMult = 1220703125ull;  // 5^13 (cg.cu:407)
constexpr int kJumpRounds = 10;            // 2^10 vectors a jump
constexpr int kMaxWidth = 32;              // nonzer + 1 <= 32

__device__ __forceinline__ uint64_t lcg_at(uint64_t seed, uint64_t k)
{
    uint64_t r = seed & kMask46, b = kMult;
    while (k) {
        if (k & 1) r = (r * b) & kMask46;  // low 46 bits of the 64-bit product
        b = (b * b) & kMask46;
        k >>= 1;
    }
    return r;
}

// One vector from pair m: accepted 1-based positions into p1 (and values
// into vv when kValues); returns the pair after its last pair, or D if the
// vector would run past pair D.
template <bool kValues>
__device__ __forceinline__ long long parse_vector(uint64_t seed, long long m, long long D, int n,
                                                  int nonzer, int shift_bits, int *p1, double *vv,
                                                  int *have_out)
{
    uint64_t x = lcg_at(seed, uint64_t(2 + 2 * m));
    int have = 0;
    while (have < nonzer) {
        if (m >= D) return D;
        const uint64_t xv = x;               // value draw
        x = (x * kMult) & kMask46;           // where draw
        const int cand = int(x >> shift_bits) + 1;
        x = (x * kMult) & kMask46;           // next pair's value draw
        m++;
        if (cand > n) continue;
        bool seen = false;
        for (int t = 0; t < have; t++) seen |= (p1[t] == cand);
        if (seen) continue;
        if (kValues) vv[have] = double(xv) * 0x1p-46;  // exact
        p1[have] = cand;
        have++;
    }
    *have_out = have;
    return m;
}

__global__ void pair_ends(uint64_t seed, long long D, int n, int nonzer, int shift_bits, int *end)
{
    int p1[kMaxWidth];
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m <= D;
         m += (long long)gridDim.x * blockDim.x) {
        int have = 0;
        end[m] = m == D ? int(D)
                        : int(parse_vector<false>(seed, m, D, n, nonzer, shift_bits, p1, nullptr, &have));
    }
}

__global__ void jump_double(long long D, const int *__restrict__ j_in, int *j_out)
{
    for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m <= D;
         m += (long long)gridDim.x * blockDim.x)
        j_out[m] = j_in[j_in[m]];
}

// One thread: heads[k] = first pair of vector k * 1024.
__global__ void chain_heads(const int *__restrict__ jump, long long D, int nheads, int *heads,
                            int *overflow)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int h = 0;
    for (int k = 0; k < nheads; k++) {
        if (h >= D) {
            *overflow = 1;
            return;
        }
        heads[k] = h;
        h = jump[h];
    }
}

// A thread per 1024 vectors: start[i] = first pair of vector i.
__global__ void chain_starts(const int *__restrict__ end, const int *__restrict__ heads, long long D,
                             int n, int *start, int *overflow)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = k << kJumpRounds;
    if (i0 >= n || *overflow) return;  // the heads are incomplete after an overflow
    const int i1 = min(n, i0 + (1 << kJumpRounds));
    int s = heads[k];
    for (int i = i0; i < i1; i++) {
        if (s < 0 || s >= D) {
            *overflow = 1;
            return;
        }
        start[i] = s;
        s = end[s];
    }
    if (s >= D) *overflow = 1;  // the last vector ran past the buffer
}

__global__ void draw_vectors(uint64_t seed, long long D, int n, int nonzer, int shift_bits,
                             const int *__restrict__ start, int width, int *count, int *pos,
                             double *val)
{
    int p1[kMaxWidth];
    double vv[kMaxWidth];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int have = 0;
        (void)parse_vector<true>(seed, start[i], D, n, nonzer, shift_bits, p1, vv, &have);
        bool set = false;
        for (int t = 0; t < have; t++)
            if (p1[t] == i + 1) {
                vv[t] = 0.5;
                set = true;
            }
        if (!set) {
            vv[have] = 0.5;
            p1[have] = i + 1;
            have++;
        }
        count[i] = have;
        for (int t = 0; t < have; t++) {
            pos[size_t(i) * width + t] = p1[t] - 1;
            val[size_t(i) * width + t] = vv[t];
        }
    }
}

// The assembly covers the rows [row0, row0 + nr) (all n, or one rank's
// block of a row-partitioned solve); arrays indexed by row below are local
// to that range, column indices stay global.

// 1a. per row: vectors touching it, and its contribution count
__global__ void row_counts(const int *__restrict__ count, const int *__restrict__ pos, int n,
                           int width, int row0, int nr, int *nvec, unsigned long long *ncontrib)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = count[i];
        for (int s = 0; s < c; s++) {
            const unsigned lr = unsigned(pos[size_t(i) * width + s] - row0);
            if (lr >= unsigned(nr)) continue;
            atomicAdd(&nvec[lr], 1);
            atomicAdd(&ncontrib[lr], (unsigned long long)c);
        }
    }
}

// 1b. per row: the (vector, entry) keys i * 32 + s, unordered
__global__ void fill_lists(const int *__restrict__ count, const int *__restrict__ pos, int n,
                           int width, int row0, int nr, const long long *__restrict__ voff,
                           int *cursor, unsigned *list)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = count[i];
        for (int s = 0; s < c; s++) {
            const unsigned lr = unsigned(pos[size_t(i) * width + s] - row0);
            if (lr >= unsigned(nr)) continue;
            const int at = atomicAdd(&cursor[lr], 1);
            list[voff[lr] + at] = unsigned(i) * 32u + unsigned(s);
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
                              int row0, int nr, int width, double rcond, double shift,
                              const long long *__restrict__ voff, const unsigned *__restrict__ list,
                              const long long *__restrict__ coff, int *ccol, double *cval)
{
    const int lane = threadIdx.x & 31;
    for (int lr = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; lr < nr;
         lr += (gridDim.x * blockDim.x) >> 5) {
        const int row = row0 + lr;
        long long at = coff[lr];
        for (long long k = voff[lr]; k < voff[lr + 1]; k++) {
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

#define GEN_TRY_IN(call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            for (void *p_ : {(void *)end, (void *)jump, (void *)heads, (void *)start,      \
                             (void *)flag})                                               \
                if (p_) cudaFree(p_);                                                     \
            return set_error(e_ == cudaErrorMemoryAllocation ? CGB_ERR_NOMEM : CGB_ERR_CUDA, \
                             "makea_device: %s: %s", #call, cudaGetErrorString(e_));       \
        }                                                                                 \
    } while (0)

namespace {

// The generator's vectors into d->count / pos / val (see the kernels above).
// The pair buffer starts at 1.3x the expected pairs and doubles while the
// chain runs past it.
int draw_on_device(double seed, int n, int nonzer, int sms, DeviceBuffers *d)
{
    int pow2 = 1, log2p = 0;
    do {
        pow2 *= 2;
        log2p++;
    } while (pow2 < n);
    const int shift_bits = 46 - log2p;
    const uint64_t useed = uint64_t(seed);
    const int nheads = (n + (1 << kJumpRounds) - 1) >> kJumpRounds;
    long long D = (long long)n * (long long)std::ceil(1.3 * nonzer * double(pow2) / n + 2.0) + 1024;
    for (int attempt = 0; attempt < 6; attempt++, D *= 2) {
        if (D + 1 > 0x7fffffffLL)
            return set_error(CGB_ERR_CAPACITY, "makea_device: %lld draw pairs overflow int32", D);
        int *end = nullptr, *jump = nullptr, *heads = nullptr, *start = nullptr, *flag = nullptr;
        GEN_TRY_IN(galloc(&end, size_t(D) + 1));
        GEN_TRY_IN(galloc(&jump, 2 * (size_t(D) + 1)));
        GEN_TRY_IN(galloc(&heads, size_t(nheads)));
        GEN_TRY_IN(galloc(&start, size_t(n)));
        GEN_TRY_IN(galloc(&flag, 1));
        GEN_TRY_IN(cudaMemset(flag, 0, sizeof(int)));
        GEN_TRY_IN(cudaMemset(heads, 0xff, sizeof(int) * size_t(nheads)));  // -1: not reached
        const int grid = 16 * sms;
        pair_ends<<<grid, 256>>>(useed, D, n, nonzer, shift_bits, end);
        const int *j_in = end;
        int *j_out = jump;
        for (int r = 0; r < kJumpRounds; r++) {
            jump_double<<<grid, 256>>>(D, j_in, j_out);
            j_in = j_out;
            j_out = (j_out == jump) ? jump + (size_t(D) + 1) : jump;
        }
        chain_heads<<<1, 32>>>(j_in, D, nheads, heads, flag);
        chain_starts<<<(nheads + 127) / 128, 128>>>(end, heads, D, n, start, flag);
        GEN_TRY_IN(cudaGetLastError());
        int overflow = 0;
        GEN_TRY_IN(cudaMemcpy(&overflow, flag, sizeof(int), cudaMemcpyDeviceToHost));
        if (!overflow) {
            draw_vectors<<<grid, 256>>>(useed, D, n, nonzer, shift_bits, start, nonzer + 1, d->count,
                                        d->pos, d->val);
            GEN_TRY_IN(cudaGetLastError());
            GEN_TRY_IN(cudaDeviceSynchronize());
        }
        for (void *p : {(void *)end, (void *)jump, (void *)heads, (void *)start, (void *)flag})
            cudaFree(p);
        if (!overflow) return CGB_OK;
    }
    return set_error(CGB_ERR_CAPACITY, "makea_device: the draw did not fit %lld pairs", D);
}

}  // namespace

#define GEN_TRY(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(e_ == cudaErrorMemoryAllocation ? CGB_ERR_NOMEM : CGB_ERR_CUDA, \
                             "makea_device: %s: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

int cgb::makea_on_device(int device, int n, int nonzer, double rcond, double shift, double seed,
                         DeviceCsr *out, int row0, int row1)
{
    if (!(rcond > 0.0) || !std::isfinite(shift))
        return set_error(CGB_ERR_INVALID, "makea_device: rcond must be > 0 and shift finite");
    if (nonzer + 1 > 32) return set_error(CGB_ERR_INVALID, "makea_device: nonzer must be <= 31");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return set_error(CGB_ERR_NO_DEVICE, "makea_device: no CUDA device %d", device);
    if (n < 2 || nonzer < 1 || nonzer >= n)
        return set_error(CGB_ERR_INVALID, "makea_device: need n >= 2, 1 <= nonzer < n");
    if (!valid_seed(seed))
        return set_error(CGB_ERR_INVALID, "makea_device: seed must be an odd integer in (1, 2^46)");
    if (row1 < 0) row1 = n;
    if (row0 < 0 || row0 >= row1 || row1 > n)
        return set_error(CGB_ERR_INVALID, "makea_device: rows [%d, %d) not within [0, %d)", row0, row1, n);
    const int nr = row1 - row0;
    GEN_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    GEN_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return set_error(CGB_ERR_NO_DEVICE, "makea_device: device %d is not sm_100", device);
    const int w = nonzer + 1, sms = prop.multiProcessorCount;
    DeviceBuffers d;
    GEN_TRY(galloc(&d.count, n));
    GEN_TRY(galloc(&d.pos, size_t(n) * w));
    GEN_TRY(galloc(&d.val, size_t(n) * w));
    GEN_TRY(galloc(&d.scale, n));
    GEN_TRY(galloc(&d.nvec, nr));
    GEN_TRY(galloc(&d.ncontrib, nr));
    {
        // the geometric weights: a running product, rounded at every step
        // as the reference's loop does (cg.cu:1695, :1755) -- host, O(n)
        std::vector<double> scale(n);
        const double ratio = std::pow(rcond, 1.0 / double(n));
        double size = 1.0;
        for (int i = 0; i < n; i++) {
            scale[i] = size;
            size = size * ratio;
        }
        GEN_TRY(cudaMemcpy(d.scale, scale.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    }
    int st = draw_on_device(seed, n, nonzer, sms, &d);
    if (st) return st;
    GEN_TRY(cudaMemset(d.nvec, 0, sizeof(int) * nr));
    GEN_TRY(cudaMemset(d.ncontrib, 0, sizeof(unsigned long long) * nr));
    const int grid = 8 * sms;
    row_counts<<<grid, 256>>>(d.count, d.pos, n, w, row0, nr, d.nvec, d.ncontrib);
    GEN_TRY(cudaGetLastError());
    // offsets (host scans of the range's counts)
    std::vector<int> nvec(nr);
    std::vector<unsigned long long> ncon(nr);
    GEN_TRY(cudaMemcpy(nvec.data(), d.nvec, sizeof(int) * nr, cudaMemcpyDeviceToHost));
    GEN_TRY(cudaMemcpy(ncon.data(), d.ncontrib, sizeof(unsigned long long) * nr, cudaMemcpyDeviceToHost));
    std::vector<long long> voff(size_t(nr) + 1, 0), coff(size_t(nr) + 1, 0);
    for (int j = 0; j < nr; j++) {
        voff[j + 1] = voff[j] + nvec[j];
        coff[j + 1] = coff[j] + (long long)ncon[j];
    }
    const long long nlist = voff[nr], ncon_total = coff[nr];
    GEN_TRY(galloc(&d.voff, size_t(nr) + 1));
    GEN_TRY(galloc(&d.coff, size_t(nr) + 1));
    GEN_TRY(galloc(&d.cursor, nr));
    GEN_TRY(galloc(&d.list, size_t(nlist)));
    GEN_TRY(galloc(&d.ccol, size_t(ncon_total)));
    GEN_TRY(galloc(&d.cval, size_t(ncon_total)));
    GEN_TRY(galloc(&d.ucount, nr));
    GEN_TRY(galloc(&d.flag, 1));
    GEN_TRY(cudaMemcpy(d.voff, voff.data(), sizeof(long long) * (size_t(nr) + 1), cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemcpy(d.coff, coff.data(), sizeof(long long) * (size_t(nr) + 1), cudaMemcpyHostToDevice));
    GEN_TRY(cudaMemset(d.cursor, 0, sizeof(int) * nr));
    GEN_TRY(cudaMemset(d.flag, 0, sizeof(int)));
    fill_lists<<<grid, 256>>>(d.count, d.pos, n, w, row0, nr, d.voff, d.cursor, d.list);
    sort_lists<<<grid, 256>>>(d.voff, nr, d.list);
    contributions<<<grid, 256>>>(d.count, d.pos, d.val, d.scale, row0, nr, w, rcond, shift, d.voff,
                                 d.list, d.coff, d.ccol, d.cval);
    fold_rows<<<std::min(nr, 16 * sms), kFoldThreads>>>(d.coff, nr, d.ccol, d.cval, d.ucount, d.flag);
    GEN_TRY(cudaGetLastError());
    int flag = 0;
    GEN_TRY(cudaMemcpy(&flag, d.flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return set_error(CGB_ERR_CAPACITY, "makea_device: a row exceeds the fold capacity");
    std::vector<int> ucount(nr);
    GEN_TRY(cudaMemcpy(ucount.data(), d.ucount, sizeof(int) * nr, cudaMemcpyDeviceToHost));
    long long nnz = 0;
    for (int j = 0; j < nr; j++) nnz += ucount[j];
    out->nnz = nnz;
    if (nnz > 0x7fffffffLL)
        return set_error(CGB_ERR_CAPACITY, "makea_device: nnz %lld of rows [%d, %d) overflows int32 rowstr",
                         nnz, row0, row1);
    std::vector<int> &rowstr = out->h_rowstr;
    rowstr.assign(size_t(nr) + 1, 0);
    for (int j = 0; j < nr; j++) rowstr[j + 1] = rowstr[j] + ucount[j];
    // the vectors and lists are spent (the copies above waited for the
    // kernels): free them before the CSR is allocated, so the peak is the
    // contributions plus the CSR
    for (int **q : {&d.count, &d.pos, &d.nvec, &d.cursor})
        if (*q) {
            cudaFree(*q);
            *q = nullptr;
        }
    for (double **q : {&d.val, &d.scale}) {
        cudaFree(*q);
        *q = nullptr;
    }
    cudaFree(d.list);
    d.list = nullptr;
    GEN_TRY(galloc(&d.rowstr, size_t(nr) + 1));
    GEN_TRY(galloc(&d.colidx, size_t(nnz)));
    GEN_TRY(galloc(&d.a, size_t(nnz)));
    GEN_TRY(cudaMemcpy(d.rowstr, rowstr.data(), sizeof(int) * (size_t(nr) + 1), cudaMemcpyHostToDevice));
    compact<<<grid, 256>>>(d.coff, d.rowstr, nr, d.ccol, d.cval, d.colidx, d.a);
    GEN_TRY(cudaGetLastError());
    GEN_TRY(cudaDeviceSynchronize());
    // hand the CSR over (the buffers' destructor skips what it no longer owns)
    out->rowstr = d.rowstr;
    out->colidx = d.colidx;
    out->a = d.a;
    d.rowstr = d.colidx = nullptr;
    d.a = nullptr;
    return CGB_OK;
}

extern "C" int cgb_makea_device(int device, int n, int nonzer, double rcond, double shift,
                                double seed, int *rowstr, int *colidx, double *a,
                                long long nz_capacity, long long *nnz_out)
{
    if (!rowstr || !nnz_out) return set_error(CGB_ERR_INVALID, "makea_device: null outputs");
    DeviceCsr csr;
    int st = makea_on_device(device, n, nonzer, rcond, shift, seed, &csr);
    *nnz_out = csr.nnz;
    if (st == CGB_OK && csr.nnz > nz_capacity)
        st = set_error(CGB_ERR_CAPACITY, "makea_device: nz_capacity %lld < nnz %lld", nz_capacity,
                       csr.nnz);
    if (st == CGB_OK && (!colidx || !a)) st = set_error(CGB_ERR_INVALID, "makea_device: null colidx/a");
    if (st == CGB_OK) {
        std::memcpy(rowstr, csr.h_rowstr.data(), sizeof(int) * (size_t(n) + 1));
        if (cudaMemcpy(colidx, csr.colidx, sizeof(int) * size_t(csr.nnz), cudaMemcpyDeviceToHost) !=
                cudaSuccess ||
            cudaMemcpy(a, csr.a, sizeof(double) * size_t(csr.nnz), cudaMemcpyDeviceToHost) != cudaSuccess)
            st = set_error(CGB_ERR_CUDA, "makea_device: copy-out failed");
    }
    for (void *p : {(void *)csr.rowstr, (void *)csr.colidx, (void *)csr.a})
        if (p) cudaFree(p);
    return st;
}

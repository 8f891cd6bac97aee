// is.cu -- the NPB IS benchmark on the GPU: ranking 2^t integer keys of
// values below 2^k by counting (GMAP/NPB-GPU CUDA/IS/is.cu: main :335-505,
// rank :725-1000, create_seq :508-566, full_verify :567-700).
//
// Keys are generated on the device: key i is (int)(2^k/4 * (r1+r2+r3+r4)),
// r the LCG's draws 4i+1 .. 4i+4 (seed 314159265, multiplier 5^13), each
// thread jumping to its run of keys (exact 64-bit integer arithmetic mod
// 2^46) -- the reference's values bit for bit.  A ranking pass: the two
// keys the benchmark rewrites each iteration and the five test keys read
// (one thread), the counts by value (atomics into a table that stays in
// L2: 32 MB at class C), their running sums by a three-phase scan (each
// CTA scans a 2048-value tile and publishes its total, one CTA scans the
// totals, each tile adds its offset), and the five test ranks checked
// against the class's table (is.cu:157-190, offsets of rank_gpu_kernel_7).
// The timed region -- ten passes -- is one CUDA graph.  Full verification
// places every key by the last running sums (a scatter whose result, the
// sorted keys, does not depend on the order of the atomics) and counts the
// out-of-order neighbours.  Counts are exact, so every result is the same
// on every run; keys, counts and the sorted keys equal the oracle's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>

#include "cgb_internal.h"

namespace cgb {
namespace is {

constexpr int kIters = 10;  // MAX_ITERATIONS (is.cu:153)
constexpr int kTests = 5;   // TEST_ARRAY_SIZE
constexpr int kThreads = 256;
constexpr int kItems = 8;                          // values a scan thread holds
constexpr int kTileVals = kThreads * kItems;       // 2048 values a scan tile
constexpr int kKeysPerThread = 16;                 // generation
constexpr uint64_t kMask46 = (uint64_t(1) << 46) - 1;
constexpr uint64_t kMult = 1220703125ull;
constexpr uint64_t kSeed = 314159265ull;

struct ClassTable {
    char name;
    int total_log2, max_log2;
    long long index[kTests], rank[kTests];
};

// is.cu:86-140 (sizes) and :157-190 (test keys and their ranks)
constexpr ClassTable kClasses[] = {
    {'S', 16, 11, {48427, 17148, 23627, 62548, 4431}, {0, 18, 346, 64917, 65463}},
    {'W', 20, 16, {357773, 934767, 875723, 898999, 404505}, {1249, 11698, 1039987, 1043896, 1048018}},
    {'A', 23, 19, {2112377, 662041, 5336171, 3642833, 4250760}, {104, 17523, 123928, 8288932, 8388264}},
    {'B', 25, 21, {41869, 812306, 5102857, 18232239, 26860214}, {33422937, 10244, 59149, 33135281, 99}},
    {'C', 27, 23, {44172927, 72999161, 74326391, 129606274, 21736814},
     {61147, 882988, 266290, 133997595, 133525895}},
    {'D', 31, 27, {1317351170, 995930646, 1157283250, 1503301535, 1453734525},
     {1, 36538729, 1978098519, 2145192618, 2147425337}},
};

struct Params {
    char cls;  // 'U': no partial checks
    long long n;
    int maxk;
    long long index[kTests], rank[kTests];
};

__device__ __forceinline__ uint64_t lcg_mul(uint64_t a, uint64_t b) { return (a * b) & kMask46; }

__device__ __forceinline__ uint64_t jump(uint64_t e)
{
    uint64_t r = kSeed, b = kMult;
    while (e) {
        if (e & 1) r = lcg_mul(r, b);
        b = lcg_mul(b, b);
        e >>= 1;
    }
    return r;
}

__global__ void k_keys(int32_t *keys, long long n, double scale)
{
    const long long i0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) * kKeysPerThread;
    if (i0 >= n) return;
    uint64_t x = jump(4 * uint64_t(i0));
    const long long i1 = min(n, i0 + kKeysPerThread);
    for (long long i = i0; i < i1; i++) {
        double s = 0.0;
        for (int d = 0; d < 4; d++) {
            x = lcg_mul(x, kMult);
            s = d == 0 ? double(x) * 0x1p-46 : s + double(x) * 0x1p-46;
        }
        keys[i] = int32_t(scale * s);
    }
}

// The iteration's two rewritten keys, then the five test keys (one thread,
// in the reference's order).
__global__ void k_prep(int32_t *keys, int it, Params P, long long *probe)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    keys[it] = it;
    keys[it + kIters] = P.maxk - it;
    for (int i = 0; i < kTests; i++) probe[i] = keys[P.index[i]];
}

__global__ void __launch_bounds__(kThreads) k_hist(const int32_t *__restrict__ keys, long long n,
                                                   unsigned *counts)
{
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x)
        atomicAdd(&counts[keys[j]], 1u);
}

// Inclusive scan of a block's values in shared memory (kThreads values).
__device__ __forceinline__ unsigned block_scan(unsigned v, unsigned *sh)
{
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        unsigned s = lane < kThreads / 32 ? sh[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kThreads / 32) sh[lane] = s;
    }
    __syncthreads();
    const unsigned before = w > 0 ? sh[w - 1] : 0u;
    __syncthreads();
    return v + before;
}

// Phase 1: each CTA scans its tile in place (inclusive) and publishes the
// tile's total.
__global__ void __launch_bounds__(kThreads) k_scan_tiles(unsigned *v, int len, unsigned *totals)
{
    __shared__ unsigned sh[32];
    const long long base = (long long)blockIdx.x * kTileVals + (long long)threadIdx.x * kItems;
    unsigned x[kItems], run = 0;
#pragma unroll
    for (int i = 0; i < kItems; i++) {
        x[i] = base + i < len ? v[base + i] : 0u;
        run += x[i];
        x[i] = run;
    }
    const unsigned before = block_scan(run, sh) - run;
#pragma unroll
    for (int i = 0; i < kItems; i++)
        if (base + i < len) v[base + i] = x[i] + before;
    if (threadIdx.x == kThreads - 1) totals[blockIdx.x] = before + run;
}

// Phase 2: one CTA turns the tile totals into exclusive offsets.
__global__ void __launch_bounds__(kThreads) k_scan_totals(unsigned *totals, int tiles)
{
    __shared__ unsigned sh[32];
    __shared__ unsigned last;
    unsigned carry = 0;
    for (int b0 = 0; b0 < tiles; b0 += kThreads) {
        const int b = b0 + threadIdx.x;
        const unsigned v = b < tiles ? totals[b] : 0u;
        const unsigned inc = block_scan(v, sh);
        if (b < tiles) totals[b] = carry + inc - v;
        if (threadIdx.x == kThreads - 1) last = inc;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
}

// Phase 3: every tile but the first adds its offset.
__global__ void __launch_bounds__(kThreads) k_scan_add(unsigned *v, int len, const unsigned *offsets)
{
    if (blockIdx.x == 0) return;
    const unsigned off = offsets[blockIdx.x];
    const long long base = (long long)blockIdx.x * kTileVals + (long long)threadIdx.x * kItems;
#pragma unroll
    for (int i = 0; i < kItems; i++)
        if (base + i < len) v[base + i] += off;
}

// Expected rank of test key i at iteration it (rank_gpu_kernel_7's table).
__device__ __forceinline__ long long expected_rank(char cls, int i, long long base, long long it)
{
    switch (cls) {
    case 'S': return i <= 2 ? base + it : base - it;
    case 'W': return i < 2 ? base + (it - 2) : base - it;
    case 'A': return i <= 2 ? base + (it - 1) : base - (it - 1);
    case 'B': return (i == 1 || i == 2 || i == 4) ? base + it : base - it;
    case 'C': return i <= 2 ? base + it : base - it;
    default: return i < 2 ? base + it : base - it;
    }
}

__global__ void k_check(const unsigned *counts, const long long *probe, Params P, int it,
                        unsigned long long *passed)
{
    if (blockIdx.x != 0 || threadIdx.x != 0 || P.cls == 'U') return;
    unsigned long long ok = 0;
    for (int i = 0; i < kTests; i++) {
        const long long k = probe[i];
        if (0 < k && k <= P.n - 1 && (long long)counts[k - 1] == expected_rank(P.cls, i, P.rank[i], it)) ok++;
    }
    *passed += ok;
}

// Full verification: each key placed by the running sums (the sorted keys
// whatever the atomics' order), then the out-of-order neighbours counted.
__global__ void __launch_bounds__(kThreads) k_scatter(const int32_t *__restrict__ keys, long long n,
                                                      unsigned *counts, int32_t *sorted)
{
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const int32_t v = keys[j];
        const unsigned at = atomicSub(&counts[v], 1u) - 1u;
        sorted[at] = v;
    }
}

__global__ void __launch_bounds__(kThreads) k_disorder(const int32_t *__restrict__ sorted, long long n,
                                                       unsigned long long *bad)
{
    unsigned long long mine = 0;
    for (long long j = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x)
        mine += sorted[j - 1] > sorted[j];
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(bad, mine);
}

}  // namespace is
}  // namespace cgb

using namespace cgb;
using namespace cgb::is;

struct cgb_is {
    int device = 0, sms = 148;
    Params P{};
    int32_t *keys = nullptr, *sorted = nullptr, *backup = nullptr;  // backup: keys[0 .. 2 kIters]
    unsigned *counts = nullptr, *totals = nullptr;
    long long *probe = nullptr;
    unsigned long long *passed = nullptr, *bad = nullptr;
    int tiles = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

#define IS_TRY(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(e_ == cudaErrorMemoryAllocation ? CGB_ERR_NOMEM : CGB_ERR_CUDA, \
                             "is: %s: %s", #call, cudaGetErrorString(e_));                \
    } while (0)

void is_release(cgb_is *s)
{
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    for (void *p : {(void *)s->keys, (void *)s->sorted, (void *)s->backup, (void *)s->counts,
                    (void *)s->totals, (void *)s->probe, (void *)s->passed, (void *)s->bad})
        if (p) cudaFree(p);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// One ranking pass (rank_gpu, is.cu:725-800) at iteration it.
void enqueue_rank(cgb_is *s, int it)
{
    const cudaStream_t st = s->stream;
    k_prep<<<1, 32, 0, st>>>(s->keys, it, s->P, s->probe);
    cudaMemsetAsync(s->counts, 0, sizeof(unsigned) * size_t(s->P.maxk), st);
    k_hist<<<8 * s->sms, kThreads, 0, st>>>(s->keys, s->P.n, s->counts);
    k_scan_tiles<<<s->tiles, kThreads, 0, st>>>(s->counts, s->P.maxk, s->totals);
    k_scan_totals<<<1, kThreads, 0, st>>>(s->totals, s->tiles);
    k_scan_add<<<s->tiles, kThreads, 0, st>>>(s->counts, s->P.maxk, s->totals);
    k_check<<<1, 32, 0, st>>>(s->counts, s->probe, s->P, it, s->passed);
}

}  // namespace

extern "C" {

int cgb_is_create(int device, char cls, int total_log2, int max_log2, cgb_is **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "is: null output");
    *out = nullptr;
    Params P{};
    P.cls = cls;
    if (cls != 'U') {
        const ClassTable *c = nullptr;
        for (const auto &t : kClasses)
            if (t.name == cls) c = &t;
        if (!c) return set_error(CGB_ERR_INVALID, "is: class must be S, W, A, B, C, D or U");
        if (c->total_log2 != total_log2 || c->max_log2 != max_log2)
            return set_error(CGB_ERR_INVALID, "is: class %c is 2^%d keys below 2^%d", cls, c->total_log2,
                             c->max_log2);
        std::memcpy(P.index, c->index, sizeof(P.index));
        std::memcpy(P.rank, c->rank, sizeof(P.rank));
    }
    if (total_log2 < 12 || total_log2 > 31 || max_log2 < 8 || max_log2 > 27)
        return set_error(CGB_ERR_INVALID, "is: 2^12 .. 2^31 keys below 2^8 .. 2^27");
    P.n = 1LL << total_log2;
    P.maxk = 1 << max_log2;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "is: no CUDA device %d", device);
    int major = 0;
    IS_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    if (major != 10) return set_error(CGB_ERR_NO_DEVICE, "is: device %d is not sm_100", device);
    IS_TRY(cudaSetDevice(device));
    cgb_is *s = new (std::nothrow) cgb_is;
    if (!s) return set_error(CGB_ERR_NOMEM, "is: allocation failed");
    s->device = device;
    s->P = P;
    IS_TRY(cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device));
    s->tiles = (P.maxk + kTileVals - 1) / kTileVals;
    const bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess &&
                    cudaEventCreate(&s->ev0) == cudaSuccess && cudaEventCreate(&s->ev1) == cudaSuccess &&
                    cudaMalloc(&s->keys, sizeof(int32_t) * size_t(P.n)) == cudaSuccess &&
                    cudaMalloc(&s->sorted, sizeof(int32_t) * size_t(P.n)) == cudaSuccess &&
                    cudaMalloc(&s->backup, sizeof(int32_t) * (2 * kIters + 1)) == cudaSuccess &&
                    cudaMalloc(&s->counts, sizeof(unsigned) * size_t(P.maxk)) == cudaSuccess &&
                    cudaMalloc(&s->totals, sizeof(unsigned) * size_t(s->tiles)) == cudaSuccess &&
                    cudaMalloc(&s->probe, sizeof(long long) * kTests) == cudaSuccess &&
                    cudaMalloc(&s->passed, sizeof(unsigned long long)) == cudaSuccess &&
                    cudaMalloc(&s->bad, sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
        is_release(s);
        return set_error(CGB_ERR_NOMEM, "is: device allocation failed (2^%d keys)", total_log2);
    }
    const long long gen_threads = (P.n + kKeysPerThread - 1) / kKeysPerThread;
    k_keys<<<unsigned((gen_threads + kThreads - 1) / kThreads), kThreads, 0, s->stream>>>(
        s->keys, P.n, double(P.maxk) / 4.0);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(s->backup, s->keys, sizeof(int32_t) * (2 * kIters + 1), cudaMemcpyDeviceToDevice,
                        s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess) {
        is_release(s);
        return set_error(CGB_ERR_CUDA, "is: key generation failed");
    }
    *out = s;
    return CGB_OK;
}

int cgb_is_destroy(cgb_is *s)
{
    is_release(s);
    return CGB_OK;
}

int cgb_is_run(cgb_is *s, long long *passed, double *device_ms)
{
    if (!s) return set_error(CGB_ERR_INVALID, "is: null instance");
    IS_TRY(cudaSetDevice(s->device));
    const cudaStream_t st = s->stream;
    if (!s->exec) {
        // the timed region (is.cu:413-440): ranking passes 1 .. 10
        cudaGraph_t graph = nullptr;
        IS_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int it = 1; it <= kIters; it++) enqueue_rank(s, it);
        const cudaError_t e1 = cudaGetLastError();
        const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return set_error(CGB_ERR_CUDA, "is: capture failed");
        }
        const cudaError_t e3 = cudaGraphInstantiate(&s->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e3 != cudaSuccess) {
            s->exec = nullptr;
            return set_error(CGB_ERR_CUDA, "is: graph instantiation failed");
        }
    }
    // the generated keys back (a run rewrites keys 1 .. 20), then main's
    // untimed pass rank(1) and the reset of the passed count
    IS_TRY(cudaMemcpyAsync(s->keys, s->backup, sizeof(int32_t) * (2 * kIters + 1), cudaMemcpyDeviceToDevice, st));
    IS_TRY(cudaMemsetAsync(s->passed, 0, sizeof(unsigned long long), st));
    enqueue_rank(s, 1);
    IS_TRY(cudaGetLastError());
    IS_TRY(cudaMemsetAsync(s->passed, 0, sizeof(unsigned long long), st));
    IS_TRY(cudaEventRecord(s->ev0, st));
    IS_TRY(cudaGraphLaunch(s->exec, st));
    IS_TRY(cudaEventRecord(s->ev1, st));
    // full verification (untimed, as the reference's)
    IS_TRY(cudaMemsetAsync(s->bad, 0, sizeof(unsigned long long), st));
    k_scatter<<<8 * s->sms, kThreads, 0, st>>>(s->keys, s->P.n, s->counts, s->sorted);
    k_disorder<<<8 * s->sms, kThreads, 0, st>>>(s->sorted, s->P.n, s->bad);
    IS_TRY(cudaGetLastError());
    unsigned long long h_passed = 0, h_bad = 0;
    IS_TRY(cudaMemcpyAsync(&h_passed, s->passed, sizeof(h_passed), cudaMemcpyDeviceToHost, st));
    IS_TRY(cudaMemcpyAsync(&h_bad, s->bad, sizeof(h_bad), cudaMemcpyDeviceToHost, st));
    IS_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    IS_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    if (passed) *passed = (long long)h_passed + (h_bad == 0 ? 1 : 0);
    if (device_ms) *device_ms = ms;
    return CGB_OK;
}

int cgb_is_read(cgb_is *s, int which, void *out, long long count)
{
    if (!s || !out || which < 0 || which > 2) return set_error(CGB_ERR_INVALID, "is: bad read");
    const long long need = which == 1 ? s->P.maxk : s->P.n;
    if (count < need) return set_error(CGB_ERR_CAPACITY, "is: %lld values needed", need);
    IS_TRY(cudaSetDevice(s->device));
    const void *src = which == 0 ? (const void *)s->keys : which == 1 ? (const void *)s->counts
                                                                       : (const void *)s->sorted;
    IS_TRY(cudaMemcpy(out, src, 4 * size_t(need), cudaMemcpyDeviceToHost));
    return CGB_OK;
}

}  // extern "C"

// ep.cu -- the NPB EP benchmark on the GPU: 2^m pairs of uniform deviates
// from one linear congruential stream, the pairs inside the unit disc turned
// into Gaussian deviates, their sums and counts in square annuli
// (GMAP/NPB-GPU CUDA/EP/ep.cu: main :114-275, gpu_kernel :276-350).
//
// The reference gives each of its 2^(m-16) threads one batch of 2^16 pairs,
// seeded S * an^kk with an = A^(2^17).  The stream is the same whichever way
// it is cut -- pair p is draws 2p + 1 and 2p + 2 after the seed S -- so here
// each thread jumps straight to its own run of pairs (A^k by squaring, in
// exact 64-bit integer arithmetic mod 2^46) and the grid holds about 2^20
// threads whatever the class, all SMs busy instead of 2^(m-16) threads.
// Each uniform is x * 2^-46, exactly the reference's value.
//
// Sums: a thread adds its pairs in order; a block adds its threads by a
// fixed tree; the last block (ticket) adds the blocks in order -- the same
// result on every run (the reference adds with atomics, in no fixed order).
// Counts are integers, summed exactly.  This file is compiled with
// -fmad=false: every product and sum rounds separately, as in the
// reference's serial code; log and sqrt are CUDA's double-precision ones.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "cgb_internal.h"

namespace cgb {
namespace ep {

constexpr int kMK = 16;  // log2 of the reference's pairs a batch (ep.cu:65)
constexpr int kNQ = 10;  // annuli (ep.cu:69)
constexpr int kThreads = 256;
constexpr uint64_t kMask46 = (uint64_t(1) << 46) - 1;
constexpr uint64_t kMult = 1220703125ull;  // A = 5^13 (ep.cu:71)
constexpr uint64_t kSeed = 271828183ull;   // S (ep.cu:72)

__device__ __forceinline__ uint64_t lcg_mul(uint64_t a, uint64_t b) { return (a * b) & kMask46; }

// kSeed * kMult^e mod 2^46
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

// Thread g takes pairs [g chunk, (g + 1) chunk).  The pairs inside the
// disc are compacted per warp before their deviates are formed: each lane
// draws one pair a step, the accepted ones go to the warp's queue in shared
// memory (ballot order), and whenever 32 are queued every lane forms one
// deviate pair -- so no lane of a log idles on a rejected pair (about 21 %
// of them).  part: per block sx, sy, then kNQ counts (as doubles, exact
// below 2^53).
constexpr int kQueue = 64;  // a warp's queue: up to 31 waiting + 32 arriving

__global__ void __launch_bounds__(kThreads) k_ep(int log_chunk, double *part, unsigned *ticket, double *out)
{
    __shared__ double ssx[kThreads], ssy[kThreads];
    __shared__ unsigned long long sq[kNQ][kThreads];
    __shared__ double qx1[kThreads / 32][kQueue], qx2[kThreads / 32][kQueue], qt[kThreads / 32][kQueue];
    __shared__ bool last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t g = uint64_t(blockIdx.x) * kThreads + tid;
    const long long chunk = 1LL << log_chunk;
    uint64_t x = jump(2 * (g << log_chunk));  // the seed before this thread's first pair
    double sx = 0.0, sy = 0.0;
    unsigned q[kNQ];
#pragma unroll
    for (int k = 0; k < kNQ; k++) q[k] = 0;
    double *wx1 = qx1[warp], *wx2 = qx2[warp], *wt = qt[warp];
    int queued = 0;  // the same in every lane of the warp
    auto deviates = [&](double x1, double x2, double t) {
        const double f = sqrt(-2.0 * log(t) / t);
        const double t3 = x1 * f, t4 = x2 * f;
        const int l = int(fmax(fabs(t3), fabs(t4)));
#pragma unroll
        for (int k = 0; k < kNQ; k++) q[k] += (l == k) ? 1u : 0u;
        sx = sx + t3;
        sy = sy + t4;
    };
    for (long long i = 0; i < chunk; i++) {
        x = lcg_mul(x, kMult);
        const double u1 = double(x) * 0x1p-46;
        x = lcg_mul(x, kMult);
        const double u2 = double(x) * 0x1p-46;
        const double x1 = 2.0 * u1 - 1.0, x2 = 2.0 * u2 - 1.0;
        const double t = x1 * x1 + x2 * x2;
        const bool keep = t <= 1.0;
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int at = queued + __popc(mask & ((1u << lane) - 1u));
            wx1[at] = x1;
            wx2[at] = x2;
            wt[at] = t;
        }
        queued += __popc(mask);
        __syncwarp();
        if (queued >= 32) {  // the newest 32: one per lane
            const int at = queued - 32 + lane;
            deviates(wx1[at], wx2[at], wt[at]);
            queued -= 32;
            __syncwarp();
        }
    }
    if (lane < queued) deviates(wx1[lane], wx2[lane], wt[lane]);
    ssx[tid] = sx;
    ssy[tid] = sy;
#pragma unroll
    for (int k = 0; k < kNQ; k++) sq[k][tid] = q[k];
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (tid < w) {
            ssx[tid] = ssx[tid] + ssx[tid + w];
            ssy[tid] = ssy[tid] + ssy[tid + w];
#pragma unroll
            for (int k = 0; k < kNQ; k++) sq[k][tid] += sq[k][tid + w];
        }
        __syncthreads();
    }
    if (tid == 0) {
        double *p = part + size_t(blockIdx.x) * (2 + kNQ);
        p[0] = ssx[0];
        p[1] = ssy[0];
        for (int k = 0; k < kNQ; k++) p[2 + k] = double(sq[k][0]);
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && tid == 0) {
        __threadfence();
        double acc[2 + kNQ] = {};
        for (unsigned b = 0; b < gridDim.x; b++)
            for (int k = 0; k < 2 + kNQ; k++) acc[k] = acc[k] + __ldcg(part + size_t(b) * (2 + kNQ) + k);
        for (int k = 0; k < 2 + kNQ; k++) out[k] = acc[k];
        *ticket = 0u;
    }
}

}  // namespace ep
}  // namespace cgb

using namespace cgb;
using namespace cgb::ep;

extern "C" int cgb_ep_run(int device, int m, double *sx, double *sy, double *q, double *device_ms)
{
    if (m < 20 || m > 40) return set_error(CGB_ERR_INVALID, "ep: m must be in [20, 40] (2^m pairs)");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "ep: no CUDA device %d", device);
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess || major != 10)
        return set_error(CGB_ERR_NO_DEVICE, "ep: device %d is not sm_100", device);
    if (cudaSetDevice(device) != cudaSuccess) return set_error(CGB_ERR_CUDA, "ep: cudaSetDevice failed");
    // about 2^20 threads: each takes 2^(m - 20) pairs (at least 2^8)
    const int log_chunk = std::max(8, m - 20);
    const long long threads = 1LL << (m - log_chunk);
    const unsigned blocks = unsigned(threads / kThreads);
    double *part = nullptr, *out = nullptr;
    unsigned *ticket = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = CGB_OK;
    if (cudaMalloc(&part, sizeof(double) * (2 + kNQ) * blocks) != cudaSuccess ||
        cudaMalloc(&out, sizeof(double) * (2 + kNQ)) != cudaSuccess ||
        cudaMalloc(&ticket, sizeof(unsigned)) != cudaSuccess || cudaMemset(ticket, 0, sizeof(unsigned)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        st = set_error(CGB_ERR_NOMEM, "ep: buffers");
    double h[2 + kNQ] = {};
    float ms = 0.f;
    if (!st) {
        cudaEventRecord(e0);
        k_ep<<<blocks, kThreads>>>(log_chunk, part, ticket, out);
        cudaEventRecord(e1);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaMemcpy(h, out, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            st = set_error(CGB_ERR_CUDA, "ep: the kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    for (void *p : {(void *)part, (void *)out, (void *)ticket})
        if (p) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) return st;
    if (sx) *sx = h[0];
    if (sy) *sy = h[1];
    if (q) std::memcpy(q, h + 2, sizeof(double) * kNQ);
    if (device_ms) *device_ms = ms;
    return CGB_OK;
}

// device_common.cuh -- device building blocks shared by the CG kernels:
// bounded grid barrier, deterministic block/grid reductions, streaming loads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cgb {

// Device status word values (first failure wins; 0 = none).
constexpr int kDevOk = 0;
constexpr int kDevTimeout = 1;    // a grid-barrier wait ran past its limit
constexpr int kDevNonFinite = 2;  // a reduction produced NaN/Inf
constexpr int kDevBadShape = 3;   // launch shape does not match the session

// Checked build (-DCGB_CHECKED, lib/libcgb_checked.so): every gather and
// stream index of the SpMVs is tested against its buffer; a failure sets
// this translation unit's check word (first failure wins, read by
// cgb_check_status) and the access is skipped -- never a trap.  In the
// normal build the test compiles to nothing.
#ifdef CGB_CHECKED
static __device__ int g_check_word;
__device__ __forceinline__ bool cgb_in_range(long long i, long long n, int code)
{
    if (i >= 0 && i < n) return true;
    atomicCAS(&g_check_word, 0, code);
    return false;
}
#define CGB_IN_RANGE(i, n, code) cgb_in_range((long long)(i), (long long)(n), (code))
#else
#define CGB_IN_RANGE(i, n, code) true
#endif
// check codes: which index left its buffer
constexpr int kCheckStream = 1;   // matrix stream entry (values / columns)
constexpr int kCheckGather = 2;   // gathered vector index (column)
constexpr int kCheckRow = 3;      // output / accumulator row
constexpr int kCheckSplit = 4;    // row range of a CTA

// State of the grid barrier: one 64-bit count of arrivals that only grows.
// A grid of G CTAs passes barrier j when the count reaches a multiple of G,
// so the count is a multiple of G between launches; the host zeroes it when
// the grid size changes (a new plan) and after a failed launch.
struct GridBarrier {
    unsigned long long *arrivals;  // CTAs arrived, over all barriers so far
    int *status;                   // device status word
    long long limit_ns;            // wait limit per barrier
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned *p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(p), "r"(v)
                 : "memory");
    return old;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p,
                                                                   unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;"
                 : "=l"(old)
                 : "l"(p), "l"(v)
                 : "memory");
    return old;
}

__device__ __forceinline__ int ld_relaxed_i32(const int *p)
{
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void raise_status(int *status, int code)
{
    atomicCAS(status, kDevOk, code);
}

// Barrier of `members` co-resident CTAs over a 64-bit count of arrivals
// that only grows (the whole grid for grid_barrier; the CTAs of one
// system's team in the batch kernel).  Thread 0 of each CTA adds its
// arrival with an acq_rel atomic, which also tells it the target (the next
// multiple of `members`); the last arriver goes on at once, the others poll
// the count with acquire loads until it reaches the target.  Every arrival
// is a release, so a CTA that sees the target sees every write made before
// the barrier by any member.  One atomic and the polls are the whole cost
// (no generation word to publish after the count): 1.36 against 2.19 us a
// barrier for 148 CTAs.  The count must be a multiple of `members` when
// the members first use it (zeroed by the host for a new grid size or
// team, and after a failed launch).  Every wait is bounded: past
// `limit_ns`, or as soon as another CTA has raised the status word, the
// barrier records kDevTimeout (first failure wins) and returns false; the
// caller then leaves the kernel.
__device__ __forceinline__ bool counted_barrier(unsigned long long *arrivals, unsigned members,
                                                int *status, long long limit_ns)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned long long g = members;
        const unsigned long long old = atom_add_acq_rel_u64(arrivals, 1ull);
        const unsigned long long target = (old / g + 1ull) * g;
        if (old + 1ull != target) {
            const unsigned long long t0 = global_ns();
            unsigned spins = 0;
            while (ld_acquire_u64(arrivals) < target) {
                if (((++spins) & 63u) == 0u) {
                    if (ld_relaxed_i32(status) != kDevOk) {
                        ok = 0;
                        break;
                    }
                    if ((long long)(global_ns() - t0) > limit_ns) {
                        raise_status(status, kDevTimeout);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid-wide barrier for a co-resident (cooperative) grid.
__device__ __forceinline__ bool grid_barrier(const GridBarrier &gb)
{
    return counted_barrier(gb.arrivals, gridDim.x, gb.status, gb.limit_ns);
}

template <int W>
__device__ __forceinline__ double group_sum(double v, unsigned mask)
{
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
    return v;
}

template <int W>
__device__ __forceinline__ float group_sum_f(float v, unsigned mask)
{
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
    return v;
}

__device__ __forceinline__ double warp_sum(double v) { return group_sum<32>(v, 0xffffffffu); }

// group_sum / group_sum_f for a group width w (a power of two <= 32) known
// only at run time: the same xor steps in the same order, so the same sums.
__device__ __forceinline__ double group_sum_rt(double v, unsigned mask, int w)
{
    for (int off = w >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
    return v;
}

__device__ __forceinline__ float group_sum_f_rt(float v, unsigned mask, int w)
{
    for (int off = w >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
    return v;
}

// Sum of `v` over the CTA, valid in thread 0.  `scratch` holds >= 32 doubles.
// Fixed shuffle/smem order: deterministic for a given launch shape.
__device__ __forceinline__ double block_sum(double v, double *scratch)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) scratch[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = (l < int(blockDim.x >> 5)) ? scratch[l] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

// Sum of the `nparts` per-CTA partials at `part`, computed identically by
// every CTA (same order), returned to all threads through `bcast`.  Reads go
// to L2 (ld.cg): the partials were written by other SMs during this launch.
// The loads of a lane's partials are all issued before the first add (one
// L2 round trip instead of one per partial); the adds keep the order
// part[lane] + part[lane + 32] + ..., so the sum is the same in every CTA.
__device__ __forceinline__ double all_partials(const double *part, int nparts, double *bcast)
{
    if (threadIdx.x < 32) {
        constexpr int kAhead = 8;  // 256 partials in one round trip
        double v[kAhead];
#pragma unroll
        for (int u = 0; u < kAhead; u++) {
            const int i = int(threadIdx.x) + 32 * u;
            v[u] = i < nparts ? __ldcg(part + i) : 0.0;
        }
        double s = 0.0;
#pragma unroll
        for (int u = 0; u < kAhead; u++)
            if (int(threadIdx.x) + 32 * u < nparts) s += v[u];
        for (int i = int(threadIdx.x) + 32 * kAhead; i < nparts; i += 32) s += __ldcg(part + i);
        s = warp_sum(s);
        if (threadIdx.x == 0) *bcast = s;
    }
    __syncthreads();
    return *bcast;
}

// Streaming (evict-first) loads for data read once per pass: the matrix.
__device__ __forceinline__ double2 ld_stream(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ int2 ld_stream(const int2 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 ld_stream(const float2 *p) { return __ldcs(p); }

// ---------------------------------------------- bulk copies and mbarriers
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Orders this thread's earlier generic-proxy accesses (and those it has
// observed) before its later async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async;" ::: "memory");
}

// 1-D bulk copy global -> shared completing on `bar`; issued by one thread.
// src, dst 16-byte aligned, bytes a multiple of 16.  Never multicast.
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

// Bounded wait for phase `parity` of `bar`; gives up after limit_ns or when
// *abort is set by another warp of the CTA.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, long long limit_ns,
                                          volatile int *abort)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (abort && *abort) return false;
        if ((long long)(global_ns() - t0) > limit_ns) return false;
    }
    return true;
}

}  // namespace cgb

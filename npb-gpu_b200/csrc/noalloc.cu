// noalloc.cu -- cgb_conj_grad_noalloc: the conj_grad solve for callers that
// cannot allocate GPU memory.
//
// Some hosts forbid device allocation on the path that calls us: an
// application whose device memory is all handed out up front by its own
// pool, a plugin whose memory budget the host process polices, or a loop
// that must not allocate at all (an allocation can synchronise the device
// or fail late).  Those callers still own their inputs and outputs; what the
// solver needs beyond them -- the p, q, r work vectors, per-CTA partial
// sums, the grid-barrier words, the row split -- lives here in one
// file-scope __device__ array of fixed size, so this entry point never calls
// cudaMalloc, cudaFree or any allocating library routine.
//
// Limits and sharing:
//   * n <= kNoallocMaxN (the work vectors' capacity); larger systems are
//     rejected with CGB_ERR_CAPACITY.  The array (about 6.3 MB) is held on
//     every GPU that loads the library until the process exits.
//   * Every call on a device uses the same array and leaves its contents
//     behind; the call clears the words that must start at zero.  Calls that
//     overlap on the GPU (two streams, or two host threads) race on the
//     array: serialise them.
//   * The first call on a device (per CUDA context) looks the array's device
//     address up (cudaGetSymbolAddress) with that device current, and caches
//     it with the SM count and the kernels' occupancy; make that first call
//     before any stream capture.
//   * The call is asynchronous: *d_rnorm and *d_status are written on the
//     stream; synchronise it before reading them.  A solve that gave up on a
//     wait leaves *d_rnorm NaN and *d_status nonzero.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "cg_kernels.cuh"
#include "cgb_internal.h"

namespace cgb {
namespace {

constexpr int kNoallocMaxN = 262144;       // largest order served (NPB classes S..C fit)
constexpr int kNoallocMaxGrid = 1024;      // CTAs of the cooperative launch
constexpr size_t kLine = 256;
constexpr size_t kHeaderBytes = 4 * kLine;  // barrier arrivals, (spare), status, trace
constexpr size_t kSplitBytes = ((kNoallocMaxGrid + 1) * sizeof(int) + kLine - 1) / kLine * kLine;
// the fixed-count FP64 kernel uses the slots below kSlotGram only
constexpr size_t kPartBytes = size_t(kSlotGram) * kNoallocMaxGrid * sizeof(double);
constexpr size_t kVecDoubles = size_t(kNoallocMaxN) + 64;
constexpr size_t kScratchBytes = kHeaderBytes + kSplitBytes + kPartBytes + 3 * kVecDoubles * sizeof(double);

}  // namespace

// The scratch array.  In host code this name is only a stand-in for the
// symbol: kernels must be given the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// What a call needs to know about the current device, looked up once per
// CUDA context (set-up) and kept: the scratch array's device address, the
// SM count and how many CTAs of each kernel instance fit on an SM.  The key
// is the context's unique id (cuCtxGetId), so a context created after a
// cudaDeviceReset -- where the library's module, and with it the array,
// is loaded again and may move -- or a driver-API context of the caller's
// gets its own set-up instead of a stale address.
using RowKernel = void (*)(OuterArgs);
constexpr int kNoallocInstances = 4;  // outer_step_fp64<16>, <8>, <4>, <2>

RowKernel noalloc_instance(int i)
{
    switch (i) {
    case 0: return outer_step_fp64<16>;
    case 1: return outer_step_fp64<8>;
    case 2: return outer_step_fp64<4>;
    default: return outer_step_fp64<2>;
    }
}

// lanes per row from the mean row length (instance index above)
int noalloc_pick(double mean_len)
{
    if (mean_len >= 40.0) return 0;
    if (mean_len >= 16.0) return 1;
    if (mean_len >= 6.0) return 2;
    return 3;
}

struct DeviceSetup {
    bool valid = false;
    unsigned long long ctx_id = 0;
    unsigned char *scratch = nullptr;
    int sm_count = 0;
    int per_sm[kNoallocInstances] = {};
};

std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// The calling thread's current context id (0 when no context is current or
// the driver entry points are unavailable; the cache is then per device).
unsigned long long current_ctx_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Set-up of `device` (current on this thread) for the current context: the
// scratch array's device address (cudaGetSymbolAddress, which also makes
// the context current if none was), the compute capability check, the SM
// count and the occupancy of each kernel instance.  Nothing here allocates.
int device_setup(int device, DeviceSetup *out)
{
    if (device < 0 || device >= 64) return set_error(CGB_ERR_NO_DEVICE, "device %d unsupported", device);
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup &d = g_setup[device];
    const unsigned long long id = current_ctx_id();
    if (d.valid && id == d.ctx_id && id != 0) {
        *out = d;
        return CGB_OK;
    }
    if (d.valid && id == 0 && d.ctx_id == 0) {  // no context ids: per device
        *out = d;
        return CGB_OK;
    }
    int major = 0, sms = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
        major != 10)
        return set_error(CGB_ERR_NO_DEVICE, "current device is not sm_100");
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1)
        return set_error(CGB_ERR_NO_DEVICE, "SM count query failed");
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
        return set_error(CGB_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    DeviceSetup fresh;
    fresh.scratch = static_cast<unsigned char *>(p);
    fresh.sm_count = sms;
    for (int i = 0; i < kNoallocInstances; i++) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, noalloc_instance(i), 512, 0) !=
                cudaSuccess ||
            per_sm < 1)
            return set_error(CGB_ERR_CUDA, "noalloc conj_grad: kernel cannot be resident");
        fresh.per_sm[i] = per_sm;
    }
    fresh.ctx_id = current_ctx_id();  // the context is current now
    fresh.valid = true;
    d = fresh;
    *out = d;
    return CGB_OK;
}

// Row split balancing (entries + 8 per row) over `grid` CTAs, on the device,
// from the caller's row pointers.
__global__ void noalloc_split(const int *__restrict__ rowstr, int n, int grid, int *split)
{
    const double total = double(rowstr[n]) + 8.0 * n;
    for (int c = threadIdx.x; c <= grid; c += blockDim.x) {
        if (c == 0) { split[0] = 0; continue; }
        if (c == grid) { split[grid] = n; continue; }
        const double target = total * c / grid;
        int lo = 0, hi = n;  // first j with rowstr[j] + 8 j >= target
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (double(rowstr[mid]) + 8.0 * mid < target) lo = mid + 1;
            else hi = mid;
        }
        split[c] = lo;
    }
}

}  // namespace
}  // namespace cgb

using namespace cgb;

extern "C" int cgb_conj_grad_noalloc(int n, long long nnz, const int *d_rowstr, const int *d_colidx,
                                     const double *d_a, const double *d_x, double *d_z,
                                     double *d_rnorm, int *d_status, void *stream)
{
    if (n < 1 || nnz < 0 || !d_rowstr || !d_colidx || !d_a || !d_x || !d_z || !d_rnorm)
        return set_error(CGB_ERR_INVALID, "noalloc conj_grad: null pointer or bad size");
    if (n > kNoallocMaxN)
        return set_error(CGB_ERR_CAPACITY,
                         "noalloc conj_grad: n = %d exceeds the scratch capacity of %d rows", n,
                         kNoallocMaxN);
    // the SpMV reads entry pairs (16-byte value loads, 8-byte index loads)
    if (reinterpret_cast<uintptr_t>(d_a) % 16 != 0 || reinterpret_cast<uintptr_t>(d_colidx) % 8 != 0)
        return set_error(CGB_ERR_INVALID,
                         "noalloc conj_grad: d_a must be 16-byte and d_colidx 8-byte aligned");
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess)
        return set_error(CGB_ERR_NO_DEVICE, "no current CUDA device");
    DeviceSetup dev;
    int st = device_setup(device, &dev);
    if (st) return st;
    unsigned char *base = dev.scratch;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    const int pick = noalloc_pick(double(nnz) / double(n));
    RowKernel kernel = noalloc_instance(pick);
    const int grid = std::max(1, std::min({dev.per_sm[pick] * dev.sm_count, n, kNoallocMaxGrid}));

    unsigned long long *arrivals = reinterpret_cast<unsigned long long *>(base);
    int *status = reinterpret_cast<int *>(base + 2 * kLine);
    StepTrace *trace = reinterpret_cast<StepTrace *>(base + 3 * kLine);
    int *split = reinterpret_cast<int *>(base + kHeaderBytes);
    double *part = reinterpret_cast<double *>(base + kHeaderBytes + kSplitBytes);
    double *vec = reinterpret_cast<double *>(base + kHeaderBytes + kSplitBytes + kPartBytes);

    // barrier words and status must start at zero.  The trace record starts
    // as NaN bytes: a solve that leaves early (a failed wait) never writes
    // it, so *d_rnorm then reads NaN rather than a stale or zero residual.
    // Everything else is written before it is read.
    if (cudaMemsetAsync(base, 0, 3 * kLine, s) != cudaSuccess ||
        cudaMemsetAsync(base + 3 * kLine, 0xff, kLine, s) != cudaSuccess)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad: clearing the scratch header failed");
    noalloc_split<<<1, 256, 0, s>>>(d_rowstr, n, grid, split);
    if (cudaGetLastError() != cudaSuccess)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad: split launch failed");

    OuterArgs A{};
    A.n = n;
    A.M.rowstr = d_rowstr;
    A.M.colidx = d_colidx;
    A.M.a = d_a;
    A.M.csr_entries = nnz;  // the caller's arrays: no padding after them
    A.M.ncols = n;
    A.x = const_cast<double *>(d_x);  // read only: finish = 0 leaves x untouched
    A.z = d_z;
    A.p = vec;
    A.q = vec + kVecDoubles;
    A.r = vec + 2 * kVecDoubles;
    A.row_split = split;
    A.part = part;
    A.gpad = kNoallocMaxGrid;
    A.gb.arrivals = arrivals;
    A.gb.status = status;
    A.gb.limit_ns = 2000000000LL;
    A.shift = 0.0;
    A.cgitmax = 25;  // cgitmax of the reference (cg.cu:666)
    A.fixed = 1;
    A.tol = 0.0;
    A.step = 0;
    A.finish = 0;
    A.trace = trace;

    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(512);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, A);
    if (e != cudaSuccess)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad launch failed: %s", cudaGetErrorString(e));
    if (cudaMemcpyAsync(d_rnorm, &trace->rnorm, sizeof(double), cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad: rnorm copy failed");
    if (d_status &&
        cudaMemcpyAsync(d_status, status, sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad: status copy failed");
    return CGB_OK;
}

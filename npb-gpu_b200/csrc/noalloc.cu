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
//   * The first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
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

std::mutex g_scratch_mu;
void *g_scratch_addr[64];

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
int scratch_address(int device, unsigned char **out)
{
    if (device < 0 || device >= 64) return set_error(CGB_ERR_NO_DEVICE, "device %d unsupported", device);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return set_error(CGB_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                             cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[device]);
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

using RowKernel = void (*)(OuterArgs);

RowKernel noalloc_kernel(double mean_len)
{
    if (mean_len >= 96.0) return outer_step_fp64<16>;
    if (mean_len >= 40.0) return outer_step_fp64<16>;
    if (mean_len >= 16.0) return outer_step_fp64<8>;
    if (mean_len >= 6.0) return outer_step_fp64<4>;
    return outer_step_fp64<2>;
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
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10)
        return set_error(CGB_ERR_NO_DEVICE, "current device is not sm_100");
    unsigned char *base = nullptr;
    int st = scratch_address(device, &base);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    RowKernel kernel = noalloc_kernel(double(nnz) / double(n));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 512, 0) != cudaSuccess ||
        per_sm < 1)
        return set_error(CGB_ERR_CUDA, "noalloc conj_grad: kernel cannot be resident");
    const int grid = std::max(1, std::min({per_sm * prop.multiProcessorCount, n, kNoallocMaxGrid}));

    unsigned long long *arrivals = reinterpret_cast<unsigned long long *>(base);
    int *status = reinterpret_cast<int *>(base + 2 * kLine);
    StepTrace *trace = reinterpret_cast<StepTrace *>(base + 3 * kLine);
    int *split = reinterpret_cast<int *>(base + kHeaderBytes);
    double *part = reinterpret_cast<double *>(base + kHeaderBytes + kSplitBytes);
    double *vec = reinterpret_cast<double *>(base + kHeaderBytes + kSplitBytes + kPartBytes);

    // barrier words, status and trace must start at zero; the rest is
    // written before it is read
    if (cudaMemsetAsync(base, 0, kHeaderBytes, s) != cudaSuccess)
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

// cgb_internal.h -- shared host-side declarations of libcgb.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/cgb.h"

namespace cgb {

// Records a formatted message as the calling thread's last error and returns
// `status` unchanged, so call sites read `return set_error(...)`.
int set_error(int status, const char *fmt, ...);

// A kernel's dynamic shared memory limit is one per process, shared by
// every session or instance that launches it: this only ever raises it, so
// an object set up for a larger problem stays launchable after a smaller
// one is set up.  `kernel` is the kernel function's address.
inline cudaError_t raise_smem_limit(const void *kernel, size_t bytes)
{
    cudaFuncAttributes fa{};
    const cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    if (size_t(fa.maxDynamicSharedSizeBytes) >= bytes) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

// Odd integer in (1, 2^46): the LCG's admissible seeds (c_randdp.cpp:70-71).
bool valid_seed(double seed);

// Generator (makea.cpp).
int makea(int n, int nonzer, double rcond, double shift, double seed, int *rowstr, int *colidx,
          double *a, long long cap, long long *nnz_out);

// The n sparse vectors of the generator (sprnvc + vecset, cg.cu:1798-1857):
// vector i has count[i] <= width entries at 0-based positions pos[i*width +
// t] with values val[i*width + t]; scale[i] is its geometric weight
// (cg.cu:1695, :1755).  Shared by the host and the GPU assembly.
struct GenVectors {
    int width = 0;                // nonzer + 1
    std::vector<int> count;
    std::vector<int> pos;
    std::vector<double> val;
    std::vector<double> scale;
};
int draw_generator_vectors(int n, int nonzer, double rcond, double seed, GenVectors &v);

// The generator's CSR left on the device (makea_gpu.cu): rowstr / colidx / a
// are device allocations the caller takes over (cudaFree), the row pointers
// are also on the host.  With a row range [row0, row1) only those rows are
// assembled (rowstr rebased to 0, columns global): one rank's block.
struct DeviceCsr {
    int *rowstr = nullptr;
    int *colidx = nullptr;
    double *a = nullptr;
    long long nnz = 0;
    std::vector<int> h_rowstr;
};
int makea_on_device(int device, int n, int nonzer, double rcond, double shift, double seed,
                    DeviceCsr *out, int row0 = 0, int row1 = -1);

}  // namespace cgb

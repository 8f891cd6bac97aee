/*
 * ref_ft_harness.cu -- wraps the reference's own FT code as a shared library.
 *
 * TEST INFRASTRUCTURE ONLY (a comparator of the bench, never the product).
 * Compiled by oracle/Makefile straight from the reference sources where they
 * lie (CUDA/FT/ft.cu and CUDA/common of GMAP/NPB-GPU); nothing of the
 * reference is copied into this repository.  One library per NPB class,
 * because ft.cu takes its sizes at compile time (setparams.cpp:797-803).
 *
 * Exported entry point (extern "C"):
 *   ref_ft_gpu    main's sequence on the GPU (ft.cu:354-412: the untimed
 *                 warm-up -- set-up, index map, initial conditions, roots,
 *                 forward transform -- then the timed region: index map,
 *                 initial conditions, roots, forward transform, niter x
 *                 (evolve, inverse transform, checksum), the sums to the
 *                 host); the checksums and the timed region's wall seconds.
 *                 main's three set-up tasks, which it runs in OpenMP
 *                 sections, run here one after the other.  The checksum
 *                 accumulators are cleared before the timed region (main
 *                 relies on fresh device memory being zero).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#define main npb_ft_reference_main
#include "FT/ft.cu"
#undef main

static double harness_now()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

extern "C" int ref_ft_niter(void) { return NITER_DEFAULT; }

extern "C" int ref_ft_gpu(double *sums_out, double *seconds)
{
    setup();
    setup_gpu();
    init_ui_gpu(u0_device, u1_device, twiddle_device);
    compute_indexmap_gpu(twiddle_device);
    compute_initial_conditions_gpu(u1_device);
    fft_init_gpu(MAXDIM);
    cudaDeviceSynchronize();
    fft_gpu(1, u1_device, u0_device);
    cudaMemset(sums_device, 0, size_sums_device);
    cudaDeviceSynchronize();
    const double t0 = harness_now();
    compute_indexmap_gpu(twiddle_device);
    compute_initial_conditions_gpu(u1_device);
    fft_init_gpu(MAXDIM);
    cudaDeviceSynchronize();
    fft_gpu(1, u1_device, u0_device);
    for (int iter = 1; iter <= niter; iter++) {
        evolve_gpu(u0_device, u1_device, twiddle_device);
        fft_gpu(-1, u1_device, u1_device);
        checksum_gpu(iter, u1_device);
    }
    cudaMemcpy(sums, sums_device, size_sums_device, cudaMemcpyDeviceToHost);
    *seconds = harness_now() - t0;
    for (int iter = 1; iter <= niter; iter++) {
        sums_out[2 * (iter - 1)] = sums[iter].real;
        sums_out[2 * (iter - 1) + 1] = sums[iter].imag;
    }
    const int ok = cudaGetLastError() == cudaSuccess;
    release_gpu();
    return ok ? niter : -1;
}

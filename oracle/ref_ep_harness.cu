/*
 * ref_ep_harness.cu -- wraps the reference's own EP code as a shared library.
 *
 * TEST INFRASTRUCTURE ONLY (a comparator of the bench, never the product).
 * Compiled by oracle/Makefile straight from the reference sources where they
 * lie (CUDA/EP/ep.cu and CUDA/common of GMAP/NPB-GPU); nothing of the
 * reference is copied into this repository.  One library per NPB class,
 * because ep.cu takes its size M at compile time (ep.cu:65-68).
 *
 * Exported entry point (extern "C"):
 *   ref_ep_gpu    main's set-up and its timed GPU region exactly as main runs
 *                 it (ep.cu:145-188: an, setup_gpu, gpu_kernel, the host's
 *                 sums of the blocks' partials), release_gpu after; the
 *                 seconds are the reference's own timer's (the launch only,
 *                 as main times it) and the wall seconds to the sums on the
 *                 host
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#define main npb_ep_reference_main
#include "EP/ep.cu"
#undef main

static double harness_now()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

extern "C" int ref_ep_m(void) { return M; }

extern "C" int ref_ep_gpu(double *sx_out, double *sy_out, double *q_out, double *seconds_launch,
                          double *seconds_wall)
{
    double t1 = A;
    for (int i = 0; i < MK + 1; i++) randlc(&t1, t1);
    const double an = t1;
    double sx = 0.0, sy = 0.0;
    for (int i = 0; i < NQ; i++) q[i] = 0.0;
    setup_gpu();
    cudaDeviceSynchronize();
    const double w0 = harness_now();
    gpu_kernel<<<blocks_per_grid, threads_per_block>>>(q_device, sx_device, sy_device, an);
    const double l1 = harness_now();
    cudaMemcpy(q_host, q_device, size_q, cudaMemcpyDeviceToHost);
    cudaMemcpy(sx_host, sx_device, size_sx, cudaMemcpyDeviceToHost);
    cudaMemcpy(sy_host, sy_device, size_sy, cudaMemcpyDeviceToHost);
    for (int block = 0; block < blocks_per_grid; block++) {
        for (int i = 0; i < NQ; i++) q[i] += q_host[block * NQ + i];
        sx += sx_host[block];
        sy += sy_host[block];
    }
    const double w1 = harness_now();
    *sx_out = sx;
    *sy_out = sy;
    for (int i = 0; i < NQ; i++) q_out[i] = q[i];
    *seconds_launch = l1 - w0;
    *seconds_wall = w1 - w0;
    release_gpu();
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

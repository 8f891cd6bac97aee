/*
 * ref_is_harness.cu -- wraps the reference's own IS code as a shared library.
 *
 * TEST INFRASTRUCTURE ONLY (a comparator of the bench, never the product).
 * Compiled by oracle/Makefile straight from the reference sources where they
 * lie (CUDA/IS/is.cu and CUDA/common of GMAP/NPB-GPU); nothing of the
 * reference is copied into this repository.  One library per NPB class,
 * because is.cu takes its class at compile time (is.cu:86-140).
 *
 * Exported entry point (extern "C"):
 *   ref_is_gpu    main's sequence on the GPU as main runs it (is.cu:345-445:
 *                 the class's test arrays, setup_gpu, create_seq_gpu, the
 *                 untimed rank_gpu(1), the timed rank_gpu(1 .. 10),
 *                 full_verify_gpu); the passed count and the wall seconds of
 *                 the ten passes, to a device synchronisation after them
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>

#define main npb_is_reference_main
#include "IS/is.cu"
#undef main

static double harness_now()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

extern "C" long long ref_is_gpu(double *seconds)
{
    const INT_TYPE *ti = nullptr, *tr = nullptr;
    switch (CLASS) {
    case 'S': ti = S_test_index_array; tr = S_test_rank_array; break;
    case 'W': ti = W_test_index_array; tr = W_test_rank_array; break;
    case 'A': ti = A_test_index_array; tr = A_test_rank_array; break;
    case 'B': ti = B_test_index_array; tr = B_test_rank_array; break;
    case 'C': ti = C_test_index_array; tr = C_test_rank_array; break;
    default: ti = D_test_index_array; tr = D_test_rank_array; break;
    }
    for (int i = 0; i < TEST_ARRAY_SIZE; i++) {
        test_index_array[i] = ti[i];
        test_rank_array[i] = tr[i];
    }
    setup_gpu();
    create_seq_gpu(314159265.00, 1220703125.00);
    rank_gpu(1);
    passed_verification = 0;
    cudaMemcpy(passed_verification_device, &passed_verification, size_passed_verification_device,
               cudaMemcpyHostToDevice);
    cudaDeviceSynchronize();
    const double t0 = harness_now();
    for (INT_TYPE iteration = 1; iteration <= MAX_ITERATIONS; iteration++) rank_gpu(iteration);
    cudaDeviceSynchronize();
    *seconds = harness_now() - t0;
    cudaMemcpy(&passed_verification, passed_verification_device, size_passed_verification_device,
               cudaMemcpyDeviceToHost);
    full_verify_gpu();
    const long long passed = (long long)passed_verification;
    release_gpu();
    return passed;
}

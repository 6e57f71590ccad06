// Host shim used only by oracle/build_ref.py to compile the reference's CUDA kernel
// sources (modules/mod_cppkernels.cpp, nonlinear/rhs_kernels.cpp,
// nonlinear/step3D_uv.kernels.cpp, modules/mod_BC.c) as plain host C++.
//
// Test infrastructure only: the result (oracle/_ref/*.so) is the reference's own
// algorithm run on the CPU, used to pin the oracle restatement and as the timed
// CPU baseline.  Nothing in the product links it.
//
// A reference kernel computes its flat thread index as
//     i = blockDim.x * blockIdx.x + threadIdx.x
// The launcher sets blockDim.x = 1, blockIdx.x = 0 and threadIdx.x = i, so each
// call of the kernel function executes exactly one CUDA thread.  The three
// "built-ins" are thread_local so that an OpenMP loop over i can run kernels
// concurrently (used only for CPU-baseline timing; pinning uses the sequential loop).
#pragma once
#include <cstdio>
#include <cmath>
#include <cstdint>

struct sfref_dim3 { unsigned int x, y, z; };
static thread_local sfref_dim3 blockDim = {1u, 1u, 1u};
static thread_local sfref_dim3 blockIdx = {0u, 0u, 0u};
static thread_local sfref_dim3 threadIdx = {0u, 0u, 0u};

#define __global__
#define __device__
#define __restrict__

// Runs `nthreads` CUDA threads of kernel `k` in flat-index order (omp <= 1), or
// spread over `omp` OpenMP threads (timing only).
template <typename K, typename... A>
static void sfref_run(K k, long nthreads, int omp, A... a) {
    if (omp <= 1) {
        for (long t = 0; t < nthreads; ++t) {
            threadIdx.x = (unsigned int)t;
            k(a...);
        }
    } else {
#pragma omp parallel for num_threads(omp) schedule(static)
        for (long t = 0; t < nthreads; ++t) {
            blockDim.x = 1u; blockIdx.x = 0u;
            threadIdx.x = (unsigned int)t;
            k(a...);
        }
    }
}

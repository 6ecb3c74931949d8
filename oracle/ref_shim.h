/*
 * ref_shim.h -- test infrastructure only (oracle).
 *
 * Lets the reference's CUDA C kernel files (_multipole_potential_kernel.cu,
 * _cylspl_potential_kernel.cu) compile unchanged as host C++ so that their
 * FP64 arithmetic can serve as a CPU checker and as the timed CPU baseline.
 * Every CUDA-only keyword becomes empty, __ldg becomes a plain load and
 * threadIdx/blockIdx/blockDim become thread-local host variables: the
 * driver (ref_driver.cpp) sets threadIdx.x = i and calls the kernel once per
 * point, one OpenMP thread per chunk of points.
 */
#pragma once
#include <math.h>
#include <stddef.h>

#define __device__
#define __global__
#define __host__
#define __constant__ static
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __ldg(p) (*(p))

struct ref_dim3 { unsigned x, y, z; };
extern thread_local ref_dim3 threadIdx;
extern thread_local ref_dim3 blockIdx;
extern thread_local ref_dim3 blockDim;

static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }

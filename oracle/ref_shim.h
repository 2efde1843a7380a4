/*
 * ref_shim.h -- test infrastructure only (the oracle), never shipped.
 *
 * Makes the reference's own CUDA sources compile and run as plain C++ on the
 * host, so that the reference's kernels and host driver can be executed here
 * as the parity oracle ("oracle/_ref").  It is force-included (g++ -include)
 * ahead of the reference headers
 *   include/lbm_model.cuh, include/global_var.cuh,
 *   include/iteration_device.cuh, include/iteration_kernel.cuh,
 *   include/iteration_host.h, src/multiphase_lbm.cu
 * which are compiled unmodified except for the lattice size macros at
 * include/lbm_model.cuh:4-6 (a compile-time constant in the reference, set by
 * the build recipe oracle/build_ref.py on a copy of the tree).
 *
 * What it supplies:
 *   - the CUDA qualifiers (__global__, __device__, __managed__) as nothing;
 *   - blockIdx / threadIdx / blockDim / gridDim as thread-local variables so
 *     one "thread" of a reference kernel can be run per lattice node from an
 *     OpenMP loop (include/iteration_kernel.cuh:9-118 reads them);
 *   - the handful of CUDA runtime calls the host driver makes
 *     (src/multiphase_lbm.cu:99-109, 579-582, 1147-1153) as host stand-ins
 *     backed by malloc/free.
 *   - std::exp / std::sqrt in the global namespace so that exp(float) picks
 *     the single-precision overload, as device code does
 *     (include/iteration_device.cuh:23, 35, 37).
 */
#ifndef MLBM_ORACLE_REF_SHIM_H_
#define MLBM_ORACLE_REF_SHIM_H_

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

using std::exp;
using std::sqrt;

#define __global__
#define __device__
#define __managed__
#define __host__

struct shim_dim3 {
  unsigned int x, y, z;
};

extern thread_local shim_dim3 blockIdx;
extern thread_local shim_dim3 threadIdx;
extern thread_local shim_dim3 blockDim;
extern thread_local shim_dim3 gridDim;

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1 };

inline const char* cudaGetErrorString(cudaError_t e) {
  return e == cudaSuccess ? "no error" : "host stand-in error";
}
inline cudaError_t cudaMallocManaged(void** p, size_t n) {
  *p = std::calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaMalloc(void** p, size_t n) {
  *p = std::calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return cudaSuccess;
}
inline cudaError_t cudaMemPrefetchAsync(const void*, size_t, int, int) {
  return cudaSuccess;
}

#endif  // MLBM_ORACLE_REF_SHIM_H_

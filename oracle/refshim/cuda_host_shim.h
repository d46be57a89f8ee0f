// Host-compilation shim for the reference solver (test infrastructure only).
//
// The reference MHD solver (src/library/mhd_solver.inl, generated from
// src/library/mhd_solver.inlrb) is CUDA C++ that runs every kernel as a
// grid-stride loop over all cells (CRYSTAL_MAP, src/library/physics_util.h:9-11)
// and stores its arrays in thrust::device_vector.  This header lets g++ compile
// that unmodified source on the host so it can serve as the oracle:
//   * CUDA qualifiers become empty, launch dimensions are stripped by the build
//     recipe (oracle/Makefile), and CRYSTAL_MAP becomes an OpenMP loop over
//     every cell (kernels write disjoint addresses, so the result is bitwise
//     the same as a serial loop);
//   * Thrust runs on its OpenMP "device" system, so device_vector is host memory
//     and cudaMemcpy is memcpy;
//   * the float overloads of fabs/sqrt/fmin/fmax/abs are brought into the global
//     namespace so `absR(x)` etc. on a float stay in float, exactly as the CUDA
//     device overloads the reference was written against do.
#pragma once

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <algorithm>

using std::abs;
using std::fabs;
using std::fmax;
using std::fmin;
using std::sqrt;
using std::floor;

#define __global__
#define __device__
#define __host__
#define __shared__

struct nmhd_shim_dim3 { unsigned x, y, z; };
static const nmhd_shim_dim3 threadIdx = {0, 0, 0};
static const nmhd_shim_dim3 blockIdx = {0, 0, 0};
static const nmhd_shim_dim3 blockDim = {1, 1, 1};
static const nmhd_shim_dim3 gridDim = {1, 1, 1};

enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3
};
typedef int cudaError_t;
static inline cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
  std::memcpy(dst, src, n);
  return 0;
}
static inline cudaError_t cudaThreadSynchronize() { return 0; }
static inline cudaError_t cudaDeviceSynchronize() { return 0; }
static inline cudaError_t cudaSetDevice(int) { return 0; }
static inline cudaError_t cudaGetDevice(int *d) { *d = 0; return 0; }

// CUDA's device min/max for floating point (used unqualified by the solver).
static inline float min(float a, float b) { return std::fmin(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline double min(double a, double b) { return std::fmin(a, b); }
static inline double max(double a, double b) { return std::fmax(a, b); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }

// CPU stand-in for the small part of the HIP runtime API that LICOM3-HIP's
// tracer.cpp and convadj.cpp use, so that those files compile unchanged with
// g++ and run on the host.  TEST INFRASTRUCTURE ONLY (builds oracle/_ref).
//
// A kernel launch runs every thread of the grid in turn on the calling host
// thread.  This is a faithful emulation for kernels whose threads write
// disjoint cells or only race with identical values, which holds for the
// kernels these two files launch.  Device memory is host memory.
#pragma once
#include <cstddef>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <cmath>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct dim3 {
  unsigned x, y, z;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};

extern thread_local dim3 threadIdx, blockIdx, blockDim, gridDim;

typedef int hipError_t;
static const hipError_t hipSuccess = 0;
enum hipMemcpyKind { hipMemcpyHostToHost = 0, hipMemcpyHostToDevice, hipMemcpyDeviceToHost, hipMemcpyDeviceToDevice };

inline hipError_t hipMemset(void* p, int v, size_t n) { std::memset(p, v, n); return hipSuccess; }
inline hipError_t hipMemcpy(void* d, const void* s, size_t n, hipMemcpyKind) {
  if (d != s) std::memmove(d, s, n);
  return hipSuccess;
}
inline hipError_t hipGetLastError() { return hipSuccess; }
inline const char* hipGetErrorString(hipError_t) { return "no error"; }
inline hipError_t hipDeviceSynchronize() { return hipSuccess; }
inline hipError_t hipGetDeviceCount(int* n) { *n = 1; return hipSuccess; }
inline hipError_t hipSetDevice(int) { return hipSuccess; }

template <class Kernel, class... Args>
void hip_cpu_launch(Kernel kernel, dim3 grid, dim3 block, Args... args) {
  gridDim = grid;
  blockDim = block;
  for (unsigned bz = 0; bz < grid.z; ++bz)
    for (unsigned by = 0; by < grid.y; ++by)
      for (unsigned bx = 0; bx < grid.x; ++bx)
        for (unsigned tz = 0; tz < block.z; ++tz)
          for (unsigned ty = 0; ty < block.y; ++ty)
            for (unsigned tx = 0; tx < block.x; ++tx) {
              blockIdx = dim3(bx, by, bz);
              threadIdx = dim3(tx, ty, tz);
              kernel(args...);
            }
}

#define hipLaunchKernelGGL(kernel, grid, block, shmem, stream, ...) \
  hip_cpu_launch(kernel, dim3(grid), dim3(block), __VA_ARGS__)

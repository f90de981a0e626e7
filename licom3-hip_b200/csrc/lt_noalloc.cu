// lt_noalloc.cu - global tracer content without any device allocation.
//
// Some host models cannot let a library call cudaMalloc: they own every byte
// of device memory through their own pool (a Fortran model whose arrays are
// placed by OpenACC/OpenMP data regions, or a coupled system that divided HBM
// between its components once at start-up and fails on any later growth).
// For them, lt_tracer_content_noalloc takes the state and the grid arrays as
// device pointers the caller already owns, writes the two tracer integrals to
// a device pointer the caller owns, and keeps its partial sums in the fixed
// array below instead of an allocated buffer.
//
// The scratch array is part of the library image: every GPU that loads the
// library holds its 2 MiB until the process exits, whether or not this entry
// point is called.  Every call on a device shares that one array, so calls
// whose work overlaps on the GPU (different streams, or threads issuing at the
// same time) race and must be ordered by the caller.  Nothing in the array
// has to start at zero: each pass writes every partial sum that the next pass
// reads, so the contents left by the previous call are never read.
//
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture begins.  Later calls look the address up again
// unless their stream is capturing, so a call after cudaDeviceReset (which
// unloads the library image from the device) finds the array where the
// reloaded image put it; inside a capture the address of the last call
// outside one is used.
//
// The sum is the same fixed binary tree as lt_tracer_content's (blocks of 2048
// consecutive wet-cell terms T*tarea*dz over k, j, i of the interior, pairs
// (t, t+stride) for stride 1024..1, repeated on the block sums), so the two
// entry points give bit-identical results on the same state.
#include <cuda_runtime.h>
#include <mutex>
#include "lt_common.cuh"

namespace lt {
namespace {

// Capacity of the scratch in doubles (2 MiB).  A tracer of n interior cells
// needs tree_sum_part_elems(n) of them, about n/2048: up to about 5.3e8 cells
// per tracer, which covers the 0.1 degree 3600 x 2302 x 55 grid (4.56e8).
constexpr long kScratchValues = 1L << 18;

// Host code may only use this name as a stand-in for the symbol: its device
// address comes from cudaGetSymbolAddress below, once per device.
static __device__ __align__(256) double g_content_scratch[kScratchValues];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Resolves the scratch address on the current device: on the first call on
// that device, and on every call whose stream is not capturing.
int scratch_on_current_device(cudaStream_t stream, double** out) {
  int dev = 0;
  LT_CUDA_OK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("lt_tracer_content_noalloc: device %d beyond the %d devices supported", dev, kMaxDevices);
    return LT_E_INVALID;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  LT_CUDA_OK(cudaStreamIsCapturing(stream, &cap));
  std::lock_guard<std::mutex> g(g_setup_mutex);
  if (!g_scratch_ptr[dev] || cap == cudaStreamCaptureStatusNone) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_content_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_content_scratch)");
    g_scratch_ptr[dev] = static_cast<double*>(ptr);
  }
  *out = g_scratch_ptr[dev];
  return LT_OK;
}

constexpr int RB = 1024;

// First pass: one block sums 2048 consecutive terms of the k-major, row-major
// interior ordering into part[blockIdx.x].
__global__ void k_content_first_static(const double* at, const double* tarea, const double* dzp, const int* kmt,
                                       int nx, int ny, int imt, long A, long n, double* part) {
  __shared__ double s[2 * RB];
  const long base = (long)blockIdx.x * 2 * RB;
  auto term = [&](long m) -> double {
    if (m >= n) return 0.0;
    const long per = (long)nx * ny;
    const int k = (int)(m / per);
    const long r = m % per;
    const int j = 2 + (int)(r / nx), i = 2 + (int)(r % nx);
    const long q = (long)j * imt + i;
    return (k < kmt[q]) ? tarea[q] * dzp[k] * at[(long)k * A + q] : 0.0;
  };
  const int t = threadIdx.x;
  s[t] = term(base + t);
  s[t + RB] = term(base + t + RB);
  for (int stride = RB; stride > 0; stride >>= 1) {
    __syncthreads();
    if (t < stride) s[t] = s[t] + s[t + stride];
  }
  if (t == 0) part[blockIdx.x] = s[0];
}

}  // namespace
}  // namespace lt

using namespace lt;

extern "C" int lt_tracer_content_noalloc(const double* at, const double* tarea, const double* dzp, const int* kmt,
                                         int nx, int ny, int km, double* out2, void* stream) {
  if (!at || !tarea || !dzp || !kmt || !out2 || nx <= 0 || ny <= 0 || km <= 0) {
    set_error("lt_tracer_content_noalloc: null pointer or non-positive size");
    return LT_E_INVALID;
  }
  const long n = (long)nx * ny * km;
  const size_t need = tree_sum_part_elems(n);
  if (need > (size_t)kScratchValues) {
    set_error("lt_tracer_content_noalloc: %d x %d x %d = %ld cells per tracer need %zu scratch values; "
              "the static scratch holds %ld (about %ld cells)",
              nx, ny, km, n, need, kScratchValues, (kScratchValues - 8) * 2 * RB);
    return LT_E_INVALID;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = nullptr;
  int rc = scratch_on_current_device(s, &part);
  if (rc) return rc;

  const int imt = nx + 4, jmt = ny + 4;
  const long A = (long)imt * jmt, F = A * km;
  const long nb = (n + 2 * RB - 1) / (2 * RB);
  for (int tr = 0; tr < 2; ++tr) {
    k_content_first_static<<<(unsigned)nb, RB, 0, s>>>(at + tr * F, tarea, dzp, kmt, nx, ny, imt, A, n, part);
    LT_LAUNCHED();
    rc = launch_tree_sum(part, nb, part + nb, out2 + tr, s);
    if (rc) return rc;
  }
  return LT_OK;
}

// gpe_norm_noalloc: the norm reduction of get_norm for callers that own all
// device memory themselves and must not have a library allocate any.
//
// Typical callers: a host whose device memory belongs to another allocator
// (a framework's caching pool, a Fortran runtime that maps its own buffers)
// and may not see foreign cudaMalloc/cudaFree calls; code running between
// steps of a captured or real-time loop where an allocation would stall or
// be illegal; and embedders that budget device memory up front.
//
// The reduction needs scratch space for one partial sum per z-plane.  That
// scratch is the file-scope array below, sized for GPE_NOALLOC_MAX_NZ planes
// (64 KiB).  It is part of this library's device image, so every GPU that
// loads the library holds it until the process exits.
//
// Host code must not use the array's name as a device address: on the host
// it is only a stand-in symbol.  The first call on each device, with that
// device current, looks up the real device address with
// cudaGetSymbolAddress and caches it per device; kernels get that pointer.
// The same first call loads both dtype instances of the reduction kernel on
// that device (cudaFuncGetAttributes), so with lazy module loading no later
// call loads code; make it before any stream capture.  The cached address is
// not refreshed after cudaDeviceReset or a primary-context reset, which this
// entry point does not support.
//
// Pointers are checked for the alignment the kernels read and write with
// (16 bytes for complex128 input, 8 for complex64 input and the output
// double) before anything is launched: a misaligned pointer is rejected
// with GPE_ERR_BADARG rather than faulting the caller's context.
//
// All calls share the one array.  Every call overwrites each partial it
// reads before reading it, so nothing has to be cleared between calls, but
// calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/gpe_cuda.h"

namespace {

static __device__ __align__(256) double g_norm_scratch[GPE_NOALLOC_MAX_NZ];

constexpr int kMaxDevices = 64;
// device address of g_norm_scratch, per device; written once under g_setup
std::atomic<double*> g_scratch_addr[kMaxDevices];
std::mutex g_setup;

// Extended closed (Numerical Recipes 4.1.14) weights of integrate_x/y/z
// (src/variables.f90:49-51, 730-840): 3/8, 7/6, 23/24 at both ends, 1 inside.
__device__ __forceinline__ double quad_weight(int q, int n) {
  double w = 1.0;
  if (q == 0) w = 3.0 / 8.0;
  if (q == 1) w = 7.0 / 6.0;
  if (q == 2) w = 23.0 / 24.0;
  if (q == n - 3) w = 23.0 / 24.0;
  if (q == n - 2) w = 7.0 / 6.0;
  if (q == n - 1) w = 3.0 / 8.0;
  return w;
}

// One block per z-plane: scratch[k] = sum_{i,j} w_i w_j |psi(i,j,k)|^2, summed
// in a fixed order (thread-strided, then a tree), so results are
// deterministic.
template <class T2>
__global__ void __launch_bounds__(256) k_plane_sums(const T2* __restrict__ psi, int nx, int ny, double* scratch) {
  __shared__ double red[256];
  const int k = blockIdx.x;
  const long long plane = (long long)nx * ny;
  const T2* p = psi + k * plane;
  double s = 0.0;
  for (long long t = threadIdx.x; t < plane; t += 256) {
    const int i = (int)(t % nx), j = (int)(t / nx);
    const double re = (double)p[t].x, im = (double)p[t].y;
    s += (quad_weight(i, nx) * quad_weight(j, ny)) * (re * re + im * im);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) scratch[k] = red[0];
}

// norm = (sum_k w_k scratch[k]) * dx * dy * dz into the caller's device word.
__global__ void __launch_bounds__(256) k_plane_total(const double* __restrict__ scratch, int nz, double dx,
                                                     double dy, double dz, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < nz; k += 256) s += quad_weight(k, nz) * scratch[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = ((red[0] * dx) * dy) * dz;
}

int reject(const char* why) {
  fprintf(stderr, "gpe_norm_noalloc: %s\n", why);
  return GPE_ERR_BADARG;
}

// Set-up of the current device (once): the scratch array's device address,
// and both reduction kernels loaded.  Returns nullptr on a CUDA error.
double* scratch_of(int dev) {
  double* p = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (p) return p;
  std::lock_guard<std::mutex> lk(g_setup);
  p = g_scratch_addr[dev].load(std::memory_order_relaxed);
  if (p) return p;
  void* addr = nullptr;
  if (cudaGetSymbolAddress(&addr, g_norm_scratch) != cudaSuccess || !addr) return nullptr;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, k_plane_sums<double2>) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, k_plane_sums<float2>) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, k_plane_total) != cudaSuccess)
    return nullptr;
  p = (double*)addr;
  g_scratch_addr[dev].store(p, std::memory_order_release);
  return p;
}

}  // namespace

extern "C" int gpe_norm_noalloc(const void* psi_dev, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, double dx,
                                double dy, double dz, double* norm_dev, void* stream) {
  if (!psi_dev || !norm_dev) return reject("null device pointer");
  if (dtype != GPE_C128 && dtype != GPE_C64) return reject("dtype must be GPE_C128 or GPE_C64");
  if (nx < 6 || ny < 6 || nz < 6) return reject("nx, ny and nz must be >= 6");
  if (nz > GPE_NOALLOC_MAX_NZ) return reject("nz exceeds GPE_NOALLOC_MAX_NZ (8192 planes of scratch)");
  const uintptr_t in_align = dtype == GPE_C128 ? 16 : 8;
  if ((uintptr_t)psi_dev % in_align != 0)
    return reject(dtype == GPE_C128 ? "psi_dev is not 16-byte aligned (complex128)"
                                    : "psi_dev is not 8-byte aligned (complex64)");
  if ((uintptr_t)norm_dev % 8 != 0) return reject("norm_dev is not 8-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GPE_ERR_CUDA;
  double* scratch = scratch_of(dev);
  if (!scratch) return GPE_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == GPE_C128)
    k_plane_sums<double2><<<nz, 256, 0, st>>>((const double2*)psi_dev, nx, ny, scratch);
  else
    k_plane_sums<float2><<<nz, 256, 0, st>>>((const float2*)psi_dev, nx, ny, scratch);
  k_plane_total<<<1, 256, 0, st>>>(scratch, nz, dx, dy, dz, norm_dev);
  return cudaGetLastError() == cudaSuccess ? GPE_OK : GPE_ERR_CUDA;
}

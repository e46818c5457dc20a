// FFT diagnostics (condensed_particles, spectrum, filtered_surface) on the
// device.  Every reduction is deterministic: per-warp shared-memory
// histograms filled in a fixed lane order, combined per block in warp order
// and over blocks in block order; no floating-point atomics.
#include <cufft.h>
#include <math.h>

#include "gpe_aux.cuh"
#include "gpe_fft.h"
#include "gpe_ic.h"

namespace gpe {

namespace {

constexpr int NS = GPE_SPECTRUM_SHELLS;
constexpr int FFT_BLOCKS = 148 * 2;
constexpr int FFT_THREADS = 256;
constexpr double PI_D = 3.1415926535897932384626433832795;

// partial layout per block: [H (nbins)] [eta (NS)] [nharm (NS)] [tot] [n0]
__host__ __device__ inline int part_width(int nbins) { return nbins + 2 * NS + 2; }

// squared modulus the way the reference takes it: abs(z)**2, abs = hypot
__device__ __forceinline__ double abs2(double re, double im) {
  const double h = hypot(re, im);
  return h * h;
}

// squared index distance of spectral index i on an n-point axis
// (io.f90:547-565, 684-699): i^2 for i <= (n-1)/2 + 1, else (n-i)^2
__device__ __forceinline__ int k2_axis(int i, int n) {
  const int n1 = n - 1;
  return i <= n1 / 2 + 1 ? i * i : (n1 - i + 1) * (n1 - i + 1);
}

// Add v into hist[bin] for every lane of the warp at once (bin < 0: no-op).
// Lanes that share a bin are summed in increasing lane order by the group's
// first lane, so the result does not depend on scheduling.
__device__ __forceinline__ void warp_bin_add(double* hist, int bin, double v, int lane) {
  const unsigned grp = __match_any_sync(0xffffffffu, bin);
  double sum = 0.0;
#pragma unroll 8
  for (int l = 0; l < 32; ++l) {
    const double x = __shfl_sync(0xffffffffu, v, l);
    if ((grp >> l) & 1u) sum += x;
  }
  if (lane == __ffs(grp) - 1 && bin >= 0) hist[bin] += sum;
  __syncwarp();
}

// Deterministic sum over the block of one value per thread; valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += scratch[q];
  return s;
}

// sum |psi|^2 over the contiguous field, one partial per block
__global__ void k_mass(const double2* __restrict__ a, long long n, double* part) {
  __shared__ double scratch[32];
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    acc += abs2(a[t].x, a[t].y);
  const double s = block_sum(acc, scratch);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Spectral sums over a = raw / sqrt(N).  Warp w of the grid owns the
// contiguous index range [w*chunk, (w+1)*chunk) and walks it 32 sites at a
// time.  tot uses the reference's real-space-indexed k grid (kq tables).
__global__ void k_spectrum(const double2* __restrict__ raw, int nx, int ny, int nz, const double* __restrict__ kq,
                           int nbins, int want_spectrum, double* part) {
  extern __shared__ double sh[];
  __shared__ double scratch[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int width = nbins + 2 * NS;
  double* wh = sh + (size_t)w * width;
  for (int b = lane; b < width; b += 32) wh[b] = 0.0;
  __syncwarp();

  const long long n = (long long)nx * ny * nz;
  const double s = sqrt((double)n);
  const double n0 = abs2(raw[0].x / s, raw[0].y / s);
  const double rho0 = n0 / (double)n;
  const double c12 = -(1.0 / 12.0);
  const double* kx = kq;
  const double* ky = kq + nx;
  const double* kz = kq + nx + ny;

  const long long tw = (long long)gridDim.x * nw;
  const long long chunk = ((n + tw - 1) / tw + 31) / 32 * 32;
  const long long t0 = ((long long)blockIdx.x * nw + w) * chunk;
  const long long t1 = min(t0 + chunk, n);
  double tot = 0.0;
  for (long long base = t0; base < t1; base += 32) {
    const long long t = base + lane;
    const bool valid = t < t1;
    int bF = -1, shell = -1;
    double v = 0.0;
    if (valid) {
      const int i = (int)(t % nx);
      const long long r = t / nx;
      const int j = (int)(r % ny);
      const int k = (int)(r / ny);
      // io.f90:343-360
      const double k2q = c12 * ((kx[i] + ky[j]) + kz[k]);
      if (k2q != 0.0) tot += (k2q + rho0) / (k2q * k2q + 2.0 * rho0 * k2q);
      if (want_spectrum) {
        v = abs2(raw[t].x / s, raw[t].y / s);
        const int k2 = k2_axis(i, nx) + k2_axis(j, ny) + k2_axis(k, nz);
        if (k2 != 0) {
          // F(kk) collects sqrt(k2) <= kk (io.f90:701-705): bin ceil(sqrt(k2))
          int b = (int)sqrt((double)k2);
          while (b * b < k2) ++b;
          while (b > 1 && (b - 1) * (b - 1) >= k2) --b;
          if (b < nbins) bF = b;
          // shells m-1 <= |log2(sqrt(k2)/(2 pi))| < m, m = 1..7 (io.f90:706-713)
          const double l2 = fabs(log(0.5 * sqrt((double)k2) / PI_D) / log(2.0));
          if (l2 < (double)NS) shell = (int)floor(l2);
        }
      }
    }
    if (want_spectrum) {
      warp_bin_add(wh, bF, v, lane);
      warp_bin_add(wh + nbins, shell, v, lane);
      warp_bin_add(wh + nbins + NS, shell, 1.0, lane);
    }
  }
  const double bt = block_sum(tot, scratch);
  __syncthreads();
  double* out = part + (size_t)blockIdx.x * part_width(nbins);
  for (int b = threadIdx.x; b < width; b += blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < nw; ++q) acc += sh[(size_t)q * width + b];
    out[b] = acc;
  }
  if (threadIdx.x == 0) {
    out[width] = bt;
    out[width + 1] = n0;
  }
}

// column sums of the per-block partials, in block order
__global__ void k_sum_columns(const double* part, int nblocks, int width, double* out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < width; c += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += part[(size_t)b * width + c];
    out[c] = acc;
  }
}

// a = raw / sqrt(N) times the filter max(1 - m k2 / kc^2, 0) (io.f90:567)
__global__ void k_filter(double2* raw, int nx, int ny, int nz, double mscale, double kc2) {
  const long long n = (long long)nx * ny * nz;
  const double s = sqrt((double)n);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const long long r = t / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    const int k2 = k2_axis(i, nx) + k2_axis(j, ny) + k2_axis(k, nz);
    const double f = fmax(1.0 - (mscale * (double)k2) / kc2, 0.0);
    raw[t].x = (raw[t].x / s) * f;
    raw[t].y = (raw[t].y / s) * f;
  }
}

__global__ void k_div(double2* a, long long n, double s) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    a[t].x = a[t].x / s;
    a[t].y = a[t].y / s;
  }
}

cudaError_t to_contiguous(const Geom& g, int esz, const void* psi_field, double2* buf, cudaStream_t st) {
  if (esz == 16) k_unpack<double2, double2><<<148 * 8, 256, 0, st>>>((const double2*)psi_field, buf, g);
  else k_unpack<float2, double2><<<148 * 8, 256, 0, st>>>((const float2*)psi_field, buf, g);
  return cudaGetLastError();
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

size_t fft_work_bytes(const gpe_params& p) {
  const size_t n = (size_t)p.nx * p.ny * p.nz;
  const int nbins = p.nx / 2 + 1;
  return round256(n * sizeof(double2)) + round256((size_t)(FFT_BLOCKS + 1) * part_width(nbins) * sizeof(double)) +
         round256((size_t)FFT_BLOCKS * sizeof(double)) + 256;
}

void fft_kq_axis(int n, int nx, double d, double* out) {
  // kc = pi, dk = 2 kc / (nx - 1) on every axis (io.f90:323-324, 345-351)
  const double kc = PI_D;
  const double dk = 2.0 * kc / (double)(nx - 1);
  const double d2 = d * d;
  for (int i = 0; i < n; ++i) {
    const double k = -kc + (double)i * dk;
    out[i] = ((-2.0 * cos(2.0 * k * d) + 32.0 * cos(k * d)) - 30.0) / d2;
  }
}

cudaError_t fft_condensed(const gpe_params& p, const Geom& g, int esz, const void* psi_field, const double* kq,
                          bool want_spectrum, void* work, size_t work_bytes, cudaStream_t st, FftDiag& out) {
  if (!work || work_bytes < fft_work_bytes(p)) return cudaErrorInvalidValue;
  const long long n = (long long)p.nx * p.ny * p.nz;
  const int nbins = p.nx / 2 + 1;
  const int width = part_width(nbins);
  double2* buf = (double2*)work;
  double* part = (double*)((char*)work + round256((size_t)n * sizeof(double2)));
  double* sums = part + (size_t)FFT_BLOCKS * width;
  double* mpart = (double*)((char*)part + round256((size_t)(FFT_BLOCKS + 1) * width * sizeof(double)));

  cudaError_t e = to_contiguous(g, esz, psi_field, buf, st);
  if (e != cudaSuccess) return e;
  k_mass<<<FFT_BLOCKS, FFT_THREADS, 0, st>>>(buf, n, mpart);
  cufftHandle plan;
  if (!plan_for(p.nx, p.ny, p.nz, &plan)) return cudaErrorUnknown;
  if (cufftSetStream(plan, st) != CUFFT_SUCCESS) return cudaErrorUnknown;
  if (cufftExecZ2Z(plan, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, CUFFT_FORWARD) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  const size_t shm = (size_t)(FFT_THREADS / 32) * (nbins + 2 * NS) * sizeof(double);
  if (shm > 48 * 1024) {
    e = cudaFuncSetAttribute(k_spectrum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    if (e != cudaSuccess) return e;
  }
  k_spectrum<<<FFT_BLOCKS, FFT_THREADS, shm, st>>>(buf, p.nx, p.ny, p.nz, kq, nbins, want_spectrum ? 1 : 0, part);
  k_sum_columns<<<(width + 255) / 256, 256, 0, st>>>(part, FFT_BLOCKS, width, sums);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;

  std::vector<double> hs(width), hm(FFT_BLOCKS);
  e = cudaMemcpyAsync(hs.data(), sums, width * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hm.data(), mpart, FFT_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  double m = 0.0;
  for (int b = 0; b < FFT_BLOCKS; ++b) m += hm[b];
  out.mass_sum = m;
  out.H.assign(hs.begin(), hs.begin() + nbins);
  for (int q = 0; q < NS; ++q) {
    out.eta[q] = hs[nbins + q];
    out.nharm[q] = hs[nbins + NS + q];
  }
  out.tot = hs[width - 2];
  // n0 is the same in every block's partial; the column sum holds FFT_BLOCKS copies
  out.n0 = 0.0;
  {
    double n0 = 0.0;
    e = cudaMemcpyAsync(&n0, part + (width - 1), sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    out.n0 = n0;
  }
  return cudaSuccess;
}

cudaError_t fft_filtered(const gpe_params& p, const Geom& g, int esz, const void* psi_field, double mscale,
                         double filter_kc, void* work, size_t work_bytes, cudaStream_t st) {
  if (!work || work_bytes < fft_work_bytes(p)) return cudaErrorInvalidValue;
  const long long n = (long long)p.nx * p.ny * p.nz;
  double2* buf = (double2*)work;
  cudaError_t e = to_contiguous(g, esz, psi_field, buf, st);
  if (e != cudaSuccess) return e;
  cufftHandle plan;
  if (!plan_for(p.nx, p.ny, p.nz, &plan)) return cudaErrorUnknown;
  if (cufftSetStream(plan, st) != CUFFT_SUCCESS) return cudaErrorUnknown;
  if (cufftExecZ2Z(plan, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, CUFFT_FORWARD) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  k_filter<<<148 * 8, 256, 0, st>>>(buf, p.nx, p.ny, p.nz, mscale, filter_kc * filter_kc);
  if (cufftExecZ2Z(plan, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  k_div<<<148 * 8, 256, 0, st>>>(buf, n, sqrt((double)n));
  return cudaGetLastError();
}

}  // namespace gpe

// FFT diagnostics on the device: the condensate, temperature and energy
// estimates of condensed_particles (src/io.f90:304-395), the shell and
// integral spectra of spectrum (src/io.f90:668-714) and the low-pass field
// of filtered_surface (src/io.f90:524-571).  The transform is the
// reference's fft (src/ic.f90:910-939): a 3-D complex DFT normalised by
// 1/sqrt(nx ny nz) in both directions, computed here with cuFFT in FP64.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/gpe_cuda.h"
#include "gpe_device.cuh"

namespace gpe {

struct FftDiag {
  double mass_sum = 0;                 // sum |psi|^2 over the grid (variables.f90:618-621)
  double n0 = 0;                       // |a(0,0,0)|^2
  double tot = 0;                      // io.f90:343-360
  double eta[GPE_SPECTRUM_SHELLS] = {};    // shell sums of |a|^2
  double nharm[GPE_SPECTRUM_SHELLS] = {};  // shell site counts
  std::vector<double> H;               // H[b]: sum of |a|^2 over sites with ceil(sqrt(k2)) = b
};

// device scratch of the diagnostics: the N-point transform plus partials
size_t fft_work_bytes(const gpe_params& p);

// Mass, n0, tot and (want_spectrum) the spectra of the psi field.
// kq = the reference's per-axis Laplacian symbols on its k grid (nx + ny + nz
// values, io.f90:347-357), device memory.
cudaError_t fft_condensed(const gpe_params& p, const Geom& g, int esz, const void* psi_field, const double* kq,
                          bool want_spectrum, void* work, size_t work_bytes, cudaStream_t st, FftDiag& out);

// filtered_surface's field: a -> a max(1 - m k2/kc^2, 0) -> inverse; the
// result (nx*ny*nz double2, x fastest) is left at the start of work.
cudaError_t fft_filtered(const gpe_params& p, const Geom& g, int esz, const void* psi_field, double mscale,
                         double filter_kc, void* work, size_t work_bytes, cudaStream_t st);

// the reference's k grid symbols for axis n with spacing d (io.f90:326-357)
void fft_kq_axis(int n, int nx, double d, double* out);

}  // namespace gpe

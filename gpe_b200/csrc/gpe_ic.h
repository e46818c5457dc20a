// Device initial conditions shared by the handle and the pool.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

#include <string>

#include "../../include/gpe_cuda.h"
#include "gpe_device.cuh"

namespace gpe {

int ic_validate(const gpe_ic* ic, std::string& why);
bool ic_needs_fft(const gpe_ic* ic);
// device scratch the generator needs (0 unless an inverse FFT is involved)
size_t ic_work_bytes(const gpe_params& p, const gpe_ic& ic);
// write the initial state (with ghosts) into psi_field on stream st
cudaError_t ic_generate(const gpe_params& p, const Geom& g, int esz, int R, const gpe_ic& ic, void* psi_field,
                        void* work, size_t work_bytes, cudaStream_t st);

// psi <- psi * IC, or |psi| * IC with modulus != 0, in place (closed-form
// factors only: the random-phase state is rejected with cudaErrorInvalidValue)
cudaError_t ic_multiply(const gpe_params& p, const Geom& g, int esz, int R, const gpe_ic& ic, void* psi_field,
                        int modulus, cudaStream_t st);

// cached 3-D Z2Z cuFFT plan for an (nz, ny, nx) grid on the current device
bool plan_for(int nx, int ny, int nz, cufftHandle* out);

}  // namespace gpe

// Stage kernels: complex64 storage, FP64 stencil compute.
#include "gpe_stage_inst.cuh"
GPE_DEFINE_LAUNCHER(f32x, float2, double)

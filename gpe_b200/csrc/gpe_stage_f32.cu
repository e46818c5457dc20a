// Stage kernels: complex64 storage, FP32 stencil compute (FP64 stage
// combinations and reductions).
#include "gpe_stage_inst.cuh"
GPE_DEFINE_LAUNCHER(f32, float2, float)

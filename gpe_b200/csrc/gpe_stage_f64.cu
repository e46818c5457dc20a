// Stage kernels: complex128 storage, FP64 compute.
#include "gpe_stage_inst.cuh"
GPE_DEFINE_LAUNCHER(f64, double2, double)

// Explicit instantiation helper: one translation unit per (storage, compute)
// pair keeps nvcc runs parallel.  Defines
//   cudaError_t launch_stage_<TAG>(int kind, int R, int ty, dim3 grid,
//                                  cudaStream_t st, const StageArgs& a)
#pragma once
#include "gpe_device.cuh"

namespace gpe {

template <class S, class C, int R, int TY>
static cudaError_t launch_kind(int kind, dim3 grid, cudaStream_t st, const StageArgs& a) {
  const dim3 block(32, TY);
  switch (kind) {
#define GPE_CASE(K) \
  case K:           \
    k_stage<S, C, R, K, TY><<<grid, block, 0, st>>>(a); \
    break;
    GPE_CASE(K_EULER)
    GPE_CASE(K_RK2_1)
    GPE_CASE(K_RK2_2)
    GPE_CASE(K_RK4_1)
    GPE_CASE(K_RK4_2)
    GPE_CASE(K_RK4_4)
    GPE_CASE(K_CK_1)
    GPE_CASE(K_CK_2)
    GPE_CASE(K_CK_3)
    GPE_CASE(K_CK_4)
    GPE_CASE(K_CK_5)
    GPE_CASE(K_CK_6)
    GPE_CASE(K_ENERGY)
#undef GPE_CASE
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class S, class C>
static cudaError_t launch_stage_impl(int kind, int R, int ty, dim3 grid, cudaStream_t st, const StageArgs& a) {
  if (ty != 8) return cudaErrorInvalidValue;
  if (R == 1) return launch_kind<S, C, 1, 8>(kind, grid, st, a);
  if (R == 2) return launch_kind<S, C, 2, 8>(kind, grid, st, a);
  return cudaErrorInvalidValue;
}

}  // namespace gpe

#define GPE_DEFINE_LAUNCHER(TAG, S, C)                                                                  \
  namespace gpe {                                                                                       \
  cudaError_t launch_stage_##TAG(int kind, int R, int ty, dim3 grid, cudaStream_t st, const StageArgs& a) { \
    return launch_stage_impl<S, C>(kind, R, ty, grid, st, a);                                           \
  }                                                                                                     \
  }

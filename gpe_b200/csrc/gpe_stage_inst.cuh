// Explicit instantiation helper: one translation unit per (storage, compute)
// pair keeps nvcc runs parallel.  Defines
//   cudaError_t launch_stage_<TAG>(int kind, int R, int ty, dim3 grid,
//                                  cudaStream_t st, const StageArgs& a)
#pragma once
#include "gpe_device.cuh"
#include "gpe_stage_tma.cuh"

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

template <class S, class C, int R, int K, int TY>
static cudaError_t launch_tma_one(dim3 grid, cudaStream_t st, const TmaMaps& m, const StageArgs& a) {
  using LY = TmaLayout<S, R, K, TY>;
  static unsigned long long attr_set = 0;  // per instantiation, one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_stage_tma<S, C, R, K, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)LY::SMEM);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set |= 1ULL << dev;
  }
  k_stage_tma<S, C, R, K, TY><<<grid, dim3(32, TY), LY::SMEM, st>>>(m, a);
  return cudaGetLastError();
}

template <class S, class C, int R, int TY>
static cudaError_t launch_tma_kind(int kind, dim3 grid, cudaStream_t st, const TmaMaps& m, const StageArgs& a) {
  switch (kind) {
#define GPE_TCASE(K) \
  case K:            \
    return launch_tma_one<S, C, R, K, TY>(grid, st, m, a);
    GPE_TCASE(K_EULER)
    GPE_TCASE(K_RK2_1)
    GPE_TCASE(K_RK2_2)
    GPE_TCASE(K_RK4_1)
    GPE_TCASE(K_RK4_2)
    GPE_TCASE(K_RK4_4)
    GPE_TCASE(K_CK_1)
    GPE_TCASE(K_CK_2)
    GPE_TCASE(K_CK_3)
    GPE_TCASE(K_CK_4)
    GPE_TCASE(K_CK_5)
    GPE_TCASE(K_CK_6)
    GPE_TCASE(K_ENERGY)
#undef GPE_TCASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <class S, class C>
static cudaError_t launch_stage_tma_impl(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                         const StageArgs& a) {
  if (ty != 8) return cudaErrorInvalidValue;
  if (R == 1) return launch_tma_kind<S, C, 1, 8>(kind, grid, st, m, a);
  if (R == 2) return launch_tma_kind<S, C, 2, 8>(kind, grid, st, m, a);
  return cudaErrorInvalidValue;
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
  cudaError_t launch_stage_tma_##TAG(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m, \
                                     const StageArgs& a) {                                              \
    return launch_stage_tma_impl<S, C>(kind, R, ty, grid, st, m, a);                                    \
  }                                                                                                     \
  }

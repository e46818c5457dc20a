// Explicit instantiation helper: one translation unit per (storage, compute)
// pair keeps nvcc runs parallel.  Defines
//   cudaError_t launch_stage_<TAG>(int kind, int R, int ty, dim3 grid,
//                                  cudaStream_t st, const StageArgs& a)
#pragma once
#include <cstdlib>
#include <memory>
#include <type_traits>

#include "gpe_device.cuh"
#include "gpe_stage_tma.cuh"

namespace gpe {

// rows of the 32 x 8 tile owned by each thread of the batched kernel
constexpr int BATCH_PY = 2;

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
    GPE_CASE(K_RK4_3)
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

template <class S, class C, int R, int K, int TY, int PY>
static cudaError_t launch_tma_one(dim3 grid, cudaStream_t st, const TmaMaps& m, const StageArgs& a) {
  using LY = TmaLayout<S, R, StageTraits<K>::NPW, TY>;
  static unsigned long long attr_set = 0;  // per instantiation, one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_stage_tma<S, C, R, K, TY, PY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::SMEM);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set |= 1ULL << dev;
  }
  k_stage_tma<S, C, R, K, TY, PY><<<grid, dim3(32, TY / PY), LY::SMEM, st>>>(m, a);
  return cudaGetLastError();
}

template <class S, class C, int R, int TY, int PY>
static cudaError_t launch_tma_kind(int kind, dim3 grid, cudaStream_t st, const TmaMaps& m, const StageArgs& a) {
  switch (kind) {
#define GPE_TCASE(K) \
  case K:            \
    return launch_tma_one<S, C, R, K, TY, PY>(grid, st, m, a);
    GPE_TCASE(K_EULER)
    GPE_TCASE(K_RK2_1)
    GPE_TCASE(K_RK2_2)
    GPE_TCASE(K_RK4_1)
    GPE_TCASE(K_RK4_2)
    GPE_TCASE(K_RK4_3)
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

template <class C, int R, int K, int TY, int PY>
static cudaError_t launch_tma_pair_one(dim3 grid, cudaStream_t st, const TmaMaps& m, const StageArgs& a) {
  using LY = TmaLayout<float2, R, StageTraits<K>::NPW, TY>;
  static unsigned long long attr_set = 0;  // per instantiation, one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !(attr_set & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_stage_tma_pair<C, R, K, TY, PY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::SMEM);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_set |= 1ULL << dev;
  }
  k_stage_tma_pair<C, R, K, TY, PY><<<grid, dim3(16, TY / PY), LY::SMEM, st>>>(m, a);
  return cudaGetLastError();
}

template <class C, int R, int TY, int PY>
static cudaError_t launch_tma_pair_kind(int kind, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                        const StageArgs& a) {
  switch (kind) {
#define GPE_PCASE(K) \
  case K:            \
    return launch_tma_pair_one<C, R, K, TY, PY>(grid, st, m, a);
    GPE_PCASE(K_EULER)
    GPE_PCASE(K_RK2_1)
    GPE_PCASE(K_RK2_2)
    GPE_PCASE(K_RK4_1)
    GPE_PCASE(K_RK4_2)
    GPE_PCASE(K_RK4_3)
    GPE_PCASE(K_RK4_4)
    GPE_PCASE(K_CK_1)
    GPE_PCASE(K_CK_2)
    GPE_PCASE(K_CK_3)
    GPE_PCASE(K_CK_4)
    GPE_PCASE(K_CK_5)
    GPE_PCASE(K_CK_6)
    GPE_PCASE(K_ENERGY)
#undef GPE_PCASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <class S, class C>
static cudaError_t launch_stage_tma_impl(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                         const StageArgs& a) {
  // ty is a TileVariant: TILE_32x8_ROW1 / TILE_32x8_ROW2 (any storage), or
  // the pair layouts (complex64 storage with FP32 stencil compute)
  if constexpr (std::is_same<S, float2>::value && std::is_same<C, float>::value) {
    if (ty == TILE_PAIR_32x8) {
      if (R == 1) return launch_tma_pair_kind<C, 1, 8, 1>(kind, grid, st, m, a);
      if (R == 2) return launch_tma_pair_kind<C, 2, 8, 1>(kind, grid, st, m, a);
    } else if (ty == TILE_PAIR_32x16) {
      if (R == 1) return launch_tma_pair_kind<C, 1, 16, 2>(kind, grid, st, m, a);
      if (R == 2) return launch_tma_pair_kind<C, 2, 16, 2>(kind, grid, st, m, a);
    }
  }
  if (ty == 8) {
    if (R == 1) return launch_tma_kind<S, C, 1, 8, 1>(kind, grid, st, m, a);
    if (R == 2) return launch_tma_kind<S, C, 2, 8, 1>(kind, grid, st, m, a);
  } else if (ty == 4) {
    if (R == 1) return launch_tma_kind<S, C, 1, 8, 2>(kind, grid, st, m, a);
    if (R == 2) return launch_tma_kind<S, C, 2, 8, 2>(kind, grid, st, m, a);
  }
  return cudaErrorInvalidValue;
}

// The batched kernel's thread layout for complex64 storage with the FP32
// stencil: two x-adjacent sites per thread (GPE_BATCH_PAIR=0 selects the
// one-site-per-column layout instead).
inline bool batch_pair_layout() {
  static const bool on = [] {
    const char* e = getenv("GPE_BATCH_PAIR");
    return !(e && atoi(e) == 0);
  }();
  return on;
}

// Item rows of the batched RK4 kernels for complex64 storage with the FP32
// stencil: 32 x 16 items with two rows of x pairs per thread (four sites),
// as the single-solve kernel; GPE_BATCH_ROWS=8 selects 32 x 8 items with one
// row per thread.  With one stencil radius per kernel the four-site body
// fits 4 CTAs per SM without spills: 44.0-44.3 against 42.4-42.6 G
// site-updates/s on the uneven mix of 32^3-160^3 solves.  Every other class
// uses 32 x 8 items.
inline int batch_rk4_f32_rows() {
  static const int rows = [] {
    const char* e = getenv("GPE_BATCH_ROWS");
    return (e && atoi(e) == 8) || !batch_pair_layout() ? 8 : 16;
  }();
  return rows;
}

__host__ __device__ constexpr bool is_rk4_kind(int k) {
  return k == K_RK4_1 || k == K_RK4_2 || k == K_RK4_3 || k == K_RK4_4;
}

// Opt the batched kernel into its dynamic shared memory once per device and
// cache how many of its CTAs fit on the device at once.
template <class S, class C, int K, int TY, bool PAIR, int RR, bool PARG = false>
static cudaError_t batch_setup(int* occupancy) {
  using LY = TmaLayout<S, RR, StageTraits<K>::NPW, TY>;
  static unsigned long long done = 0;
  static int occ[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return cudaErrorInvalidDevice;
  if (!(done & (1ULL << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_stage_batch<S, C, K, TY, BATCH_PY, PAIR, RR, PARG>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LY::SMEM);
    if (e != cudaSuccess) return e;
    int nsm = 0, per = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_stage_batch<S, C, K, TY, BATCH_PY, PAIR, RR, PARG>,
                                                      batch_threads<TY, BATCH_PY, PAIR>(), LY::SMEM);
    if (e != cudaSuccess) return e;
    occ[dev] = nsm * (per > 0 ? per : 1);
    done |= 1ULL << dev;
  }
  if (occupancy) *occupancy = occ[dev];
  return cudaSuccess;
}

// One launch; with at most BATCH_PARAM_SOLVES solves their stage arguments
// go into the launch's parameter space (the PARG kernel), else the kernel
// reads them from the device table.  FP32 Cash-Karp stages keep the table
// path: their item bodies read the arguments so often per site that
// constant-cache reads cost more than the registers they free (a batch of
// 16 FP32 RKF45 solves: 9.8 against 10.5 G accepted site-updates/s; FP64
// Cash-Karp gains 14 %, the RK4 stages 4 %).
template <class S, class C, int K, int TY, bool PAIR, int RR>
static cudaError_t launch_batch_one(int grid, cudaStream_t st, const BatchLaunch& b) {
  using LY = TmaLayout<S, RR, StageTraits<K>::NPW, TY>;
  const dim3 block = PAIR ? dim3(16, 8) : dim3(32, TY / BATCH_PY);
  constexpr bool kParamArgs = !(sizeof(C) == sizeof(float) && K >= K_CK_1 && K <= K_CK_6);
  if constexpr (kParamArgs) {
    if (b.htab && b.ns >= 1 && b.ns <= BATCH_PARAM_SOLVES) {
      cudaError_t e = batch_setup<S, C, K, TY, PAIR, RR, true>(nullptr);
      if (e != cudaSuccess) return e;
      thread_local std::unique_ptr<BatchArgs> pa;  // 32 KB staging, copied by the launch
      if (!pa) pa.reset(new BatchArgs);
      for (int q = 0; q < b.ns; ++q) pa->a[q] = b.htab[q].args;
      k_stage_batch<S, C, K, TY, BATCH_PY, PAIR, RR, true>
          <<<grid, block, LY::SMEM, st>>>(b.tab, b.items, b.order, b.nitems, b.queue, b.partials, *pa);
      return cudaGetLastError();
    }
  }
  cudaError_t e = batch_setup<S, C, K, TY, PAIR, RR, false>(nullptr);
  if (e != cudaSuccess) return e;
  k_stage_batch<S, C, K, TY, BATCH_PY, PAIR, RR, false>
      <<<grid, block, LY::SMEM, st>>>(b.tab, b.items, b.order, b.nitems, b.queue, b.partials, NoBatchArgs{});
  return cudaGetLastError();
}

// CTAs of the kernel launch_batch_one would launch for b that fit on the
// device at once (b.ns picks the parameter-space or the table kernel).
template <class S, class C, int K, int TY, bool PAIR, int RR>
static cudaError_t batch_occupancy(const BatchLaunch& b, int* occupancy) {
  constexpr bool kParamArgs = !(sizeof(C) == sizeof(float) && K >= K_CK_1 && K <= K_CK_6);
  if constexpr (kParamArgs) {
    if (b.ns >= 1 && b.ns <= BATCH_PARAM_SOLVES) return batch_setup<S, C, K, TY, PAIR, RR, true>(occupancy);
  }
  return batch_setup<S, C, K, TY, PAIR, RR, false>(occupancy);
}

template <class S, class C, int K, int RR>
static cudaError_t launch_batch_kind_r(int grid, cudaStream_t st, const BatchLaunch& b, int* occupancy) {
  if constexpr (std::is_same<S, float2>::value && std::is_same<C, float>::value) {
    if constexpr (is_rk4_kind(K)) {
      if (batch_rk4_f32_rows() == 16) {
        if (grid <= 0) return batch_occupancy<S, C, K, 16, true, RR>(b, occupancy);
        return launch_batch_one<S, C, K, 16, true, RR>(grid, st, b);
      }
    }
    if (batch_pair_layout()) {
      if (grid <= 0) return batch_occupancy<S, C, K, 8, true, RR>(b, occupancy);
      return launch_batch_one<S, C, K, 8, true, RR>(grid, st, b);
    }
  }
  if (grid <= 0) return batch_occupancy<S, C, K, 8, false, RR>(b, occupancy);
  return launch_batch_one<S, C, K, 8, false, RR>(grid, st, b);
}

template <class S, class C, int K>
static cudaError_t launch_batch_kind(int R, int grid, cudaStream_t st, const BatchLaunch& b, int* occupancy) {
  if (R == 1) return launch_batch_kind_r<S, C, K, 1>(grid, st, b, occupancy);
  if (R == 2) return launch_batch_kind_r<S, C, K, 2>(grid, st, b, occupancy);
  return cudaErrorInvalidValue;
}

template <class S, class C>
static cudaError_t launch_batch_impl(int kind, int R, int grid, cudaStream_t st, const BatchLaunch& b,
                                     int* occupancy) {
  switch (kind) {
#define GPE_BCASE(K) \
  case K:            \
    return launch_batch_kind<S, C, K>(R, grid, st, b, occupancy);
    GPE_BCASE(K_RK4_1)
    GPE_BCASE(K_RK4_2)
    GPE_BCASE(K_RK4_3)
    GPE_BCASE(K_RK4_4)
    GPE_BCASE(K_CK_1)
    GPE_BCASE(K_CK_2)
    GPE_BCASE(K_CK_3)
    GPE_BCASE(K_CK_4)
    GPE_BCASE(K_CK_5)
    GPE_BCASE(K_CK_6)
#undef GPE_BCASE
    default:
      return cudaErrorInvalidValue;
  }
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
  int batch_rows_##TAG(int kind) {                                                                      \
    return (std::is_same<S, float2>::value && std::is_same<C, float>::value && is_rk4_kind(kind))          \
               ? batch_rk4_f32_rows()                                                                    \
               : 8;                                                                                      \
  }                                                                                                       \
  cudaError_t launch_batch_##TAG(int kind, int R, int grid, cudaStream_t st, const BatchLaunch& b,      \
                                 int* occupancy) {                                                     \
    return launch_batch_impl<S, C>(kind, R, grid, st, b, occupancy);                                    \
  }                                                                                                     \
  }

// Fused stage kernel, TMA version (sm_100a).
//
// Same per-site work as k_stage (site_stage), but every input plane reaches
// shared memory through the Tensor Memory Accelerator: one
// cp.async.bulk.tensor.3d per plane tile, completion tracked by an mbarrier
// per ring slot.  Two rings per CTA:
//   * stencil ring, NSS slots: tile (32 + 4) x (TY + 2R) of the stencil input
//     (x halo of 2 keeps every box start 16-byte aligned also for complex64;
//     y halo R).  z neighbours come from a per-thread register queue fed from
//     the tile centres, x/y neighbours straight from the tile.
//   * point-wise ring, NPS slots: tiles 32 x TY of psi / acc / K_j.
// One elected thread issues the copies NSS-(R+1) (stencil) and NPS-1
// (point-wise) planes ahead of use, so the memory pipeline is deep without
// spending registers on prefetch.  Boxes that stick out of the ghost-padded
// tensor are zero-filled by the TMA unit (loads only; nothing is stored with
// TMA).  Every mbarrier wait is bounded: on expiry the CTA records an error
// in a.status, drains the copies it issued (bounded again) and returns.
#pragma once
#include <cuda.h>

#include "gpe_device.cuh"

namespace gpe {

constexpr int TMA_TX = 32;
constexpr int TMA_HX = 2;

struct TmaMaps {
  CUtensorMap in;     // stencil input: box (2*(TMA_TX+2*TMA_HX)) x (TY+2R) x 1 scalars
  CUtensorMap pw[5];  // point-wise inputs: box (2*TMA_TX) x TY x 1 scalars
};

// box sizes shared by host (tensor-map encoding) and device (expect_tx)
__host__ __device__ constexpr int tma_stencil_w() { return TMA_TX + 2 * TMA_HX; }
__host__ __device__ constexpr int tma_stencil_h(int ty, int R) { return ty + 2 * R; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after ~2^31 SM cycles (about a second) or 2^26
// polls, whichever comes first.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 0; it < (1 << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > (1LL << 31)) break;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

template <class S, int R, int KIND, int TY>
struct TmaLayout {
  static constexpr int NPW = StageTraits<KIND>::NPW;
  static constexpr int NSS = 2 * R + 2;                       // stencil ring slots
  static constexpr int NPS = 3;                               // point-wise ring slots
  static constexpr uint32_t ST_BYTES = tma_stencil_w() * (TY + 2 * R) * sizeof(S);
  static constexpr uint32_t PW1_BYTES = TMA_TX * TY * sizeof(S);
  static constexpr uint32_t ST_SLOT = (ST_BYTES + 127) / 128 * 128;
  static constexpr uint32_t PW_SLOT = (NPW * PW1_BYTES + 127) / 128 * 128;
  static constexpr uint32_t BAR_BYTES = 128;
  // dynamic shared memory: barriers + rings + 128 B of alignment slack
  static constexpr uint32_t SMEM = BAR_BYTES + NSS * ST_SLOT + (NPW > 0 ? NPS * PW_SLOT : 0) + 128;
};

template <class S, class C, int R, int KIND, int TY>
__global__ void __launch_bounds__(32 * TY) k_stage_tma(const __grid_constant__ TmaMaps maps, const StageArgs a) {
  using T = StageTraits<KIND>;
  using LY = TmaLayout<S, R, KIND, TY>;
  constexpr int TX = TMA_TX, HX = TMA_HX, TW = tma_stencil_w();
  constexpr int NT = TX * TY, NSS = LY::NSS, NPS = LY::NPS, NPW = T::NPW;

  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_abort;
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* sbar = (uint64_t*)smem;   // NSS stencil barriers
  uint64_t* pbar = sbar + NSS;        // NPS point-wise barriers
  unsigned char* sring = smem + LY::BAR_BYTES;
  unsigned char* pring = sring + NSS * LY::ST_SLOT;

  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = blockIdx.x * TX + tx;
  const int j = blockIdx.y * TY + ty;
  const int kb = blockIdx.z * a.zc;
  const int ke = min(kb + a.zc, g.nz);
  const int M = ke - kb;          // planes updated by this CTA
  const int L = M + 2 * R;        // stencil planes read: kb-R .. ke+R-1
  const bool active = (i < g.nx) && (j < g.ny);
  const long long col = (long long)(j + 2) * g.px + g.xoff + i;

  // box origins in the padded tensor, in scalars (x) / rows (y) / planes (z)
  const int cxs = 2 * (g.xoff + blockIdx.x * TX - HX);
  const int cys = blockIdx.y * TY - R + 2;
  const int cxp = 2 * (g.xoff + blockIdx.x * TX);
  const int cyp = blockIdx.y * TY + 2;

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < NSS; ++s) mbar_init(&sbar[s], 1);
    for (int s = 0; s < NPS; ++s) mbar_init(&pbar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  int issued_s = 0, issued_p = 0;  // meaningful in thread 0 only
  auto issue_stencil = [&](int l) {
    const int s = l % NSS;
    mbar_arrive_expect_tx(&sbar[s], LY::ST_BYTES);
    tma_load_3d(sring + s * LY::ST_SLOT, &maps.in, &sbar[s], cxs, cys, kb - R + l + 2);
    issued_s = l + 1;
  };
  auto issue_pw = [&](int m) {
    if constexpr (NPW > 0) {
      const int s = m % NPS;
      mbar_arrive_expect_tx(&pbar[s], NPW * LY::PW1_BYTES);
#pragma unroll
      for (int f = 0; f < NPW; ++f)
        tma_load_3d(pring + s * LY::PW_SLOT + f * LY::PW1_BYTES, &maps.pw[f], &pbar[s], cxp, cyp, kb + m + 2);
      issued_p = m + 1;
    }
  };
  // on a timed-out wait: flag the error, let every copy this CTA issued land
  // (bounded), then leave
  auto drain = [&](int waited_s, int waited_p) {
    if (tid == 0) {
      atomicExch(a.status, 1);
      for (int l = waited_s; l < issued_s; ++l) mbar_wait_bounded(&sbar[l % NSS], (l / NSS) & 1);
      for (int m = waited_p; m < issued_p; ++m) mbar_wait_bounded(&pbar[m % NPS], (m / NPS) & 1);
    }
    __syncthreads();
  };

  if (tid == 0) {
    for (int l = 0; l < min(NSS, L); ++l) issue_stencil(l);
    for (int m = 0; m < min(NPS, M); ++m) issue_pw(m);
  }

  const int cofs = (ty + R) * TW + tx + HX;  // this thread's centre in a stencil tile
  S q[2 * R + 1];
  bool ok = true;
#pragma unroll
  for (int l = 0; l < 2 * R; ++l) {
    ok &= mbar_wait_bounded(&sbar[l % NSS], (l / NSS) & 1);
    q[l] = ((const S*)(sring + (l % NSS) * LY::ST_SLOT))[cofs];
  }
  if (!ok) s_abort = 1;
  __syncthreads();
  if (s_abort) {
    drain(2 * R, 0);
    return;
  }
  if (tid == 0) {
    fence_proxy_async();
    for (int l = 0; l < R; ++l)
      if (l + NSS < L) issue_stencil(l + NSS);
  }

  const ColumnConsts cc = column_consts(a, i, j, R, active);
  double r_norm = 0.0, r_en = 0.0, r_err = 0.0;

  for (int m = 0; m < M; ++m) {
    const int k = kb + m;
    const int lc = m + R, ll = m + 2 * R;
    bool okw = mbar_wait_bounded(&sbar[ll % NSS], (ll / NSS) & 1);
    q[2 * R] = ((const S*)(sring + (ll % NSS) * LY::ST_SLOT))[cofs];
    const S* pws = nullptr;
    if constexpr (NPW > 0) {
      okw &= mbar_wait_bounded(&pbar[m % NPS], (m / NPS) & 1);
      pws = (const S*)(pring + (m % NPS) * LY::PW_SLOT);
    }
    if (!okw) s_abort = 1;

    if (active && okw) {
      const S* tile = (const S*)(sring + (lc % NSS) * LY::ST_SLOT);
      Nb<C> n;
      n.c0 = to_c<C>(q[R]);
      n.xm1 = to_c<C>(tile[cofs - 1]);
      n.xp1 = to_c<C>(tile[cofs + 1]);
      n.ym1 = to_c<C>(tile[cofs - TW]);
      n.yp1 = to_c<C>(tile[cofs + TW]);
      n.zm1 = to_c<C>(q[R - 1]);
      n.zp1 = to_c<C>(q[R + 1]);
      if constexpr (R == 2) {
        n.xm2 = to_c<C>(tile[cofs - 2]);
        n.xp2 = to_c<C>(tile[cofs + 2]);
        n.ym2 = to_c<C>(tile[cofs - 2 * TW]);
        n.yp2 = to_c<C>(tile[cofs + 2 * TW]);
        n.zm2 = to_c<C>(q[0]);
        n.zp2 = to_c<C>(q[4]);
      } else {
        n.xm2 = n.xp2 = n.ym2 = n.yp2 = n.zm2 = n.zp2 = cx<C>{0, 0};
      }
      S pv[NPW > 0 ? NPW : 1];
#pragma unroll
      for (int f = 0; f < NPW; ++f) pv[f] = pws[f * (TX * TY) + tid];
      site_stage<S, C, R, KIND>(a, n, pv, i, j, k, col, cc, r_norm, r_en, r_err);
    }
#pragma unroll
    for (int d = 0; d < 2 * R; ++d) q[d] = q[d + 1];

    __syncthreads();  // every thread is done with stencil slot lc and point-wise slot m
    if (s_abort) {
      drain(ll + 1, m + 1);
      return;
    }
    if (tid == 0) {
      fence_proxy_async();
      if (lc + NSS < L) issue_stencil(lc + NSS);
      if (m + NPS < M) issue_pw(m + NPS);
    }
  }

  if (a.partials) block_reduce_store<NT>(r_norm, r_en, r_err, a.partials);
}

}  // namespace gpe

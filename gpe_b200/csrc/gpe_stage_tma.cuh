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

#include <type_traits>

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

// Bounded wait: gives up after ~2^31 SM cycles (about a second) or
// max_polls polls, whichever comes first.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int max_polls = 1 << 26) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 0; it < max_polls; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > (1LL << 31)) break;
  }
  return false;
}

// Device status word values (StageArgs::status).  STATUS_EXPIRE_TEST is set
// by the host only (gpe_test_expire_waits): while it stands, every work item
// first waits, with a short limit, on a barrier that nothing arrives at, so
// that the timeout path (abort, drain the issued copies, return) runs; the
// word keeps the value until the host reads and clears it.
constexpr int STATUS_OK = 0;
constexpr int STATUS_WAIT_EXPIRED = 1;
constexpr int STATUS_EXPIRE_TEST = 2;
constexpr int EXPIRE_TEST_POLLS = 1 << 10;

// Copy stage arguments from the device table through the read-only path.
__device__ __forceinline__ StageArgs __ldg_args(const StageArgs* p) {
  StageArgs a;
  const uint4* src = reinterpret_cast<const uint4*>(p);
  uint4* dst = reinterpret_cast<uint4*>(&a);
#pragma unroll
  for (int q = 0; q < (int)(sizeof(StageArgs) / sizeof(uint4)); ++q) dst[q] = __ldg(src + q);
  return a;
}

// Order a tensor map that sits in global memory (written by the host
// between launches) before the async proxy reads it.
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((uint64_t)map) : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

template <class S>
__host__ __device__ constexpr uint32_t tma_st_bytes(int R, int TY) {
  return (uint32_t)(tma_stencil_w() * (TY + 2 * R) * sizeof(S));
}
template <class S>
__host__ __device__ constexpr uint32_t tma_pw1_bytes(int TY) {
  return (uint32_t)(TMA_TX * TY * sizeof(S));
}
__host__ __device__ constexpr uint32_t round128(uint32_t b) { return (b + 127) / 128 * 128; }

// Shared-memory layout of the two rings.  RMAX sizes the stencil slots (a
// batched launch mixes R = 1 and R = 2 solves in the same rings).
template <class S, int RMAX, int NPW, int TY>
struct TmaLayout {
  static constexpr int NSS = 2 * RMAX + 2;  // stencil ring slots
  static constexpr int NPS = 3;             // point-wise ring slots
  static constexpr int NEVER_BAR = 15;      // barrier nothing arrives at (timeout test), last of 16
  static constexpr uint32_t ST_SLOT = round128(tma_st_bytes<S>(RMAX, TY));
  static constexpr uint32_t PW_SLOT = round128(NPW * tma_pw1_bytes<S>(TY));
  static constexpr uint32_t BAR_BYTES = 128;
  static_assert(NSS + NPS <= NEVER_BAR, "ring barriers overlap the never-arriving one");
  // dynamic shared memory: barriers + rings + 128 B of alignment slack
  static constexpr uint32_t SMEM = BAR_BYTES + NSS * ST_SLOT + (NPW > 0 ? NPS * PW_SLOT : 0) + 128;
};

// Ring state of one CTA.  Loads are numbered globally over the CTA's
// lifetime (a persistent CTA processes many work items): load G sits in
// slot G % NSS and completes phase G / NSS of that slot's barrier.
struct TmaRing {
  uint64_t* sbar;
  uint64_t* pbar;
  uint64_t* nbar;  // no thread or copy ever arrives here
  unsigned char* sring;
  unsigned char* pring;
  int sbase, pbase;  // loads issued for earlier work items
};

template <class LY>
__device__ __forceinline__ TmaRing tma_ring_setup(unsigned char* smem_raw, int* s_abort) {
  // align by pointer arithmetic on the __shared__ array itself (an integer
  // round trip would hide the state space and turn every ring read into a
  // generic load)
  unsigned char* smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  TmaRing rg;
  rg.sbar = (uint64_t*)smem;
  rg.pbar = rg.sbar + LY::NSS;
  rg.nbar = rg.sbar + LY::NEVER_BAR;
  rg.sring = smem + LY::BAR_BYTES;
  rg.pring = rg.sring + LY::NSS * LY::ST_SLOT;
  rg.sbase = rg.pbase = 0;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    *s_abort = 0;
    for (int s = 0; s < LY::NSS; ++s) mbar_init(&rg.sbar[s], 1);
    for (int s = 0; s < LY::NPS; ++s) mbar_init(&rg.pbar[s], 1);
    mbar_init(rg.nbar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  return rg;
}

// One work item: the 32 x TY tile (bx, by) of planes [bz*zc, bz*zc+zc) of one
// solve, processed by 32 x (TY/PY) threads, each owning PY rows of the tile
// (rows ty, ty + TY/PY, ...) so that the per-plane waits, barrier and ring
// bookkeeping are shared by PY sites.  Returns false when a bounded wait
// expired (the caller must stop; the copies this item issued have been
// drained and a.status set).
// Unroll factor of the single-solve kernels' z march.  RK4 stages at
// 256^3, 2 against 1: +0.7 % complex64 (pair kernel), +1.2 % complex128;
// 3 against 2: -0.9 % complex64, +0.5 % complex128.  The Cash-Karp stages
// of the 192^2 x 384 RKF45 solve lose 1.5 % with 3 (complex128), so the
// other schemes keep 1, as does the persistent batched kernel (2 cost 1 %
// on the uneven batch).
template <class S, int KIND>
__host__ __device__ constexpr int single_zu() {
  return (KIND == K_RK4_1 || KIND == K_RK4_2 || KIND == K_RK4_3 || KIND == K_RK4_4) ? (sizeof(S) == 16 ? 3 : 2)
                                                                                     : 1;
}

// ZU: unroll factor of the z march (the z-queue shifts are renamed across
// ZU planes); see single_zu.
template <class S, class C, int R, int KIND, int TY, int PY, class LY, int ZU = 1>
__device__ __forceinline__ bool tma_item(const TmaMaps& maps, const StageArgs& a, int bx, int by, int bz,
                                         TmaRing& rg, int* s_abort, double& r_norm, double& r_en,
                                         double& r_err) {
  using T = StageTraits<KIND>;
  constexpr int TX = TMA_TX, HX = TMA_HX, TW = tma_stencil_w(), TYT = TY / PY;
  constexpr int NSS = LY::NSS, NPS = LY::NPS, NPW = T::NPW;
  constexpr uint32_t ST_BYTES = tma_st_bytes<S>(R, TY), PW1 = tma_pw1_bytes<S>(TY);
  static_assert(TY % PY == 0, "PY must divide TY");

  const Geom& g = a.g;
  const int tx = threadIdx.x, tyt = threadIdx.y, tid = tyt * TX + tx;
  const int i = bx * TX + tx;
  const int kb = bz * a.zc;
  const int ke = min(kb + a.zc, g.nz);
  const int M = ke - kb;    // planes updated by this item
  const int L = M + 2 * R;  // stencil planes read: kb-R .. ke+R-1
  const int SB = rg.sbase, PB = rg.pbase;

  // box origins in the padded tensor, in scalars (x) / rows (y) / planes (z)
  const int cxs = 2 * (g.xoff + bx * TX - HX);
  const int cys = by * TY - R + 2;
  const int cxp = 2 * (g.xoff + bx * TX);
  const int cyp = by * TY + 2;

  int issued_s = 0, issued_p = 0;  // meaningful in thread 0 only
  auto issue_stencil = [&](int l) {
    const int G = SB + l, s = G % NSS;
    mbar_arrive_expect_tx(&rg.sbar[s], ST_BYTES);
    tma_load_3d(rg.sring + s * LY::ST_SLOT, &maps.in, &rg.sbar[s], cxs, cys, kb - R + l + 2);
    issued_s = l + 1;
  };
  auto issue_pw = [&](int m) {
    if constexpr (NPW > 0) {
      const int G = PB + m, s = G % NPS;
      mbar_arrive_expect_tx(&rg.pbar[s], NPW * PW1);
#pragma unroll
      for (int f = 0; f < NPW; ++f)
        tma_load_3d(rg.pring + s * LY::PW_SLOT + f * PW1, &maps.pw[f], &rg.pbar[s], cxp, cyp, kb + m + 2);
      issued_p = m + 1;
    }
  };
  auto swait = [&](int l) { return mbar_wait_bounded(&rg.sbar[(SB + l) % NSS], ((SB + l) / NSS) & 1); };
  auto pwait = [&](int m) { return mbar_wait_bounded(&rg.pbar[(PB + m) % NPS], ((PB + m) / NPS) & 1); };
  // on a timed-out wait: flag the error, let every copy this item issued land
  // (bounded), then leave
  auto drain = [&](int waited_s, int waited_p) {
    if (tid == 0) {
      atomicCAS(a.status, STATUS_OK, STATUS_WAIT_EXPIRED);  // a standing test value stays
      for (int l = waited_s; l < issued_s; ++l) swait(l);
      for (int m = waited_p; m < issued_p; ++m) pwait(m);
    }
    __syncthreads();
  };

  if (tid == 0) {
    for (int l = 0; l < min(NSS, L); ++l) issue_stencil(l);
    for (int m = 0; m < min(NPS, M); ++m) issue_pw(m);
  }

  // per owned row: grid row, activity, centre offset in a stencil tile
  int jr[PY], cofs[PY];
  bool act[PY];
  long long o[PY];  // element offset of (i, j, k)
  ColumnConsts<C> cc[PY];
#pragma unroll
  for (int r = 0; r < PY; ++r) {
    const int ty = tyt + r * TYT;
    jr[r] = by * TY + ty;
    act[r] = (i < g.nx) && (jr[r] < g.ny);
    cofs[r] = (ty + R) * TW + tx + HX;
    o[r] = (long long)(kb + 2) * g.pz + (long long)(jr[r] + 2) * g.px + g.xoff + i;
    cc[r] = column_consts<C>(a, i, jr[r], R, act[r]);
  }
  // does this tile hold a site with an x or y ghost?  Ghosts come from the
  // index ranges [0, R] and [n-1-R, n-1] of an axis only.
  const bool xyg = (bx * TX <= R) || (bx * TX + TX - 1 >= g.nx - 1 - R) || (by * TY <= R) ||
                   (by * TY + TY - 1 >= g.ny - 1 - R);

  auto stile = [&](int l) { return (const S*)(rg.sring + ((SB + l) % NSS) * LY::ST_SLOT); };
  S q[PY][2 * R + 1];  // z queue of each owned row: planes k-R .. k+R
  bool ok = true;
  // timeout test (host-armed only): wait, with a short limit, on the barrier
  // nothing arrives at; it expires and the item takes the abort path below
  // with its first copies in flight
  if (*(volatile const int*)a.status == STATUS_EXPIRE_TEST)
    ok = mbar_wait_bounded(rg.nbar, 0, EXPIRE_TEST_POLLS);
#pragma unroll
  for (int l = 0; l < 2 * R; ++l) {
    ok &= swait(l);
    const S* tl = stile(l);
#pragma unroll
    for (int r = 0; r < PY; ++r) q[r][l] = tl[cofs[r]];
  }
  if (!ok) *s_abort = 1;
  __syncthreads();
  if (*s_abort) {
    drain(0, 0);
    return false;
  }
  if (tid == 0) {
    fence_proxy_async();
    for (int l = 0; l < R; ++l)
      if (l + NSS < L) issue_stencil(l + NSS);
  }

  // ring cursors (slot, phase parity) of the lead plane, the centre plane
  // and the point-wise plane, advanced incrementally
  int sl_s = (SB + 2 * R) % NSS, sl_p = ((SB + 2 * R) / NSS) & 1;
  int sc_s = (SB + R) % NSS;
  int pw_s = PB % NPS, pw_p = (PB / NPS) & 1;

#pragma unroll ZU
  for (int m = 0; m < M; ++m) {
    const int k = kb + m;
    const int lc = m + R, ll = m + 2 * R;
    bool okw = mbar_wait_bounded(&rg.sbar[sl_s], sl_p);
    {
      const S* tl = (const S*)(rg.sring + sl_s * LY::ST_SLOT);
#pragma unroll
      for (int r = 0; r < PY; ++r) q[r][2 * R] = tl[cofs[r]];
    }
    const S* pws = nullptr;
    if constexpr (NPW > 0) {
      okw &= mbar_wait_bounded(&rg.pbar[pw_s], pw_p);
      pws = (const S*)(rg.pring + pw_s * LY::PW_SLOT);
    }
    if (!okw) *s_abort = 1;

    if (okw) {
      const S* tile = (const S*)(rg.sring + sc_s * LY::ST_SLOT);
      const int gz = (k <= R || k >= g.nz - 1 - R) ? zghost_pos(k, g.nz, R, a.bcs, a.zghost) : NOGHOST;
      // each row's neighbourhood is reduced to its Laplacian (and, with
      // Urhs, x-derivative) right after its loads, so one row's neighbours
      // are live at a time
      cx<C> lap[PY], c0v[PY], dpx[PY];
      S pv[PY][NPW > 0 ? NPW : 1];
#pragma unroll
      for (int r = 0; r < PY; ++r) {
        const int c0 = cofs[r];
        Nb<C> n;
        n.c0 = to_c<C>(q[r][R]);
        n.xm1 = to_c<C>(tile[c0 - 1]);
        n.xp1 = to_c<C>(tile[c0 + 1]);
        n.ym1 = to_c<C>(tile[c0 - TW]);
        n.yp1 = to_c<C>(tile[c0 + TW]);
        n.zm1 = to_c<C>(q[r][R - 1]);
        n.zp1 = to_c<C>(q[r][R + 1]);
        if constexpr (R == 2) {
          n.xm2 = to_c<C>(tile[c0 - 2]);
          n.xp2 = to_c<C>(tile[c0 + 2]);
          n.ym2 = to_c<C>(tile[c0 - 2 * TW]);
          n.yp2 = to_c<C>(tile[c0 + 2 * TW]);
          n.zm2 = to_c<C>(q[r][0]);
          n.zp2 = to_c<C>(q[r][4]);
        } else {
          n.xm2 = n.xp2 = n.ym2 = n.yp2 = n.zm2 = n.zp2 = cx<C>{0, 0};
        }
        lap[r] = site_lap<C, R>(a, n);
        c0v[r] = n.c0;
        dpx[r] = a.has_urhs ? site_dpx<C, R>(a, n) : cx<C>{0, 0};
        const int pofs = (tyt + r * TYT) * TX + tx;
#pragma unroll
        for (int f = 0; f < NPW; ++f) pv[r][f] = pws[f * (TX * TY) + pofs];
      }
      constexpr int NPWX = NPW > 0 ? NPW : 1;
      if constexpr (KIND == K_ENERGY) {
        sites_update<S, C, R, KIND, PY, NPWX>(a, lap, c0v, dpx, pv, act, i, jr, k, o, gz, cc, r_norm, r_en, r_err);
      } else {
        // the sites store their own values only; face ghosts are copied
        // after them, by tiles that touch an x/y face and on the first and
        // last R + 1 planes only (uniform branches, the site code stays one)
        S ns[PY];
        sites_update<S, C, R, KIND, PY, NPWX, false, false>(a, lap, c0v, dpx, pv, act, i, jr, k, o, gz, cc, r_norm,
                                                           r_en, r_err, ns);
        S* out = (S*)a.out;
        if (xyg) {
#pragma unroll
          for (int r = 0; r < PY; ++r)
            if (act[r]) {
              if (cc[r].gx != NOGHOST) out[o[r] + (cc[r].gx - i)] = ns[r];
              if (cc[r].gy != NOGHOST) out[o[r] + (long long)(cc[r].gy - jr[r]) * g.px] = ns[r];
            }
        }
        if (gz != NOGHOST) {
          const long long zo = (long long)(gz - k) * g.pz;
#pragma unroll
          for (int r = 0; r < PY; ++r)
            if (act[r]) out[o[r] + zo] = ns[r];
        }
      }
    }
#pragma unroll
    for (int r = 0; r < PY; ++r) {
#pragma unroll
      for (int d = 0; d < 2 * R; ++d) q[r][d] = q[r][d + 1];
      o[r] += g.pz;
    }
    if (++sl_s == NSS) { sl_s = 0; sl_p ^= 1; }
    if (++sc_s == NSS) sc_s = 0;
    if (++pw_s == NPS) { pw_s = 0; pw_p ^= 1; }

    __syncthreads();  // every thread is done with stencil slot lc and point-wise slot m
    if (*s_abort) {
      drain(ll, m);
      return false;
    }
    if (tid == 0) {
      fence_proxy_async();
      if (lc + NSS < L) issue_stencil(lc + NSS);
      if (m + NPS < M) issue_pw(m + NPS);
    }
  }
  rg.sbase = SB + L;
  rg.pbase = PB + (NPW > 0 ? M : 0);
  return true;
}

// Single-solve stage kernel: one work item per CTA (grid = tiles x z-chunks).
template <class S, class C, int R, int KIND, int TY, int PY>
__global__ void __launch_bounds__(32 * TY / PY) k_stage_tma(const __grid_constant__ TmaMaps maps,
                                                           const StageArgs a) {
  using LY = TmaLayout<S, R, StageTraits<KIND>::NPW, TY>;
  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_abort;
  TmaRing rg = tma_ring_setup<LY>(smem_raw, &s_abort);
  double r_norm = 0.0, r_en = 0.0, r_err = 0.0;
  if (!tma_item<S, C, R, KIND, TY, PY, LY, single_zu<S, KIND>()>(maps, a, blockIdx.x, blockIdx.y, blockIdx.z, rg,
                                                                  &s_abort, r_norm,
                                           r_en, r_err))
    return;
  if (a.partials) block_reduce_store<32 * TY / PY>(r_norm, r_en, r_err, a.partials);
}

// ---------------------------------------------------------------------------
// Two x-adjacent sites per thread, complex64 storage.  The 32 x TY tile is
// processed by 16 x (TY/PY) threads; thread (tx, tyt) owns the sites
// (2tx, 2tx+1) of rows tyt + r*TY/PY.  Every shared-memory read of the
// stencil and point-wise tiles moves both sites of a pair (one 16-byte word),
// so a pair takes three reads for its x neighbourhood and one per y
// neighbour row instead of eight single-site reads per site, and the stage
// outputs leave as 16-byte stores.  The per-site arithmetic is sites_stage,
// the same as the one-site-per-column kernels, so results are identical.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 lds_pair(const float2* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
// store the sites (i, i+1) of a pair; i+1 inside the grid implies i is
__device__ __forceinline__ void st_pair(float2* p, float2 v0, float2 v1, bool act0, bool act1) {
  if (act1)
    *reinterpret_cast<float4*>(p) = make_float4(v0.x, v0.y, v1.x, v1.y);
  else if (act0)
    *p = v0;
}

template <class C, int R, int KIND, int TY, int PY, class LY, int ZU = 1>
__device__ __forceinline__ bool tma_item_pair(const TmaMaps& maps, const StageArgs& a, int bx, int by, int bz,
                                              TmaRing& rg, int* s_abort, double& r_norm, double& r_en,
                                              double& r_err) {
  using S = float2;
  using T = StageTraits<KIND>;
  constexpr int TX = TMA_TX, HX = TMA_HX, TW = tma_stencil_w(), TXT = TX / 2, TYT = TY / PY;
  constexpr int NSS = LY::NSS, NPS = LY::NPS, NPW = T::NPW;
  constexpr int NS = 2 * PY;  // sites per thread: site 2r + s is x = i0 + s of owned row r
  constexpr uint32_t ST_BYTES = tma_st_bytes<S>(R, TY), PW1 = tma_pw1_bytes<S>(TY);
  static_assert(TY % PY == 0, "PY must divide TY");
  static_assert(HX % 2 == 0 && TW % 2 == 0, "pairs must stay 16-byte aligned in the tiles");

  const Geom& g = a.g;
  const int tx = threadIdx.x, tyt = threadIdx.y, tid = tyt * TXT + tx;
  const int i0 = bx * TX + 2 * tx;
  const int kb = bz * a.zc;
  const int ke = min(kb + a.zc, g.nz);
  const int M = ke - kb;
  const int L = M + 2 * R;
  const int SB = rg.sbase, PB = rg.pbase;

  const int cxs = 2 * (g.xoff + bx * TX - HX);
  const int cys = by * TY - R + 2;
  const int cxp = 2 * (g.xoff + bx * TX);
  const int cyp = by * TY + 2;

  int issued_s = 0, issued_p = 0;
  auto issue_stencil = [&](int l) {
    const int G = SB + l, s = G % NSS;
    mbar_arrive_expect_tx(&rg.sbar[s], ST_BYTES);
    tma_load_3d(rg.sring + s * LY::ST_SLOT, &maps.in, &rg.sbar[s], cxs, cys, kb - R + l + 2);
    issued_s = l + 1;
  };
  auto issue_pw = [&](int m) {
    if constexpr (NPW > 0) {
      const int G = PB + m, s = G % NPS;
      mbar_arrive_expect_tx(&rg.pbar[s], NPW * PW1);
#pragma unroll
      for (int f = 0; f < NPW; ++f)
        tma_load_3d(rg.pring + s * LY::PW_SLOT + f * PW1, &maps.pw[f], &rg.pbar[s], cxp, cyp, kb + m + 2);
      issued_p = m + 1;
    }
  };
  auto swait = [&](int l) { return mbar_wait_bounded(&rg.sbar[(SB + l) % NSS], ((SB + l) / NSS) & 1); };
  auto pwait = [&](int m) { return mbar_wait_bounded(&rg.pbar[(PB + m) % NPS], ((PB + m) / NPS) & 1); };
  auto drain = [&](int waited_s, int waited_p) {
    if (tid == 0) {
      atomicCAS(a.status, STATUS_OK, STATUS_WAIT_EXPIRED);  // a standing test value stays
      for (int l = waited_s; l < issued_s; ++l) swait(l);
      for (int m = waited_p; m < issued_p; ++m) pwait(m);
    }
    __syncthreads();
  };

  if (tid == 0) {
    for (int l = 0; l < min(NSS, L); ++l) issue_stencil(l);
    for (int m = 0; m < min(NPS, M); ++m) issue_pw(m);
  }

  int jr[PY], cofs[PY], pofs[PY], jq[NS];
  bool act[NS];
  long long o[PY], oq[NS];
  ColumnConsts<C> cc[NS];
#pragma unroll
  for (int r = 0; r < PY; ++r) {
    const int ty = tyt + r * TYT;
    jr[r] = by * TY + ty;
    cofs[r] = (ty + R) * TW + 2 * tx + HX;
    pofs[r] = ty * TX + 2 * tx;
    o[r] = (long long)(kb + 2) * g.pz + (long long)(jr[r] + 2) * g.px + g.xoff + i0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const int q = 2 * r + s;
      act[q] = (i0 + s < g.nx) && (jr[r] < g.ny);
      jq[q] = jr[r];
      oq[q] = o[r] + s;
      cc[q] = column_consts<C>(a, i0 + s, jr[r], R, act[q]);
    }
  }
  const bool xyg = (bx * TX <= R) || (bx * TX + TX - 1 >= g.nx - 1 - R) || (by * TY <= R) ||
                   (by * TY + TY - 1 >= g.ny - 1 - R);

  auto stile = [&](int l) { return (const S*)(rg.sring + ((SB + l) % NSS) * LY::ST_SLOT); };
  float4 q[PY][2 * R + 1];  // z queue of each owned row's pair: planes k-R .. k+R
  bool ok = true;
  if (*(volatile const int*)a.status == STATUS_EXPIRE_TEST) ok = mbar_wait_bounded(rg.nbar, 0, EXPIRE_TEST_POLLS);
#pragma unroll
  for (int l = 0; l < 2 * R; ++l) {
    ok &= swait(l);
    const S* tl = stile(l);
#pragma unroll
    for (int r = 0; r < PY; ++r) q[r][l] = lds_pair(tl + cofs[r]);
  }
  if (!ok) *s_abort = 1;
  __syncthreads();
  if (*s_abort) {
    drain(0, 0);
    return false;
  }
  if (tid == 0) {
    fence_proxy_async();
    for (int l = 0; l < R; ++l)
      if (l + NSS < L) issue_stencil(l + NSS);
  }

  int sl_s = (SB + 2 * R) % NSS, sl_p = ((SB + 2 * R) / NSS) & 1;
  int sc_s = (SB + R) % NSS;
  int pw_s = PB % NPS, pw_p = (PB / NPS) & 1;

#pragma unroll ZU
  for (int m = 0; m < M; ++m) {
    const int k = kb + m;
    const int lc = m + R, ll = m + 2 * R;
    bool okw = mbar_wait_bounded(&rg.sbar[sl_s], sl_p);
    {
      const S* tl = (const S*)(rg.sring + sl_s * LY::ST_SLOT);
#pragma unroll
      for (int r = 0; r < PY; ++r) q[r][2 * R] = lds_pair(tl + cofs[r]);
    }
    const S* pws = nullptr;
    if constexpr (NPW > 0) {
      okw &= mbar_wait_bounded(&rg.pbar[pw_s], pw_p);
      pws = (const S*)(rg.pring + pw_s * LY::PW_SLOT);
    }
    if (!okw) *s_abort = 1;

    if (okw) {
      const S* tile = (const S*)(rg.sring + sc_s * LY::ST_SLOT);
      const int gz = (k <= R || k >= g.nz - 1 - R) ? zghost_pos(k, g.nz, R, a.bcs, a.zghost) : NOGHOST;
      constexpr int NPWX = NPW > 0 ? NPW : 1;
      // each row's neighbourhoods are reduced to Laplacians (and, with
      // Urhs, x-derivatives) right after its loads, so only one row's
      // neighbours are live at a time
      cx<C> lap[NS], c0[NS], dpx[NS];
      S pv[NS][NPWX];
#pragma unroll
      for (int r = 0; r < PY; ++r) {
        const S* c = tile + cofs[r];
        const float4 xl = lds_pair(c - 2), xr = lds_pair(c + 2), cc4 = q[r][R];
        const float4 ym1 = lds_pair(c - TW), yp1 = lds_pair(c + TW);
        Nb<C> n0, n1;
        n0.c0 = to_c<C>(lo2(cc4));
        n1.c0 = to_c<C>(hi2(cc4));
        n0.xm1 = to_c<C>(hi2(xl));
        n0.xp1 = to_c<C>(hi2(cc4));
        n1.xm1 = to_c<C>(lo2(cc4));
        n1.xp1 = to_c<C>(lo2(xr));
        n0.ym1 = to_c<C>(lo2(ym1));
        n1.ym1 = to_c<C>(hi2(ym1));
        n0.yp1 = to_c<C>(lo2(yp1));
        n1.yp1 = to_c<C>(hi2(yp1));
        n0.zm1 = to_c<C>(lo2(q[r][R - 1]));
        n1.zm1 = to_c<C>(hi2(q[r][R - 1]));
        n0.zp1 = to_c<C>(lo2(q[r][R + 1]));
        n1.zp1 = to_c<C>(hi2(q[r][R + 1]));
        if constexpr (R == 2) {
          const float4 ym2 = lds_pair(c - 2 * TW), yp2 = lds_pair(c + 2 * TW);
          n0.xm2 = to_c<C>(lo2(xl));
          n1.xm2 = to_c<C>(hi2(xl));
          n0.xp2 = to_c<C>(lo2(xr));
          n1.xp2 = to_c<C>(hi2(xr));
          n0.ym2 = to_c<C>(lo2(ym2));
          n1.ym2 = to_c<C>(hi2(ym2));
          n0.yp2 = to_c<C>(lo2(yp2));
          n1.yp2 = to_c<C>(hi2(yp2));
          n0.zm2 = to_c<C>(lo2(q[r][0]));
          n1.zm2 = to_c<C>(hi2(q[r][0]));
          n0.zp2 = to_c<C>(lo2(q[r][4]));
          n1.zp2 = to_c<C>(hi2(q[r][4]));
        } else {
          n0.xm2 = n0.xp2 = n0.ym2 = n0.yp2 = n0.zm2 = n0.zp2 = cx<C>{0, 0};
          n1.xm2 = n1.xp2 = n1.ym2 = n1.yp2 = n1.zm2 = n1.zp2 = cx<C>{0, 0};
        }
        lap[2 * r] = site_lap<C, R>(a, n0);
        lap[2 * r + 1] = site_lap<C, R>(a, n1);
        c0[2 * r] = n0.c0;
        c0[2 * r + 1] = n1.c0;
        dpx[2 * r] = dpx[2 * r + 1] = cx<C>{0, 0};
        if (a.has_urhs) {
          dpx[2 * r] = site_dpx<C, R>(a, n0);
          dpx[2 * r + 1] = site_dpx<C, R>(a, n1);
        }
#pragma unroll
        for (int f = 0; f < NPW; ++f) {
          const float4 w = lds_pair(pws + f * (TX * TY) + pofs[r]);
          pv[2 * r][f] = lo2(w);
          pv[2 * r + 1][f] = hi2(w);
        }
      }
      S ns[NS], ax[NS];
      sites_update<S, C, R, KIND, NS, NPWX, false, false, false>(a, lap, c0, dpx, pv, act, i0, jq, k, oq, gz, cc,
                                                                  r_norm, r_en, r_err, ns, ax);
      if constexpr (KIND != K_ENERGY) {
        S* out = (S*)a.out;
#pragma unroll
        for (int r = 0; r < PY; ++r) st_pair(out + o[r], ns[2 * r], ns[2 * r + 1], act[2 * r], act[2 * r + 1]);
        if constexpr (KIND == K_RK4_2) {
#pragma unroll
          for (int r = 0; r < PY; ++r)
            st_pair((S*)a.acc + o[r], ax[2 * r], ax[2 * r + 1], act[2 * r], act[2 * r + 1]);
        }
        if constexpr (KIND >= K_CK_1 && KIND <= K_CK_5) {
#pragma unroll
          for (int r = 0; r < PY; ++r)
            st_pair((S*)a.kout + o[r], ax[2 * r], ax[2 * r + 1], act[2 * r], act[2 * r + 1]);
        }
        // face ghosts after the sites, in uniform branches (see tma_item)
        if (xyg) {
#pragma unroll
          for (int q2 = 0; q2 < NS; ++q2)
            if (act[q2]) {
              const long long os = o[q2 / 2] + (q2 & 1);
              if (cc[q2].gx != NOGHOST) out[os + (cc[q2].gx - (i0 + (q2 & 1)))] = ns[q2];
              if (cc[q2].gy != NOGHOST) out[os + (long long)(cc[q2].gy - jr[q2 / 2]) * g.px] = ns[q2];
            }
        }
        if (gz != NOGHOST) {
          const long long zo = (long long)(gz - k) * g.pz;
#pragma unroll
          for (int r = 0; r < PY; ++r)
            st_pair(out + o[r] + zo, ns[2 * r], ns[2 * r + 1], act[2 * r], act[2 * r + 1]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < PY; ++r) {
#pragma unroll
      for (int d = 0; d < 2 * R; ++d) q[r][d] = q[r][d + 1];
      o[r] += g.pz;
    }
    if (++sl_s == NSS) { sl_s = 0; sl_p ^= 1; }
    if (++sc_s == NSS) sc_s = 0;
    if (++pw_s == NPS) { pw_s = 0; pw_p ^= 1; }

    __syncthreads();
    if (*s_abort) {
      drain(ll, m);
      return false;
    }
    if (tid == 0) {
      fence_proxy_async();
      if (lc + NSS < L) issue_stencil(lc + NSS);
      if (m + NPS < M) issue_pw(m + NPS);
    }
  }
  rg.sbase = SB + L;
  rg.pbase = PB + (NPW > 0 ? M : 0);
  return true;
}

// Single-solve stage kernel with two x-adjacent sites per thread
// (complex64 storage): one work item per CTA, 16 x TY/PY threads.
template <class C, int R, int KIND, int TY, int PY>
__global__ void __launch_bounds__(16 * TY / PY) k_stage_tma_pair(const __grid_constant__ TmaMaps maps,
                                                                const StageArgs a) {
  using LY = TmaLayout<float2, R, StageTraits<KIND>::NPW, TY>;
  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_abort;
  TmaRing rg = tma_ring_setup<LY>(smem_raw, &s_abort);
  double r_norm = 0.0, r_en = 0.0, r_err = 0.0;
  if (!tma_item_pair<C, R, KIND, TY, PY, LY, single_zu<float2, KIND>()>(maps, a, blockIdx.x, blockIdx.y, blockIdx.z,
                                                                       rg, &s_abort, r_norm,
                                             r_en, r_err))
    return;
  if (a.partials) block_reduce_store<16 * TY / PY>(r_norm, r_en, r_err, a.partials);
}

// ---------------------------------------------------------------------------
// Batched, persistent stage kernel: many independent solves (any sizes, BCs,
// orders 2 and 4) advanced by one launch per stage.  Work item w = tile
// (bx, by, bz) of solve items[w].solve.  CTAs take items from a work queue:
// an atomic counter (zero at launch) indexes `order`, which lists the items
// largest first, so the launch ends with small items spread over all CTAs
// instead of a few CTAs finishing a long tail.  Per-solve stage arguments
// and tensor maps live in a device table.  Reductions go to per-item
// partials (indexed by w, whichever CTA runs the item), summed per solve by
// k_finalize_ranges in a fixed order, so a solve's results depend neither on
// what else is in the batch nor on the schedule.
// ---------------------------------------------------------------------------
struct alignas(64) BatchStage {
  TmaMaps maps;
  StageArgs args;
};

struct BatchItem {
  int solve, bx, by, bz;
};

// The per-solve stage arguments of one batched launch as a kernel parameter
// (32 KB of parameter space, read through the constant cache): up to
// BATCH_PARAM_SOLVES solves.  Items index it by their solve, and the item
// body reads its arguments from there as the single-solve kernels read
// theirs.  Loaded per item from the global table into registers instead,
// they keep the kernel at its 128-register bound, and the stages of one
// 256^3 solve in a pool take 6-8 % longer (a launch with more solves keeps
// that path).
constexpr int BATCH_PARAM_SOLVES = 60;
struct BatchArgs {
  StageArgs a[BATCH_PARAM_SOLVES];
};
struct NoBatchArgs {};
static_assert(sizeof(BatchArgs) + 256 <= 32764, "batched launch parameters exceed the 32 KB parameter space");
template <bool PARG>
using BatchArgsOf = typename std::conditional<PARG, BatchArgs, NoBatchArgs>::type;

// One batched launch: tab = the device rows of the ns solves (stage
// arguments + tensor maps), htab = the same rows on the host.
struct BatchLaunch {
  const BatchStage* tab;
  const BatchStage* htab;
  int ns;
  const BatchItem* items;
  const int* order;
  int nitems;
  int* queue;
  double* partials;
};

// CTAs per SM the batched kernels' registers are fitted to (each kernel
// carries the item body of one stencil radius).  RK4: 4 CTAs of 128 threads
// for the complex64 pair layout on 32 x 16 items (four sites per thread, as
// its single-solve form) and at FP64, 6 for FP32 on 32 x 8 items;
// Cash-Karp: 4 at FP32 (+8 % against unbounded on a batch of RKF45 solves)
// and 3 at FP64 (stages 3-6 are held to 2 CTAs by shared memory anyway).
template <class C, int KIND, int TY = 8>
__host__ __device__ constexpr int batch_min_blocks() {
  return (KIND == K_RK4_1 || KIND == K_RK4_2 || KIND == K_RK4_3 || KIND == K_RK4_4)
             ? (sizeof(C) == 4 ? (TY == 16 ? 4 : 6) : 4)
         : (KIND >= K_CK_1 && KIND <= K_CK_6) ? (sizeof(C) == 4 ? 4 : 3)
                                              : 1;
}

// Threads of a batched CTA: 32 x TY/PY, or with the pair layout 16 x 8 (one
// row per thread on 32 x 8 items, two rows on 32 x 16 items).
template <int TY, int PY, bool PAIR>
__host__ __device__ constexpr int batch_threads() {
  return PAIR ? 128 : 32 * TY / PY;
}

// PAIR (complex64 storage with the FP32 stencil only): 16 x 8 threads, each
// with two x-adjacent sites in TY/8 rows of the 32 x TY item tile
// (tma_item_pair); otherwise 32 x TY/PY threads with PY rows each.  RR is
// the stencil radius of every solve the launch serves (a pool keeps solves
// of the two FD orders in separate classes): one item body per kernel, and
// rings sized for that radius.
template <class S, class C, int KIND, int TY, int PY, bool PAIR, int RR, bool PARG>
__global__ void __launch_bounds__(batch_threads<TY, PY, PAIR>(), (batch_min_blocks<C, KIND, PAIR ? TY : 8>()))
    k_stage_batch(const BatchStage* __restrict__ tab, const BatchItem* __restrict__ items,
                  const int* __restrict__ order, int nitems, int* queue, double* partials,
                  const __grid_constant__ BatchArgsOf<PARG> pa) {
  static_assert(!PAIR || (sizeof(S) == 8 && sizeof(C) == 4 && (TY == 8 || TY == 16)),
                "the pair layout is for complex64 / FP32 on 32 x 8 or 32 x 16 items");
  static_assert(RR == 1 || RR == 2, "stencil radius 1 or 2");
  constexpr int PYP = TY / 8;  // rows per thread of the pair layout
  using LY = TmaLayout<S, RR, StageTraits<KIND>::NPW, TY>;
  constexpr int NT = batch_threads<TY, PY, PAIR>();
  extern __shared__ unsigned char smem_raw[];
  __shared__ int s_abort;
  __shared__ int s_w[2];  // item taken from the queue, double-buffered by turn parity
  TmaRing rg = tma_ring_setup<LY>(smem_raw, &s_abort);
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  int fenced = -1;  // solve whose tensor maps thread 0 has acquired (they do not change within a launch)
  for (int turn = 0;; ++turn) {
    if (tid == 0) {
      const int q = atomicAdd(queue, 1);
      s_w[turn & 1] = q < nitems ? order[q] : -1;
    }
    __syncthreads();
    const int w = s_w[turn & 1];
    if (w < 0) break;
    const BatchItem it = items[w];
    const BatchStage* bs = tab + it.solve;
    if (tid == 0 && it.solve != fenced) {
      tensormap_acquire(&bs->maps.in);
      for (int f = 0; f < StageTraits<KIND>::NPW; ++f) tensormap_acquire(&bs->maps.pw[f]);
      fenced = it.solve;
    }
    double r_norm = 0.0, r_en = 0.0, r_err = 0.0;
    auto run = [&](const StageArgs& sa) {
      if constexpr (PAIR)
        return tma_item_pair<C, RR, KIND, TY, PYP, LY>(bs->maps, sa, it.bx, it.by, it.bz, rg, &s_abort, r_norm,
                                                       r_en, r_err);
      else
        return tma_item<S, C, RR, KIND, TY, PY, LY>(bs->maps, sa, it.bx, it.by, it.bz, rg, &s_abort, r_norm, r_en,
                                                    r_err);
    };
    bool ok;
    if constexpr (PARG) {
      ok = run(pa.a[it.solve]);  // parameter space: the host puts at most BATCH_PARAM_SOLVES rows there
    } else {
      // the item's arguments in registers (read-only path, same address for
      // every thread); a shared-memory copy would be re-read after every
      // barrier of the z march
      const StageArgs sa = __ldg_args(&bs->args);
      ok = run(sa);
    }
    if (!ok) return;
    if (partials) block_reduce_store_at<NT>(r_norm, r_en, r_err, partials, w);
  }
}

}  // namespace gpe

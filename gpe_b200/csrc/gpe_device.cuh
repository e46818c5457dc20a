// Device side of the B200 Gross-Pitaevskii stepper: the fused RK stage
// kernel (stencil + GP right-hand side + stage combination + reductions).
//
// Reference path restated here (anthonyyoud/gpe):
//   src/derivs.f90:25-64, 146-272   2nd/4th order centred differences
//   src/derivs.f90:276-398          boundary index maps (see ghost_pos)
//   src/variables.f90:55-71         laplacian = dxx + dyy + dzz
//   src/solve.f90:382-440           get_rhs, equations 1-4
//   src/solve.f90:57-378            Euler / RK2 / RK4 / Cash-Karp stages
//   src/variables.f90:554-604       get_norm, energy
//
// HBM layout (one solve, one field): a ghost-padded array
//   elem(i,j,k) = (k+2)*pz + (j+2)*px + XOFF + i,
//   i in [-2, nx+1], j in [-2, ny+1], k in [-2, nz+1],
// with XOFF = 128 B / sizeof(element) so that x = 0 of every row starts on a
// 128-byte boundary and px a multiple of XOFF.  The producer of every field
// that is read through the stencil writes, next to each interior value, the
// face ghosts that the boundary conditions map onto it; the stencil then has
// no boundary logic at all.  Periodic and reflective BCs differ only in
// where the producer writes ghosts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpe {

enum StageKind : int {
  K_EULER = 0,
  K_RK2_1,
  K_RK2_2,
  K_RK4_1,
  K_RK4_2,
  K_RK4_4,
  K_CK_1,
  K_CK_2,
  K_CK_3,
  K_CK_4,
  K_CK_5,
  K_CK_6,
  K_ENERGY,  // no stores: energy of the input state only
  K_RK4_3,
  K_NUM
};

// Thread layouts of the single-solve TMA stage kernel over a 32-column tile.
// The values of the first two are the kernels' threads in y (the tile is
// 32 x 8 either way); the pair layouts give every thread two x-adjacent
// sites (complex64 storage only).
enum TileVariant : int {
  TILE_32x8_ROW1 = 8,    // 32 x 8 threads, one site per plane each
  TILE_32x8_ROW2 = 4,    // 32 x 4 threads, two rows each
  TILE_PAIR_32x8 = 16,   // 16 x 8 threads, one x pair each
  TILE_PAIR_32x16 = 32,  // 16 x 8 threads on a 32 x 16 tile, an x pair in two rows each
};
__host__ __device__ constexpr int tile_rows(int v) { return v == TILE_PAIR_32x16 ? 16 : 8; }
__host__ __device__ constexpr bool tile_is_pair(int v) { return v == TILE_PAIR_32x8 || v == TILE_PAIR_32x16; }

// reduction slots in the per-block partials: [norm, energy, errmax]
enum { RED_NORM = 0, RED_ENERGY = 1, RED_ERR = 2, RED_SLOTS = 3 };

struct Geom {
  int nx, ny, nz;
  int xoff;             // elements before x = 0 in a row
  long long px, pz;     // row and plane pitch in elements
};

struct alignas(16) StageArgs {
  Geom g;
  int R;                // stencil radius: 1 (order 2) or 2 (order 4)
  int bcs;              // 1 periodic, 2 reflective
  int eqn;              // 1..4
  int zc;               // z planes per block
  int want_norm, want_energy;
  int has_urhs, has_diss;
  const void* in;       // stencil input (ghost-padded)
  const void* psi;      // psi_n, read point-wise
  void* acc;            // RK4 accumulator (read/write point-wise)
  void* out;            // stencil output for the next stage (+ ghosts)
  void* kout;           // Cash-Karp: K_m = dt*f for this stage
  const void* kin[5];   // Cash-Karp: K_1..K_{m-1}
  double cf_r[2], cf_i[2];  // complex stage coefficients
  double b[6];              // real Cash-Karp coefficients of this stage
  double dte_r, dte_i;      // dt at entry of rkqs (psi_scal)
  double inv_adt;           // 1/|dt| of this attempt (psi_scal)
  // stencil constants
  double ixx, iyy, izz;     // 1/dx2 (order 2) or 1/(12 dx2) (order 4)
  double ix1;               // 1/(2dx) (order 2) or 1/(12dx) (order 4)
  double g_nl, mu, gamma, urhs, diss_amp;
  // per-axis tables, length n of each axis
  const double *vx, *vy, *vz;   // om^2 x^2 (Vtrap pieces)
  const double *sx, *sy, *sz;   // 1 + tanh(x-a)tanh(x+a) (diss pieces)
  const double *wx, *wy, *wz;   // norm quadrature weights
  const double *cx, *cy, *cz;   // coordinates (sphere)
  double* partials;             // [nblocks][RED_SLOTS]
  int* status;                  // device status word: non-zero = a bounded wait expired
  int zghost;                   // z ghosts the producer writes: bit 0 below the grid, bit 1 above
  int eqn4_plain;               // eqn 4 with V = 0 and gamma = 0 (the trap and damping terms vanish)
  // The FP32 stencil's copies of the constants above, each the double
  // rounded once to float on the host (set_f32_constants), so that the
  // kernels convert nothing per site or per plane
  float f_ixx, f_iyy, f_izz, f_ix1;
  float f_g_nl, f_mu, f_gamma, f_urhs, f_diss_amp;
  float f_cf_r[2], f_cf_i[2];
  float f_b[6];
  float f_pad;
};

// The stencil's compute-type copy of a stage constant: the float copy for
// the FP32 stencil, the double itself for FP64.
template <class C>
__host__ __device__ __forceinline__ C cval(double d, float f) {
  if constexpr (sizeof(C) == sizeof(float)) return f;
  else return (C)d;
}

// Fill the float copies of a's constants (round to nearest, as the device's
// (float) conversion of the same double).
inline void set_f32_constants(StageArgs& a) {
  a.f_ixx = (float)a.ixx;
  a.f_iyy = (float)a.iyy;
  a.f_izz = (float)a.izz;
  a.f_ix1 = (float)a.ix1;
  a.f_g_nl = (float)a.g_nl;
  a.f_mu = (float)a.mu;
  a.f_gamma = (float)a.gamma;
  a.f_urhs = (float)a.urhs;
  a.f_diss_amp = (float)a.diss_amp;
  for (int q = 0; q < 2; ++q) {
    a.f_cf_r[q] = (float)a.cf_r[q];
    a.f_cf_i[q] = (float)a.cf_i[q];
  }
  for (int q = 0; q < 6; ++q) a.f_b[q] = (float)a.b[q];
  a.f_pad = 0.0f;
}

static_assert(sizeof(StageArgs) % 16 == 0, "StageArgs is copied in 16-byte words");

template <class S>
struct Stor;
template <>
struct Stor<double2> {
  using R = double;
  static constexpr int XOFF = 8;
};
template <>
struct Stor<float2> {
  using R = float;
  static constexpr int XOFF = 16;
};

template <class C>
struct cx {
  C r, i;
};

template <class C, class S>
__device__ __forceinline__ cx<C> to_c(const S& v) {
  return cx<C>{(C)v.x, (C)v.y};
}
template <class S, class C>
__device__ __forceinline__ S to_s(const cx<C>& v) {
  S s;
  s.x = (typename Stor<S>::R)v.r;
  s.y = (typename Stor<S>::R)v.i;
  return s;
}
template <class S>
__device__ __forceinline__ S szero() {
  S s;
  s.x = 0;
  s.y = 0;
  return s;
}

// Read-only, non-coherent global load for inputs no thread writes in the
// same launch.
template <class S>
__device__ __forceinline__ S ldro(const S* p) {
  return __ldg(p);
}

constexpr int NOGHOST = -1000000;

// Ghost position written next to interior index q of an axis with n points,
// stencil radius R (derivs.f90:276-398 restated as ghost cells):
//   periodic:   ghost(q+n) = psi(q) for q < R;  ghost(q-n) = psi(q) for q >= n-R
//   reflective: ghost(-q) = psi(q) for 1 <= q <= R;
//               ghost(2(n-1)-q) = psi(q) for n-1-R <= q <= n-2
// (even mirror about the end node: x_{-1} = x_1, x_{n+1} = x_{n-1}).
// For n >= 6 at most one ghost exists per axis.
__host__ __device__ __forceinline__ int ghost_pos(int q, int n, int R, int bcs) {
  if (bcs == 1) {
    if (q < R) return q + n;
    if (q >= n - R) return q - n;
  } else {
    if (q >= 1 && q <= R) return -q;
    if (q >= n - 1 - R && q <= n - 2) return 2 * (n - 1) - q;
  }
  return NOGHOST;
}

// ghost_pos for the z axis of a grid that may be one z-slab of a larger
// one: ghosts that land below the slab (q < 0) are written only with bit 0
// of zmask, those above (q >= n) only with bit 1.  A whole grid uses 3; a
// slab whose face borders another slab leaves that face to the halo exchange.
__host__ __device__ __forceinline__ int zghost_pos(int k, int n, int R, int bcs, int zmask) {
  const int q = ghost_pos(k, n, R, bcs);
  if (q == NOGHOST) return q;
  return (q < 0 ? (zmask & 1) : (zmask & 2)) ? q : NOGHOST;
}

// 2nd derivative along one axis, expression order of derivs.f90:164-181
template <class C, int R>
__device__ __forceinline__ cx<C> d2(cx<C> m2, cx<C> m1, cx<C> c0, cx<C> p1, cx<C> p2, C inv) {
  cx<C> o;
  if constexpr (R == 1) {
    o.r = ((p1.r - (C)2 * c0.r) + m1.r) * inv;
    o.i = ((p1.i - (C)2 * c0.i) + m1.i) * inv;
  } else {
    o.r = ((((-p2.r + (C)16 * p1.r) - (C)30 * c0.r) + (C)16 * m1.r) - m2.r) * inv;
    o.i = ((((-p2.i + (C)16 * p1.i) - (C)30 * c0.i) + (C)16 * m1.i) - m2.i) * inv;
  }
  return o;
}

// 1st derivative (derivs.f90:43, 54-57)
template <class C, int R>
__device__ __forceinline__ cx<C> d1(cx<C> m2, cx<C> m1, cx<C> p1, cx<C> p2, C inv) {
  cx<C> o;
  if constexpr (R == 1) {
    o.r = (p1.r - m1.r) * inv;
    o.i = (p1.i - m1.i) * inv;
  } else {
    o.r = (((-p2.r + (C)8 * p1.r) - (C)8 * m1.r) + m2.r) * inv;
    o.i = (((-p2.i + (C)8 * p1.i) - (C)8 * m1.i) + m2.i) * inv;
  }
  return o;
}

__device__ __forceinline__ cx<double> cmuld(double ar, double ai, cx<double> b) {
  return cx<double>{ar * b.r - ai * b.i, ar * b.i + ai * b.r};
}

// Store v at interior (i,j,k) of a ghost-padded field and at its face ghosts.
template <class S>
__device__ __forceinline__ void store_with_ghosts(S* f, const Geom& g, long long col, int i, int j, int k, int gx,
                                                  int gy, int gz, S v) {
  const long long pl = (long long)(k + 2) * g.pz;
  f[pl + col] = v;
  if (gx != NOGHOST) f[pl + (long long)(j + 2) * g.px + g.xoff + gx] = v;
  if (gy != NOGHOST) f[pl + (long long)(gy + 2) * g.px + g.xoff + i] = v;
  if (gz != NOGHOST) f[(long long)(gz + 2) * g.pz + col] = v;
}

// Same with the centre offset o of (i,j,k) already known.  XY = false / Z =
// false leave the x/y / z ghosts to the caller (the TMA kernels copy them in
// a separate pass that interior tiles and planes skip).
template <bool XY = true, bool Z = true, class S>
__device__ __forceinline__ void store_at(S* f, const Geom& g, long long o, int i, int j, int k, int gx, int gy,
                                         int gz, S v) {
  f[o] = v;
  if constexpr (XY) {
    if (gx != NOGHOST) f[o + (gx - i)] = v;
    if (gy != NOGHOST) f[o + (long long)(gy - j) * g.px] = v;
  }
  if constexpr (Z) {
    if (gz != NOGHOST) f[o + (long long)(gz - k) * g.pz] = v;
  }
}

// Deterministic block sum of up to RED_SLOTS values (fixed shuffle and warp
// order), thread 0 writes the block's partials.  Slot RED_ERR is a max.
template <int NT>
__device__ __forceinline__ void block_reduce_store_at(double v0, double v1, double v2, double* partials,
                                                      long long b);

template <int NT>
__device__ __forceinline__ void block_reduce_store(double v0, double v1, double v2, double* partials) {
  const long long b = blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
  block_reduce_store_at<NT>(v0, v1, v2, partials, b);
}

// Same, writing the partials of slot b (a work-item index in batched launches).
template <int NT>
__device__ __forceinline__ void block_reduce_store_at(double v0, double v1, double v2, double* partials,
                                                      long long b) {
  __shared__ double red[NT / 32][RED_SLOTS];
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v0 += __shfl_down_sync(0xffffffffu, v0, o);
    v1 += __shfl_down_sync(0xffffffffu, v1, o);
    v2 = fmax(v2, __shfl_down_sync(0xffffffffu, v2, o));
  }
  if ((tid & 31) == 0) {
    red[tid >> 5][0] = v0;
    red[tid >> 5][1] = v1;
    red[tid >> 5][2] = v2;
  }
  __syncthreads();
  if (tid == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < NT / 32; ++w) {
      s0 += red[w][0];
      s1 += red[w][1];
      s2 = fmax(s2, red[w][2]);
    }
    partials[b * RED_SLOTS + 0] = s0;
    partials[b * RED_SLOTS + 1] = s1;
    partials[b * RED_SLOTS + 2] = s2;
  }
}

// ---------------------------------------------------------------------------
// Per-stage data flow (which point-wise fields a stage reads).
// ---------------------------------------------------------------------------
template <int KIND>
struct StageTraits {
  static constexpr bool HAS_PSI = (KIND == K_RK2_2 || KIND == K_RK4_2 || KIND == K_RK4_3 ||
                                   (KIND >= K_CK_2 && KIND <= K_CK_6));
  static constexpr bool HAS_ACC = (KIND == K_RK4_4);
  // Cash-Karp K inputs: stages 2..5 read K_1..K_{m-1}; stage 6 reads K1, K3,
  // K4, K5 (K2 only enters with the zero weights c2 = dc2 = 0).
  static constexpr int NK = (KIND >= K_CK_2 && KIND <= K_CK_5) ? (KIND - K_CK_1) : (KIND == K_CK_6 ? 4 : 0);
  static constexpr int NPW = (HAS_PSI ? 1 : 0) + (HAS_ACC ? 1 : 0) + NK;  // point-wise input fields
  static constexpr bool FIRST = (KIND == K_ENERGY || KIND == K_EULER || KIND == K_RK2_1 || KIND == K_RK4_1 ||
                                 KIND == K_CK_1);
};

// stencil neighbourhood of one site
template <class C>
struct Nb {
  cx<C> c0, xm1, xp1, xm2, xp2, ym1, yp1, ym2, yp2, zm1, zp1, zm2, zp2;
};

// Per-column constants hoisted out of the z loop, in the stencil's compute
// type C (the FP32 stencil keeps them as floats: fewer registers per site).
template <class C>
struct ColumnConsts {
  double wxy;  // norm quadrature weight wx wy
  C vc;        // trap: vx + vy (FP64), or 0.5 (vx + vy) rounded once (FP32)
  C sxy;       // sponge: sx + sy
  C rxy2;      // sphere: x^2 + y^2
  int gx, gy;  // x / y ghost positions (ghost_pos)
};

template <class C>
__device__ __forceinline__ ColumnConsts<C> column_consts(const StageArgs& a, int i, int j, int R, bool active) {
  ColumnConsts<C> c;
  c.wxy = active ? a.wx[i] * a.wy[j] : 0.0;
  const double vxy = (active && a.eqn == 4) ? a.vx[i] + a.vy[j] : 0.0;
  c.vc = sizeof(C) == sizeof(double) ? (C)vxy : (C)(0.5 * vxy);
  c.sxy = (C)((active && a.has_diss) ? a.sx[i] + a.sy[j] : 0.0);
  c.rxy2 = (C)((active && a.eqn == 3) ? a.cx[i] * a.cx[i] + a.cy[j] * a.cy[j] : 0.0);
  c.gx = ghost_pos(i, a.g.nx, R, a.bcs);
  c.gy = ghost_pos(j, a.g.ny, R, a.bcs);
  return c;
}

// GP right-hand side (solve.f90:414-437) at the PY sites (i, j_r, k) of one
// thread.  Every statement runs over all PY sites inside the (warp-uniform)
// equation branches, so the sites' dependency chains interleave.  The
// column parts of the trap, dissipation and sphere terms come hoisted in cc;
// the sums keep the reference's left-to-right order.
template <class C, int PY>
__device__ __forceinline__ void gp_rhs_n(const StageArgs& a, const cx<C> (&p)[PY], const cx<C> (&lap)[PY],
                                         const cx<C> (&dpx)[PY], const ColumnConsts<C> (&cc)[PY], int k,
                                         cx<C> (&r)[PY]) {
  C n2[PY];
#pragma unroll
  for (int q = 0; q < PY; ++q) n2[q] = p[q].r * p[q].r + p[q].i * p[q].i;
  if (a.eqn == 4) {
    // -(i + gamma) * (-0.5 lap + V psi + g |psi|^2 psi - mu psi).  V in
    // FP64 as 0.5 ((vx + vy) + vz); in FP32 compute as the sum of the
    // column's and the plane's halves, each rounded once to float (no FP64
    // operations or conversions per site)
    const C g = cval<C>(a.g_nl, a.f_g_nl), mu = cval<C>(a.mu, a.f_mu), gm = cval<C>(a.gamma, a.f_gamma);
    if (a.eqn4_plain) {
      // V = 0, gamma = 0: the same sums without their zero terms (the
      // results agree bit for bit up to the sign of a zero)
#pragma unroll
      for (int q = 0; q < PY; ++q) {
        const C wr = (-(C)0.5 * lap[q].r + g * (n2[q] * p[q].r)) - mu * p[q].r;
        const C wi = (-(C)0.5 * lap[q].i + g * (n2[q] * p[q].i)) - mu * p[q].i;
        r[q].r = wi;
        r[q].i = -wr;
      }
      return;
    }
    const double vz = a.vz[k];
    const float vzh = (float)(0.5 * vz);
#pragma unroll
    for (int q = 0; q < PY; ++q) {
      C v;
      if constexpr (sizeof(C) == sizeof(double)) v = (C)(0.5 * (cc[q].vc + vz));
      else v = cc[q].vc + vzh;
      const C wr = ((-(C)0.5 * lap[q].r + v * p[q].r) + g * (n2[q] * p[q].r)) - mu * p[q].r;
      const C wi = ((-(C)0.5 * lap[q].i + v * p[q].i) + g * (n2[q] * p[q].i)) - mu * p[q].i;
      r[q].r = wi - gm * wr;
      r[q].i = -wr - gm * wi;
    }
  } else if (a.eqn == 2) {
    // i (lap - |psi|^2 psi) + U dpsi/dx
#pragma unroll
    for (int q = 0; q < PY; ++q) {
      const C cr = lap[q].r - n2[q] * p[q].r, ci = lap[q].i - n2[q] * p[q].i;
      r[q].r = -ci;
      r[q].i = cr;
    }
    if (a.has_urhs) {
      const C u = cval<C>(a.urhs, a.f_urhs);
#pragma unroll
      for (int q = 0; q < PY; ++q) {
        r[q].r += u * dpx[q].r;
        r[q].i += u * dpx[q].i;
      }
    }
  } else {
    // 0.5 (i + diss) (lap + (1 - |psi|^2) psi) + U dpsi/dx   [eqn 3: * sphere]
    C dd[PY];
#pragma unroll
    for (int q = 0; q < PY; ++q) dd[q] = 0;
    if (a.has_diss) {
      const double sz = a.sz[k];
      if constexpr (sizeof(C) == sizeof(double)) {
#pragma unroll
        for (int q = 0; q < PY; ++q) dd[q] = 0.5 * (a.diss_amp * (cc[q].sxy + sz));
      } else {
        const C amp = cval<C>(a.diss_amp, a.f_diss_amp), szf = (C)sz;
#pragma unroll
        for (int q = 0; q < PY; ++q) dd[q] = (C)0.5 * (amp * (cc[q].sxy + szf));
      }
    }
#pragma unroll
    for (int q = 0; q < PY; ++q) {
      const C sf = (C)1 - n2[q];
      const C cr = lap[q].r + sf * p[q].r, ci = lap[q].i + sf * p[q].i;
      r[q].r = dd[q] * cr - (C)0.5 * ci;
      r[q].i = dd[q] * ci + (C)0.5 * cr;
    }
    if (a.has_urhs) {
      const C u = cval<C>(a.urhs, a.f_urhs);
#pragma unroll
      for (int q = 0; q < PY; ++q) {
        r[q].r += u * dpx[q].r;
        r[q].i += u * dpx[q].i;
      }
    }
    if (a.eqn == 3) {
      const double zz = a.cz[k];
#pragma unroll
      for (int q = 0; q < PY; ++q) {
        C sp;
        if constexpr (sizeof(C) == sizeof(double)) {
          sp = 0.5 * (1.0 + tanh((sqrt(cc[q].rxy2 + zz * zz) - 10.0) - 2.0));
        } else {
          const C zf = (C)zz;
          sp = (C)0.5 * ((C)1 + tanhf((sqrtf(cc[q].rxy2 + zf * zf) - (C)10) - (C)2));
        }
        r[q].r *= sp;
        r[q].i *= sp;
      }
    }
  }
}

// Laplacian of one site from its neighbourhood.  FP64: the reference's
// expression order (derivs.f90:164-181, then laplacian = dxx + dyy + dzz,
// variables.f90:55-71).  FP32 stencil: each axis's bracket keeps the
// reference's order, so the cancellation of a smooth field happens inside it
// at the scale of one axis, and the three brackets are scaled and summed with
// one multiply and two fused multiply-adds, (iz Dz + (iy Dy + ix Dx)): 15
// instead of 17 operations per component.
template <class C, int R>
__device__ __forceinline__ cx<C> site_lap(const StageArgs& a, const Nb<C>& b) {
  cx<C> lap;
  if constexpr (sizeof(C) == sizeof(double)) {
    const cx<C> lxx = d2<C, R>(b.xm2, b.xm1, b.c0, b.xp1, b.xp2, cval<C>(a.ixx, a.f_ixx));
    const cx<C> lyy = d2<C, R>(b.ym2, b.ym1, b.c0, b.yp1, b.yp2, cval<C>(a.iyy, a.f_iyy));
    const cx<C> lzz = d2<C, R>(b.zm2, b.zm1, b.c0, b.zp1, b.zp2, cval<C>(a.izz, a.f_izz));
    lap.r = (lxx.r + lyy.r) + lzz.r;
    lap.i = (lxx.i + lyy.i) + lzz.i;
  } else {
    const C ix = cval<C>(a.ixx, a.f_ixx), iy = cval<C>(a.iyy, a.f_iyy), iz = cval<C>(a.izz, a.f_izz);
    auto axis = [](C m2, C m1, C c, C p1, C p2) -> C {
      if constexpr (R == 1) return (p1 - (C)2 * c) + m1;
      else return ((((-p2 + (C)16 * p1) - (C)30 * c) + (C)16 * m1) - m2);
    };
    const C dxr = axis(b.xm2.r, b.xm1.r, b.c0.r, b.xp1.r, b.xp2.r);
    const C dxi = axis(b.xm2.i, b.xm1.i, b.c0.i, b.xp1.i, b.xp2.i);
    const C dyr = axis(b.ym2.r, b.ym1.r, b.c0.r, b.yp1.r, b.yp2.r);
    const C dyi = axis(b.ym2.i, b.ym1.i, b.c0.i, b.yp1.i, b.yp2.i);
    const C dzr = axis(b.zm2.r, b.zm1.r, b.c0.r, b.zp1.r, b.zp2.r);
    const C dzi = axis(b.zm2.i, b.zm1.i, b.c0.i, b.zp1.i, b.zp2.i);
    lap.r = fmaf(iz, dzr, fmaf(iy, dyr, ix * dxr));
    lap.i = fmaf(iz, dzi, fmaf(iy, dyi, ix * dxi));
  }
  return lap;
}

// First x-derivative of one site (only read when Urhs != 0).
template <class C, int R>
__device__ __forceinline__ cx<C> site_dpx(const StageArgs& a, const Nb<C>& b) {
  return d1<C, R>(b.xm2, b.xm1, b.xp1, b.xp2, cval<C>(a.ix1, a.f_ix1));
}

// Everything a stage does at the PY interior sites (i, j_q, k) of one thread
// once their Laplacians (lap), x-derivatives (dpx, read only when Urhs != 0),
// centre values (c0) and point-wise inputs are in registers: GP right-hand
// side, the stage combination, the stores (with ghosts) and the fused
// reductions.  pw[q][] holds site q's point-wise inputs in the order psi,
// acc, K... of StageTraits; o[q] is the element offset of (i, j_q, k);
// gz = ghost_pos(k, nz, R, bcs).  Sites with act[q] false (outside the grid)
// are computed but neither stored nor reduced, which keeps the arithmetic
// free of per-site branches.  MAIN = false stores nothing: the stencil
// output of each site comes back in ns_out, and the second output of the
// stage (Q of RK4 stage 2, K_m of Cash-Karp stages 1-5) in aux_out, for
// callers that store neighbouring sites together.
template <class S, class C, int R, int KIND, int PY, int NPWX, bool GXY = true, bool GZ = true, bool MAIN = true>
__device__ __forceinline__ void sites_update(const StageArgs& a, const cx<C> (&lap)[PY], const cx<C> (&c0)[PY],
                                             const cx<C> (&dpx_in)[PY], const S (&pw)[PY][NPWX],
                                             const bool (&act)[PY], int i, const int (&j)[PY], int k,
                                             const long long (&o)[PY], int gz, const ColumnConsts<C> (&cc)[PY],
                                             double& r_norm, double& r_en, double& r_err, S* ns_out = nullptr,
                                             S* aux_out = nullptr) {
  using T = StageTraits<KIND>;
  const Geom& g = a.g;
  if constexpr (T::FIRST) {
    if (a.want_energy) {
      // real(-lap * conjg(psi) + 0.5 |psi|^4)   (variables.f90:591-592)
#pragma unroll
      for (int q = 0; q < PY; ++q) {
        const double cr = (double)c0[q].r, ci = (double)c0[q].i;
        const double n2 = cr * cr + ci * ci;
        const double e = (-(double)lap[q].r * cr - (double)lap[q].i * ci) + 0.5 * (n2 * n2);
        if (act[q]) r_en += e;
      }
    }
  }
  if constexpr (KIND != K_ENERGY) {
    cx<C> f[PY];
    gp_rhs_n<C, PY>(a, c0, lap, dpx_in, cc, k, f);
    S* out = (S*)a.out;
    constexpr bool FINAL = (KIND == K_EULER || KIND == K_RK2_2 || KIND == K_RK4_4 || KIND == K_CK_6);
    S ns[PY];  // the stored stencil output of each site

#pragma unroll
    for (int q = 0; q < PY; ++q) {
      S pv = szero<S>(), av = szero<S>();
      {
        int m = 0;
        if constexpr (T::HAS_PSI) pv = pw[q][m++];
        if constexpr (T::HAS_ACC) av = pw[q][m++];
      }
      constexpr int K0 = (T::HAS_PSI ? 1 : 0) + (T::HAS_ACC ? 1 : 0);
      const double cr = (double)c0[q].r, ci = (double)c0[q].i;
      const cx<double> fd{(double)f[q].r, (double)f[q].i};

      if constexpr (KIND == K_EULER || KIND == K_RK2_1 || KIND == K_RK4_1 || KIND == K_RK2_2 ||
                    KIND == K_RK4_2 || KIND == K_RK4_3 || KIND == K_RK4_4) {
        // out = base + cf0 * f, with base = psi_n (pv), the stencil centre,
        // or for RK4 stage 4 a third of (accumulator + centre).  Outputs that
        // are a new psi (Euler, RK2 stage 2, RK4 stage 4) are formed in FP64;
        // intermediate stage inputs in the stencil's compute type C
        // (identical to FP64 when C = double).
        //
        // RK4 runs in a reduced-traffic form of classical RK4 (h = dt):
        //   s1: A = psi + h/2 k1
        //   s2: B = psi + h/2 k2,  Q = (psi + A) + h k2  (= 2psi + h/2 k1 + h k2)
        //   s3: A = psi + h k3
        //   s4: psi' = (Q + A)/3 + h/6 k4  (= psi + h (k1/6 + k2/3 + k3/3 + k4/6))
        // so that stage 1 reads 1 field, stage 3 reads 2 and stage 4 reads 2
        // (solve.f90:124-148 keeps k1..k4; the sum is the same).  The only
        // division by 3 sits in the FP64 update of stage 4.
        constexpr double THIRD = 1.0 / 3.0;
        if constexpr (FINAL || sizeof(C) == sizeof(double)) {
          cx<double> base;
          if constexpr (KIND == K_RK2_2 || KIND == K_RK4_2 || KIND == K_RK4_3) {
            base = to_c<double>(pv);
          } else if constexpr (KIND == K_RK4_4) {
            const cx<double> qv = to_c<double>(av);
            base = cx<double>{(qv.r + cr) * THIRD, (qv.i + ci) * THIRD};
          } else {
            base = cx<double>{cr, ci};
          }
          const cx<double> t0 = cmuld(a.cf_r[0], a.cf_i[0], fd);
          ns[q] = to_s<S>(cx<double>{base.r + t0.r, base.i + t0.i});
        } else {
          const cx<C> base = (KIND == K_RK2_2 || KIND == K_RK4_2 || KIND == K_RK4_3) ? to_c<C>(pv) : c0[q];
          const C ar = cval<C>(a.cf_r[0], a.f_cf_r[0]), ai = cval<C>(a.cf_i[0], a.f_cf_i[0]);
          ns[q] = to_s<S>(cx<C>{base.r + (ar * f[q].r - ai * f[q].i), base.i + (ar * f[q].i + ai * f[q].r)});
        }
        if constexpr (MAIN) {
          if (act[q]) store_at<GXY, GZ>(out, g, o[q], i, j[q], k, cc[q].gx, cc[q].gy, gz, ns[q]);
        }
        if constexpr (KIND == K_RK4_2) {
          // Q = (psi + A) + h k2 in the stencil's compute type: Q is rounded
          // to S either way, and no third enters here (a C-rounded 1/3 would
          // scale psi by a biased factor every step); cf1 = h
          S qs;
          if constexpr (sizeof(C) == sizeof(double)) {
            const cx<double> pd = to_c<double>(pv);
            const cx<double> t1 = cmuld(a.cf_r[1], a.cf_i[1], fd);
            qs = to_s<S>(cx<double>{(pd.r + cr) + t1.r, (pd.i + ci) + t1.i});
          } else {
            const cx<C> pc = to_c<C>(pv);
            const C br = cval<C>(a.cf_r[1], a.f_cf_r[1]), bi = cval<C>(a.cf_i[1], a.f_cf_i[1]);
            qs = to_s<S>(cx<C>{(pc.r + c0[q].r) + (br * f[q].r - bi * f[q].i),
                               (pc.i + c0[q].i) + (br * f[q].i + bi * f[q].r)});
          }
          if constexpr (MAIN) {
            if (act[q]) ((S*)a.acc)[o[q]] = qs;
          } else {
            aux_out[q] = qs;
          }
        }
      } else if constexpr (KIND != K_CK_6 && sizeof(C) != sizeof(double)) {
        // Cash-Karp stages 1-5 in the stencil's compute type: K_m = dt f and
        // tmp = psi + sum_j b_j K_j feed the next stencil only
        const C kr = cval<C>(a.cf_r[0], a.f_cf_r[0]), ki = cval<C>(a.cf_i[0], a.f_cf_i[0]);
        const cx<C> Km{kr * f[q].r - ki * f[q].i, kr * f[q].i + ki * f[q].r};
        const S Ks = to_s<S>(Km);
        if constexpr (MAIN) {
          if (act[q]) ((S*)a.kout)[o[q]] = Ks;
        } else {
          aux_out[q] = Ks;
        }
        const cx<C> Kmc = to_c<C>(Ks);
        const cx<C> pc = (KIND == K_CK_1) ? c0[q] : to_c<C>(pv);
        C tr = pc.r, ti = pc.i;
#pragma unroll
        for (int m = 0; m < T::NK; ++m) {
          const cx<C> km = to_c<C>(pw[q][K0 + m]);
          tr = tr + cval<C>(a.b[m], a.f_b[m]) * km.r;
          ti = ti + cval<C>(a.b[m], a.f_b[m]) * km.i;
        }
        tr = tr + cval<C>(a.b[T::NK], a.f_b[T::NK]) * Kmc.r;
        ti = ti + cval<C>(a.b[T::NK], a.f_b[T::NK]) * Kmc.i;
        ns[q] = to_s<S>(cx<C>{tr, ti});
        if constexpr (MAIN) {
          if (act[q]) store_at<GXY, GZ>(out, g, o[q], i, j[q], k, cc[q].gx, cc[q].gy, gz, ns[q]);
        }
      } else {
        // Cash-Karp stage m: K_m = dt * f ; tmp = psi + sum_j b_j K_j
        const cx<double> Km = cmuld(a.cf_r[0], a.cf_i[0], fd);
        const S Ks = to_s<S>(Km);
        const cx<double> Kmd = to_c<double>(Ks);
        const cx<double> pd = (KIND == K_CK_1) ? cx<double>{cr, ci} : to_c<double>(pv);
        if constexpr (KIND != K_CK_6) {
          if constexpr (MAIN) {
            if (act[q]) ((S*)a.kout)[o[q]] = Ks;
          } else {
            aux_out[q] = Ks;
          }
          double tr = pd.r, ti = pd.i;
#pragma unroll
          for (int m = 0; m < T::NK; ++m) {
            const cx<double> km = to_c<double>(pw[q][K0 + m]);
            tr = tr + a.b[m] * km.r;
            ti = ti + a.b[m] * km.i;
          }
          tr = tr + a.b[T::NK] * Kmd.r;
          ti = ti + a.b[T::NK] * Kmd.i;
          ns[q] = to_s<S>(cx<double>{tr, ti});
          if constexpr (MAIN) {
            if (act[q]) store_at<GXY, GZ>(out, g, o[q], i, j[q], k, cc[q].gx, cc[q].gy, gz, ns[q]);
          }
        } else {
          // kin = K1, K3, K4, K5; c2 = c5 = 0 and dc2 = 0 (solve.f90:270-281)
          // contribute exact zeros and are skipped.
          const cx<double> k1 = to_c<double>(pw[q][K0]), k3 = to_c<double>(pw[q][K0 + 1]);
          const cx<double> k4 = to_c<double>(pw[q][K0 + 2]), k5 = to_c<double>(pw[q][K0 + 3]);
          const double C1 = 37.0 / 378.0, C3 = 250.0 / 621.0, C4 = 125.0 / 594.0, C6 = 512.0 / 1771.0;
          const double DC1 = C1 - 2825.0 / 27648.0, DC3 = C3 - 18575.0 / 48384.0;
          const double DC4 = C4 - 13525.0 / 55296.0, DC5 = 0.0 - 277.0 / 14336.0, DC6 = C6 - 0.25;
          const double nr = (((pd.r + C1 * k1.r) + C3 * k3.r) + C4 * k4.r) + C6 * Kmd.r;
          const double ni = (((pd.i + C1 * k1.i) + C3 * k3.i) + C4 * k4.i) + C6 * Kmd.i;
          ns[q] = to_s<S>(cx<double>{nr, ni});
          if constexpr (MAIN) {
            if (act[q]) store_at<GXY, GZ>(out, g, o[q], i, j[q], k, cc[q].gx, cc[q].gy, gz, ns[q]);
          }
          const double er = (((DC1 * k1.r + DC3 * k3.r) + DC4 * k4.r) + DC5 * k5.r) + DC6 * Kmd.r;
          const double ei = (((DC1 * k1.i + DC3 * k3.i) + DC4 * k4.i) + DC5 * k5.i) + DC6 * Kmd.i;
          // psi_scal = |psi| + dt_entry |f| + 1e-30 (complex), |f| = |K1|/|dt|
          const double fa = hypot(k1.r, k1.i) * a.inv_adt;
          const double sr = (hypot(pd.r, pd.i) + a.dte_r * fa) + 1e-30;
          const double si = a.dte_i * fa;
          const double ratio = hypot(er, ei) / hypot(sr, si);
          if (act[q]) r_err = fmax(r_err, ratio);  // maxval(abs(err/psi_scal)); host divides by eps
        }
      }
    }
    if (ns_out) {
#pragma unroll
      for (int q = 0; q < PY; ++q) ns_out[q] = ns[q];
    }
    if constexpr (FINAL) {
      if (a.want_norm) {
        const double wz = a.wz[k];
#pragma unroll
        for (int q = 0; q < PY; ++q) {
          const double sr = (double)ns[q].x, si = (double)ns[q].y;
          const double v = (cc[q].wxy * wz) * (sr * sr + si * si);
          if (act[q]) r_norm += v;
        }
      }
    }
  }
}

// sites_update from the PY sites' stencil neighbourhoods.
template <class S, class C, int R, int KIND, int PY, int NPWX, bool GXY = true, bool GZ = true, bool MAIN = true>
__device__ __forceinline__ void sites_stage(const StageArgs& a, const Nb<C> (&n)[PY], const S (&pw)[PY][NPWX],
                                            const bool (&act)[PY], int i, const int (&j)[PY], int k,
                                            const long long (&o)[PY], int gz, const ColumnConsts<C> (&cc)[PY],
                                            double& r_norm, double& r_en, double& r_err, S* ns_out = nullptr,
                                            S* aux_out = nullptr) {
  cx<C> lap[PY], c0[PY], dpx[PY];
#pragma unroll
  for (int q = 0; q < PY; ++q) {
    lap[q] = site_lap<C, R>(a, n[q]);
    c0[q] = n[q].c0;
    dpx[q] = cx<C>{0, 0};
  }
  if (a.has_urhs) {
#pragma unroll
    for (int q = 0; q < PY; ++q) dpx[q] = site_dpx<C, R>(a, n[q]);
  }
  sites_update<S, C, R, KIND, PY, NPWX, GXY, GZ, MAIN>(a, lap, c0, dpx, pw, act, i, j, k, o, gz, cc, r_norm, r_en,
                                                       r_err, ns_out, aux_out);
}

// Single-site form (one site per thread).
template <class S, class C, int R, int KIND>
__device__ __forceinline__ void site_stage(const StageArgs& a, const Nb<C>& n, const S* pw, int i, int j, int k,
                                           long long o, int gz, const ColumnConsts<C>& cc, double& r_norm,
                                           double& r_en, double& r_err) {
  constexpr int NPWX = StageTraits<KIND>::NPW > 0 ? StageTraits<KIND>::NPW : 1;
  const Nb<C> nn[1] = {n};
  S pv[1][NPWX];
#pragma unroll
  for (int f = 0; f < StageTraits<KIND>::NPW; ++f) pv[0][f] = pw[f];
  const bool act[1] = {true};
  const int jj[1] = {j};
  const long long oo[1] = {o};
  const ColumnConsts<C> c1[1] = {cc};
  sites_stage<S, C, R, KIND, 1, NPWX>(a, nn, pv, act, i, jj, k, oo, gz, c1, r_norm, r_en, r_err);
}

// ---------------------------------------------------------------------------
// The fused stage kernel (load/store-unit version).
//
// Block = 32 (x) x TY (y) threads owning an x-y tile and marching over zc
// planes in z.  Per plane: the centre plane's tile plus a radius-R halo sits
// in shared memory (x and y neighbours); the z neighbours of each column sit
// in a register queue of 2R+1 values.  The next plane of the queue and the
// next halo are prefetched one iteration ahead, so every element of the
// stencil input is read from HBM about once per stage; halo re-reads hit L2.
// ---------------------------------------------------------------------------
template <class S, class C, int R, int KIND, int TY>
__global__ void __launch_bounds__(32 * TY) k_stage(const StageArgs a) {
  using T = StageTraits<KIND>;
  constexpr int TX = 32, NT = TX * TY;
  constexpr int TW = TX + 2 * R, TH = TY + 2 * R;
  constexpr int NH = 2 * R * TX + 2 * R * TY;  // halo points per plane
  constexpr int HPT = (NH + NT - 1) / NT;      // halo points per thread
  constexpr int NPW = T::NPW > 0 ? T::NPW : 1;

  __shared__ S tile[TH * TW];

  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = blockIdx.x * TX + tx;
  const int j = blockIdx.y * TY + ty;
  const int kb = blockIdx.z * a.zc;
  const int ke = min(kb + a.zc, g.nz);
  const bool ldok = (i <= g.nx + 1) && (j <= g.ny + 1);
  const bool active = (i < g.nx) && (j < g.ny);
  const long long col = (long long)(j + 2) * g.px + g.xoff + i;
  const S* __restrict__ in = (const S*)a.in;

  // halo bookkeeping
  long long hcol[HPT];
  int hsm[HPT];
  bool hok[HPT];
#pragma unroll
  for (int h = 0; h < HPT; ++h) {
    const int p = tid + h * NT;
    int hy = 0, hx = 0;
    if (p < 2 * R * TX) {
      const int r = p / TX, c = p % TX;
      hy = r < R ? r : TY + r;
      hx = R + c;
    } else {
      const int q = p - 2 * R * TX;
      const int r = q / (2 * R), c = q % (2 * R);
      hy = R + r;
      hx = c < R ? c : TX + c;
    }
    const int gi = blockIdx.x * TX + hx - R, gj = blockIdx.y * TY + hy - R;
    hok[h] = (p < NH) && gi >= -2 && gi <= g.nx + 1 && gj >= -2 && gj <= g.ny + 1;
    hsm[h] = (p < NH) ? hy * TW + hx : 0;
    hcol[h] = (long long)(gj + 2) * g.px + g.xoff + gi;
  }
  const ColumnConsts<C> cc = column_consts<C>(a, i, j, R, active);

  // point-wise input pointers in StageTraits order
  const S* pwp[NPW];
  {
    int q = 0;
    if constexpr (T::HAS_PSI) pwp[q++] = (const S*)a.psi;
    if constexpr (T::HAS_ACC) pwp[q++] = (const S*)a.acc;
#pragma unroll
    for (int m = 0; m < T::NK; ++m) pwp[q++] = (const S*)a.kin[m];
  }

  // z queue and halo of the first plane
  S q[2 * R + 1];
#pragma unroll
  for (int d = 0; d <= 2 * R; ++d) q[d] = ldok ? ldro(in + (long long)(kb - R + d + 2) * g.pz + col) : szero<S>();
  S hv[HPT];
#pragma unroll
  for (int h = 0; h < HPT; ++h) hv[h] = hok[h] ? ldro(in + (long long)(kb + 2) * g.pz + hcol[h]) : szero<S>();
  S pv[NPW];
#pragma unroll
  for (int m = 0; m < T::NPW; ++m)
    pv[m] = active ? ldro(pwp[m] + (long long)(kb + 2) * g.pz + col) : szero<S>();

  double r_norm = 0.0, r_en = 0.0, r_err = 0.0;

  for (int k = kb; k < ke; ++k) {
    const bool more = (k + 1 < ke);
    // prefetch the next iteration's loads
    S qn = szero<S>();
    S hn[HPT];
    S pn[NPW];
    if (more) {
      if (ldok) qn = ldro(in + (long long)(k + R + 3) * g.pz + col);
#pragma unroll
      for (int h = 0; h < HPT; ++h) hn[h] = hok[h] ? ldro(in + (long long)(k + 3) * g.pz + hcol[h]) : szero<S>();
#pragma unroll
      for (int m = 0; m < T::NPW; ++m)
        pn[m] = active ? ldro(pwp[m] + (long long)(k + 3) * g.pz + col) : szero<S>();
    }

    __syncthreads();
    tile[(ty + R) * TW + tx + R] = q[R];
#pragma unroll
    for (int h = 0; h < HPT; ++h)
      if (tid + h * NT < NH) tile[hsm[h]] = hv[h];
    __syncthreads();

    if (active) {
      const int ts = (ty + R) * TW + tx + R;
      Nb<C> n;
      n.c0 = to_c<C>(q[R]);
      n.xm1 = to_c<C>(tile[ts - 1]);
      n.xp1 = to_c<C>(tile[ts + 1]);
      n.ym1 = to_c<C>(tile[ts - TW]);
      n.yp1 = to_c<C>(tile[ts + TW]);
      n.zm1 = to_c<C>(q[R - 1]);
      n.zp1 = to_c<C>(q[R + 1]);
      if constexpr (R == 2) {
        n.xm2 = to_c<C>(tile[ts - 2]);
        n.xp2 = to_c<C>(tile[ts + 2]);
        n.ym2 = to_c<C>(tile[ts - 2 * TW]);
        n.yp2 = to_c<C>(tile[ts + 2 * TW]);
        n.zm2 = to_c<C>(q[0]);
        n.zp2 = to_c<C>(q[4]);
      } else {
        n.xm2 = n.xp2 = n.ym2 = n.yp2 = n.zm2 = n.zp2 = cx<C>{0, 0};
      }
      site_stage<S, C, R, KIND>(a, n, pv, i, j, k, (long long)(k + 2) * g.pz + col, zghost_pos(k, g.nz, R, a.bcs, a.zghost),
                                cc, r_norm, r_en, r_err);
    }

    // rotate the queue
#pragma unroll
    for (int d = 0; d < 2 * R; ++d) q[d] = q[d + 1];
    q[2 * R] = qn;
#pragma unroll
    for (int h = 0; h < HPT; ++h) hv[h] = hn[h];
#pragma unroll
    for (int m = 0; m < T::NPW; ++m) pv[m] = pn[m];
  }

  if (a.partials) block_reduce_store<NT>(r_norm, r_en, r_err, a.partials);
}

}  // namespace gpe

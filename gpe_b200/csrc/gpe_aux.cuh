// Auxiliary kernels: layout conversion between the caller's contiguous
// interior array and the ghost-padded device fields, stand-alone norm,
// deterministic finalisation of block partials, and renormalisation.
#pragma once
#include "gpe_device.cuh"

namespace gpe {

// contiguous interior (complex T2, [k][j][i]) -> ghost-padded field S with
// its face ghosts (the halo exchange of gpe.f90:173-176, done once)
template <class S, class T2>
__global__ void k_pack(const T2* __restrict__ src, S* __restrict__ dst, Geom g, int R, int bcs, int zmask = 3) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long r = t / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const T2 v = src[t];
    S s;
    s.x = (typename Stor<S>::R)v.x;
    s.y = (typename Stor<S>::R)v.y;
    const long long col = (long long)(j + 2) * g.px + g.xoff + i;
    store_with_ghosts(dst, g, col, i, j, k, ghost_pos(i, g.nx, R, bcs), ghost_pos(j, g.ny, R, bcs),
                      zghost_pos(k, g.nz, R, bcs, zmask), s);
  }
}

// ghost-padded field -> contiguous interior
template <class S, class T2>
__global__ void k_unpack(const S* __restrict__ src, T2* __restrict__ dst, Geom g) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long r = t / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const S v = src[(long long)(k + 2) * g.pz + (long long)(j + 2) * g.px + g.xoff + i];
    T2 o;
    o.x = v.x;
    o.y = v.y;
    dst[t] = o;
  }
}

// get_norm partials (variables.f90:554-576): w_i w_j w_k |psi|^2 per block,
// same tiling as the stage kernel so the sum order is fixed.
template <class S>
__global__ void __launch_bounds__(256) k_norm(const S* __restrict__ f, Geom g, int zc, const double* __restrict__ wx,
                                               const double* __restrict__ wy, const double* __restrict__ wz,
                                               double* partials) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  const int kb = blockIdx.z * zc, ke = min(kb + zc, g.nz);
  double s = 0.0;
  if (i < g.nx && j < g.ny) {
    const double wxy = wx[i] * wy[j];
    const long long col = (long long)(j + 2) * g.px + g.xoff + i;
    for (int k = kb; k < ke; ++k) {
      const S v = __ldg(f + (long long)(k + 2) * g.pz + col);
      const double vr = (double)v.x, vi = (double)v.y;
      s += (wxy * wz[k]) * (vr * vr + vi * vi);
    }
  }
  block_reduce_store<256>(s, 0.0, 0.0, partials);
}

// Sum (slots 0,1) and max (slot 2) of nb block partials in a fixed order.
static __global__ void __launch_bounds__(256) k_finalize(const double* __restrict__ partials, long long nb, double* out) {
  __shared__ double s0[256], s1[256], s2[256];
  const int t = threadIdx.x;
  double a = 0.0, b = 0.0, c = 0.0;
  for (long long q = t; q < nb; q += 256) {
    a += partials[q * RED_SLOTS + 0];
    b += partials[q * RED_SLOTS + 1];
    c = fmax(c, partials[q * RED_SLOTS + 2]);
  }
  s0[t] = a;
  s1[t] = b;
  s2[t] = c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) {
      s0[t] += s0[t + w];
      s1[t] += s1[t + w];
      s2[t] = fmax(s2[t], s2[t + w]);
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = s0[0];
    out[1] = s1[0];
    out[2] = s2[0];
  }
}

// Per-solve sums of work-item partials: block s reduces items
// [first[s], first[s+1]) in a fixed order (thread-strided, then a tree), so a
// solve's result depends only on its own items.
static __global__ void __launch_bounds__(256) k_finalize_ranges(const double* __restrict__ partials,
                                                         const int* __restrict__ first, double* out) {
  __shared__ double s0[256], s1[256], s2[256];
  const int sv = blockIdx.x, t = threadIdx.x;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int q = first[sv] + t; q < first[sv + 1]; q += 256) {
    a += partials[(long long)q * RED_SLOTS + 0];
    b += partials[(long long)q * RED_SLOTS + 1];
    c = fmax(c, partials[(long long)q * RED_SLOTS + 2]);
  }
  s0[t] = a;
  s1[t] = b;
  s2[t] = c;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (t < w) {
      s0[t] += s0[t + w];
      s1[t] += s1[t + w];
      s2[t] = fmax(s2[t], s2[t + w]);
    }
    __syncthreads();
  }
  if (t == 0) {
    out[sv * RED_SLOTS + 0] = s0[0];
    out[sv * RED_SLOTS + 1] = s1[0];
    out[sv * RED_SLOTS + 2] = s2[0];
  }
}

// Face ghosts of a field whose interior was just written (for example by a
// strided host-to-device copy): every interior site writes its ghost copies.
template <class S>
__global__ void k_fill_ghosts(S* f, Geom g, int R, int bcs) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long r = t / g.nx;
    const int j = (int)(r % g.ny);
    const int k = (int)(r / g.ny);
    const int gx = ghost_pos(i, g.nx, R, bcs), gy = ghost_pos(j, g.ny, R, bcs), gz = ghost_pos(k, g.nz, R, bcs);
    if (gx == NOGHOST && gy == NOGHOST && gz == NOGHOST) continue;
    const long long col = (long long)(j + 2) * g.px + g.xoff + i;
    const long long pl = (long long)(k + 2) * g.pz;
    const S v = f[pl + col];
    if (gx != NOGHOST) f[pl + (long long)(j + 2) * g.px + g.xoff + gx] = v;
    if (gy != NOGHOST) f[pl + (long long)(gy + 2) * g.px + g.xoff + i] = v;
    if (gz != NOGHOST) f[(long long)(gz + 2) * g.pz + col] = v;
  }
}

// renormalise (variables.f90:715-726): var = sqrt(nn)*var/sqrt(norm), over
// the whole padded buffer (ghost copies scale identically)
template <class S>
__global__ void k_scale(S* f, long long n, double a, double b) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    S v = f[t];
    v.x = (typename Stor<S>::R)(((double)v.x * a) / b);
    v.y = (typename Stor<S>::R)(((double)v.y * a) / b);
    f[t] = v;
  }
}

}  // namespace gpe

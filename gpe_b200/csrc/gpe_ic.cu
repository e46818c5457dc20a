// Initial conditions generated on the device (gpe_set_ic,
// gpe_pool_submit_ic).  Each site evaluates the reference's closed-form
// initial states (src/ic.f90) in FP64 and the product is written straight
// into the solve's ghost-padded psi field, ghosts included.  The seeded
// random-phase state is a spectrum built in place, one inverse cuFFT and a
// rescale to mean density 1.
#include <cuda_runtime.h>
#include <cufft.h>

#include <map>
#include <mutex>
#include <tuple>

#include "gpe_ic.h"

namespace gpe {

namespace {

constexpr double kPi = 3.1415926535897932384626433832795;

struct IcGrid {
  int nx, ny, nz;
  double xl, yl, zl, dx, dy, dz;
  double mu, g, omx, omy, omz, scal;
};

__device__ __forceinline__ double coord(double lo, double d, int q) { return lo + (double)q * d; }

// get_rr (src/ic.f90:893-906)
__device__ __forceinline__ double rr_of(double r) {
  const double r2 = r * r, r4 = r2 * r2;
  return sqrt((0.3437 + 0.0286 * r2) / ((1.0 + 0.3333 * r2) + 0.0286 * r4));
}

// get_r / get_theta (src/ic.f90:735-889) for a line along dir
__device__ __forceinline__ void line_geom(const gpe_line& vl, double sc, double x, double y, double z, double* r,
                                          double* th) {
  const double eps = 2.220446049250313e-16;
  double s1 = 0.0, s2 = 0.0;
  if (fabs(vl.ll) < eps) {
    s1 = 1.0;
    s2 = 1.0;
  }
  double a, b;
  if (vl.dir == 'x') {
    a = y - vl.y0 - vl.amp1 * sin(2.0 * kPi * (x - vl.x0) / (vl.ll + s1));
    b = z - vl.z0 - vl.amp2 * cos(2.0 * kPi * (x - vl.x0) / (vl.ll + s2));
  } else if (vl.dir == 'y') {
    a = z - vl.z0 - vl.amp1 * sin(2.0 * kPi * (y - vl.y0) / (vl.ll + s1));
    b = x - vl.x0 - vl.amp2 * cos(2.0 * kPi * (y - vl.y0) / (vl.ll + s2));
  } else {
    a = x - vl.x0 - vl.amp1 * sin(2.0 * kPi * (z - vl.z0) / (vl.ll + s1));
    b = y - vl.y0 - vl.amp2 * cos(2.0 * kPi * (z - vl.z0) / (vl.ll + s2));
  }
  *r = sqrt(sc * (a * a) + sc * (b * b));
  *th = vl.sgn * atan2(sc * b, sc * a);
}

// vortex_ring (src/ic.f90:357-514)
__device__ __forceinline__ void ring_val(const gpe_ring& vr, double sc, double x, double y, double z, double* re,
                                         double* im) {
  double u, v, w, u0, v0, w0;
  if (vr.plane[0] == 'x' && vr.plane[1] == 'y') { u = x; v = y; w = z; u0 = vr.x0; v0 = vr.y0; w0 = vr.z0; }
  else if (vr.plane[0] == 'x' && vr.plane[1] == 'z') { u = x; v = z; w = y; u0 = vr.x0; v0 = vr.z0; w0 = vr.y0; }
  else { u = y; v = z; w = x; u0 = vr.y0; v0 = vr.z0; w0 = vr.x0; }
  const double theta = atan2(v - v0, u - u0);
  const double s = sqrt((u - u0) * (u - u0) + (v - v0) * (v - v0)) - vr.r1 * sin((double)vr.kk * theta);
  const double dist = vr.amp * cos((double)vr.mm * theta);
  const double pp = w - vr.r1 * cos((double)vr.kk * theta);
  const double A = sc * (pp - w0), Bp = sc * ((s + vr.r0) - dist), Bm = sc * ((s - vr.r0) - dist);
  const double q1 = rr_of(sqrt(A * A + Bp * Bp)), q2 = rr_of(sqrt(A * A + Bm * Bm));
  const double z1r = A + vr.dir * 0.0 * Bp, z1i = vr.dir * Bp;
  const double z2r = A - vr.dir * 0.0 * Bm, z2i = -(vr.dir * Bm);
  const double tr = (q1 * z1r) * q2, ti = (q1 * z1i) * q2;
  *re = tr * z2r - ti * z2i;
  *im = tr * z2i + ti * z2r;
}

// pade_pulse_ring (src/ic.f90:518-587): the Pade approximations of the
// rarefaction pulse (pulse = true) and of the axisymmetric vortex ring that
// move along x (N. G. Berloff, J. Phys. A 37, 1617 (2004)), centred at x0
// with the axis through (y0, z0) and radius r0.  a(1..9), U and m are the
// published coefficients the reference's get_consts lists for the two cases
// (src/ic.f90:572-581); the same numbers give the same state.
__device__ __forceinline__ void pade_val(bool pulse, const gpe_pulse& pp, double x, double y, double z, double* re,
                                         double* im) {
  const double a1 = pulse ? -0.79792 : -1.1, a2 = pulse ? 0.00388059 : 0.0170524;
  const double a3 = pulse ? 0.00882276 : 0.0289452, a4 = pulse ? -0.7981 : -0.953;
  const double a5 = pulse ? -0.012783 : -0.0049767, a6 = pulse ? -0.0574092 : -0.0594346;
  const double a7 = pulse ? 0.0399 : 0.04, a8 = pulse ? 0.199 : 0.21, a9 = pulse ? 0.0058 : 0.00612;
  const double U = pulse ? 0.63 : 0.6, m = pulse ? 8.37 : 8.97;
  const double p74 = 7.0 / 4.0;
  const double one_2u = 1.0 - 2.0 * (U * U);
  const double ma9 = m * pow(a9, p74);
  const double s = sqrt((y - pp.y0) * (y - pp.y0) + (z - pp.z0) * (z - pp.z0));  // get_s, ic.f90:804-820
  const double xs = x - pp.x0;
  const double x2 = xs * xs, s2 = (s - pp.r0) * (s - pp.r0);
  const double t = x2 + one_2u * s2;
  const double denom = pow(((1.0 + a8 * x2) + a7 * s2) + a9 * (t * t), p74);
  *re = 1.0 + ((((a1 + a3 * x2) + a2 * s2) + (ma9 * U) * (2.0 * x2 - one_2u * s2)) * t) / denom;
  *im = (xs * (((a4 + a6 * x2) + a5 * s2) - ma9 * (t * t))) / denom;
}

// vortex_pair (src/ic.f90:591-636): the Pade approximation of a vortex pair
// in the x-y plane, the same in every z plane; coefficients as listed there.
__device__ __forceinline__ void pair_val(double x, double y, double* re, double* im) {
  const double a0 = -1.14026, a1 = -0.150112, a2 = -0.0294564;
  const double b0 = -0.830953, b1 = -0.108296, b2 = -0.073641;
  const double c0 = 0.35022, c1 = 0.03032, c2 = 0.15905, c3 = 0.04123, c4 = 0.01402;
  const double x2 = x * x, y2 = y * y, x4 = x2 * x2, y4 = y2 * y2;
  const double denom = ((((1.0 + c0 * x2) + c1 * x4) + c2 * y2) + (c3 * x2) * y2) + c4 * y4;
  *re = 1.0 + ((a0 + a1 * x2) + a2 * y2) / denom;
  *im = (x * ((b0 + b1 * x2) + b2 * y2)) / denom;
}

// The product of the closed-form factors of ic at (x, y, z), factors taken
// left to right as the reference's init_cond expression multiplies them.
__device__ __forceinline__ void ic_product(const gpe_ic& ic, const IcGrid& G, double x, double y, double z,
                                           double* out_r, double* out_i) {
    double pr = 1.0, pi = 0.0;
    for (int q = 0; q < ic.nfactors; ++q) {
      double fr = 1.0, fi = 0.0;
      switch (ic.factor[q]) {
        case GPE_IC_FERMI: {
          const double v = 0.5 * (((G.omx * G.omx) * (x * x) + (G.omy * G.omy) * (y * y)) + (G.omz * G.omz) * (z * z));
          const double a = (G.mu - v) / G.g;
          fr = a >= 0.0 ? sqrt(a) : 0.0;
          break;
        }
        case GPE_IC_LINE: {
          double r, th;
          line_geom(ic.line, G.scal, x, y, z, &r, &th);
          const double a = ic.line.imprint_phase ? 1.0 : 1.0 - exp(-0.7 * pow(r, 1.15));
          fr = a * cos(th);
          fi = a * sin(th);
          break;
        }
        case GPE_IC_LINE_PADE: {
          double r, th;
          line_geom(ic.line, G.scal, x, y, z, &r, &th);
          const double a = r * rr_of(r);
          fr = a * cos(th);
          fi = a * sin(th);
          break;
        }
        case GPE_IC_RING:
          ring_val(ic.ring, G.scal, x, y, z, &fr, &fi);
          break;
        case GPE_IC_PADE_PULSE:
        case GPE_IC_PADE_RING:
          pade_val(ic.factor[q] == GPE_IC_PADE_PULSE, ic.pulse, x, y, z, &fr, &fi);
          break;
        case GPE_IC_VORTEX_PAIR:
          pair_val(x, y, &fr, &fi);
          break;
        case GPE_IC_SPHERE:  // ic.f90:640-662 (rad = 10, eps1 = 2)
          fr = 0.5 * (1.0 + tanh((sqrt((x * x + y * y) + z * z) - 10.0) - 2.0));
          break;
        case GPE_IC_SPHERE2:  // ic.f90:666-684 (amp = 100, width = 10)
          fr = 100.0 * exp(-((x * x + y * y) + z * z) / 10.0);
          break;
        case GPE_IC_WALL:  // ic.f90:688-709 (pos = -30)
          fr = z <= -30.0 ? 0.0 : 1.0;
          break;
        default:
          break;
      }
      const double nr = pr * fr - pi * fi, ni = pr * fi + pi * fr;
      pr = nr;
      pi = ni;
    }
    *out_r = pr;
    *out_i = pi;
}

template <class S>
__global__ void k_ic_closed_form(S* f, Geom g, int R, int bcs, IcGrid G, gpe_ic ic) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long rq = t / g.nx;
    const int j = (int)(rq % g.ny);
    const int k = (int)(rq / g.ny);
    const double x = coord(G.xl, G.dx, i), y = coord(G.yl, G.dy, j), z = coord(G.zl, G.dz, k);
    double pr, pi;
    ic_product(ic, G, x, y, z, &pr, &pi);
    S s;
    s.x = (typename Stor<S>::R)pr;
    s.y = (typename Stor<S>::R)pi;
    store_with_ghosts(f, g, (long long)(j + 2) * g.px + g.xoff + i, i, j, k, ghost_pos(i, g.nx, R, bcs),
                      ghost_pos(j, g.ny, R, bcs), ghost_pos(k, g.nz, R, bcs), s);
  }
}

// psi <- psi * IC (modulus = 0: the state_restart product with init_cond,
// src/ic.f90:160-162) or psi <- |psi| * IC (modulus = 1:
// imprint_vortex_line, src/variables.f90:1166-1180), in FP64 per site, the
// new value stored with its ghosts.
template <class S>
__global__ void k_ic_multiply(S* f, Geom g, int R, int bcs, IcGrid G, gpe_ic ic, int modulus) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long rq = t / g.nx;
    const int j = (int)(rq % g.ny);
    const int k = (int)(rq / g.ny);
    const double x = coord(G.xl, G.dx, i), y = coord(G.yl, G.dy, j), z = coord(G.zl, G.dz, k);
    double pr, pi;
    ic_product(ic, G, x, y, z, &pr, &pi);
    const long long col = (long long)(j + 2) * g.px + g.xoff + i;
    const S v = f[(long long)(k + 2) * g.pz + col];
    double ar = (double)v.x, ai = (double)v.y;
    if (modulus) {
      ar = hypot(ar, ai);
      ai = 0.0;
    }
    S s;
    s.x = (typename Stor<S>::R)(ar * pr - ai * pi);
    s.y = (typename Stor<S>::R)(ar * pi + ai * pr);
    store_with_ghosts(f, g, col, i, j, k, ghost_pos(i, g.nx, R, bcs), ghost_pos(j, g.ny, R, bcs),
                      ghost_pos(k, g.nz, R, bcs), s);
  }
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + (idx + 1ULL) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// psi_hat(m) = exp(i 2 pi u_m) for |k_m| < kc, else 0; modes in numpy's
// fftfreq order, u_m from SplitMix64 over the linear mode index
__global__ void k_random_spectrum(double2* buf, int nx, int ny, int nz, double dx, double dy, double dz,
                                  unsigned long long seed, double kc) {
  const long long n = (long long)nx * ny * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const long long rq = t / nx;
    const int j = (int)(rq % ny);
    const int k = (int)(rq / ny);
    const int mi = i < (nx + 1) / 2 ? i : i - nx, mj = j < (ny + 1) / 2 ? j : j - ny, mk = k < (nz + 1) / 2 ? k : k - nz;
    const double kx = 2.0 * kPi * mi / (nx * dx), ky = 2.0 * kPi * mj / (ny * dy), kz = 2.0 * kPi * mk / (nz * dz);
    const double k2 = (kz * kz + ky * ky) + kx * kx;
    double2 v = make_double2(0.0, 0.0);
    if (k2 < kc * kc) {
      const double u = (double)(splitmix64(seed, (unsigned long long)t) >> 11) * (1.0 / 9007199254740992.0);
      const double th = 2.0 * kPi * u;
      v = make_double2(cos(th), sin(th));
    }
    buf[t] = v;
  }
}

// sum |psi|^2 over the buffer (fixed-order block partials, then one block)
__global__ void __launch_bounds__(256) k_sumsq(const double2* __restrict__ buf, long long n, double* part) {
  __shared__ double red[256];
  double s = 0.0;
  for (long long t = blockIdx.x * 256LL + threadIdx.x; t < n; t += 256LL * gridDim.x)
    s += buf[t].x * buf[t].x + buf[t].y * buf[t].y;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(256) k_sum_parts(double* part, int nb) {
  __shared__ double red[256];
  double s = 0.0;
  for (int q = threadIdx.x; q < nb; q += 256) s += part[q];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[nb] = red[0];
}

// psi = buf * sqrt(n / sum|buf|^2) into the padded field with ghosts
template <class S>
__global__ void k_pack_scaled(const double2* __restrict__ buf, const double* __restrict__ total, S* f, Geom g,
                              int R, int bcs) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  const double sc = 1.0 / sqrt(*total / (double)n);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx);
    const long long rq = t / g.nx;
    const int j = (int)(rq % g.ny);
    const int k = (int)(rq / g.ny);
    S s;
    s.x = (typename Stor<S>::R)(buf[t].x * sc);
    s.y = (typename Stor<S>::R)(buf[t].y * sc);
    store_with_ghosts(f, g, (long long)(j + 2) * g.px + g.xoff + i, i, j, k, ghost_pos(i, g.nx, R, bcs),
                      ghost_pos(j, g.ny, R, bcs), ghost_pos(k, g.nz, R, bcs), s);
  }
}

// 3-D Z2Z plans, one per (device, grid), created on first use
std::mutex g_plan_mu;
std::map<std::tuple<int, int, int, int>, cufftHandle> g_plans;

}  // namespace

bool plan_for(int nx, int ny, int nz, cufftHandle* out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto key = std::make_tuple(dev, nx, ny, nz);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) {
    *out = it->second;
    return true;
  }
  cufftHandle p;
  if (cufftPlan3d(&p, nz, ny, nx, CUFFT_Z2Z) != CUFFT_SUCCESS) return false;
  g_plans[key] = p;
  *out = p;
  return true;
}

int ic_validate(const gpe_ic* ic, std::string& why) {
  if (!ic || ic->nfactors < 1 || ic->nfactors > 4) {
    why = "gpe_ic: nfactors must be 1..4";
    return GPE_ERR_BADARG;
  }
  for (int q = 0; q < ic->nfactors; ++q) {
    const int f = ic->factor[q];
    if (f < GPE_IC_UNIFORM || f > GPE_IC_WALL) {
      why = "gpe_ic: unknown factor";
      return GPE_ERR_BADARG;
    }
    if (f == GPE_IC_RANDOM_PHASE && ic->nfactors != 1) {
      why = "gpe_ic: the random-phase state must be the only factor";
      return GPE_ERR_BADARG;
    }
    if (f == GPE_IC_RING) {
      const char* p = ic->ring.plane;
      const bool ok = (p[0] == 'x' && p[1] == 'y') || (p[0] == 'x' && p[1] == 'z') || (p[0] == 'y' && p[1] == 'z');
      if (!ok) {
        why = "ERROR: Unrecognised vortex ring plane.";  // src/ic.f90:510
        return GPE_ERR_BADARG;
      }
    }
    if (f == GPE_IC_LINE || f == GPE_IC_LINE_PADE) {
      const double eps = 2.220446049250313e-16;
      if (fabs(ic->line.ll) < eps && (fabs(ic->line.amp1) >= eps || fabs(ic->line.amp2) >= eps)) {
        why = "ERROR: vortex line disturbance wavelength is zero, but amplitude is non-zero.";  // ic.f90:755
        return GPE_ERR_BADARG;
      }
      if (ic->line.dir != 'x' && ic->line.dir != 'y' && ic->line.dir != 'z') {
        why = "gpe_ic: line direction must be x, y or z";
        return GPE_ERR_BADARG;
      }
    }
  }
  return GPE_OK;
}

bool ic_needs_fft(const gpe_ic* ic) { return ic->nfactors == 1 && ic->factor[0] == GPE_IC_RANDOM_PHASE; }

IcGrid ic_grid(const gpe_params& p) {
  IcGrid G;
  G.nx = p.nx;
  G.ny = p.ny;
  G.nz = p.nz;
  G.xl = -p.xr;
  G.yl = -p.yr;
  G.zl = -p.zr;
  G.dx = (p.xr - G.xl) / (p.nx - 1);
  G.dy = (p.yr - G.yl) / (p.ny - 1);
  G.dz = (p.zr - G.zl) / (p.nz - 1);
  G.mu = p.mu;
  G.g = p.g;
  G.omx = p.omx;
  G.omy = p.omy;
  G.omz = p.omz;
  G.scal = p.scal;
  return G;
}

cudaError_t ic_multiply(const gpe_params& p, const Geom& g, int esz, int R, const gpe_ic& ic, void* psi_field,
                        int modulus, cudaStream_t st) {
  if (ic_needs_fft(&ic)) return cudaErrorInvalidValue;
  const IcGrid G = ic_grid(p);
  const int nb = 148 * 8;
  if (esz == 16) k_ic_multiply<double2><<<nb, 256, 0, st>>>((double2*)psi_field, g, R, p.bcs, G, ic, modulus);
  else k_ic_multiply<float2><<<nb, 256, 0, st>>>((float2*)psi_field, g, R, p.bcs, G, ic, modulus);
  return cudaGetLastError();
}

cudaError_t ic_generate(const gpe_params& p, const Geom& g, int esz, int R, const gpe_ic& ic, void* psi_field,
                        void* work, size_t work_bytes, cudaStream_t st) {
  const IcGrid G = ic_grid(p);
  const int nb = 148 * 8;
  if (!ic_needs_fft(&ic)) {
    if (esz == 16) k_ic_closed_form<double2><<<nb, 256, 0, st>>>((double2*)psi_field, g, R, p.bcs, G, ic);
    else k_ic_closed_form<float2><<<nb, 256, 0, st>>>((float2*)psi_field, g, R, p.bcs, G, ic);
    return cudaGetLastError();
  }
  const long long n = (long long)p.nx * p.ny * p.nz;
  const size_t need = (size_t)n * sizeof(double2) + 1024 * sizeof(double) + 256;
  if (!work || work_bytes < need) return cudaErrorInvalidValue;
  double2* buf = (double2*)work;
  double* part = (double*)((char*)work + (((size_t)n * sizeof(double2) + 255) & ~size_t(255)));
  k_random_spectrum<<<nb, 256, 0, st>>>(buf, p.nx, p.ny, p.nz, G.dx, G.dy, G.dz, (unsigned long long)ic.seed, ic.kc);
  cufftHandle plan;
  if (!plan_for(p.nx, p.ny, p.nz, &plan)) return cudaErrorUnknown;
  if (cufftSetStream(plan, st) != CUFFT_SUCCESS) return cudaErrorUnknown;
  if (cufftExecZ2Z(plan, (cufftDoubleComplex*)buf, (cufftDoubleComplex*)buf, CUFFT_INVERSE) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  const int nbs = 1000;
  k_sumsq<<<nbs, 256, 0, st>>>(buf, n, part);
  k_sum_parts<<<1, 256, 0, st>>>(part, nbs);
  if (esz == 16) k_pack_scaled<double2><<<nb, 256, 0, st>>>(buf, part + nbs, (double2*)psi_field, g, R, p.bcs);
  else k_pack_scaled<float2><<<nb, 256, 0, st>>>(buf, part + nbs, (float2*)psi_field, g, R, p.bcs);
  return cudaGetLastError();
}

size_t ic_work_bytes(const gpe_params& p, const gpe_ic& ic) {
  if (!ic_needs_fft(&ic)) return 0;
  const size_t n = (size_t)p.nx * p.ny * p.nz;
  return ((n * sizeof(double2) + 255) & ~size_t(255)) + 1024 * sizeof(double) + 256;
}

}  // namespace gpe

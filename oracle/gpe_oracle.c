/*
 * CPU oracle: plain-C FP64 restatement of the reference's time-stepper path
 * (anthonyyoud/gpe src/solve.f90, src/derivs.f90, src/variables.f90,
 * src/ic.f90) for a single process.  TEST INFRASTRUCTURE ONLY -- see
 * gpe_oracle.h for who may load it and for its parity status ("parity
 * unpinned" by reference artefacts; pinned by analytic known answers).
 *
 * Expression order follows the Fortran statement by statement.  Complex
 * arithmetic is written out in reals the way gfortran lowers it:
 *   complex*complex  -> (ac - bd, ad + bc)          (no NaN fix-up)
 *   complex/real, real*complex -> componentwise
 *   complex/complex  -> Smith's algorithm (R. L. Smith, CACM 5(8) 1962)
 *   abs(complex)     -> hypot
 * Build with -ffp-contract=off: the reference is built with
 * -O3 -march=corei7 (src/Makefile.inc.linux:20), which has no FMA.
 */
#include "gpe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct or_ctx {
  or_params p;
  int nx, ny, nz, nx1, ny1, nz1;
  double xl, yl, zl, dx, dy, dz, dx2, dy2, dz2;
  double *x, *y, *z;
  /* derivative index maps (derivs.f90:276-398) per axis, [indx][0..3] =
   * minus(1), minus(2), plus(1), plus(2) */
  int *mx, *my, *mz;
  size_t nint, nhal;
  double *hold, *htmp;          /* halo'd psi%old / tmp (0:nx1,-2:ny+1,-2:nz+1) */
  double *kk[6];                /* stage arrays (interior) */
  double *tmpv, *errv, *scal;   /* rkqs work arrays */
  double *dxx, *dyy, *dzz, *lap, *dpx;
  double *diss, *vt, *sph;      /* real interior */
  int faithful_cost;            /* recompute diss/Vtrap/sphere per RHS */
};

/* ------------------------------------------------------------------ */
/* threads                                                             */

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* index helpers                                                        */

static inline size_t IX(const or_ctx *c, int i, int j, int k) {
  return ((size_t)k * c->ny + (size_t)j) * c->nx + (size_t)i;
}
/* halo'd array: j in [-2, ny+1], k in [-2, nz+1] (gpe.f90:59) */
static inline size_t HX(const or_ctx *c, int i, int j, int k) {
  return ((size_t)(k + 2) * (c->ny + 4) + (size_t)(j + 2)) * c->nx + (size_t)i;
}

/* derivs.f90:276-317 second_index */
static void second_index(int indx, int n, int bcs, int x_deriv, int mn[2], int pl[2]) {
  if (bcs == 1) {
    mn[0] = indx - 1;
    pl[0] = indx + 1;
    if (x_deriv) {
      if (indx == 0) { mn[0] = n; pl[0] = 1; }
      if (indx == n) { mn[0] = n - 1; pl[0] = 0; }
    }
  } else {
    mn[0] = indx - 1;
    pl[0] = indx + 1;
    if (indx == 0) { mn[0] = 1; pl[0] = 1; }
    if (indx == n) { mn[0] = n - 1; pl[0] = n - 1; }
  }
  mn[1] = 0;
  pl[1] = 0;
}

/* derivs.f90:321-398 fourth_index */
static void fourth_index(int indx, int n, int bcs, int x_deriv, int mn[2], int pl[2]) {
  mn[0] = indx - 1; mn[1] = indx - 2;
  pl[0] = indx + 1; pl[1] = indx + 2;
  if (bcs == 1) {
    if (x_deriv) {
      if (indx == 0)     { mn[0] = n;     mn[1] = n - 1; pl[0] = 1; pl[1] = 2; }
      if (indx == 1)     { mn[0] = 0;     mn[1] = n;     pl[0] = 2; pl[1] = 3; }
      if (indx == n - 1) { mn[0] = n - 2; mn[1] = n - 3; pl[0] = n; pl[1] = 0; }
      if (indx == n)     { mn[0] = n - 1; mn[1] = n - 2; pl[0] = 0; pl[1] = 1; }
    }
  } else {
    if (indx == 0)     { mn[0] = 1;     mn[1] = 2;     pl[0] = 1;     pl[1] = 2; }
    if (indx == 1)     { mn[0] = 0;     mn[1] = 1;     pl[0] = 2;     pl[1] = 3; }
    if (indx == n - 1) { mn[0] = n - 2; mn[1] = n - 3; pl[0] = n;     pl[1] = n - 1; }
    if (indx == n)     { mn[0] = n - 1; mn[1] = n - 2; pl[0] = n - 1; pl[1] = n - 2; }
  }
}

static int *make_map(int npts, int bcs, int order, int x_deriv) {
  int *m = (int *)malloc(sizeof(int) * 4 * (size_t)npts);
  for (int i = 0; i < npts; i++) {
    int mn[2], pl[2];
    if (order == 2) second_index(i, npts - 1, bcs, x_deriv, mn, pl);
    else fourth_index(i, npts - 1, bcs, x_deriv, mn, pl);
    m[4 * i + 0] = mn[0]; m[4 * i + 1] = mn[1];
    m[4 * i + 2] = pl[0]; m[4 * i + 3] = pl[1];
  }
  return m;
}

/* ------------------------------------------------------------------ */
/* set-up                                                               */

/* ic.f90:32-69 get_grid */
static void get_grid(or_ctx *c) {
  c->xl = -c->p.xr; c->yl = -c->p.yr; c->zl = -c->p.zr;
  c->dx = (c->p.xr - c->xl) / c->nx1;
  c->dy = (c->p.yr - c->yl) / c->ny1;
  c->dz = (c->p.zr - c->zl) / c->nz1;
  c->dx2 = c->dx * c->dx;
  c->dy2 = c->dy * c->dy;
  c->dz2 = c->dz * c->dz;
  for (int i = 0; i < c->nx; i++) c->x[i] = c->xl + (double)i * c->dx;
  for (int j = 0; j < c->ny; j++) c->y[j] = c->yl + (double)j * c->dy;
  for (int k = 0; k < c->nz; k++) c->z[k] = c->zl + (double)k * c->dz;
}

static void compute_diss(or_ctx *c);
static void compute_vtrap(or_ctx *c, double *out);
static void compute_sphere(or_ctx *c);

or_ctx *or_create(const or_params *prm) {
  if (prm->nx < 6 || prm->ny < 6 || prm->nz < 6) return NULL;
  if (prm->order != 2 && prm->order != 4) return NULL;
  if (prm->bcs != 1 && prm->bcs != 2) return NULL;
  if (prm->eqn < 1 || prm->eqn > 4) return NULL;
  if (prm->scheme < 0 || prm->scheme > 3) return NULL;
  or_ctx *c = (or_ctx *)calloc(1, sizeof(or_ctx));
  c->p = *prm;
  c->nx = prm->nx; c->ny = prm->ny; c->nz = prm->nz;
  c->nx1 = c->nx - 1; c->ny1 = c->ny - 1; c->nz1 = c->nz - 1;
  c->x = (double *)malloc(sizeof(double) * c->nx);
  c->y = (double *)malloc(sizeof(double) * c->ny);
  c->z = (double *)malloc(sizeof(double) * c->nz);
  get_grid(c);
  c->mx = make_map(c->nx, prm->bcs, prm->order, 1);
  c->my = make_map(c->ny, prm->bcs, prm->order, 0);
  c->mz = make_map(c->nz, prm->bcs, prm->order, 0);
  c->nint = (size_t)c->nx * c->ny * c->nz;
  c->nhal = (size_t)c->nx * (c->ny + 4) * (c->nz + 4);
  /* gpe.f90:133 psi%old = 0; automatic arrays are never read in their
   * halos under reflective BCs, so zero-initialised memory is equivalent */
  c->hold = (double *)calloc(2 * c->nhal, sizeof(double));
  c->htmp = (double *)calloc(2 * c->nhal, sizeof(double));
  for (int s = 0; s < 6; s++) c->kk[s] = (double *)calloc(2 * c->nint, sizeof(double));
  c->tmpv = (double *)calloc(2 * c->nint, sizeof(double));
  c->errv = (double *)calloc(2 * c->nint, sizeof(double));
  c->scal = (double *)calloc(2 * c->nint, sizeof(double));
  c->dxx = (double *)calloc(2 * c->nint, sizeof(double));
  c->dyy = (double *)calloc(2 * c->nint, sizeof(double));
  c->dzz = (double *)calloc(2 * c->nint, sizeof(double));
  c->lap = (double *)calloc(2 * c->nint, sizeof(double));
  c->dpx = (double *)calloc(2 * c->nint, sizeof(double));
  c->diss = (double *)calloc(c->nint, sizeof(double));
  c->vt = (double *)calloc(c->nint, sizeof(double));
  c->sph = (double *)calloc(c->nint, sizeof(double));
  c->faithful_cost = 0;
  compute_diss(c);
  compute_vtrap(c, c->vt);
  compute_sphere(c);
  return c;
}

void or_destroy(or_ctx *c) {
  if (!c) return;
  free(c->x); free(c->y); free(c->z);
  free(c->mx); free(c->my); free(c->mz);
  free(c->hold); free(c->htmp);
  for (int s = 0; s < 6; s++) free(c->kk[s]);
  free(c->tmpv); free(c->errv); free(c->scal);
  free(c->dxx); free(c->dyy); free(c->dzz); free(c->lap); free(c->dpx);
  free(c->diss); free(c->vt); free(c->sph);
  free(c);
}

/* When set, diss(), Vtrap() and sphere() are rebuilt on every RHS call as
 * the reference does (solve.f90:401-409, ic.f90:713-731, ic.f90:640-662);
 * the values are identical either way, only the CPU cost differs. */
void or_set_faithful_cost(or_ctx *c, int on) { c->faithful_cost = on; }

void or_get_grid(const or_ctx *c, double *x, double *y, double *z, double *dxyz) {
  if (x) memcpy(x, c->x, sizeof(double) * c->nx);
  if (y) memcpy(y, c->y, sizeof(double) * c->ny);
  if (z) memcpy(z, c->z, sizeof(double) * c->nz);
  if (dxyz) { dxyz[0] = c->dx; dxyz[1] = c->dy; dxyz[2] = c->dz; }
}

/* solve.f90:397-409 */
static void compute_diss(or_ctx *c) {
  const double a = c->x[c->nx - 3], b = c->y[c->ny - 3], cc = c->z[c->nz - 3];
  const double amp = c->p.diss_amp;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double xi = c->x[i], yj = c->y[j], zk = c->z[k];
        c->diss[IX(c, i, j, k)] =
            amp * (((1.0 + tanh(xi - a) * tanh(xi + a)) + (1.0 + tanh(yj - b) * tanh(yj + b))) +
                   (1.0 + tanh(zk - cc) * tanh(zk + cc)));
      }
}

/* ic.f90:713-731 Vtrap */
static void compute_vtrap(or_ctx *c, double *out) {
  const double o1 = c->p.omx, o2 = c->p.omy, o3 = c->p.omz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double xi = c->x[i], yj = c->y[j], zk = c->z[k];
        out[IX(c, i, j, k)] = 0.5 * (((o1 * o1) * (xi * xi) + (o2 * o2) * (yj * yj)) + (o3 * o3) * (zk * zk));
      }
}

void or_vtrap(or_ctx *c, double *out) { compute_vtrap(c, out); }

/* ic.f90:640-662 sphere (rad = 10, eps1 = 2) */
static void compute_sphere(or_ctx *c) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double xi = c->x[i], yj = c->y[j], zk = c->z[k];
        c->sph[IX(c, i, j, k)] = 0.5 * (1.0 + tanh((sqrt((xi * xi + yj * yj) + zk * zk) - 10.0) - 2.0));
      }
}

/* ------------------------------------------------------------------ */
/* halos                                                                */

/* Copy an interior array into the halo'd layout and fill the halos the way
 * gpe.f90:167-176 (copy + send_recv_z + pack_y/send_recv_y/unpack_y) does on
 * one rank: periodic BCs wrap with period ny / nz (variables.f90:123-128);
 * reflective BCs leave the halos untouched (never read, derivs.f90:365). */
static void fill_halo(or_ctx *c, double *h) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  if (c->p.bcs != 1) return;
  /* send_recv_z: planes ke-1, ks+1 first, then ke, ks, for j in js..je */
  for (int j = 0; j < ny; j++) {
    memcpy(&h[2 * HX(c, 0, j, -2)], &h[2 * HX(c, 0, j, nz - 2)], sizeof(double) * 2 * nx);
    memcpy(&h[2 * HX(c, 0, j, nz + 1)], &h[2 * HX(c, 0, j, 1)], sizeof(double) * 2 * nx);
    memcpy(&h[2 * HX(c, 0, j, -1)], &h[2 * HX(c, 0, j, nz - 1)], sizeof(double) * 2 * nx);
    memcpy(&h[2 * HX(c, 0, j, nz)], &h[2 * HX(c, 0, j, 0)], sizeof(double) * 2 * nx);
  }
  /* pack_y / send_recv_y / unpack_y for k in kks..kke = 0..nz-1 */
  for (int k = 0; k < nz; k++) {
    memcpy(&h[2 * HX(c, 0, -2, k)], &h[2 * HX(c, 0, ny - 2, k)], sizeof(double) * 4 * nx);
    memcpy(&h[2 * HX(c, 0, ny, k)], &h[2 * HX(c, 0, 0, k)], sizeof(double) * 4 * nx);
  }
}

static void to_halo(or_ctx *c, const double *in, double *h) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      memcpy(&h[2 * HX(c, 0, j, k)], &in[2 * IX(c, 0, j, k)], sizeof(double) * 2 * c->nx);
  fill_halo(c, h);
}

/* ------------------------------------------------------------------ */
/* derivatives: derivs.f90:25-64 (deriv_x), 146-272 (deriv_xx/yy/zz)    */

static void deriv_x(or_ctx *c, const double *f, double *fx) {
  const int *m = c->mx;
  const double dx = c->dx;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        const double *fm1 = &f[2 * HX(c, m[4 * i + 0], j, k)];
        const double *fp1 = &f[2 * HX(c, m[4 * i + 2], j, k)];
        double *o = &fx[2 * IX(c, i, j, k)];
        if (c->p.order == 2) {
          for (int r = 0; r < 2; r++) o[r] = (fp1[r] - fm1[r]) / (2.0 * dx);
        } else {
          const double *fm2 = &f[2 * HX(c, m[4 * i + 1], j, k)];
          const double *fp2 = &f[2 * HX(c, m[4 * i + 3], j, k)];
          for (int r = 0; r < 2; r++)
            o[r] = (((-fp2[r] + 8.0 * fp1[r]) - 8.0 * fm1[r]) + fm2[r]) / (12.0 * dx);
        }
      }
}

/* axis 0 = x (index map per i), 1 = y (per j), 2 = z (per k) */
static void deriv_2(or_ctx *c, const double *f, double *out, int axis) {
  const int order = c->p.order;
  const double d2 = axis == 0 ? c->dx2 : axis == 1 ? c->dy2 : c->dz2;
  const int *m = axis == 0 ? c->mx : axis == 1 ? c->my : c->mz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        int q = axis == 0 ? i : axis == 1 ? j : k;
        size_t cm1, cm2, cp1, cp2;
        if (axis == 0) {
          cm1 = HX(c, m[4 * q], j, k); cm2 = HX(c, m[4 * q + 1], j, k);
          cp1 = HX(c, m[4 * q + 2], j, k); cp2 = HX(c, m[4 * q + 3], j, k);
        } else if (axis == 1) {
          cm1 = HX(c, i, m[4 * q], k); cm2 = HX(c, i, m[4 * q + 1], k);
          cp1 = HX(c, i, m[4 * q + 2], k); cp2 = HX(c, i, m[4 * q + 3], k);
        } else {
          cm1 = HX(c, i, j, m[4 * q]); cm2 = HX(c, i, j, m[4 * q + 1]);
          cp1 = HX(c, i, j, m[4 * q + 2]); cp2 = HX(c, i, j, m[4 * q + 3]);
        }
        const double *f0 = &f[2 * HX(c, i, j, k)];
        double *o = &out[2 * IX(c, i, j, k)];
        if (order == 2) {
          for (int r = 0; r < 2; r++)
            o[r] = ((f[2 * cp1 + r] - 2.0 * f0[r]) + f[2 * cm1 + r]) / d2;
        } else {
          for (int r = 0; r < 2; r++)
            o[r] = ((((-f[2 * cp2 + r] + 16.0 * f[2 * cp1 + r]) - 30.0 * f0[r]) + 16.0 * f[2 * cm1 + r]) -
                    f[2 * cm2 + r]) /
                   (12.0 * d2);
        }
      }
}

/* variables.f90:55-71 */
static void laplacian_h(or_ctx *c, const double *h, double *lap) {
  deriv_2(c, h, c->dxx, 0);
  deriv_2(c, h, c->dyy, 1);
  deriv_2(c, h, c->dzz, 2);
#pragma omp parallel for schedule(static)
  for (size_t n = 0; n < 2 * c->nint; n++) lap[n] = (c->dxx[n] + c->dyy[n]) + c->dzz[n];
}

void or_laplacian(or_ctx *c, const double *psi, double *out) {
  to_halo(c, psi, c->htmp);
  laplacian_h(c, c->htmp, out);
}

void or_deriv_x(or_ctx *c, const double *psi, double *out) {
  to_halo(c, psi, c->htmp);
  deriv_x(c, c->htmp, out);
}

/* ------------------------------------------------------------------ */
/* solve.f90:382-440 get_rhs (input halo'd, output interior)             */

static void get_rhs_h(or_ctx *c, const double *h, double *rhs) {
  const int eqn = c->p.eqn;
  if (c->faithful_cost) {
    compute_diss(c);
    if (eqn == 4) compute_vtrap(c, c->vt);
    if (eqn == 3) compute_sphere(c);
  }
  deriv_x(c, h, c->dpx);
  laplacian_h(c, h, c->lap);
  const double U = c->p.Urhs, g = c->p.g, mu = c->p.mu, gam = c->p.gamma;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k);
        const double *f = &h[2 * HX(c, i, j, k)];
        const double pr = f[0], pi = f[1];
        const double lr = c->lap[2 * n], li = c->lap[2 * n + 1];
        const double dr = c->dpx[2 * n], di = c->dpx[2 * n + 1];
        double rr, ri;
        if (eqn == 1 || eqn == 3) {
          /* 0.5*(eye+diss) * (lap + (1-abs(psi)**2)*psi) + Urhs*dpsidx */
          double a = 0.5 * c->diss[n], b = 0.5 * 1.0;
          double h2 = hypot(pr, pi);
          double s = 1.0 - h2 * h2;
          double cr = lr + s * pr, ci = li + s * pi;
          rr = (a * cr - b * ci) + U * dr;
          ri = (a * ci + b * cr) + U * di;
          if (eqn == 3) {
            double sp = c->sph[n];
            rr = rr * sp;
            ri = ri * sp;
          }
        } else if (eqn == 2) {
          /* eye * (lap - abs(psi)**2*psi) + Urhs*dpsidx */
          double h2 = hypot(pr, pi);
          double s = h2 * h2;
          double cr = lr - s * pr, ci = li - s * pi;
          rr = -ci + U * dr;
          ri = cr + U * di;
        } else {
          /* -eye * (-0.5*lap + Vtrap*psi + g*(abs(psi**2)*psi) - mu*psi);
           * with gamma != 0: -(eye+gamma) * (...) */
          double v = c->vt[n];
          double sqr = pr * pr - pi * pi, sqi = pr * pi + pi * pr;
          double a2 = hypot(sqr, sqi);
          double wr = ((-0.5 * lr + v * pr) + g * (a2 * pr)) - mu * pr;
          double wi = ((-0.5 * li + v * pi) + g * (a2 * pi)) - mu * pi;
          if (gam == 0.0) {
            rr = wi;
            ri = -wr;
          } else {
            double ar = -gam, ai = -1.0;
            rr = ar * wr - ai * wi;
            ri = ar * wi + ai * wr;
          }
        }
        rhs[2 * n] = rr;
        rhs[2 * n + 1] = ri;
      }
}

void or_get_rhs(or_ctx *c, const double *psi, double *rhs) {
  to_halo(c, psi, c->htmp);
  get_rhs_h(c, c->htmp, rhs);
}

/* ------------------------------------------------------------------ */
/* schemes: solve.f90:57-378                                            */

static inline void cmul(double ar, double ai, double br, double bi, double *r, double *i) {
  *r = ar * br - ai * bi;
  *i = ar * bi + ai * br;
}

/* complex/complex as gfortran expands it with -fcx-fortran-rules:
 * Smith's algorithm */
static inline void cdiv(double ar, double ai, double br, double bi, double *r, double *i) {
  if (fabs(br) < fabs(bi)) {
    double ratio = br / bi;
    double div = (br * ratio) + bi;
    *r = ((ar * ratio) + ai) / div;
    *i = ((ai * ratio) - ar) / div;
  } else {
    double ratio = bi / br;
    double div = (bi * ratio) + br;
    *r = ((ai * ratio) + ar) / div;
    *i = (ai - (ar * ratio)) / div;
  }
}

/* interior of the halo'd array into an interior array */
static void from_halo(or_ctx *c, const double *h, double *out) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      memcpy(&out[2 * IX(c, 0, j, k)], &h[2 * HX(c, 0, j, k)], sizeof(double) * 2 * c->nx);
}

/* solve.f90:57-74 */
static void euler(or_ctx *c, double *psi, or_clock *clk) {
  double *old = c->hold, *rhs = c->kk[0];
  get_rhs_h(c, old, rhs);
  const double dr = clk->dt_re, di = clk->dt_im;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        double tr, ti;
        cmul(dr, di, rhs[2 * n], rhs[2 * n + 1], &tr, &ti);
        psi[2 * n] = old[2 * h] + tr;
        psi[2 * n + 1] = old[2 * h + 1] + ti;
      }
  clk->t = clk->t + clk->dt_re;
  clk->im_t = clk->im_t + fabs(clk->dt_im);
}

/* tmp(interior) = old + (fac*dt) * kk ; then halo fill (send_recv_z/y) */
static void stage_combo(or_ctx *c, const double *old, const double *k, double fac, double dr,
                        double di, double *tmp) {
  const double hr = fac * dr, hi = fac * di;
#pragma omp parallel for collapse(2) schedule(static)
  for (int kz = 0; kz < c->nz; kz++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, kz), h = HX(c, i, j, kz);
        double tr, ti;
        cmul(hr, hi, k[2 * n], k[2 * n + 1], &tr, &ti);
        tmp[2 * h] = old[2 * h] + tr;
        tmp[2 * h + 1] = old[2 * h + 1] + ti;
      }
  fill_halo(c, tmp);
}

/* solve.f90:78-105 */
static void rk2(or_ctx *c, double *psi, or_clock *clk) {
  double *old = c->hold, *tmp = c->htmp, *k1 = c->kk[0], *k2 = c->kk[1];
  const double dr = clk->dt_re, di = clk->dt_im;
  get_rhs_h(c, old, k1);
  stage_combo(c, old, k1, 0.5, dr, di, tmp);
  get_rhs_h(c, tmp, k2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        double tr, ti;
        cmul(dr, di, k2[2 * n], k2[2 * n + 1], &tr, &ti);
        psi[2 * n] = old[2 * h] + tr;
        psi[2 * n + 1] = old[2 * h + 1] + ti;
      }
  clk->t = clk->t + clk->dt_re;
  clk->im_t = clk->im_t + fabs(clk->dt_im);
}

/* solve.f90:109-154 */
static void rk4(or_ctx *c, double *psi, or_clock *clk) {
  double *old = c->hold, *tmp = c->htmp;
  double *k1 = c->kk[0], *k2 = c->kk[1], *k3 = c->kk[2], *k4 = c->kk[3];
  const double dr = clk->dt_re, di = clk->dt_im;
  get_rhs_h(c, old, k1);
  stage_combo(c, old, k1, 0.5, dr, di, tmp);
  get_rhs_h(c, tmp, k2);
  stage_combo(c, old, k2, 0.5, dr, di, tmp);
  get_rhs_h(c, tmp, k3);
  stage_combo(c, old, k3, 1.0, dr, di, tmp);
  get_rhs_h(c, tmp, k4);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        double sr = ((k1[2 * n] / 6.0 + k2[2 * n] / 3.0) + k3[2 * n] / 3.0) + k4[2 * n] / 6.0;
        double si = ((k1[2 * n + 1] / 6.0 + k2[2 * n + 1] / 3.0) + k3[2 * n + 1] / 3.0) + k4[2 * n + 1] / 6.0;
        double tr, ti;
        cmul(dr, di, sr, si, &tr, &ti);
        psi[2 * n] = old[2 * h] + tr;
        psi[2 * n + 1] = old[2 * h + 1] + ti;
      }
  clk->t = clk->t + clk->dt_re;
  clk->im_t = clk->im_t + fabs(clk->dt_im);
}

/* Cash-Karp tableau, solve.f90:255-281 */
static const double b21 = 0.2, b31 = 0.075, b32 = 0.225, b41 = 0.3, b42 = -0.9, b43 = 1.2;
#define B51 (-11.0 / 54.0)
#define B52 2.5
#define B53 (-70.0 / 27.0)
#define B54 (35.0 / 27.0)
#define B61 (1631.0 / 55296.0)
#define B62 (175.0 / 512.0)
#define B63 (575.0 / 13824.0)
#define B64 (44275.0 / 110592.0)
#define B65 (253.0 / 4096.0)
#define C1 (37.0 / 378.0)
#define C2 0.0
#define C3 (250.0 / 621.0)
#define C4 (125.0 / 594.0)
#define C5 0.0
#define C6 (512.0 / 1771.0)
#define DC1 (C1 - 2825.0 / 27648.0)
#define DC2 (C2 - 0.0)
#define DC3 (C3 - 18575.0 / 48384.0)
#define DC4 (C4 - 13525.0 / 55296.0)
#define DC5 (C5 - 277.0 / 14336.0)
#define DC6 (C6 - 0.25)

/* kk(s) = dt*kk(s) in place */
static void scale_dt(or_ctx *c, double *k, double dr, double di) {
#pragma omp parallel for schedule(static)
  for (size_t n = 0; n < c->nint; n++) {
    double tr, ti;
    cmul(dr, di, k[2 * n], k[2 * n + 1], &tr, &ti);
    k[2 * n] = tr;
    k[2 * n + 1] = ti;
  }
}

/* solve.f90:248-378 rkck: new, err interior */
static void rkck(or_ctx *c, const double *old, double *newv, double *err, double dr, double di) {
  double *tmp = c->htmp;
  double **K = c->kk;
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  get_rhs_h(c, old, K[0]);
  scale_dt(c, K[0], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++) tmp[2 * h + r] = old[2 * h + r] + b21 * K[0][2 * n + r];
      }
  fill_halo(c, tmp);
  get_rhs_h(c, tmp, K[1]);
  scale_dt(c, K[1], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++)
          tmp[2 * h + r] = (old[2 * h + r] + b31 * K[0][2 * n + r]) + b32 * K[1][2 * n + r];
      }
  fill_halo(c, tmp);
  get_rhs_h(c, tmp, K[2]);
  scale_dt(c, K[2], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++)
          tmp[2 * h + r] =
              ((old[2 * h + r] + b41 * K[0][2 * n + r]) + b42 * K[1][2 * n + r]) + b43 * K[2][2 * n + r];
      }
  fill_halo(c, tmp);
  get_rhs_h(c, tmp, K[3]);
  scale_dt(c, K[3], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++)
          tmp[2 * h + r] = (((old[2 * h + r] + B51 * K[0][2 * n + r]) + B52 * K[1][2 * n + r]) +
                            B53 * K[2][2 * n + r]) +
                           B54 * K[3][2 * n + r];
      }
  fill_halo(c, tmp);
  get_rhs_h(c, tmp, K[4]);
  scale_dt(c, K[4], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++)
          tmp[2 * h + r] = ((((old[2 * h + r] + B61 * K[0][2 * n + r]) + B62 * K[1][2 * n + r]) +
                             B63 * K[2][2 * n + r]) +
                            B64 * K[3][2 * n + r]) +
                           B65 * K[4][2 * n + r];
      }
  fill_halo(c, tmp);
  get_rhs_h(c, tmp, K[5]);
  scale_dt(c, K[5], dr, di);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        for (int r = 0; r < 2; r++) {
          size_t q = 2 * n + r;
          newv[q] = (((((old[2 * h + r] + C1 * K[0][q]) + C2 * K[1][q]) + C3 * K[2][q]) + C4 * K[3][q]) +
                     C5 * K[4][q]) +
                    C6 * K[5][q];
          err[q] = ((((DC1 * K[0][q] + DC2 * K[1][q]) + DC3 * K[2][q]) + DC4 * K[3][q]) + DC5 * K[4][q]) +
                   DC6 * K[5][q];
        }
      }
}

static const double EPS_RK = 1e-6, SAFETY = 0.9, DT_DECREASE = -0.25, DT_INCREASE = -0.20;

/* solve.f90:158-244 rkqs */
static void rkqs(or_ctx *c, double *psi, or_clock *clk) {
  const double *in = c->hold;
  const double errcon = pow(5.0 / SAFETY, 1.0 / DT_INCREASE);
  double dr = clk->dt_re, di = clk->dt_im;
  /* psi_scal = abs(in) + dt*abs(rhs) + 1e-30 */
  get_rhs_h(c, in, c->scal);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k), h = HX(c, i, j, k);
        double a = hypot(in[2 * h], in[2 * h + 1]);
        double f = hypot(c->scal[2 * n], c->scal[2 * n + 1]);
        c->scal[2 * n] = (a + dr * f) + 1e-30;
        c->scal[2 * n + 1] = di * f;
      }
  double errmax;
  for (;;) {
    rkck(c, in, c->tmpv, c->errv, dr, di);
    errmax = 0.0;
    for (size_t n = 0; n < c->nint; n++) {
      double qr, qi;
      cdiv(c->errv[2 * n], c->errv[2 * n + 1], c->scal[2 * n], c->scal[2 * n + 1], &qr, &qi);
      double a = hypot(qr, qi);
      if (a > errmax) errmax = a;
    }
    errmax = errmax / EPS_RK;
    if (errmax <= 1.0) break;
    clk->rejected++;
    /* dt_temp = safety*dt*(errmax**dt_decrease) */
    double e = pow(errmax, DT_DECREASE);
    double tr = (SAFETY * dr) * e, ti = (SAFETY * di) * e;
    double adt = hypot(dr, di);
    double m = fmax(hypot(tr, ti), 0.1 * adt);
    if (!c->p.real_time) { dr = 0.0; di = -m; }
    else { dr = m; di = 0.0; }
  }
  double nr, ni;
  if (errmax > errcon) {
    double e = pow(errmax, DT_INCREASE);
    nr = (SAFETY * dr) * e;
    ni = (SAFETY * di) * e;
  } else {
    nr = 5.0 * dr;
    ni = 5.0 * di;
  }
  clk->t = clk->t + dr;
  clk->dt_re = nr;
  clk->dt_im = ni;
  clk->im_t = clk->im_t + fabs(ni); /* uses the NEW dt (solve.f90:229) */
  clk->errmax = errmax;
  memcpy(psi, c->tmpv, sizeof(double) * 2 * c->nint);
}

void or_solver(or_ctx *c, double *psi, or_clock *clk) {
  /* gpe.f90:167-176: psi%old = psi%new + halo exchange */
  to_halo(c, psi, c->hold);
  switch (c->p.scheme) {
    case 0: euler(c, psi, clk); break;
    case 1: rk2(c, psi, clk); break;
    case 2: rk4(c, psi, clk); break;
    default: rkqs(c, psi, clk); break;
  }
  clk->p += 1;
}

void or_run(or_ctx *c, double *psi, or_clock *clk, int64_t nsteps) {
  for (int64_t s = 0; s < nsteps; s++) or_solver(c, psi, clk);
}

/* ------------------------------------------------------------------ */
/* reductions: variables.f90:554-604, 715-840                           */

static const double QC1 = 3.0 / 8.0, QC2 = 7.0 / 6.0, QC3 = 23.0 / 24.0;

double or_get_norm(or_ctx *c, const double *psi) {
  const int nx = c->nx, ny = c->ny, nz = c->nz;
  double *xint = (double *)malloc(sizeof(double) * (size_t)ny * nz);
  double *yint = (double *)malloc(sizeof(double) * (size_t)nz);
  /* integrate_x (variables.f90:730-753) */
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) {
      const double *row = &psi[2 * IX(c, 0, j, k)];
#define IV(ii) (hypot(row[2 * (ii)], row[2 * (ii) + 1]) * hypot(row[2 * (ii)], row[2 * (ii) + 1]))
      double s = 0.0;
      for (int i = 3; i <= nx - 4; i++) s = s + IV(i);
      xint[(size_t)k * ny + j] =
          ((((((QC1 * IV(0) + QC2 * IV(1)) + QC3 * IV(2)) + s) + QC3 * IV(nx - 3)) + QC2 * IV(nx - 2)) +
           QC1 * IV(nx - 1)) *
          c->dx;
#undef IV
    }
  /* integrate_y (variables.f90:757-798) */
  for (int k = 0; k < nz; k++) {
    double s = 0.0;
    for (int j = 0; j < ny; j++) {
      double v = xint[(size_t)k * ny + j], t = v;
      if (j == 0) t = QC1 * v;
      if (j == 1) t = QC2 * v;
      if (j == 2) t = QC3 * v;
      if (j == ny - 3) t = QC3 * v;
      if (j == ny - 2) t = QC2 * v;
      if (j == ny - 1) t = QC1 * v;
      s = s + t;
    }
    yint[k] = s * c->dy;
  }
  /* integrate_z (variables.f90:802-840) */
  double s = 0.0;
  for (int k = 0; k < nz; k++) {
    double v = yint[k], t = v;
    if (k == 0) t = QC1 * v;
    if (k == 1) t = QC2 * v;
    if (k == 2) t = QC3 * v;
    if (k == nz - 3) t = QC3 * v;
    if (k == nz - 2) t = QC2 * v;
    if (k == nz - 1) t = QC1 * v;
    s = s + t;
  }
  free(xint);
  free(yint);
  return s * c->dz;
}

double or_energy(or_ctx *c, const double *psi) {
  to_halo(c, psi, c->htmp);
  laplacian_h(c, c->htmp, c->lap);
  double s = 0.0;
  for (size_t n = 0; n < c->nint; n++) {
    double pr = psi[2 * n], pi = psi[2 * n + 1];
    double ar = -c->lap[2 * n], ai = -c->lap[2 * n + 1];
    /* real(-lap * conjg(psi) + 0.5*abs(psi)**4) */
    double re = ar * pr - ai * (-pi);
    double h = hypot(pr, pi);
    double h2 = h * h;
    s = s + (re + 0.5 * (h2 * h2));
  }
  return ((s * c->dx) * c->dy) * c->dz;
}

void or_renormalise(or_ctx *c, double *psi, double norm) {
  const double a = sqrt(c->p.nn), b = sqrt(norm);
  for (size_t n = 0; n < 2 * c->nint; n++) psi[n] = (a * psi[n]) / b;
}

/* ------------------------------------------------------------------ */
/* initial conditions: ic.f90                                           */

/* ic.f90:893-906 get_rr */
void or_get_rr(const double *r, double *rr, int64_t n) {
  for (int64_t q = 0; q < n; q++) {
    double r2 = r[q] * r[q];
    double r4 = r2 * r2;
    rr[q] = sqrt((0.3437 + 0.0286 * r2) / ((1.0 + 0.3333 * r2) + 0.0286 * r4));
  }
}

static double rr1(double r) {
  double rr;
  or_get_rr(&r, &rr, 1);
  return rr;
}

/* ic.f90:357-514 vortex_ring; plane in {xy, xz, yz} */
int or_vortex_ring(or_ctx *c, const or_ring *vr, double *out) {
  int pl;
  if (vr->plane[0] == 'x' && vr->plane[1] == 'y') pl = 0;
  else if (vr->plane[0] == 'x' && vr->plane[1] == 'z') pl = 1;
  else if (vr->plane[0] == 'y' && vr->plane[1] == 'z') pl = 2;
  else return -1;
  const double sc = c->p.scal;
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double xi = c->x[i], yj = c->y[j], zk = c->z[k];
        double u, v, w, u0, v0, w0; /* in-plane (u, v), normal w */
        if (pl == 0) { u = xi; v = yj; w = zk; u0 = vr->x0; v0 = vr->y0; w0 = vr->z0; }
        else if (pl == 1) { u = xi; v = zk; w = yj; u0 = vr->x0; v0 = vr->z0; w0 = vr->y0; }
        else { u = yj; v = zk; w = xi; u0 = vr->y0; v0 = vr->z0; w0 = vr->x0; }
        double theta = atan2(v - v0, u - u0);
        double s = sqrt((u - u0) * (u - u0) + (v - v0) * (v - v0)) - vr->r1 * sin((double)vr->kk * theta);
        double dist = vr->amp * cos((double)vr->mm * theta);
        double pp = w - vr->r1 * cos((double)vr->kk * theta);
        double A = sc * (pp - w0);
        double Bp = sc * ((s + vr->r0) - dist);
        double Bm = sc * ((s - vr->r0) - dist);
        double d1 = sqrt(A * A + Bp * Bp);
        double d2 = sqrt(A * A + Bm * Bm);
        double q1 = rr1(d1), q2 = rr1(d2);
        /* rr1*(A + dir*eye*Bp) * rr2 * (A - dir*eye*Bm) */
        double z1r = A + vr->dir * 0.0 * Bp, z1i = vr->dir * Bp;
        double z2r = A - vr->dir * 0.0 * Bm, z2i = -(vr->dir * Bm);
        double tr = (q1 * z1r) * q2, ti = (q1 * z1i) * q2;
        double orr, oi;
        cmul(tr, ti, z2r, z2i, &orr, &oi);
        out[2 * IX(c, i, j, k)] = orr;
        out[2 * IX(c, i, j, k) + 1] = oi;
      }
  return 0;
}

/* ic.f90:735-800 get_r and ic.f90:824-889 get_theta; returns X, Y, r, theta */
static int line_geom(or_ctx *c, const or_line *vl, int i, int j, int k, double *r, double *theta) {
  const double PI = 3.1415926535897932384626433832795;
  double safe1 = 0.0, safe2 = 0.0;
  const double eps = 2.220446049250313e-16;
  if (fabs(vl->ll) < eps) {
    if (fabs(vl->amp1) < eps) safe1 = 1.0; else return -1;
    if (fabs(vl->amp2) < eps) safe2 = 1.0; else return -1;
  }
  const double sc = c->p.scal;
  double xi = c->x[i], yj = c->y[j], zk = c->z[k];
  double a, b; /* r: first / second transverse coordinate */
  if (vl->dir == 'x') {
    a = yj - vl->y0 - vl->amp1 * sin(2.0 * PI * (xi - vl->x0) / (vl->ll + safe1));
    b = zk - vl->z0 - vl->amp2 * cos(2.0 * PI * (xi - vl->x0) / (vl->ll + safe2));
  } else if (vl->dir == 'y') {
    a = zk - vl->z0 - vl->amp1 * sin(2.0 * PI * (yj - vl->y0) / (vl->ll + safe1));
    b = xi - vl->x0 - vl->amp2 * cos(2.0 * PI * (yj - vl->y0) / (vl->ll + safe2));
  } else if (vl->dir == 'z') {
    a = xi - vl->x0 - vl->amp1 * sin(2.0 * PI * (zk - vl->z0) / (vl->ll + safe1));
    b = yj - vl->y0 - vl->amp2 * cos(2.0 * PI * (zk - vl->z0) / (vl->ll + safe2));
  } else {
    return -1;
  }
  /* get_r: sqrt(scal*a**2 + scal*b**2); get_theta: sgn*atan2(scal*b, scal*a) */
  *r = sqrt(sc * (a * a) + sc * (b * b));
  *theta = vl->sgn * atan2(sc * b, sc * a);
  return 0;
}

/* ic.f90:332-353 vortex_line with amp(r) = 1 - exp(-0.7 r**1.15) (ic.f90:314-328) */
int or_vortex_line(or_ctx *c, const or_line *vl, double *out) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double r, th;
        if (line_geom(c, vl, i, j, k, &r, &th)) return -1;
        double a = vl->imprint_phase ? 1.0 : 1.0 - exp(-0.7 * pow(r, 1.15));
        size_t n = IX(c, i, j, k);
        out[2 * n] = a * cos(th);
        out[2 * n + 1] = a * sin(th);
      }
  return 0;
}

/* straight vortex line with the Pade core: R(r) e^{i theta}, R(r) = r*get_rr(r) */
int or_vortex_line_pade(or_ctx *c, const or_line *vl, double *out) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double r, th;
        if (line_geom(c, vl, i, j, k, &r, &th)) return -1;
        double a = r * rr1(r);
        size_t n = IX(c, i, j, k);
        out[2 * n] = a * cos(th);
        out[2 * n + 1] = a * sin(th);
      }
  return 0;
}

/* ic.f90:278-310 fermi (mu_tf = mu) */
void or_fermi(or_ctx *c, double *out) {
  double *v = (double *)malloc(sizeof(double) * c->nint);
  compute_vtrap(c, v);
  for (size_t n = 0; n < c->nint; n++) {
    double f = (c->p.mu - v[n]) / c->p.g;
    out[2 * n] = f >= 0.0 ? sqrt(f) : 0.0;
    out[2 * n + 1] = 0.0;
  }
  free(v);
}

/* ic.f90:518-587 pade_pulse_ring.  get_consts (ic.f90:563-585) lists a(1..9),
 * U and m for 'ring' and 'pulse'; denom, uu and vv are evaluated per site as
 * the loop at ic.f90:537-555 writes them, with s = get_s (ic.f90:804-820). */
int or_pade_pulse_ring(or_ctx *c, int pulse, double x0, double y0, double z0, double r0, double *out) {
  static const double ring_a[9] = {-1.1, 0.0170524, 0.0289452, -0.953, -0.0049767, -0.0594346, 0.04, 0.21,
                                   0.00612};
  static const double pulse_a[9] = {-0.79792, 0.00388059, 0.00882276, -0.7981, -0.012783, -0.0574092, 0.0399,
                                    0.199, 0.0058};
  const double *a = pulse ? pulse_a : ring_a;
  const double U = pulse ? 0.63 : 0.6, m = pulse ? 8.37 : 8.97;
  const double pw = 7.0 / 4.0;
  const double one_2u = 1.0 - 2.0 * (U * U);
  const double a9p = pow(a[8], pw);
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++) {
      double dy = c->y[j] - y0, dz = c->z[k] - z0;
      double sjk = sqrt(dy * dy + dz * dz);
      double s2 = (sjk - r0) * (sjk - r0);
      for (int i = 0; i < c->nx; i++) {
        double xs = c->x[i] - x0;
        double x2 = xs * xs;
        double t = x2 + one_2u * s2;
        double denom = pow(((1.0 + a[7] * x2) + a[6] * s2) + a[8] * (t * t), pw);
        double uu = 1.0 + ((((a[0] + a[2] * x2) + a[1] * s2) + ((m * a9p) * U) * (2.0 * x2 - one_2u * s2)) * t) /
                              denom;
        double vv = (xs * (((a[3] + a[5] * x2) + a[4] * s2) - (m * a9p) * (t * t))) / denom;
        size_t n = IX(c, i, j, k);
        out[2 * n] = uu;
        out[2 * n + 1] = vv;
      }
    }
  return 0;
}

/* ic.f90:591-636 vortex_pair (the same in every z plane) */
void or_vortex_pair(or_ctx *c, double *out) {
  const double a0 = -1.14026, a1 = -0.150112, a2 = -0.0294564;
  const double b0 = -0.830953, b1 = -0.108296, b2 = -0.073641;
  const double c0 = 0.35022, c1 = 0.03032, c2 = 0.15905, c3 = 0.04123, c4 = 0.01402;
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double x = c->x[i], y = c->y[j];
        double x2 = x * x, y2 = y * y;
        double denom = ((((1.0 + c0 * x2) + c1 * (x2 * x2)) + c2 * y2) + (c3 * x2) * y2) + c4 * (y2 * y2);
        size_t n = IX(c, i, j, k);
        out[2 * n] = 1.0 + ((a0 + a1 * x2) + a2 * y2) / denom;
        out[2 * n + 1] = (x * ((b0 + b1 * x2) + b2 * y2)) / denom;
      }
}

/* ic.f90:640-662 sphere, 666-684 sphere2, 688-709 wall (real factors) */
void or_sphere(or_ctx *c, double *out) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double x = c->x[i], y = c->y[j], z = c->z[k];
        size_t n = IX(c, i, j, k);
        out[2 * n] = 0.5 * (1.0 + tanh((sqrt((x * x + y * y) + z * z) - 10.0) - 2.0));
        out[2 * n + 1] = 0.0;
      }
}

void or_sphere2(or_ctx *c, double *out) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        double x = c->x[i], y = c->y[j], z = c->z[k];
        size_t n = IX(c, i, j, k);
        out[2 * n] = 100.0 * exp(-((x * x + y * y) + z * z) / 10.0);
        out[2 * n + 1] = 0.0;
      }
}

void or_wall(or_ctx *c, double *out) {
  for (int k = 0; k < c->nz; k++)
    for (int j = 0; j < c->ny; j++)
      for (int i = 0; i < c->nx; i++) {
        size_t n = IX(c, i, j, k);
        out[2 * n] = c->z[k] <= -30.0 ? 0.0 : 1.0;
        out[2 * n + 1] = 0.0;
      }
}

void or_cmul(const double *a, const double *b, double *out, int64_t n) {
  for (int64_t q = 0; q < n; q++) {
    double r, i;
    cmul(a[2 * q], a[2 * q + 1], b[2 * q], b[2 * q + 1], &r, &i);
    out[2 * q] = r;
    out[2 * q + 1] = i;
  }
}

/*
 * CPU oracle for the Gross-Pitaevskii time-stepper: a plain-C, FP64
 * restatement of the reference Fortran (anthonyyoud/gpe, src/) for one
 * process (nyprocs = nzprocs = 1).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * checker (or as the timed stand-in for the reference's CPU path).  The
 * product (gpe_b200, libgpe_cuda.so) never links, loads or calls it.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors
 * for this path, and its Fortran cannot be compiled in this image (no
 * gfortran, MPI, 2DECOMP&FFT or FFTW).  Parity of this restatement is
 * therefore UNPINNED by reference artefacts; it is pinned instead by
 * analytic known-answer tests derived from the reference's own formulas
 * (tests/golden/make_golden.py, tests/test_oracle_kat.py).
 *
 * Arrays are complex128 stored as interleaved (re, im) doubles in the
 * reference's column-major order psi(0:nx-1, 0:ny-1, 0:nz-1), i.e. C order
 * [k][j][i][2].
 */
#ifndef GPE_ORACLE_H
#define GPE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;
  double xr, yr, zr;
  int scheme;     /* 0 euler, 1 rk2, 2 rk4, 3 rk45   (parameters.f90:28) */
  int eqn;        /* eqn_to_solve 1..4               (solve.f90:414)   */
  int bcs;        /* 1 periodic, 2 reflective        (derivs.f90:285)  */
  int order;      /* 2 or 4                          (derivs.f90:35)   */
  int real_time;  /* dt = tau or -i tau              (gpe.f90:78-82)   */
  double tau;
  double Urhs, diss_amp, scal, g, mu, nn, omx, omy, omz;
  double gamma;   /* damped-GPE extension of eqn 4 (0 = reference eqn 4) */
} or_params;

typedef struct {
  double t, im_t, dt_re, dt_im;
  int64_t p;
  double errmax;  /* last accepted RKF45 error norm */
  int64_t rejected;
} or_clock;

typedef struct or_ctx or_ctx;

or_ctx *or_create(const or_params *prm);
void or_destroy(or_ctx *c);
void or_set_threads(int n);
int or_get_threads(void);
/* rebuild diss/Vtrap/sphere on every RHS call as the reference does
 * (same values; only the CPU cost differs) */
void or_set_faithful_cost(or_ctx *c, int on);

/* ic.f90:32-69 get_grid */
void or_get_grid(const or_ctx *c, double *x, double *y, double *z, double *dxyz);

/* derivs.f90 + variables.f90:55-71 on an interior array (halos filled from
 * the boundary conditions like the reference's halo exchange) */
void or_laplacian(or_ctx *c, const double *psi, double *out);
void or_deriv_x(or_ctx *c, const double *psi, double *out);
/* solve.f90:382-440 get_rhs */
void or_get_rhs(or_ctx *c, const double *psi, double *rhs);

/* solve.f90:25-53 solver() + its time update; psi updated in place.
 * For rk45 the clock's dt is updated as rkqs does. */
void or_solver(or_ctx *c, double *psi, or_clock *clk);
/* n calls of or_solver */
void or_run(or_ctx *c, double *psi, or_clock *clk, int64_t nsteps);

/* variables.f90:554-576, 580-604, 715-726 */
double or_get_norm(or_ctx *c, const double *psi);
double or_energy(or_ctx *c, const double *psi);
void or_renormalise(or_ctx *c, double *psi, double norm);

/* ic.f90 initial conditions (interior arrays) */
typedef struct {
  char plane[3];
  double x0, y0, z0, r0, amp;
  int mm;
  double r1;
  int kk;
  double dir;
} or_ring;
typedef struct {
  double x0, y0, z0, amp1, amp2, ll, sgn;
  char dir;
  int imprint_phase;
} or_line;
void or_get_rr(const double *r, double *rr, int64_t n);
int or_vortex_ring(or_ctx *c, const or_ring *vr, double *out);
int or_vortex_line(or_ctx *c, const or_line *vl, double *out);
void or_fermi(or_ctx *c, double *out);
void or_vtrap(or_ctx *c, double *out);
/* straight vortex line with the Pade core R(r) = r*get_rr(r) */
int or_vortex_line_pade(or_ctx *c, const or_line *vl, double *out);
/* ic.f90:518-587 pade_pulse_ring: pulse != 0 for 'pulse', 0 for 'ring' */
int or_pade_pulse_ring(or_ctx *c, int pulse, double x0, double y0, double z0, double r0, double *out);
/* ic.f90:591-636 vortex_pair; 640-662 sphere; 666-684 sphere2; 688-709 wall */
void or_vortex_pair(or_ctx *c, double *out);
void or_sphere(or_ctx *c, double *out);
void or_sphere2(or_ctx *c, double *out);
void or_wall(or_ctx *c, double *out);
/* complex product a*b elementwise into out (ic.in products) */
void or_cmul(const double *a, const double *b, double *out, int64_t n);

#ifdef __cplusplus
}
#endif
#endif

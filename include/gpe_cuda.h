/*
 * gpe_cuda.h -- C ABI of the B200 (sm_100a) Gross-Pitaevskii time-stepper.
 *
 * This is the drop-in boundary for the reference's (anthonyyoud/gpe) time
 * stepping path.  In the reference the path is reached through Fortran module
 * procedures that read module globals (src/parameters.f90:24-129); here the
 * same quantities travel in a POD struct and the state lives on the GPU
 * inside an opaque handle.  Every entry point below names the reference
 * interface it replaces.
 *
 * Conventions
 *   - Return 0 (GPE_OK) on success, a negative GPE_ERR_* on failure.  The
 *     reference has no return codes: a host maps any non-zero value onto its
 *     emergency_stop(gpe_last_error(h)) (src/error.f90:24-46), which keeps the
 *     ERROR / RUNNING file semantics unchanged.
 *   - Host arrays are the reference's interior arrays psi(0:nx-1,0:ny-1,
 *     0:nz-1), Fortran column-major (x fastest), complex (re, im) pairs:
 *     GPE_C128 = complex(8) / double[2], GPE_C64 = complex(4) / float[2].
 *   - A handle is not thread-safe; use one host thread per handle.  Distinct
 *     handles are independent and each owns its own CUDA stream.
 *   - There is no CPU fallback: without a usable sm_100 GPU, gpe_create
 *     fails with GPE_ERR_CUDA.
 */
#ifndef GPE_CUDA_H
#define GPE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPE_OK 0
#define GPE_ERR_BADARG (-1)
#define GPE_ERR_CUDA (-2)
#define GPE_ERR_NONFINITE (-3)
#define GPE_ERR_TIMEOUT (-4)
#define GPE_ERR_NOMEM (-5)
#define GPE_ERR_NOMEM_BUDGET (-6)
#define GPE_ERR_STATE (-7)

/* time-stepping schemes (src/solve.f90:34-50, run.in `scheme`) */
#define GPE_EULER 0
#define GPE_RK2 1
#define GPE_RK4 2
#define GPE_RK45 3

/* element types of host arrays and of device storage */
#define GPE_C128 0
#define GPE_C64 1

/* Compute type used by the stencil when storage is GPE_C64 */
#define GPE_COMPUTE_AUTO 0
#define GPE_COMPUTE_F32 1
#define GPE_COMPUTE_F64 2

/*
 * Run parameters.  Field meanings follow the reference's namelists
 * (src/parameters.f90:40-87) and compile-time grid (src/parameters.in:22-30).
 * The grid is node-inclusive and symmetric, x_i = -xr + i*2xr/(nx-1)
 * (src/ic.f90:32-69).
 */
typedef struct {
  int32_t nx, ny, nz;      /* grid points per axis (>= 6)                     */
  int32_t scheme;          /* GPE_EULER | GPE_RK2 | GPE_RK4 | GPE_RK45        */
  int32_t eqn;             /* eqn_to_solve 1..4 (src/solve.f90:414-437)       */
  int32_t bcs;             /* 1 periodic, 2 reflective                        */
  int32_t order;           /* 2 or 4                                          */
  int32_t real_time;       /* 1: dt = tau, 0: dt = -i tau (src/gpe.f90:78-82) */
  int32_t storage;         /* GPE_C128 | GPE_C64 device storage of psi/stages */
  int32_t compute;         /* GPE_COMPUTE_* (GPE_C64 storage only)            */
  int32_t tile_zc;         /* z planes per CTA work item; 0 = library default  */
                           /* (single solve: enough items to fill the GPU;    */
                           /*  pooled solve: 16 up to nz = 48, else 32)       */
  int32_t reserved;        /* must be 0                                        */
  double xr, yr, zr;       /* half box lengths                                 */
  double tau;              /* |dt| (run.in tau)                                */
  double Urhs, diss_amp, scal, g, mu, nn, omx, omy, omz;
  double gamma;            /* damped eqn 4: rhs = -(i+gamma)(...); 0 = eqn 4  */
  double eps, safety, dt_decrease, dt_increase; /* RKF45 control; 0 selects the
                              reference constants 1e-6, 0.9, -0.25, -0.2
                              (src/parameters.f90:90-93)                      */
} gpe_params;

/*
 * In/out record of gpe_step.  t, im_t, dt and p are the reference's globals
 * (src/parameters.f90:117-129) and are advanced exactly as solver() does.
 */
typedef struct {
  double t, im_t;          /* in/out                                           */
  double dt_re, dt_im;     /* in/out; RKF45 returns the next trial step        */
  int64_t p;               /* in/out step index                                */
  int64_t accepted;        /* out: steps taken in this call                    */
  int64_t rejected;        /* out: RKF45 rejected attempts in this call        */
  double errmax;           /* out: last accepted RKF45 error norm              */
  double norm;             /* out: get_norm of the final state (want_norm)     */
  double energy;           /* out: energy of the state entering the call       */
  int32_t want_norm;       /* in                                               */
  int32_t want_energy;     /* in                                               */
} gpe_step_info;

typedef struct gpe_handle gpe_handle;

/* Replaces the set-up of src/gpe.f90:59-88 (allocate psi%old/psi%new, dt,
 * get_grid).  Allocates all device state for one solve. */
int gpe_create(const gpe_params* p, gpe_handle** out);

/* Frees the handle's device memory and stream (src/gpe.f90:296-304). */
void gpe_destroy(gpe_handle* h);

/* Message for the last failure on this handle (h may be NULL: the last
 * failure of gpe_create on this thread).  Feeds emergency_stop. */
const char* gpe_last_error(const gpe_handle* h);

/* Copy the host interior array in / out (replaces psi%new assignment from
 * ics(), src/gpe.f90:107, and the reads of psi%new by io.f90's writers).
 * dtype is GPE_C128 or GPE_C64; synchronous. */
int gpe_set_state(gpe_handle* h, const void* psi, int32_t dtype);
int gpe_get_state(gpe_handle* h, void* psi, int32_t dtype);

/* Same as above with a device pointer to a contiguous interior array. */
int gpe_set_state_device(gpe_handle* h, const void* psi_dev, int32_t dtype);
int gpe_get_state_device(gpe_handle* h, void* psi_dev, int32_t dtype);

/* nsteps x (solver(psi%old, psi%new) + its time update), src/solve.f90:25-53
 * called from src/gpe.f90:230, including the halo exchange of
 * src/gpe.f90:173-176 (replaced by in-kernel boundary conditions).
 * RKF45 follows rkqs (src/solve.f90:158-244) including its quirks.
 * Returns after the device work completes. */
int gpe_step(gpe_handle* h, int64_t nsteps, gpe_step_info* io);

/* Enqueue nsteps fixed-step steps (Euler/RK2/RK4) on the handle's stream
 * without waiting; io's clock is advanced on return.  gpe_sync waits. */
int gpe_step_async(gpe_handle* h, int64_t nsteps, gpe_step_info* io);
int gpe_sync(gpe_handle* h);

/* Asynchronous forms of gpe_set_state / gpe_get_state for a pipeline of
 * solves: the host<->device transfer runs on the handle's copy stream
 * through device staging buffers, ordered with the handle's stream by
 * events, so the transfers of one solve overlap the steps of the next.
 * Both return at once.  psi must be page-locked (gpe_host_alloc) and must
 * not be touched until gpe_sync returns.  gpe_wait_copies orders the
 * handle's stream after every transfer issued so far (no host wait), e.g.
 * before recording a timing event; gpe_sync waits for the transfers too. */
int gpe_set_state_async(gpe_handle* h, const void* psi, int32_t dtype);
int gpe_get_state_async(gpe_handle* h, void* psi, int32_t dtype);
int gpe_wait_copies(gpe_handle* h);

/* get_norm (src/variables.f90:554-576) of the current state. */
int gpe_norm(gpe_handle* h, double* norm);
/* energy (src/variables.f90:580-604), un-normalised: io.f90:202 divides the
 * value by nx*ny*nz before writing energy.dat. */
int gpe_energy(gpe_handle* h, double* energy);
/* renormalise (src/variables.f90:715-726): psi = sqrt(nn)*psi/sqrt(norm). */
int gpe_renormalise(gpe_handle* h, double norm);

/* get_grid results (src/ic.f90:32-69): x[nx], y[ny], z[nz], dxyz[3];
 * any pointer may be NULL. */
int gpe_get_grid(const gpe_handle* h, double* x, double* y, double* z, double* dxyz);

/* The CUDA stream (cudaStream_t) all of the handle's work runs on. */
int gpe_get_stream(const gpe_handle* h, void** stream);

/*
 * Initial conditions generated on the device (replaces the host-side
 * ics()/ic.in evaluation, src/ic.f90:84-113, for the products ic.in can
 * express).  The state is the product of up to four factors, each one of:
 */
#define GPE_IC_UNIFORM 0      /* 1                                                 */
#define GPE_IC_FERMI 1        /* fermi(): sqrt(max(mu - V, 0)/g), src/ic.f90:278  */
#define GPE_IC_LINE 2         /* vortex_line(vl), core 1-exp(-0.7 r^1.15), :332   */
#define GPE_IC_RING 3         /* vortex_ring(vr), Pade core, src/ic.f90:357       */
#define GPE_IC_LINE_PADE 4    /* straight line with the Pade core r*get_rr(r)     */
#define GPE_IC_RANDOM_PHASE 5 /* seeded spectrum |k| < kc, inverse FFT, mean
                                 density 1 (must be the only factor)               */
#define GPE_IC_PADE_PULSE 6   /* pade_pulse_ring('pulse', x0, y0, z0, r0): Pade
                                 rarefaction pulse moving along x, ic.f90:518      */
#define GPE_IC_PADE_RING 7    /* pade_pulse_ring('ring', x0, y0, z0, r0): Pade
                                 axisymmetric vortex ring moving along x, :518     */
#define GPE_IC_VORTEX_PAIR 8  /* vortex_pair(): Pade vortex pair in x-y, :591     */
#define GPE_IC_SPHERE 9       /* sphere(): 0.5(1 + tanh(r - 12)), :640            */
#define GPE_IC_SPHERE2 10     /* sphere2(): 100 exp(-r^2/10), :666                */
#define GPE_IC_WALL 11        /* wall(): 0 for z <= -30, else 1, :688             */

typedef struct {              /* ring_param, src/parameters.in:54-68 */
  double x0, y0, z0, r0, amp, r1, dir;
  int32_t mm, kk;
  char plane[4];              /* "xy", "xz" or "yz" */
  int32_t reserved;
} gpe_ring;

typedef struct {              /* line_param, src/parameters.in:32-43 */
  double x0, y0, z0, amp1, amp2, ll, sgn;
  int32_t imprint_phase;
  char dir;                   /* 'x', 'y' or 'z' */
  char reserved[3];
} gpe_line;

typedef struct {              /* arguments of pade_pulse_ring, src/ic.f90:518-524 */
  double x0, y0, z0;          /* centre; the axis of symmetry is the x line through (y0, z0) */
  double r0;                  /* ring radius (distance of the core from the axis) */
} gpe_pulse;

typedef struct {
  int32_t nfactors;           /* 1..4 */
  int32_t factor[4];          /* GPE_IC_* */
  int32_t reserved;
  gpe_ring ring;
  gpe_line line;
  uint64_t seed;              /* GPE_IC_RANDOM_PHASE */
  double kc;                  /* GPE_IC_RANDOM_PHASE cutoff |k| < kc */
  gpe_pulse pulse;            /* GPE_IC_PADE_PULSE / GPE_IC_PADE_RING (one set per product) */
} gpe_ic;

/* Set the handle's state to the initial condition (no host array). */
int gpe_set_ic(gpe_handle* h, const gpe_ic* ic);

/* Multiply the current state by an initial-condition product, on the device
 * in FP64 per site: modulus = 0 gives psi <- psi * IC, the restart product
 * with ic.in of state_restart (src/ic.f90:160-162, multiply_ic_restart);
 * modulus = 1 gives psi <- |psi| * IC, imprint_vortex_line
 * (src/variables.f90:1166-1180, imprint_vl, applied at src/gpe.f90:272).
 * Closed-form factors only (a random-phase factor is GPE_ERR_BADARG). */
int gpe_multiply_ic(gpe_handle* h, const gpe_ic* ic, int32_t modulus);

/* FFT diagnostics of the current state, computed on the device in FP64
 * (cuFFT), with the reference's transform a = DFT(psi)/sqrt(nx ny nz)
 * (src/ic.f90:910-939).
 *
 * gpe_condensed replaces condensed_particles (src/io.f90:304-395): the
 * record of mass.dat plus, when eta/nharm/F are non-NULL, the spectra of
 * spectrum (src/io.f90:668-714): the mean occupation eta[m] of the 7 shells
 * m-1 <= |log2(|k|/2pi)| < m (already divided by the shell's site count
 * nharm[m], as written to spectrum/spectrum<p>.dat) and the integral
 * distribution F[kk-1] = sum over 0 < |k| <= kk of |a|^2, kk = 1..nF, with
 * nF = nx/2 (idf/idf<p>.dat).  |k| is the integer index distance of the
 * reference.  Sums are deterministic (fixed order on the device). */
typedef struct {
  double M;        /* mass: sum |psi|^2 dx dy dz (src/variables.f90:608-628)   */
  double n0;       /* |a(0,0,0)|^2                                             */
  double rho0;     /* n0 / (nx ny nz)                                          */
  double tot;      /* sum (k2 + rho0)/(k2^2 + 2 rho0 k2) (src/io.f90:343-360)  */
  double temp;     /* (M - n0)/tot                                             */
  double temp2;    /* (M/(8 xr yr zr) - n0/V)/tot                              */
  double H;        /* E0 + temp (V - 1), E0 = (M^2 + (M - n0)^2)/(2V)          */
  double mass_density; /* M/(8 xr yr zr), column 3 of mass.dat                */
} gpe_condensed_info;

#define GPE_SPECTRUM_SHELLS 7

int gpe_condensed(gpe_handle* h, gpe_condensed_info* info, double* eta, int32_t* nharm, double* F, int32_t nF);

/* filtered_surface (src/io.f90:524-571): the state low-passed in spectral
 * space, a -> a max(1 - m k2 / filter_kc^2, 0), transformed back; written to
 * the host buffer out (nx*ny*nz complex, x fastest, dtype GPE_C128 or
 * GPE_C64).  m = 1 for the reference's periodic saves, fscale * ind in
 * post-processing (src/io.f90:540-544). */
int gpe_filtered(gpe_handle* h, double m, double filter_kc, void* out, int32_t dtype);

/* ---------------------------------------------------------------------------
 * z-slab decomposition of one solve over several GPUs (the reference's MPI
 * domain decomposition, src/variables.f90:203-375 + src/mpi.f90, with the z
 * split only).  Slab r of n owns global planes [k0, k0 + nzl) (the first
 * nz % n slabs get one plane more; every slab needs >= 6).  p describes the
 * GLOBAL grid.  After every stage the R boundary planes of the stage output
 * go to the neighbour slabs' ghost planes; norms, energies and the RKF45
 * error norm are reduced over the slabs, so every slab takes the same step
 * control decisions.  gpe_set_state / gpe_get_state / gpe_get_site work on
 * the handle's own slab (nx * ny * nzl, local k); every slab of a solve must
 * make the same calls in the same order (set_state, step, norm, energy).
 *
 * Transports (exactly one of nccl_id / hub):
 *   nccl_id: one process (rank) per GPU.  Rank 0 calls gpe_slab_nccl_id and
 *            sends the 128 bytes to the others (MPI_Bcast, a file, a
 *            torch.distributed store); the exchange is ncclSend/ncclRecv on
 *            the handle's stream.  NCCL is loaded at run time.
 *   hub:     the n slabs live in one process on one device, each handle
 *            driven by its own host thread; they share the hub's stream.
 *            gpe_destroy of a hub slab is collective too (all slabs of the
 *            hub call it), and the hub outlives its slabs.
 * gpe_set_ic and the FFT diagnostics are not available on slab handles. */
typedef struct gpe_slab_hub gpe_slab_hub;

int gpe_slab_nccl_id(void* id128);
int gpe_slab_hub_create(int32_t nslabs, gpe_slab_hub** out);
void gpe_slab_hub_destroy(gpe_slab_hub* hub);
int gpe_create_slab(const gpe_params* p, int32_t rank, int32_t nranks, const void* nccl_id, gpe_slab_hub* hub,
                    gpe_handle** out);
int gpe_slab_extent(const gpe_handle* h, int32_t* k0, int32_t* nzl);
int gpe_slab_partition(int32_t nz, int32_t nranks, int32_t rank, int32_t* k0, int32_t* nzl);

/* Asynchronous snapshots for checkpoint writers (end_state, dens, filtered
 * files: src/io.f90:480-520, 831-882).  gpe_snapshot_begin copies the
 * current state (interior, dtype) on the device, in stream order, and
 * streams it to a pinned host buffer owned by the handle on a separate
 * stream; it returns at once and stepping may continue.  gpe_snapshot_wait
 * blocks until the copy has landed and returns the buffer (nx*ny*nz
 * complex, x fastest), valid until the next gpe_snapshot_begin.  It touches
 * no other handle state, so a writer thread may call it while another
 * thread steps the handle; gpe_snapshot_begin itself belongs to the
 * stepping thread.  No reference counterpart: the reference writes from the
 * live array and stalls the time loop meanwhile. */
int gpe_snapshot_begin(gpe_handle* h, int32_t dtype);
int gpe_snapshot_wait(gpe_handle* h, const void** host_data, size_t* bytes);

/* One site of the current state, (re, im) in FP64: the probe of save_time
 * (src/io.f90:136-184, psi at (nx/2, ny/2, nz/2) into psi_time.dat). */
int gpe_get_site(gpe_handle* h, int32_t i, int32_t j, int32_t k, double* re_im);

/* Stage-kernel kinds reported by gpe_profile_get (one fused kernel each). */
#define GPE_KIND_EULER 0
#define GPE_KIND_RK2_1 1
#define GPE_KIND_RK2_2 2
#define GPE_KIND_RK4_1 3
#define GPE_KIND_RK4_2 4
#define GPE_KIND_RK4_4 5
#define GPE_KIND_CK_1 6
#define GPE_KIND_CK_6 11
#define GPE_KIND_ENERGY 12
#define GPE_KIND_RK4_3 13
#define GPE_NUM_KINDS 14

/* Instrumentation (no reference counterpart; the reference has no tracing
 * beyond timestep.dat, src/solve.f90:234-241): with enable = 1, every stage
 * kernel launch is bracketed by CUDA events on the handle's stream and its
 * device time accumulated per kind; enable resets the totals. */
int gpe_profile(gpe_handle* h, int32_t enable);
/* Total device ms and launch count of one kind since gpe_profile(h, 1), and
 * the kind's algorithmic HBM bytes per grid site per launch (one read of
 * each input field, one write of each output field). */
int gpe_profile_get(gpe_handle* h, int32_t kind, double* total_ms, int64_t* launches, double* bytes_per_site);

/* Testing aid for the timeout path (the reference's counterpart is the
 * emergency_stop convention of src/error.f90:24-46 that a host applies to
 * GPE_ERR_TIMEOUT).  Arms the handle's device status word so that every
 * stage-kernel work item queued after this call first waits, with a short
 * limit, on a shared-memory barrier that nothing arrives at: the wait
 * expires, the CTA lets the copies it has issued land (bounded wait) and
 * returns without storing anything.  The next gpe_step / gpe_sync that reads
 * the word returns GPE_ERR_TIMEOUT and clears it; the handle stays usable.
 * After any GPE_ERR_TIMEOUT the state is unspecified: set it again. */
int gpe_test_expire_waits(gpe_handle* h);

/*
 * Batched solves and serving (no reference counterpart: the reference runs
 * exactly one solve per MPI job).  A pool owns one device arena of
 * budget_bytes.  gpe_pool_submit admits a solve if its state fits in the
 * free part of the arena (else GPE_ERR_NOMEM_BUDGET: retry after results
 * have been polled); the solve joins the running batch at the next
 * gpe_pool_step.  gpe_pool_step advances every active solve by up to
 * max_steps steps with one persistent launch per Runge-Kutta stage per
 * (precision, scheme) class over all their tiles, then retires the solves
 * that reached their step count: the final state is copied to the caller's
 * psi_out buffer (same element type as the solve's storage) and a
 * gpe_result is queued for gpe_pool_poll.  Supported schemes: RK4 and RK45.
 * Each solve evolves exactly as it would alone (same arithmetic per site,
 * per-solve reductions in a fixed order).
 */
typedef struct gpe_pool gpe_pool;

typedef struct {
  uint64_t tag;
  int32_t status;          /* GPE_OK or the error that stopped this solve      */
  int32_t reserved;
  int64_t steps, rejected; /* accepted steps; RKF45 rejected attempts          */
  double t, im_t, dt_re, dt_im;
  double norm;             /* get_norm of the final state                       */
  double submit_s, start_s, finish_s; /* host seconds since gpe_pool_create   */
} gpe_result;

int gpe_pool_create(int64_t budget_bytes, gpe_pool** out);
int gpe_pool_submit(gpe_pool* pool, const gpe_params* p, const void* psi0, int32_t dtype, int64_t nsteps,
                    uint64_t tag, void* psi_out);
/* Same, with the initial state generated on the device from an IC spec. */
int gpe_pool_submit_ic(gpe_pool* pool, const gpe_params* p, const gpe_ic* ic, int64_t nsteps, uint64_t tag,
                       void* psi_out);
int gpe_pool_step(gpe_pool* pool, int64_t max_steps, int32_t* n_active);
int gpe_pool_poll(gpe_pool* pool, gpe_result* out, int32_t max, int32_t* n_out);
int64_t gpe_pool_free_bytes(const gpe_pool* pool);
/* Arena bytes one solve with these parameters needs (state + tables). */
int64_t gpe_pool_solve_bytes(const gpe_params* p);
const char* gpe_pool_last_error(const gpe_pool* pool);
/* The pool's form of gpe_test_expire_waits: the next gpe_pool_step returns
 * GPE_ERR_TIMEOUT, and the solves it was advancing are retired with status
 * GPE_ERR_TIMEOUT in their results (what a genuine expiry does too); solves
 * submitted afterwards run normally. */
int gpe_pool_test_expire_waits(gpe_pool* pool);

/* Page-locked host memory (cudaMallocHost) for the psi0 / out buffers of
 * gpe_pool_submit and the host arrays of gpe_set_state / gpe_get_state:
 * copies to and from it run at DMA speed and asynchronously, where pageable
 * memory is staged by the driver.  NULL on failure. */
void* gpe_host_alloc(size_t bytes);
void gpe_host_free(void* p);
void gpe_pool_destroy(gpe_pool* pool);

/* Bytes of device memory a solve with these parameters allocates. */
int64_t gpe_state_bytes(const gpe_params* p);

/*
 * gpe_norm_noalloc -- no counterpart in the reference.  The same weighted
 * integral as gpe_norm (extended closed quadrature times dx*dy*dz), for a
 * caller-owned device array, without allocating any device memory.
 *
 * For callers that cannot let a library allocate on the GPU: hosts whose
 * device memory is owned by another allocator (a framework's caching pool,
 * a runtime that maps its own buffers) and must not see foreign
 * cudaMalloc/cudaFree traffic; loops that must not stall or fail on an
 * allocation between steps; embedders that fix their device-memory budget
 * up front.  The caller passes the input (contiguous interior psi in the
 * reference's order, complex128 or complex64 by dtype) and the output (one
 * double in device memory); the work is queued on `stream` (NULL = the
 * legacy default stream) and the call does not wait for it.
 *
 * Scratch: one partial sum per z-plane in a fixed array inside the library
 * (GPE_NOALLOC_MAX_NZ doubles, 64 KiB), resident on every GPU that loads the
 * library until the process exits.  nz > GPE_NOALLOC_MAX_NZ (or nx, ny,
 * nz < 6, a bad dtype, a NULL pointer) returns GPE_ERR_BADARG and prints the
 * reason on stderr, and so does a psi_dev that is not aligned to its element
 * (16 bytes for complex128, 8 for complex64) or a norm_dev that is not
 * 8-byte aligned; nothing is launched then.  The first call on a device
 * looks up the array's device address and loads the kernels of both dtypes
 * there; make it before any stream capture.  A device reset after that
 * first call is not supported.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.
 */
#define GPE_NOALLOC_MAX_NZ 8192
int gpe_norm_noalloc(const void* psi_dev, int32_t dtype, int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                     double dz, double* norm_dev, void* stream);

/* Library build/version string. */
const char* gpe_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GPE_CUDA_H */

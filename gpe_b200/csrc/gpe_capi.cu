// C ABI of the B200 Gross-Pitaevskii time-stepper (include/gpe_cuda.h).
//
// One handle = one solve (or one z-slab of a decomposed solve): ghost-padded
// device fields, per-axis tables, a stream, reduction buffers.  gpe_step()
// enqueues one fused stage kernel per Runge-Kutta stage (steps without
// reductions as a replayed graph of one step); the time bookkeeping follows
// the reference's solver() routines (src/solve.f90:57-244) on the host, in
// FP64.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpe_cuda.h"
#include "gpe_aux.cuh"
#include "gpe_device.cuh"
#include "gpe_stage_tma.cuh"
#include "gpe_common.h"
#include "gpe_fft.h"
#include "gpe_ic.h"
#include "gpe_slab.h"

namespace gpe {
cudaError_t launch_stage_f64(int kind, int R, int ty, dim3 grid, cudaStream_t st, const StageArgs& a);
cudaError_t launch_stage_f32(int kind, int R, int ty, dim3 grid, cudaStream_t st, const StageArgs& a);
cudaError_t launch_stage_f32x(int kind, int R, int ty, dim3 grid, cudaStream_t st, const StageArgs& a);
cudaError_t launch_stage_tma_f64(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                 const StageArgs& a);
cudaError_t launch_stage_tma_f32(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                 const StageArgs& a);
cudaError_t launch_stage_tma_f32x(int kind, int R, int ty, dim3 grid, cudaStream_t st, const TmaMaps& m,
                                  const StageArgs& a);
}  // namespace gpe

using namespace gpe;
using gpe::CK_B;

namespace {

thread_local std::string g_create_err;

enum { CM_F64 = 0, CM_F32 = 1, CM_F32X = 2 };
enum { T_VX, T_VY, T_VZ, T_SX, T_SY, T_SZ, T_WX, T_WY, T_WZ, T_CX, T_CY, T_CZ, T_NUM };

}  // namespace

struct gpe_handle {
  gpe_params p{};
  int dev = 0;
  cudaStream_t st = nullptr;
  Geom g{};
  int R = 2;
  int esz = 16;
  int cmode = CM_F64;
  long long nelem = 0;  // padded elements per field
  std::vector<void*> fields;
  int cur = 0;  // index of the field holding psi
  double* tables = nullptr;
  std::vector<double> x, y, z;
  double dx = 0, dy = 0, dz = 0;
  double* part_a = nullptr;  // block partials (energy / first reduction)
  double* part_b = nullptr;  // block partials (norm / errmax)
  long long npart = 0;       // partials of one stage launch (one per CTA of grid)
  dim3 norm_grid;            // k_norm's grid: 32 x 8 tiles x z-chunks
  long long norm_npart = 0;  // its partials
  double* dres = nullptr;    // [6] finalised reductions
  double* hres = nullptr;    // pinned mirror of dres
  void* staging = nullptr;
  size_t staging_bytes = 0;
  int zc = 8;
  dim3 grid;
  std::string err;
  // optional per-kernel timing (gpe_profile): event pairs around launches
  bool prof = false;
  std::vector<cudaEvent_t> ev;     // pool, 2 per launch
  std::vector<int> ev_kind;        // kind of each pending pair
  size_t ev_used = 0;              // pairs in flight
  double prof_ms[K_NUM] = {0};
  long long prof_n[K_NUM] = {0};
  // kernel variant: true = TMA plane pipeline (k_stage_tma), false = k_stage
  bool use_tma = true;
  int tma_ty = TILE_32x8_ROW2;  // thread layout of the TMA stage kernel (TileVariant)
  std::vector<CUtensorMap> map_halo, map_pw;  // per field
  int* status = nullptr;                      // device status word
  // FFT diagnostics: transform scratch + the reference's k-grid symbols
  void* fft_work = nullptr;
  size_t fft_work_bytes = 0;
  double* fft_kq = nullptr;
  // z-slab decomposition (gpe_create_slab): this handle owns planes
  // [k0, k0 + p.nz) of a grid of nz_global planes and exchanges R boundary
  // planes with slab_down / slab_up (-1 = a global face) after every stage
  int rank = 0, nranks = 1, k0 = 0, nz_global = 0;
  int slab_down = -1, slab_up = -1;
  bool slab = false;
  int zghost = 3;          // z ghosts the stage kernels write (StageArgs::zghost)
  void* nccl = nullptr;    // ncclComm_t of the NCCL transport
  gpe::SlabHub* hub = nullptr;
  bool own_stream = true;
  std::string xerr;        // detail of a failed exchange, appended to the next error
  // asynchronous snapshots (gpe_snapshot_begin/wait): a device copy of the
  // interior streamed to pinned host memory on its own stream
  void* snap_dev = nullptr;
  void* snap_host = nullptr;
  size_t snap_cap = 0, snap_bytes = 0;
  cudaStream_t snap_st = nullptr;
  cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
  bool snap_pending = false;
  // one captured RK4/RK2 step without reductions, replayed by gpe_step
  // (the stage arguments, dt included, are baked into the graph)
  cudaGraphExec_t step_graph = nullptr;
  double graph_dr = 0, graph_di = 0;
  // asynchronous state copies (gpe_set_state_async / gpe_get_state_async):
  // host <-> staging transfers on a copy stream, pack/unpack on the solve's
  // stream, ordered by events so transfers overlap the steps around them
  cudaStream_t cp_st = nullptr;   // host -> device transfers
  cudaStream_t cp2_st = nullptr;  // device -> host transfers (a stream each, so neither queues behind the other)
  void *in_stage = nullptr, *out_stage = nullptr;
  size_t in_cap = 0, out_cap = 0;
  cudaEvent_t ev_packed = nullptr, ev_in = nullptr, ev_unpacked = nullptr, ev_out = nullptr;
  bool copies_pending = false;
};

struct gpe_slab_hub {
  gpe::SlabHub hub;
};

namespace {

int fail(gpe_handle* h, int code, const std::string& msg) {
  if (h) {
    h->err = msg;
    if (!h->xerr.empty()) {
      h->err += " (" + h->xerr + ")";
      h->xerr.clear();
    }
  } else {
    g_create_err = msg;
  }
  return code;
}



#define CU(h, call)                                                                        \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail((h), GPE_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                         " at " #call);                                    \
  } while (0)

int validate(const gpe_params* p, std::string& why) { return validate_params(p, why); }
void layout(const gpe_params* p, Geom& g, int& esz) { param_layout(p, g, esz); }
int nfields(int scheme) { return scheme_fields(scheme); }
int choose_zc(const Geom& g, int tile_h, int esz) { return default_zc(g, tile_h, esz); }
bool encode_field_maps(gpe_handle* h, void* base, CUtensorMap* halo, CUtensorMap* pw) {
  return encode_maps(base, h->g, h->esz, h->R, halo, pw, tile_rows(h->tma_ty));
}

int field_of(const gpe_handle* h, const void* p) {
  for (size_t f = 0; f < h->fields.size(); ++f)
    if (h->fields[f] == p) return (int)f;
  return -1;
}

cudaError_t launch_raw(gpe_handle* h, int kind, const StageArgs& a_in) {
  StageArgs a = a_in;
  a.status = h->status;
  set_f32_constants(a);
  if (!h->use_tma) {
    switch (h->cmode) {
      case CM_F64: return launch_stage_f64(kind, h->R, 8, h->grid, h->st, a);
      case CM_F32: return launch_stage_f32(kind, h->R, 8, h->grid, h->st, a);
      default: return launch_stage_f32x(kind, h->R, 8, h->grid, h->st, a);
    }
  }
  TmaMaps m;
  memset(&m, 0, sizeof(m));
  const int fin = field_of(h, a.in);
  if (fin < 0) return cudaErrorInvalidValue;
  m.in = h->map_halo[fin];
  // point-wise inputs in the order of StageTraits: psi, acc, K...
  const bool has_psi = (kind == K_RK2_2 || kind == K_RK4_2 || kind == K_RK4_3 || (kind >= K_CK_2 && kind <= K_CK_6));
  const bool has_acc = (kind == K_RK4_4);
  const int nk = (kind >= K_CK_2 && kind <= K_CK_5) ? (kind - K_CK_1) : (kind == K_CK_6 ? 4 : 0);
  int q = 0;
  const void* pws[7];
  if (has_psi) pws[q++] = a.psi;
  if (has_acc) pws[q++] = a.acc;
  for (int t = 0; t < nk; ++t) pws[q++] = a.kin[t];
  for (int t = 0; t < q; ++t) {
    const int f = field_of(h, pws[t]);
    if (f < 0) return cudaErrorInvalidValue;
    m.pw[t] = h->map_pw[f];
  }
  switch (h->cmode) {
    case CM_F64: return launch_stage_tma_f64(kind, h->R, h->tma_ty, h->grid, h->st, m, a);
    case CM_F32: return launch_stage_tma_f32(kind, h->R, h->tma_ty, h->grid, h->st, m, a);
    default: return launch_stage_tma_f32x(kind, h->R, h->tma_ty, h->grid, h->st, m, a);
  }
}

// Halo exchange of field f of a z-slab handle: the R planes next to each
// face go to the neighbour slab's ghost planes (the role of send_recv_z,
// src/variables.f90:203-256).  Planes are contiguous (pz elements each).
cudaError_t slab_exchange(gpe_handle* h, int f) {
  if (!h->slab || f < 0) return cudaSuccess;
  const size_t plane = (size_t)h->g.pz * h->esz;
  const int R = h->R, nzl = h->p.nz;
  const size_t bytes = (size_t)R * plane;
  char* base = (char*)h->fields[f];
  char* lo_send = base + 2 * plane;                    // k = 0 .. R-1
  char* hi_send = base + (size_t)(nzl + 2 - R) * plane;  // k = nzl-R .. nzl-1
  char* lo_recv = base + (size_t)(2 - R) * plane;      // k = -R .. -1
  char* hi_recv = base + (size_t)(nzl + 2) * plane;    // k = nzl .. nzl+R-1
  if (h->nccl) {
    // sends to down/up, then receives from up/down: with down == up (two
    // ranks, or one rank on a periodic axis) the pairs match in this order
    const NcclXfer xs[4] = {{h->slab_down, lo_send, nullptr, bytes},
                            {h->slab_up, hi_send, nullptr, bytes},
                            {h->slab_up, nullptr, hi_recv, bytes},
                            {h->slab_down, nullptr, lo_recv, bytes}};
    if (nccl_exchange(h->nccl, xs, 4, h->st, h->xerr) != 0) return cudaErrorUnknown;
    return cudaSuccess;
  }
  SlabHub* hub = h->hub;
  if (!hub->barrier(hub->timeout_s)) {
    h->xerr = "a z-slab of the hub stopped calling in (barrier timeout)";
    return cudaErrorTimeout;
  }
  if (h->slab_up >= 0) {
    const gpe_handle* u = hub->slabs[h->slab_up];
    cudaError_t e = cudaMemcpyAsync(hi_recv, (const char*)u->fields[f] + 2 * plane, bytes,
                                    cudaMemcpyDeviceToDevice, h->st);
    if (e != cudaSuccess) return e;
  }
  if (h->slab_down >= 0) {
    const gpe_handle* d = hub->slabs[h->slab_down];
    cudaError_t e = cudaMemcpyAsync(lo_recv, (const char*)d->fields[f] + (size_t)(d->p.nz + 2 - R) * plane, bytes,
                                    cudaMemcpyDeviceToDevice, h->st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_prof(gpe_handle* h, int kind, const StageArgs& a);

// A stage launch; on a z-slab handle its output's boundary planes are
// exchanged before anything reads them.
cudaError_t launch(gpe_handle* h, int kind, const StageArgs& a) {
  cudaError_t e = launch_prof(h, kind, a);
  if (e != cudaSuccess || !h->slab || !a.out) return e;
  return slab_exchange(h, field_of(h, a.out));
}

cudaError_t launch_prof(gpe_handle* h, int kind, const StageArgs& a) {
  if (!h->prof) return launch_raw(h, kind, a);
  if (2 * (h->ev_used + 1) > h->ev.size()) {
    for (int q = 0; q < 64; ++q) {
      cudaEvent_t e;
      cudaError_t rc = cudaEventCreate(&e);
      if (rc != cudaSuccess) return rc;
      h->ev.push_back(e);
    }
  }
  cudaEvent_t e0 = h->ev[2 * h->ev_used], e1 = h->ev[2 * h->ev_used + 1];
  cudaEventRecord(e0, h->st);
  cudaError_t rc = launch_raw(h, kind, a);
  cudaEventRecord(e1, h->st);
  if (h->ev_kind.size() <= h->ev_used) h->ev_kind.resize(h->ev_used + 1);
  h->ev_kind[h->ev_used] = kind;
  h->ev_used++;
  return rc;
}

// after a stream synchronisation: fold the pending event pairs into totals
void prof_resolve(gpe_handle* h) {
  for (size_t q = 0; q < h->ev_used; ++q) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->ev[2 * q], h->ev[2 * q + 1]) == cudaSuccess) {
      h->prof_ms[h->ev_kind[q]] += ms;
      h->prof_n[h->ev_kind[q]] += 1;
    }
  }
  h->ev_used = 0;
}

// Per-axis tables of the solve.  A z-slab takes its rows of the global
// grid's tables (coordinates, trap, sponge and quadrature weights all belong
// to the global z axis).
void build_tables(gpe_handle* h, std::vector<double>& t) {
  std::vector<double>* xyz[3] = {&h->x, &h->y, &h->z};
  double d[3];
  if (!h->slab) {
    build_axis_tables(h->p, t, xyz, d);
  } else {
    gpe_params pg = h->p;
    pg.nz = h->nz_global;
    std::vector<double> tg, zg;
    std::vector<double>* xyzg[3] = {&h->x, &h->y, &zg};
    build_axis_tables(pg, tg, xyzg, d);
    const size_t ng = (size_t)pg.nx + pg.ny + pg.nz, nl = (size_t)h->p.nx + h->p.ny + h->p.nz;
    const size_t nxy = (size_t)pg.nx + pg.ny;
    t.assign(nl * 4, 0.0);
    for (int b = 0; b < 4; ++b) {
      for (size_t q = 0; q < nxy; ++q) t[b * nl + q] = tg[b * ng + q];
      for (int k = 0; k < h->p.nz; ++k) t[b * nl + nxy + k] = tg[b * ng + nxy + h->k0 + k];
    }
    h->z.assign(zg.begin() + h->k0, zg.begin() + h->k0 + h->p.nz);
  }
  h->dx = d[0];
  h->dy = d[1];
  h->dz = d[2];
}

StageArgs base_args(gpe_handle* h) {
  const double d[3] = {h->dx, h->dy, h->dz};
  StageArgs a = make_base_args(h->p, h->g, h->R, h->zc, d, h->tables);
  a.zghost = h->zghost;
  return a;
}

int finalize_into(gpe_handle* h, const double* part, int slot, long long nparts = -1) {
  k_finalize<<<1, 256, 0, h->st>>>(part, nparts < 0 ? h->npart : nparts, h->dres + 3 * slot);
  CU(h, cudaGetLastError());
  return GPE_OK;
}

// A stage kernel whose bounded mbarrier wait expired leaves a non-zero
// status word; report it as GPE_ERR_TIMEOUT (and clear it).
int check_status(gpe_handle* h) {
  int st = 0;
  CU(h, cudaMemcpy(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    CU(h, cudaMemset(h->status, 0, sizeof(int)));
    return fail(h, GPE_ERR_TIMEOUT, "a stage kernel's bounded wait for its TMA copies expired");
  }
  return GPE_OK;
}

int fetch_results(gpe_handle* h) {
  // z-slabs: norms and energies are sums over the slabs, errmax a maximum
  // (the MPI_ALLREDUCE of src/variables.f90:554-604, src/solve.f90:189-190)
  if (h->nccl && nccl_reduce_results(h->nccl, h->dres, h->st, h->xerr) != 0)
    return fail(h, GPE_ERR_CUDA, "z-slab reduction failed");
  CU(h, cudaMemcpyAsync(h->hres, h->dres, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  if (h->prof) prof_resolve(h);
  if (h->hub && h->hub->n > 1) {
    SlabHub* hub = h->hub;
    for (int q = 0; q < 6; ++q) hub->vals[h->rank][q] = h->hres[q];
    if (!hub->barrier(hub->timeout_s))
      return fail(h, GPE_ERR_TIMEOUT, "a z-slab of the hub stopped calling in (barrier timeout)");
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int r = 0; r < hub->n; ++r)
      for (int q = 0; q < 6; ++q)
        v[q] = (q == 2 || q == 5) ? std::max(v[q], hub->vals[r][q]) : v[q] + hub->vals[r][q];
    if (!hub->barrier(hub->timeout_s))
      return fail(h, GPE_ERR_TIMEOUT, "a z-slab of the hub stopped calling in (barrier timeout)");
    for (int q = 0; q < 6; ++q) h->hres[q] = v[q];
  }
  return check_status(h);
}

double rk_param(double v, double def) { return v != 0.0 ? v : def; }

void default_dt(const gpe_params& p, gpe_step_info* io) {
  if (io->dt_re == 0.0 && io->dt_im == 0.0) {
    if (p.real_time) { io->dt_re = p.tau; io->dt_im = 0.0; }
    else { io->dt_re = 0.0; io->dt_im = -p.tau; }
  }
}

// One fixed-step step (Euler / RK2 / RK4) enqueued on the stream.
int enqueue_fixed_step(gpe_handle* h, double dr, double di, bool energy, bool norm) {
  StageArgs a = base_args(h);
  void** F = h->fields.data();
  const int sc = h->p.scheme;
  if (sc == GPE_RK4) {
    void *psi = F[0], *A = F[1], *B = F[2], *Q = F[3];
    // s1: k1 = f(psi); A = psi + dt/2 k1
    a.in = psi; a.out = A;
    a.cf_r[0] = 0.5 * dr; a.cf_i[0] = 0.5 * di;
    a.want_energy = energy;
    a.partials = energy ? h->part_a : nullptr;
    CU(h, launch(h, K_RK4_1, a));
    if (energy && finalize_into(h, h->part_a, 0)) return GPE_ERR_CUDA;
    a.want_energy = 0;
    a.partials = nullptr;
    // s2: k2 = f(A); B = psi + dt/2 k2; Q = (psi + A) + dt k2
    a.in = A; a.psi = psi; a.out = B; a.acc = Q;
    a.cf_r[0] = 0.5 * dr; a.cf_i[0] = 0.5 * di;
    a.cf_r[1] = dr; a.cf_i[1] = di;
    CU(h, launch(h, K_RK4_2, a));
    // s3: k3 = f(B); A = psi + dt k3
    a.in = B; a.out = A;
    a.cf_r[0] = dr; a.cf_i[0] = di;
    CU(h, launch(h, K_RK4_3, a));
    // s4: k4 = f(A); psi = (Q + A)/3 + dt/6 k4 (psi itself is not read)
    a.in = A; a.psi = nullptr; a.out = psi;
    a.cf_r[0] = dr / 6.0; a.cf_i[0] = di / 6.0;
    a.want_norm = norm;
    a.partials = norm ? h->part_b : nullptr;
    CU(h, launch(h, K_RK4_4, a));
    if (norm && finalize_into(h, h->part_b, 1)) return GPE_ERR_CUDA;
    return GPE_OK;
  }
  if (sc == GPE_RK2) {
    void *psi = F[0], *A = F[1];
    a.in = psi; a.out = A;
    a.cf_r[0] = 0.5 * dr; a.cf_i[0] = 0.5 * di;
    a.want_energy = energy;
    a.partials = energy ? h->part_a : nullptr;
    CU(h, launch(h, K_RK2_1, a));
    if (energy && finalize_into(h, h->part_a, 0)) return GPE_ERR_CUDA;
    a.want_energy = 0;
    a.in = A; a.psi = psi; a.out = psi;
    a.cf_r[0] = dr; a.cf_i[0] = di;
    a.want_norm = norm;
    a.partials = norm ? h->part_b : nullptr;
    CU(h, launch(h, K_RK2_2, a));
    if (norm && finalize_into(h, h->part_b, 1)) return GPE_ERR_CUDA;
    return GPE_OK;
  }
  // Euler: new = old + dt f(old), written into the other buffer
  void *psi = F[h->cur], *nw = F[1 - h->cur];
  a.in = psi; a.out = nw;
  a.cf_r[0] = dr; a.cf_i[0] = di;
  a.want_energy = energy;
  a.want_norm = norm;
  if (energy && !norm) {
    a.partials = h->part_a;
    CU(h, launch(h, K_EULER, a));
    if (finalize_into(h, h->part_a, 0)) return GPE_ERR_CUDA;
  } else {
    a.partials = norm ? h->part_b : nullptr;
    CU(h, launch(h, K_EULER, a));
    if (norm && finalize_into(h, h->part_b, 1)) return GPE_ERR_CUDA;
    // one kernel produced both sums: move the energy into its slot
    if (energy) CU(h, cudaMemcpyAsync(h->dres + 1, h->dres + 4, sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  }
  h->cur = 1 - h->cur;
  return GPE_OK;
}

// RKF45 = rkqs (src/solve.f90:158-244) with Cash-Karp stages (248-378)
int rk45_step(gpe_handle* h, gpe_step_info* io, bool energy, bool norm) {
  const gpe_params& p = h->p;
  const double eps = rk_param(p.eps, 1e-6), safety = rk_param(p.safety, 0.9);
  const double dtdec = rk_param(p.dt_decrease, -0.25), dtinc = rk_param(p.dt_increase, -0.2);
  const double errcon = pow(5.0 / safety, 1.0 / dtinc);
  double dr = io->dt_re, di = io->dt_im;
  const double dte_r = dr, dte_i = di;  // psi_scal uses the dt at entry (solve.f90:178)
  void** F = h->fields.data();
  void* psi = F[h->cur];
  void* pnew = F[1 - h->cur];
  void *A = F[2], *B = F[3];
  void* K[5] = {F[4], F[5], F[6], F[7], F[8]};
  double errmax = 0.0;
  bool first = true;
  for (int attempt = 0;; ++attempt) {
    if (attempt > 10000) return fail(h, GPE_ERR_STATE, "rkqs: no acceptable step after 10000 attempts");
    StageArgs a = base_args(h);
    a.cf_r[0] = dr;
    a.cf_i[0] = di;
    a.psi = psi;
    void* ins[6] = {psi, A, B, A, B, A};
    void* outs[6] = {A, B, A, B, A, pnew};
    for (int m = 0; m < 6; ++m) {
      a.in = ins[m];
      a.out = outs[m];
      for (int q = 0; q < 5; ++q) a.b[q] = 0.0;
      a.kout = m < 5 ? K[m] : nullptr;
      if (m < 5) {
        for (int q = 0; q <= m; ++q) a.b[q] = CK_B[m][q];
        for (int q = 0; q < m; ++q) a.kin[q] = K[q];
      } else {
        a.kin[0] = K[0]; a.kin[1] = K[2]; a.kin[2] = K[3]; a.kin[3] = K[4];
        a.dte_r = dte_r;
        a.dte_i = dte_i;
        a.inv_adt = 1.0 / hypot(dr, di);
        a.want_norm = norm;
      }
      a.want_energy = (m == 0 && energy && first);
      a.partials = (m == 5) ? h->part_b : (a.want_energy ? h->part_a : nullptr);
      CU(h, launch(h, K_CK_1 + m, a));
      if (a.want_energy && finalize_into(h, h->part_a, 0)) return GPE_ERR_CUDA;
    }
    if (finalize_into(h, h->part_b, 1)) return GPE_ERR_CUDA;
    if (int rc = fetch_results(h)) return rc;
    first = false;
    errmax = h->hres[5] / eps;
    if (!std::isfinite(errmax)) return fail(h, GPE_ERR_NONFINITE, "rkqs: non-finite error norm");
    if (errmax <= 1.0) break;
    io->rejected++;
    const double e = pow(errmax, dtdec);
    const double tr = (safety * dr) * e, ti = (safety * di) * e;
    const double m = std::max(hypot(tr, ti), 0.1 * hypot(dr, di));
    // real time <=> dt on the real axis (src/solve.f90:197-201 tests the
    // real_time flag; dt is (tau, 0) exactly when it is set, also after the
    // imaginary-to-real switch of src/gpe.f90:264)
    if (!(di == 0.0)) { dr = 0.0; di = -m; }
    else { dr = m; di = 0.0; }
  }
  double nr, ni;
  if (errmax > errcon) {
    const double e = pow(errmax, dtinc);
    nr = (safety * dr) * e;
    ni = (safety * di) * e;
  } else {
    nr = 5.0 * dr;
    ni = 5.0 * di;
  }
  io->t = io->t + dr;
  io->dt_re = nr;
  io->dt_im = ni;
  io->im_t = io->im_t + fabs(ni);  // the new dt, as src/solve.f90:229
  io->errmax = errmax;
  h->cur = 1 - h->cur;
  return GPE_OK;
}

int norm_now(gpe_handle* h, double* out) {
  const Geom& g = h->g;
  const size_t ntot = (size_t)h->p.nx + h->p.ny + h->p.nz;
  const double* w = h->tables + 2 * ntot;
  if (h->esz == 16)
    k_norm<double2><<<h->norm_grid, dim3(32, 8), 0, h->st>>>((const double2*)h->fields[h->cur], g, h->zc, w,
                                                             w + g.nx, w + g.nx + g.ny, h->part_b);
  else
    k_norm<float2><<<h->norm_grid, dim3(32, 8), 0, h->st>>>((const float2*)h->fields[h->cur], g, h->zc, w,
                                                            w + g.nx, w + g.nx + g.ny, h->part_b);
  CU(h, cudaGetLastError());
  if (int rc = finalize_into(h, h->part_b, 1, h->norm_npart)) return rc;
  if (int rc = fetch_results(h)) return rc;
  *out = ((h->hres[3] * h->dx) * h->dy) * h->dz;
  return GPE_OK;
}

int ensure_staging(gpe_handle* h, size_t bytes) {
  if (h->staging_bytes >= bytes) return GPE_OK;
  if (h->staging) cudaFree(h->staging);
  h->staging = nullptr;
  h->staging_bytes = 0;
  CU(h, cudaMalloc(&h->staging, bytes));
  h->staging_bytes = bytes;
  return GPE_OK;
}

int pack_from_device(gpe_handle* h, const void* src, int dtype) {
  const int nb = 148 * 8;
  void* dst = h->fields[h->cur];
  const int zm = h->zghost;
  if (h->esz == 16) {
    if (dtype == GPE_C128) k_pack<double2, double2><<<nb, 256, 0, h->st>>>((const double2*)src, (double2*)dst, h->g, h->R, h->p.bcs, zm);
    else k_pack<double2, float2><<<nb, 256, 0, h->st>>>((const float2*)src, (double2*)dst, h->g, h->R, h->p.bcs, zm);
  } else {
    if (dtype == GPE_C128) k_pack<float2, double2><<<nb, 256, 0, h->st>>>((const double2*)src, (float2*)dst, h->g, h->R, h->p.bcs, zm);
    else k_pack<float2, float2><<<nb, 256, 0, h->st>>>((const float2*)src, (float2*)dst, h->g, h->R, h->p.bcs, zm);
  }
  CU(h, cudaGetLastError());
  CU(h, slab_exchange(h, h->cur));
  return GPE_OK;
}

int unpack_to_device(gpe_handle* h, void* dst, int dtype) {
  const int nb = 148 * 8;
  const void* src = h->fields[h->cur];
  if (h->esz == 16) {
    if (dtype == GPE_C128) k_unpack<double2, double2><<<nb, 256, 0, h->st>>>((const double2*)src, (double2*)dst, h->g);
    else k_unpack<double2, float2><<<nb, 256, 0, h->st>>>((const double2*)src, (float2*)dst, h->g);
  } else {
    if (dtype == GPE_C128) k_unpack<float2, double2><<<nb, 256, 0, h->st>>>((const float2*)src, (double2*)dst, h->g);
    else k_unpack<float2, float2><<<nb, 256, 0, h->st>>>((const float2*)src, (float2*)dst, h->g);
  }
  CU(h, cudaGetLastError());
  return GPE_OK;
}

size_t interior_bytes(const gpe_handle* h, int dtype) {
  return (size_t)h->p.nx * h->p.ny * h->p.nz * (dtype == GPE_C128 ? 16 : 8);
}

int check_dtype(gpe_handle* h, int dtype) {
  if (dtype != GPE_C128 && dtype != GPE_C64) return fail(h, GPE_ERR_BADARG, "dtype must be GPE_C128 or GPE_C64");
  return GPE_OK;
}

}  // namespace

extern "C" {

const char* gpe_version(void) { return "gpe_b200 0.1 (sm_100a)"; }

int64_t gpe_state_bytes(const gpe_params* p) {
  std::string why;
  if (validate(p, why)) return -1;
  Geom g;
  int esz;
  layout(p, g, esz);
  return (int64_t)padded_elems(g) * esz * nfields(p->scheme);
}

}  // extern "C"

namespace {

// which z-slab of a decomposed solve a handle is (null: the whole grid)
struct SlabSpec {
  int rank, nranks;
  const void* nccl_id;
  SlabHub* hub;
};

int create_impl(const gpe_params* p, const SlabSpec* sp, gpe_handle** out) {
  if (!out) return fail(nullptr, GPE_ERR_BADARG, "null output handle pointer");
  *out = nullptr;
  std::string why;
  if (int rc = validate(p, why)) return fail(nullptr, rc, why);
  int k0 = 0, nzl = p->nz;
  if (sp) {
    if (sp->nranks < 1 || sp->rank < 0 || sp->rank >= sp->nranks)
      return fail(nullptr, GPE_ERR_BADARG, "gpe_create_slab: rank must be in [0, nranks)");
    if ((sp->nccl_id != nullptr) == (sp->hub != nullptr))
      return fail(nullptr, GPE_ERR_BADARG, "gpe_create_slab: give exactly one of nccl_id and hub");
    if (sp->hub && sp->hub->n != sp->nranks)
      return fail(nullptr, GPE_ERR_BADARG, "gpe_create_slab: the hub was created for another number of slabs");
    slab_partition(p->nz, sp->nranks, sp->rank, &k0, &nzl);
    if (nzl < 6) return fail(nullptr, GPE_ERR_BADARG, "gpe_create_slab: every z-slab needs at least 6 planes");
    if (sp->hub) {
      int dev = 0;
      cudaGetDevice(&dev);
      if (dev != sp->hub->dev)
        return fail(nullptr, GPE_ERR_BADARG, "gpe_create_slab: the hub's slabs share its device and stream");
    }
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(nullptr, GPE_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  gpe_handle* h = new gpe_handle();
  h->p = *p;
  h->nz_global = p->nz;
  if (sp) {
    // local geometry of the slab; neighbours and the z faces whose ghosts
    // the kernels write: a periodic axis is a ring of slabs (one slab
    // exchanges with itself), a reflective axis mirrors at its two ends
    h->slab = true;
    h->rank = sp->rank;
    h->nranks = sp->nranks;
    h->k0 = k0;
    h->p.nz = nzl;
    if (p->bcs == 1) {
      h->slab_down = (sp->rank + sp->nranks - 1) % sp->nranks;
      h->slab_up = (sp->rank + 1) % sp->nranks;
      h->zghost = 0;
    } else {
      h->slab_down = sp->rank > 0 ? sp->rank - 1 : -1;
      h->slab_up = sp->rank < sp->nranks - 1 ? sp->rank + 1 : -1;
      h->zghost = (sp->rank == 0 ? 1 : 0) | (sp->rank == sp->nranks - 1 ? 2 : 0);
    }
  }
  const gpe_params& pl = h->p;
  cudaGetDevice(&h->dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, h->dev) != cudaSuccess || prop.major < 10) {
    delete h;
    return fail(nullptr, GPE_ERR_CUDA, "an sm_100 (Blackwell) device is required");
  }
  layout(&pl, h->g, h->esz);
  h->R = p->order / 2;
  h->cmode = p->storage == GPE_C128 ? CM_F64 : (p->compute == GPE_COMPUTE_F64 ? CM_F32X : CM_F32);
  h->nelem = padded_elems(h->g);
  // thread layout: complex64 storage with the FP32 stencil takes two
  // x-adjacent sites per thread (16-byte shared-memory reads and stores)
  if (const char* e = getenv("GPE_KERNEL")) h->use_tma = strcmp(e, "ldg") != 0;
  if (h->cmode == CM_F32 && h->use_tma) h->tma_ty = TILE_PAIR_32x16;
  if (const char* e = getenv("GPE_ROWS_PER_THREAD")) h->tma_ty = atoi(e) == 1 ? TILE_32x8_ROW1 : TILE_32x8_ROW2;
  if (const char* e = getenv("GPE_TILE")) {
    const int v = atoi(e);
    if (v == TILE_32x8_ROW1 || v == TILE_32x8_ROW2 || (h->cmode == CM_F32 && h->use_tma && tile_is_pair(v)))
      h->tma_ty = v;
  }
  const int th = tile_rows(h->tma_ty);
  h->zc = p->tile_zc > 0 ? std::min(p->tile_zc, pl.nz) : choose_zc(h->g, th, h->esz);
  h->grid = dim3((pl.nx + 31) / 32, (pl.ny + th - 1) / th, (pl.nz + h->zc - 1) / h->zc);
  h->npart = (long long)h->grid.x * h->grid.y * h->grid.z;
  h->norm_grid = dim3((pl.nx + 31) / 32, (pl.ny + 7) / 8, (pl.nz + h->zc - 1) / h->zc);
  h->norm_npart = (long long)h->norm_grid.x * h->norm_grid.y * h->norm_grid.z;
  const long long npart_alloc = std::max(h->npart, h->norm_npart);
  auto bail = [&](int rc) {
    std::string m = h->err;
    gpe_destroy(h);
    return fail(nullptr, rc, m);
  };
  if (sp && sp->hub) {
    h->hub = sp->hub;
    h->st = sp->hub->st;
    h->own_stream = false;
  } else if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
    h->err = "cudaStreamCreate failed";
    return bail(GPE_ERR_CUDA);
  }
  const int nf = nfields(p->scheme);
  h->fields.assign(nf, nullptr);
  for (int f = 0; f < nf; ++f) {
    if (cudaMalloc(&h->fields[f], (size_t)h->nelem * h->esz) != cudaSuccess) {
      cudaGetLastError();
      h->err = "out of device memory allocating the solve's fields";
      return bail(GPE_ERR_NOMEM);
    }
    cudaMemsetAsync(h->fields[f], 0, (size_t)h->nelem * h->esz, h->st);
  }
  if (h->use_tma) {
    h->map_halo.resize(nf);
    h->map_pw.resize(nf);
    for (int f = 0; f < nf; ++f)
      if (!encode_field_maps(h, h->fields[f], &h->map_halo[f], &h->map_pw[f])) {
        h->err = "cuTensorMapEncodeTiled failed (driver entry point unavailable or bad layout)";
        return bail(GPE_ERR_CUDA);
      }
  }
  if (cudaMalloc(&h->status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    h->err = "out of device memory (status word)";
    return bail(GPE_ERR_NOMEM);
  }
  cudaMemsetAsync(h->status, 0, sizeof(int), h->st);
  std::vector<double> tab;
  build_tables(h, tab);
  if (cudaMalloc(&h->tables, tab.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->part_a, npart_alloc * RED_SLOTS * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->part_b, npart_alloc * RED_SLOTS * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->dres, 6 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->hres, 6 * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    h->err = "out of memory allocating tables / reduction buffers";
    return bail(GPE_ERR_NOMEM);
  }
  cudaMemcpyAsync(h->tables, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->st);
  cudaMemsetAsync(h->dres, 0, 6 * sizeof(double), h->st);
  if (cudaStreamSynchronize(h->st) != cudaSuccess) {
    h->err = "initialisation failed";
    return bail(GPE_ERR_CUDA);
  }
  if (sp && sp->nccl_id && nccl_comm_init(&h->nccl, sp->nranks, sp->nccl_id, sp->rank, h->err) != 0)
    return bail(GPE_ERR_CUDA);
  if (sp && sp->hub) {
    std::lock_guard<std::mutex> lk(sp->hub->mu);
    sp->hub->slabs[sp->rank] = h;
  }
  *out = h;
  return GPE_OK;
}

}  // namespace

extern "C" {

int gpe_create(const gpe_params* p, gpe_handle** out) { return create_impl(p, nullptr, out); }

int gpe_create_slab(const gpe_params* p, int32_t rank, int32_t nranks, const void* nccl_id, gpe_slab_hub* hub,
                    gpe_handle** out) {
  const SlabSpec sp{rank, nranks, nccl_id, hub ? &hub->hub : nullptr};
  return create_impl(p, &sp, out);
}

int gpe_slab_partition(int32_t nz, int32_t nranks, int32_t rank, int32_t* k0, int32_t* nzl) {
  if (nz < 1 || nranks < 1 || rank < 0 || rank >= nranks || !k0 || !nzl) return GPE_ERR_BADARG;
  int a = 0, b = 0;
  slab_partition(nz, nranks, rank, &a, &b);
  *k0 = a;
  *nzl = b;
  return GPE_OK;
}

int gpe_slab_extent(const gpe_handle* h, int32_t* k0, int32_t* nzl) {
  if (!h || !k0 || !nzl) return GPE_ERR_BADARG;
  *k0 = h->k0;
  *nzl = h->p.nz;
  return GPE_OK;
}

int gpe_slab_nccl_id(void* id128) {
  if (!id128) return fail(nullptr, GPE_ERR_BADARG, "null id buffer");
  std::string why;
  if (nccl_unique_id(id128, why) != 0) return fail(nullptr, GPE_ERR_CUDA, why);
  return GPE_OK;
}

int gpe_slab_hub_create(int32_t nranks, gpe_slab_hub** out) {
  if (!out || nranks < 1) return fail(nullptr, GPE_ERR_BADARG, "gpe_slab_hub_create: bad arguments");
  gpe_slab_hub* hb = new gpe_slab_hub();
  hb->hub.n = nranks;
  cudaGetDevice(&hb->hub.dev);
  hb->hub.slabs.assign(nranks, nullptr);
  hb->hub.vals.assign(nranks, std::array<double, 6>{});
  // seconds a slab waits at a hub barrier for the others (a slab that stops
  // calling in breaks the hub and every slab's next call returns
  // GPE_ERR_TIMEOUT)
  if (const char* e = getenv("GPE_HUB_TIMEOUT_S")) hb->hub.timeout_s = atof(e) > 0 ? atof(e) : 120.0;
  if (cudaStreamCreateWithFlags(&hb->hub.st, cudaStreamNonBlocking) != cudaSuccess) {
    delete hb;
    return fail(nullptr, GPE_ERR_CUDA, "cudaStreamCreate failed");
  }
  *out = hb;
  return GPE_OK;
}

void gpe_slab_hub_destroy(gpe_slab_hub* hb) {
  if (!hb) return;
  cudaSetDevice(hb->hub.dev);
  cudaStreamSynchronize(hb->hub.st);
  cudaStreamDestroy(hb->hub.st);
  delete hb;
}

void gpe_destroy(gpe_handle* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  // the slabs of a hub read each other's fields: every slab must be done
  // enqueueing exchanges before any of them frees its memory (collective)
  if (h->hub && h->hub->slabs[h->rank] == h) h->hub->barrier(h->hub->timeout_s);
  if (h->st) cudaStreamSynchronize(h->st);
  for (void* f : h->fields)
    if (f) cudaFree(f);
  if (h->tables) cudaFree(h->tables);
  if (h->part_a) cudaFree(h->part_a);
  if (h->part_b) cudaFree(h->part_b);
  if (h->dres) cudaFree(h->dres);
  if (h->hres) cudaFreeHost(h->hres);
  if (h->staging) cudaFree(h->staging);
  if (h->status) cudaFree(h->status);
  if (h->fft_work) cudaFree(h->fft_work);
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
  for (cudaStream_t c : {h->cp_st, h->cp2_st})
    if (c) {
      cudaStreamSynchronize(c);
      cudaStreamDestroy(c);
    }
  for (cudaEvent_t e : {h->ev_packed, h->ev_in, h->ev_unpacked, h->ev_out})
    if (e) cudaEventDestroy(e);
  if (h->in_stage) cudaFree(h->in_stage);
  if (h->out_stage) cudaFree(h->out_stage);
  if (h->snap_st) {
    cudaStreamSynchronize(h->snap_st);
    cudaStreamDestroy(h->snap_st);
  }
  if (h->snap_ready) cudaEventDestroy(h->snap_ready);
  if (h->snap_done) cudaEventDestroy(h->snap_done);
  if (h->snap_dev) cudaFree(h->snap_dev);
  if (h->snap_host) cudaFreeHost(h->snap_host);
  if (h->st && h->own_stream) cudaStreamDestroy(h->st);
  if (h->nccl) nccl_comm_destroy(h->nccl);
  if (h->hub) {
    std::lock_guard<std::mutex> lk(h->hub->mu);
    if (h->hub->slabs[h->rank] == h) h->hub->slabs[h->rank] = nullptr;
  }
  delete h;
}

const char* gpe_last_error(const gpe_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int gpe_set_state(gpe_handle* h, const void* psi, int32_t dtype) {
  if (!h || !psi) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  const size_t bytes = interior_bytes(h, dtype);
  if (int rc = ensure_staging(h, bytes)) return rc;
  CU(h, cudaMemcpyAsync(h->staging, psi, bytes, cudaMemcpyHostToDevice, h->st));
  if (int rc = pack_from_device(h, h->staging, dtype)) return rc;
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_get_state(gpe_handle* h, void* psi, int32_t dtype) {
  if (!h || !psi) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  const size_t bytes = interior_bytes(h, dtype);
  if (int rc = ensure_staging(h, bytes)) return rc;
  if (int rc = unpack_to_device(h, h->staging, dtype)) return rc;
  CU(h, cudaMemcpyAsync(psi, h->staging, bytes, cudaMemcpyDeviceToHost, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_set_state_device(gpe_handle* h, const void* psi_dev, int32_t dtype) {
  if (!h || !psi_dev) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  if (int rc = pack_from_device(h, psi_dev, dtype)) return rc;
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_get_state_device(gpe_handle* h, void* psi_dev, int32_t dtype) {
  if (!h || !psi_dev) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  if (int rc = unpack_to_device(h, psi_dev, dtype)) return rc;
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

// Graph of one fixed step for the current dt (captured on first use and
// whenever dt changes).  Only for schemes that keep psi in place.
static int ensure_step_graph(gpe_handle* h, double dr, double di) {
  if (h->step_graph && h->graph_dr == dr && h->graph_di == di) return GPE_OK;
  if (h->step_graph) {
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  CU(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue_fixed_step(h, dr, di, false, false);
  const cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (rc != GPE_OK) {
    if (e == cudaSuccess && g) cudaGraphDestroy(g);
    return rc;
  }
  CU(h, e);
  const cudaError_t ei = cudaGraphInstantiate(&h->step_graph, g, 0);
  cudaGraphDestroy(g);
  CU(h, ei);
  h->graph_dr = dr;
  h->graph_di = di;
  return GPE_OK;
}

static bool use_step_graphs(const gpe_handle* h) {
  static const bool off = [] {
    const char* e = getenv("GPE_GRAPHS");
    return e && atoi(e) == 0;
  }();
  return !off && !h->prof && !h->slab && (h->p.scheme == GPE_RK4 || h->p.scheme == GPE_RK2);
}

static int step_impl(gpe_handle* h, int64_t nsteps, gpe_step_info* io, bool wait) {
  if (!h || !io || nsteps < 0) return fail(h, GPE_ERR_BADARG, "bad gpe_step arguments");
  CU(h, cudaSetDevice(h->dev));
  default_dt(h->p, io);
  io->accepted = 0;
  io->rejected = 0;
  const bool want_e = io->want_energy != 0, want_n = io->want_norm != 0;
  if (h->p.scheme == GPE_RK45) {
    if (!wait) return fail(h, GPE_ERR_BADARG, "gpe_step_async does not support rk45");
    for (int64_t s = 0; s < nsteps; ++s) {
      if (int rc = rk45_step(h, io, want_e && s == 0, want_n && s == nsteps - 1)) return rc;
      io->p += 1;
      io->accepted += 1;
    }
  } else {
    const double dr = io->dt_re, di = io->dt_im;
    // steps without reductions replay a captured graph (one launch instead of
    // one per stage); the first step of a call runs plainly, so every kernel
    // has been loaded and configured before any capture
    const bool graphs = use_step_graphs(h) && nsteps >= 3;
    for (int64_t s = 0; s < nsteps; ++s) {
      const bool e = want_e && s == 0, n = want_n && s == nsteps - 1;
      if (graphs && s > 0 && !e && !n) {
        if (int rc = ensure_step_graph(h, dr, di)) return rc;
        CU(h, cudaGraphLaunch(h->step_graph, h->st));
      } else if (int rc = enqueue_fixed_step(h, dr, di, e, n)) {
        return rc;
      }
      io->t = io->t + dr;
      io->im_t = io->im_t + fabs(di);
      io->p += 1;
      io->accepted += 1;
    }
    if (!wait) return GPE_OK;
    if (int rc = fetch_results(h)) return rc;
  }
  if (want_e && nsteps > 0) io->energy = ((h->hres[1] * h->dx) * h->dy) * h->dz;
  if (want_n && nsteps > 0) {
    io->norm = ((h->hres[3] * h->dx) * h->dy) * h->dz;
    if (!std::isfinite(io->norm)) return fail(h, GPE_ERR_NONFINITE, "non-finite norm: the solution blew up");
  }
  return GPE_OK;
}

int gpe_step(gpe_handle* h, int64_t nsteps, gpe_step_info* io) { return step_impl(h, nsteps, io, true); }

int gpe_step_async(gpe_handle* h, int64_t nsteps, gpe_step_info* io) { return step_impl(h, nsteps, io, false); }

// copy stream, staging buffers and events of the asynchronous state copies
static int ensure_async_copies(gpe_handle* h, size_t bytes) {
  if (!h->cp_st) {
    CU(h, cudaStreamCreateWithFlags(&h->cp_st, cudaStreamNonBlocking));
    CU(h, cudaStreamCreateWithFlags(&h->cp2_st, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&h->ev_packed, &h->ev_in, &h->ev_unpacked, &h->ev_out})
      CU(h, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    // record every event once so that the first waits on them are no-ops
    for (cudaEvent_t e : {h->ev_packed, h->ev_unpacked}) CU(h, cudaEventRecord(e, h->st));
    CU(h, cudaEventRecord(h->ev_in, h->cp_st));
    CU(h, cudaEventRecord(h->ev_out, h->cp2_st));
  }
  if (h->in_cap < bytes || h->out_cap < bytes) {
    CU(h, cudaStreamSynchronize(h->st));
    CU(h, cudaStreamSynchronize(h->cp_st));
    CU(h, cudaStreamSynchronize(h->cp2_st));
    if (h->in_stage) cudaFree(h->in_stage);
    if (h->out_stage) cudaFree(h->out_stage);
    h->in_stage = h->out_stage = nullptr;
    h->in_cap = h->out_cap = 0;
    CU(h, cudaMalloc(&h->in_stage, bytes));
    CU(h, cudaMalloc(&h->out_stage, bytes));
    h->in_cap = h->out_cap = bytes;
  }
  return GPE_OK;
}

int gpe_set_state_async(gpe_handle* h, const void* psi, int32_t dtype) {
  if (!h || !psi) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  const size_t bytes = interior_bytes(h, dtype);
  if (int rc = ensure_async_copies(h, bytes)) return rc;
  // the previous pack must be done with the input staging buffer
  CU(h, cudaStreamWaitEvent(h->cp_st, h->ev_packed, 0));
  CU(h, cudaMemcpyAsync(h->in_stage, psi, bytes, cudaMemcpyHostToDevice, h->cp_st));
  CU(h, cudaEventRecord(h->ev_in, h->cp_st));
  CU(h, cudaStreamWaitEvent(h->st, h->ev_in, 0));
  if (int rc = pack_from_device(h, h->in_stage, dtype)) return rc;
  CU(h, cudaEventRecord(h->ev_packed, h->st));
  h->copies_pending = true;
  return GPE_OK;
}

int gpe_get_state_async(gpe_handle* h, void* psi, int32_t dtype) {
  if (!h || !psi) return fail(h, GPE_ERR_BADARG, "null argument");
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  const size_t bytes = interior_bytes(h, dtype);
  if (int rc = ensure_async_copies(h, bytes)) return rc;
  // the previous transfer must be done with the output staging buffer
  CU(h, cudaStreamWaitEvent(h->st, h->ev_out, 0));
  if (int rc = unpack_to_device(h, h->out_stage, dtype)) return rc;
  CU(h, cudaEventRecord(h->ev_unpacked, h->st));
  CU(h, cudaStreamWaitEvent(h->cp2_st, h->ev_unpacked, 0));
  CU(h, cudaMemcpyAsync(psi, h->out_stage, bytes, cudaMemcpyDeviceToHost, h->cp2_st));
  CU(h, cudaEventRecord(h->ev_out, h->cp2_st));
  h->copies_pending = true;
  return GPE_OK;
}

int gpe_wait_copies(gpe_handle* h) {
  if (!h) return GPE_ERR_BADARG;
  if (!h->cp_st) return GPE_OK;
  CU(h, cudaSetDevice(h->dev));
  CU(h, cudaStreamWaitEvent(h->st, h->ev_out, 0));
  CU(h, cudaStreamWaitEvent(h->st, h->ev_in, 0));
  return GPE_OK;
}

int gpe_sync(gpe_handle* h) {
  if (!h) return GPE_ERR_BADARG;
  CU(h, cudaSetDevice(h->dev));
  if (h->cp_st) {
    CU(h, cudaStreamSynchronize(h->cp_st));
    CU(h, cudaStreamSynchronize(h->cp2_st));
    h->copies_pending = false;
  }
  CU(h, cudaStreamSynchronize(h->st));
  if (h->prof) prof_resolve(h);
  return check_status(h);
}

int gpe_test_expire_waits(gpe_handle* h) {
  if (!h) return GPE_ERR_BADARG;
  CU(h, cudaSetDevice(h->dev));
  static const int v = STATUS_EXPIRE_TEST;
  CU(h, cudaMemcpyAsync(h->status, &v, sizeof(int), cudaMemcpyHostToDevice, h->st));
  return GPE_OK;
}

int gpe_profile(gpe_handle* h, int32_t enable) {
  if (!h) return GPE_ERR_BADARG;
  CU(h, cudaSetDevice(h->dev));
  CU(h, cudaStreamSynchronize(h->st));
  prof_resolve(h);
  h->prof = enable != 0;
  for (int k = 0; k < K_NUM; ++k) {
    h->prof_ms[k] = 0.0;
    h->prof_n[k] = 0;
  }
  return GPE_OK;
}

int gpe_profile_get(gpe_handle* h, int32_t kind, double* total_ms, int64_t* launches, double* bytes_per_site) {
  if (!h || kind < 0 || kind >= K_NUM) return fail(h, GPE_ERR_BADARG, "bad profile kind");
  CU(h, cudaSetDevice(h->dev));
  CU(h, cudaStreamSynchronize(h->st));
  prof_resolve(h);
  if (total_ms) *total_ms = h->prof_ms[kind];
  if (launches) *launches = h->prof_n[kind];
  if (bytes_per_site) *bytes_per_site = (double)kind_elems(kind) * h->esz;
  return GPE_OK;
}

int gpe_norm(gpe_handle* h, double* norm) {
  if (!h || !norm) return fail(h, GPE_ERR_BADARG, "null argument");
  CU(h, cudaSetDevice(h->dev));
  return norm_now(h, norm);
}

int gpe_energy(gpe_handle* h, double* energy) {
  if (!h || !energy) return fail(h, GPE_ERR_BADARG, "null argument");
  CU(h, cudaSetDevice(h->dev));
  StageArgs a = base_args(h);
  a.in = h->fields[h->cur];
  a.want_energy = 1;
  a.partials = h->part_a;
  CU(h, launch(h, K_ENERGY, a));
  if (int rc = finalize_into(h, h->part_a, 0)) return rc;
  if (int rc = fetch_results(h)) return rc;
  *energy = ((h->hres[1] * h->dx) * h->dy) * h->dz;
  return GPE_OK;
}

// FFT scratch on first use: transform buffer + partials, then the k tables
static int ensure_fft(gpe_handle* h) {
  if (h->fft_work) return GPE_OK;
  const size_t need = fft_work_bytes(h->p);
  const int nk = h->p.nx + h->p.ny + h->p.nz;
  if (cudaMalloc(&h->fft_work, need + nk * sizeof(double)) != cudaSuccess) {
    h->fft_work = nullptr;
    return fail(h, GPE_ERR_NOMEM, "cudaMalloc failed for the FFT diagnostics scratch");
  }
  h->fft_work_bytes = need;
  h->fft_kq = (double*)((char*)h->fft_work + need);
  std::vector<double> kq(nk);
  fft_kq_axis(h->p.nx, h->p.nx, h->dx, kq.data());
  fft_kq_axis(h->p.ny, h->p.nx, h->dy, kq.data() + h->p.nx);
  fft_kq_axis(h->p.nz, h->p.nx, h->dz, kq.data() + h->p.nx + h->p.ny);
  CU(h, cudaMemcpy(h->fft_kq, kq.data(), nk * sizeof(double), cudaMemcpyHostToDevice));
  return GPE_OK;
}

int gpe_condensed(gpe_handle* h, gpe_condensed_info* info, double* eta, int32_t* nharm, double* F, int32_t nF) {
  if (!h || !info) return fail(h, GPE_ERR_BADARG, "null argument");
  if (h->slab) return fail(h, GPE_ERR_BADARG, "gpe_condensed: not available on a z-slab handle");
  if (F && nF != h->p.nx / 2) return fail(h, GPE_ERR_BADARG, "gpe_condensed: nF must be nx/2");
  CU(h, cudaSetDevice(h->dev));
  if (int rc = ensure_fft(h)) return rc;
  const bool spec = eta || nharm || F;
  FftDiag d;
  CU(h, fft_condensed(h->p, h->g, h->esz, h->fields[h->cur], h->fft_kq, spec, h->fft_work, h->fft_work_bytes,
                      h->st, d));
  // io.f90:331-381, in the reference's expression order
  const double V = (double)h->p.nx * (double)h->p.ny * (double)h->p.nz;
  const long long Vi = (long long)h->p.nx * h->p.ny * h->p.nz;
  const double M = ((d.mass_sum * h->dx) * h->dy) * h->dz;
  const double vol8 = ((8.0 * h->p.xr) * h->p.yr) * h->p.zr;
  info->M = M;
  info->n0 = d.n0;
  info->rho0 = d.n0 / V;
  info->tot = d.tot;
  info->temp = (M - d.n0) / d.tot;
  const double E0 = (1.0 / (double)(2 * Vi)) * (M * M + (M - d.n0) * (M - d.n0));
  info->H = E0 + info->temp * (double)(Vi - 1);
  info->temp2 = ((M / vol8) - (d.n0 / V)) / d.tot;
  info->mass_density = M / vol8;
  for (int m = 0; m < GPE_SPECTRUM_SHELLS; ++m) {
    const double e = d.eta[m];
    const double c = d.nharm[m];
    if (nharm) nharm[m] = (int32_t)c;
    if (eta) eta[m] = (e == 0.0) ? e : e / c;
  }
  if (F) {
    double acc = 0.0;
    for (int kk = 1; kk <= nF; ++kk) {
      acc += d.H[kk];
      F[kk - 1] = acc;
    }
  }
  return GPE_OK;
}

int gpe_filtered(gpe_handle* h, double m, double filter_kc, void* out, int32_t dtype) {
  if (!h || !out) return fail(h, GPE_ERR_BADARG, "null argument");
  if (h->slab) return fail(h, GPE_ERR_BADARG, "gpe_filtered: not available on a z-slab handle");
  if (!(filter_kc > 0.0)) return fail(h, GPE_ERR_BADARG, "gpe_filtered: filter_kc must be > 0");
  if (dtype != GPE_C128 && dtype != GPE_C64) return fail(h, GPE_ERR_BADARG, "gpe_filtered: bad dtype");
  CU(h, cudaSetDevice(h->dev));
  if (int rc = ensure_fft(h)) return rc;
  CU(h, fft_filtered(h->p, h->g, h->esz, h->fields[h->cur], m, filter_kc, h->fft_work, h->fft_work_bytes, h->st));
  const size_t n = (size_t)h->p.nx * h->p.ny * h->p.nz;
  if (dtype == GPE_C128) {
    CU(h, cudaMemcpyAsync(out, h->fft_work, n * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
  } else {
    std::vector<double2> tmp(n);
    CU(h, cudaMemcpyAsync(tmp.data(), h->fft_work, n * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
    float2* o = (float2*)out;
    for (size_t t = 0; t < n; ++t) o[t] = make_float2((float)tmp[t].x, (float)tmp[t].y);
  }
  return GPE_OK;
}

int gpe_renormalise(gpe_handle* h, double norm) {
  if (!h || !(norm > 0)) return fail(h, GPE_ERR_BADARG, "norm must be > 0");
  CU(h, cudaSetDevice(h->dev));
  const double a = sqrt(h->p.nn), b = sqrt(norm);
  if (h->esz == 16) k_scale<double2><<<148 * 8, 256, 0, h->st>>>((double2*)h->fields[h->cur], h->nelem, a, b);
  else k_scale<float2><<<148 * 8, 256, 0, h->st>>>((float2*)h->fields[h->cur], h->nelem, a, b);
  CU(h, cudaGetLastError());
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_set_ic(gpe_handle* h, const gpe_ic* ic) {
  if (!h) return GPE_ERR_BADARG;
  if (h->slab) return fail(h, GPE_ERR_BADARG, "gpe_set_ic: not available on a z-slab handle (use gpe_set_state)");
  std::string why;
  if (int rc = ic_validate(ic, why)) return fail(h, rc, why);
  CU(h, cudaSetDevice(h->dev));
  const size_t wb = ic_work_bytes(h->p, *ic);
  if (wb)
    if (int rc = ensure_staging(h, wb)) return rc;
  CU(h, ic_generate(h->p, h->g, h->esz, h->R, *ic, h->fields[h->cur], h->staging, h->staging_bytes, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_multiply_ic(gpe_handle* h, const gpe_ic* ic, int32_t modulus) {
  if (!h) return GPE_ERR_BADARG;
  if (h->slab) return fail(h, GPE_ERR_BADARG, "gpe_multiply_ic: not available on a z-slab handle");
  std::string why;
  if (int rc = ic_validate(ic, why)) return fail(h, rc, why);
  if (ic_needs_fft(ic))
    return fail(h, GPE_ERR_BADARG, "gpe_multiply_ic: the random-phase state cannot multiply a state");
  CU(h, cudaSetDevice(h->dev));
  CU(h, ic_multiply(h->p, h->g, h->esz, h->R, *ic, h->fields[h->cur], modulus != 0, h->st));
  CU(h, cudaStreamSynchronize(h->st));
  return GPE_OK;
}

int gpe_get_grid(const gpe_handle* h, double* x, double* y, double* z, double* dxyz) {
  if (!h) return GPE_ERR_BADARG;
  if (x) memcpy(x, h->x.data(), sizeof(double) * h->x.size());
  if (y) memcpy(y, h->y.data(), sizeof(double) * h->y.size());
  if (z) memcpy(z, h->z.data(), sizeof(double) * h->z.size());
  if (dxyz) {
    dxyz[0] = h->dx;
    dxyz[1] = h->dy;
    dxyz[2] = h->dz;
  }
  return GPE_OK;
}

int gpe_snapshot_begin(gpe_handle* h, int32_t dtype) {
  if (!h) return GPE_ERR_BADARG;
  if (int rc = check_dtype(h, dtype)) return rc;
  CU(h, cudaSetDevice(h->dev));
  const size_t bytes = interior_bytes(h, dtype);
  if (!h->snap_st) {
    CU(h, cudaStreamCreateWithFlags(&h->snap_st, cudaStreamNonBlocking));
    CU(h, cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
    CU(h, cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
  }
  if (h->snap_cap < bytes) {
    // the previous snapshot's copy must be done with the old buffers
    CU(h, cudaStreamSynchronize(h->snap_st));
    if (h->snap_dev) cudaFree(h->snap_dev);
    if (h->snap_host) cudaFreeHost(h->snap_host);
    h->snap_dev = h->snap_host = nullptr;
    h->snap_cap = 0;
    CU(h, cudaMalloc(&h->snap_dev, bytes));
    CU(h, cudaMallocHost(&h->snap_host, bytes));
    h->snap_cap = bytes;
  } else if (h->snap_pending) {
    // the device copy of the new snapshot must not overwrite the buffer the
    // previous transfer still reads (device-side order, the host does not wait)
    CU(h, cudaStreamWaitEvent(h->st, h->snap_done, 0));
  }
  if (int rc = unpack_to_device(h, h->snap_dev, dtype)) return rc;
  CU(h, cudaEventRecord(h->snap_ready, h->st));
  CU(h, cudaStreamWaitEvent(h->snap_st, h->snap_ready, 0));
  CU(h, cudaMemcpyAsync(h->snap_host, h->snap_dev, bytes, cudaMemcpyDeviceToHost, h->snap_st));
  CU(h, cudaEventRecord(h->snap_done, h->snap_st));
  h->snap_bytes = bytes;
  h->snap_pending = true;
  return GPE_OK;
}

int gpe_snapshot_wait(gpe_handle* h, const void** host_data, size_t* bytes) {
  if (!h || !host_data || !bytes) return GPE_ERR_BADARG;
  if (!h->snap_pending) return GPE_ERR_STATE;
  if (cudaEventSynchronize(h->snap_done) != cudaSuccess) return GPE_ERR_CUDA;
  *host_data = h->snap_host;
  *bytes = h->snap_bytes;
  return GPE_OK;
}

int gpe_get_site(gpe_handle* h, int32_t i, int32_t j, int32_t k, double* re_im) {
  if (!h || !re_im) return fail(h, GPE_ERR_BADARG, "null argument");
  if (i < 0 || i >= h->p.nx || j < 0 || j >= h->p.ny || k < 0 || k >= h->p.nz)
    return fail(h, GPE_ERR_BADARG, "gpe_get_site: index outside the grid");
  CU(h, cudaSetDevice(h->dev));
  const long long o = (long long)(k + 2) * h->g.pz + (long long)(j + 2) * h->g.px + h->g.xoff + i;
  const char* src = (const char*)h->fields[h->cur] + o * h->esz;
  if (h->esz == 16) {
    CU(h, cudaMemcpyAsync(re_im, src, 16, cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
  } else {
    float v[2];
    CU(h, cudaMemcpyAsync(v, src, 8, cudaMemcpyDeviceToHost, h->st));
    CU(h, cudaStreamSynchronize(h->st));
    re_im[0] = v[0];
    re_im[1] = v[1];
  }
  return GPE_OK;
}

int gpe_get_stream(const gpe_handle* h, void** stream) {
  if (!h || !stream) return GPE_ERR_BADARG;
  *stream = (void*)h->st;
  return GPE_OK;
}

}  // extern "C"

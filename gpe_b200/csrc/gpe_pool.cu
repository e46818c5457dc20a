// Batched solves and serving: the gpe_pool_* entry points of
// include/gpe_cuda.h.
//
// A pool owns one device arena (the HBM budget).  Each admitted solve gets
// its ghost-padded fields and per-axis tables from the arena.  Active solves
// are grouped into classes by (storage/compute mode, scheme family); each
// class keeps a work list of (solve, tile, z-chunk) items and a device table
// of per-solve stage arguments and tensor maps.  One persistent launch of
// k_stage_batch per Runge-Kutta stage advances every solve of a class; the
// RK4 step of a class is captured once into a CUDA graph and replayed.
// RKF45 solves share their attempts: after each attempt every solve's error
// norm is read back and that solve alone accepts or rejects (rkqs,
// src/solve.f90:158-244), so per-solve time steps diverge freely.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "../../include/gpe_cuda.h"
#include "gpe_aux.cuh"
#include "gpe_common.h"
#include "gpe_ic.h"

namespace gpe {
cudaError_t launch_batch_f64(int kind, int R, int grid, cudaStream_t st, const BatchLaunch& b, int* occupancy);
cudaError_t launch_batch_f32(int kind, int R, int grid, cudaStream_t st, const BatchLaunch& b, int* occupancy);
cudaError_t launch_batch_f32x(int kind, int R, int grid, cudaStream_t st, const BatchLaunch& b, int* occupancy);
int batch_rows_f64(int kind);
int batch_rows_f32(int kind);
int batch_rows_f32x(int kind);
}  // namespace gpe

using namespace gpe;

namespace {

enum { CM_F64 = 0, CM_F32 = 1, CM_F32X = 2, NCM = 3 };
// Classes of solves that share launches: (precision mode, stencil radius) x
// scheme family.  Solves of the two FD orders run in separate classes, so
// each batched kernel carries one item body and rings sized for its radius.
constexpr int NCLS = NCM * 2;
inline int class_of(int cmode, int R) { return cmode * 2 + (R - 1); }
inline int class_cmode(int cls) { return cls / 2; }
inline int class_radius(int cls) { return cls % 2 + 1; }
enum { FAM_RK4 = 0, FAM_RK45 = 1, NFAM = 2 };

// First-fit allocator over [0, total) with coalescing; 256-byte granules.
class Arena {
 public:
  void init(size_t total) {
    free_.clear();
    free_[0] = total;
    total_ = total;
    used_ = 0;
  }
  static size_t round(size_t n) { return (n + 255) & ~size_t(255); }
  bool alloc(size_t n, size_t* off) {
    n = round(n);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, start = it->first + n;
      free_.erase(it);
      if (rest) free_[start] = rest;
      used_ += n;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    n = round(n);
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t free_bytes() const { return total_ - used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t total_ = 0, used_ = 0;
};

struct Solve {
  uint64_t tag = 0;
  gpe_params p{};
  Geom g{};
  int R = 2, esz = 16, cmode = CM_F64, fam = FAM_RK4, nf = 4;
  size_t off = 0, bytes = 0, field_bytes = 0;
  void* f[9] = {};
  double* tables = nullptr;
  double d[3] = {};
  int zc = 8, ntx = 1, nty = 1, ntz = 1;
  int tile_h = 8;  // rows of the solve's 32-column work items (its class's kernel layout)
  int64_t nsteps = 0, done = 0, rejected = 0, quota = 0;
  double t = 0, im_t = 0, dr = 0, di = 0, dte_r = 0, dte_i = 0, errmax = 0, norm = 0;
  int64_t p_index = 0;
  int cur = 0;  // RKF45: field holding psi (0 or 1)
  void* out = nullptr;
  int status = GPE_OK;
  double t_submit = 0, t_start = -1;
  CUtensorMap halo[9], pw[9];
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t c = std::max<size_t>(n, 16) * 2;
    cudaError_t e = cudaMalloc(&p, c * sizeof(T));
    if (e == cudaSuccess) cap = c;
    return e;
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

template <class T>
struct HostPinned {
  T* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t c = std::max<size_t>(n, 16) * 2;
    cudaError_t e = cudaMallocHost(&p, c * sizeof(T));
    if (e == cudaSuccess) cap = c;
    return e;
  }
  void free() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

struct Class {
  std::vector<Solve*> solves;
  bool dirty = true;
  DevBuf<BatchStage> tab;   // [stage][solve]
  DevBuf<BatchItem> items;
  DevBuf<int> order;        // item indices, largest items first (the work queue's order)
  DevBuf<int> queue;        // one work-queue counter per stage launch, zeroed before each step
  DevBuf<int> first;        // [solve + 1] item ranges
  DevBuf<double> part;      // [item][RED_SLOTS]
  DevBuf<double> res;       // [solve][RED_SLOTS]
  HostPinned<BatchStage> htab;
  HostPinned<double> hres;
  HostPinned<int> hstatus;  // device status word after the class's last RKF45 attempt
  std::vector<BatchItem> hitems;
  std::vector<int> horder;
  // the solves (in order) the device work list was built for; an RKF45 class
  // keeps it across attempts while no solve joins or leaves (dirty stays false)
  std::vector<Solve*> built_for;
  std::vector<int> hfirst;
  int nitems = 0;
  // RK4 step graphs: without reductions, and with the per-solve norm (the
  // last step of a chunk)
  cudaGraph_t graph = nullptr, graph_n = nullptr;
  cudaGraphExec_t gexec = nullptr, gexec_n = nullptr;
  cudaStream_t st = nullptr;  // classes run concurrently, one stream each
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (gexec_n) cudaGraphExecDestroy(gexec_n);
    if (graph_n) cudaGraphDestroy(graph_n);
    gexec = gexec_n = nullptr;
    graph = graph_n = nullptr;
  }
};

double now_s(const std::chrono::steady_clock::time_point& t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

size_t tables_bytes(const gpe_params& p) { return (size_t)(p.nx + p.ny + p.nz) * 4 * sizeof(double); }

}  // namespace

struct gpe_pool {
  int dev = 0;
  cudaStream_t st = nullptr;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  Arena alloc;
  int* d_status = nullptr;
  std::vector<Solve*> pending;
  Class cls[NCLS][NFAM];
  std::deque<gpe_result> done;
  std::string err;
  std::chrono::steady_clock::time_point t0;
};

namespace {

int pfail(gpe_pool* P, int code, const std::string& msg) {
  if (P) P->err = msg;
  return code;
}

#define PCU(P, call)                                                                               \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return pfail((P), GPE_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #call); \
  } while (0)

int cmode_of(const gpe_params& p) {
  if (p.storage == GPE_C128) return CM_F64;
  return p.compute == GPE_COMPUTE_F64 ? CM_F32X : CM_F32;
}

cudaError_t launch_batch(int cls, int kind, int grid, cudaStream_t st, const BatchLaunch& b, int* occ) {
  const int R = class_radius(cls);
  switch (class_cmode(cls)) {
    case CM_F64: return launch_batch_f64(kind, R, grid, st, b, occ);
    case CM_F32: return launch_batch_f32(kind, R, grid, st, b, occ);
    default: return launch_batch_f32x(kind, R, grid, st, b, occ);
  }
}

// rows of the work items of a (precision, scheme family) class
int batch_rows(int cmode, int fam) {
  const int kind = fam == FAM_RK45 ? K_CK_1 : K_RK4_1;
  switch (cmode) {
    case CM_F64: return batch_rows_f64(kind);
    case CM_F32: return batch_rows_f32(kind);
    default: return batch_rows_f32x(kind);
  }
}

// Persistent grid of a class's launch: as many CTAs as fit on the device at
// once (of the kernel variant its ns solves select), at most one per item.
int grid_for(int cls, int kind, int nitems, int ns) {
  int occ = 0;
  BatchLaunch q{};
  q.ns = ns;
  launch_batch(cls, kind, 0, nullptr, q, &occ);
  return std::max(1, std::min(nitems, occ));
}

// Copy a contiguous host interior into field f of a solve, then its ghosts.
int upload_state(gpe_pool* P, Solve* s, const void* psi, int fidx) {
  cudaMemcpy3DParms m;
  memset(&m, 0, sizeof(m));
  m.srcPtr = make_cudaPitchedPtr(const_cast<void*>(psi), (size_t)s->g.nx * s->esz, (size_t)s->g.nx * s->esz,
                                 (size_t)s->g.ny);
  m.dstPtr = make_cudaPitchedPtr(s->f[fidx], (size_t)s->g.px * s->esz, (size_t)s->g.px * s->esz,
                                 (size_t)(s->g.ny + 4));
  m.dstPos = make_cudaPos((size_t)s->g.xoff * s->esz, 2, 2);
  m.extent = make_cudaExtent((size_t)s->g.nx * s->esz, (size_t)s->g.ny, (size_t)s->g.nz);
  m.kind = cudaMemcpyHostToDevice;
  PCU(P, cudaMemcpy3DAsync(&m, P->st));
  if (s->esz == 16)
    k_fill_ghosts<double2><<<148 * 4, 256, 0, P->st>>>((double2*)s->f[fidx], s->g, s->R, s->p.bcs);
  else
    k_fill_ghosts<float2><<<148 * 4, 256, 0, P->st>>>((float2*)s->f[fidx], s->g, s->R, s->p.bcs);
  PCU(P, cudaGetLastError());
  return GPE_OK;
}

int download_state(gpe_pool* P, Solve* s, int fidx) {
  cudaMemcpy3DParms m;
  memset(&m, 0, sizeof(m));
  m.srcPtr = make_cudaPitchedPtr(s->f[fidx], (size_t)s->g.px * s->esz, (size_t)s->g.px * s->esz,
                                 (size_t)(s->g.ny + 4));
  m.srcPos = make_cudaPos((size_t)s->g.xoff * s->esz, 2, 2);
  m.dstPtr = make_cudaPitchedPtr(s->out, (size_t)s->g.nx * s->esz, (size_t)s->g.nx * s->esz, (size_t)s->g.ny);
  m.extent = make_cudaExtent((size_t)s->g.nx * s->esz, (size_t)s->g.ny, (size_t)s->g.nz);
  m.kind = cudaMemcpyDeviceToHost;
  PCU(P, cudaMemcpy3DAsync(&m, P->st));
  return GPE_OK;
}

// Per-solve stage table entry: arguments + tensor maps of the fields the
// stage reads.  pw fields in StageTraits order.
BatchStage make_stage(gpe_pool* P, Solve* s, int kind, int fin, int fout, std::initializer_list<int> pwf) {
  BatchStage b;
  memset(&b, 0, sizeof(b));
  b.args = make_base_args(s->p, s->g, s->R, s->zc, s->d, s->tables);
  b.args.status = P->d_status;
  b.args.in = s->f[fin];
  b.args.out = fout >= 0 ? s->f[fout] : nullptr;
  b.maps.in = s->halo[fin];
  int q = 0;
  for (int fi : pwf) b.maps.pw[q++] = s->pw[fi];
  (void)kind;
  return b;
}

// RK4 tables: 4 stages (fields psi=0, A=1, B=2, Q=3) of the reduced-traffic
// RK4 form of site_stage: A = psi + h/2 k1; B = psi + h/2 k2,
// Q = (psi + A) + h k2; A = psi + h k3; psi = (Q + A)/3 + h/6 k4
void rk4_tables(gpe_pool* P, Solve* s, BatchStage* t4) {
  const double dr = s->dr, di = s->di;
  BatchStage b = make_stage(P, s, K_RK4_1, 0, 1, {});
  b.args.cf_r[0] = 0.5 * dr; b.args.cf_i[0] = 0.5 * di;
  t4[0] = b;
  b = make_stage(P, s, K_RK4_2, 1, 2, {0});
  b.args.psi = s->f[0];
  b.args.acc = s->f[3];
  b.args.cf_r[0] = 0.5 * dr; b.args.cf_i[0] = 0.5 * di;
  b.args.cf_r[1] = dr; b.args.cf_i[1] = di;
  t4[1] = b;
  b = make_stage(P, s, K_RK4_3, 2, 1, {0});
  b.args.psi = s->f[0];
  b.args.cf_r[0] = dr; b.args.cf_i[0] = di;
  t4[2] = b;
  b = make_stage(P, s, K_RK4_4, 1, 0, {3});
  b.args.acc = s->f[3];
  b.args.cf_r[0] = dr / 6.0; b.args.cf_i[0] = di / 6.0;
  b.args.want_norm = 1;
  t4[3] = b;
}

// RKF45 tables for one attempt: fields psi/psi_new = cur/1-cur, A=2, B=3, K1..K5=4..8
void rk45_tables(gpe_pool* P, Solve* s, BatchStage* t6) {
  const int psi = s->cur, pnew = 1 - s->cur;
  const int ins[6] = {psi, 2, 3, 2, 3, 2};
  const int outs[6] = {2, 3, 2, 3, 2, pnew};
  for (int m = 0; m < 6; ++m) {
    BatchStage b;
    if (m == 0) b = make_stage(P, s, K_CK_1, ins[m], outs[m], {});
    else if (m == 1) b = make_stage(P, s, K_CK_2, ins[m], outs[m], {psi, 4});
    else if (m == 2) b = make_stage(P, s, K_CK_3, ins[m], outs[m], {psi, 4, 5});
    else if (m == 3) b = make_stage(P, s, K_CK_4, ins[m], outs[m], {psi, 4, 5, 6});
    else if (m == 4) b = make_stage(P, s, K_CK_5, ins[m], outs[m], {psi, 4, 5, 6, 7});
    else b = make_stage(P, s, K_CK_6, ins[m], outs[m], {psi, 4, 6, 7, 8});
    b.args.psi = s->f[psi];
    b.args.cf_r[0] = s->dr;
    b.args.cf_i[0] = s->di;
    if (m < 5) {
      b.args.kout = s->f[4 + m];
      for (int q = 0; q <= m; ++q) b.args.b[q] = CK_B[m][q];
      for (int q = 0; q < m; ++q) b.args.kin[q] = s->f[4 + q];
    } else {
      b.args.kin[0] = s->f[4];
      b.args.kin[1] = s->f[6];
      b.args.kin[2] = s->f[7];
      b.args.kin[3] = s->f[8];
      b.args.dte_r = s->dte_r;
      b.args.dte_i = s->dte_i;
      b.args.inv_adt = 1.0 / hypot(s->dr, s->di);
      b.args.want_norm = 1;
    }
    t6[m] = b;
  }
}

// Work list of the given solves (in order) into the class buffers.
int build_items(gpe_pool* P, Class& c, const std::vector<Solve*>& sv) {
  c.built_for = sv;
  c.hitems.clear();
  c.hfirst.assign(1, 0);
  for (Solve* s : sv) {
    for (int bz = 0; bz < s->ntz; ++bz)
      for (int by = 0; by < s->nty; ++by)
        for (int bx = 0; bx < s->ntx; ++bx) c.hitems.push_back(BatchItem{(int)c.hfirst.size() - 1, bx, by, bz});
    c.hfirst.push_back((int)c.hitems.size());
  }
  c.nitems = (int)c.hitems.size();
  // work-queue order: largest items first (planes x sites in the tile, plus
  // the 2R halo planes every item reads), ties in item order
  std::vector<double> cost(c.hitems.size());
  for (size_t w = 0; w < c.hitems.size(); ++w) {
    const BatchItem& it = c.hitems[w];
    const Solve* s = sv[it.solve];
    const int m = std::min(s->zc, s->g.nz - it.bz * s->zc);
    const int cols = std::min(32, s->g.nx - it.bx * 32), rows = std::min(s->tile_h, s->g.ny - it.by * s->tile_h);
    cost[w] = (double)(m + 2 * s->R) * cols * rows;
  }
  c.horder.resize(c.hitems.size());
  for (size_t w = 0; w < c.horder.size(); ++w) c.horder[w] = (int)w;
  std::stable_sort(c.horder.begin(), c.horder.end(), [&](int u, int v) { return cost[u] > cost[v]; });
  PCU(P, c.items.ensure(c.hitems.size()));
  PCU(P, c.order.ensure(c.horder.size()));
  PCU(P, c.queue.ensure(8));
  PCU(P, c.first.ensure(c.hfirst.size()));
  PCU(P, c.part.ensure(c.hitems.size() * RED_SLOTS));
  PCU(P, c.res.ensure(sv.size() * RED_SLOTS));
  PCU(P, c.hres.ensure(sv.size() * RED_SLOTS));
  PCU(P, cudaMemcpyAsync(c.items.p, c.hitems.data(), c.hitems.size() * sizeof(BatchItem), cudaMemcpyHostToDevice,
                         c.st));
  PCU(P, cudaMemcpyAsync(c.order.p, c.horder.data(), c.horder.size() * sizeof(int), cudaMemcpyHostToDevice, c.st));
  PCU(P, cudaMemcpyAsync(c.first.p, c.hfirst.data(), c.hfirst.size() * sizeof(int), cudaMemcpyHostToDevice, c.st));
  return GPE_OK;
}

int check_status(gpe_pool* P) {
  int st = 0;
  PCU(P, cudaMemcpy(&st, P->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    PCU(P, cudaMemset(P->d_status, 0, sizeof(int)));
    return pfail(P, GPE_ERR_TIMEOUT, "a batched stage kernel's bounded wait for its TMA copies expired");
  }
  return GPE_OK;
}

int ensure_stream(gpe_pool* P, Class& c) {
  if (!c.st) PCU(P, cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
  return GPE_OK;
}

// Capture one RK4 step of a class: the queue reset and four batched
// launches; with_norm: stage 4 reads table row 3 (norm on) and writes the
// partials, else row 4 (norm off) and no partials.
int capture_rk4_step(gpe_pool* P, Class& c, int cm, int ns, const int* grids, bool with_norm,
                     cudaGraph_t* graph, cudaGraphExec_t* gexec) {
  const int kinds[4] = {K_RK4_1, K_RK4_2, K_RK4_3, K_RK4_4};
  PCU(P, cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaMemsetAsync(c.queue.p, 0, 4 * sizeof(int), c.st);
  for (int m = 0; m < 4 && e == cudaSuccess; ++m) {
    const int row = (m == 3 && !with_norm) ? 4 : m;
    e = launch_batch(cm, kinds[m], grids[m], c.st,
                     BatchLaunch{c.tab.p + (size_t)row * ns, c.htab.p + (size_t)row * ns, ns, c.items.p, c.order.p,
                                 c.nitems, c.queue.p + m, (m == 3 && with_norm) ? c.part.p : nullptr},
                     nullptr);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(c.st, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return pfail(P, GPE_ERR_CUDA, std::string("capturing the batched RK4 step failed: ") +
                                      cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  *graph = g;
  PCU(P, cudaGraphInstantiate(gexec, g, 0));
  return GPE_OK;
}

// Enqueue `chunk` RK4 steps of every solve of an RK4 class on the class's
// stream (each step a captured graph of four batched launches; only the last
// one forms the per-solve norm of the result), then the norm's finalisation;
// returns without waiting.
int rk4_enqueue(gpe_pool* P, int cm, int64_t chunk) {
  Class& c = P->cls[cm][FAM_RK4];
  const int ns = (int)c.solves.size();
  if (int rc = ensure_stream(P, c)) return rc;
  if (c.dirty) {
    c.drop_graph();
    PCU(P, cudaStreamSynchronize(c.st));
    if (int rc = build_items(P, c, c.solves)) return rc;
    // table rows: stages 1-4, then stage 4 without the norm
    PCU(P, c.tab.ensure((size_t)5 * ns));
    PCU(P, c.htab.ensure((size_t)5 * ns));
    std::vector<BatchStage> t4(4);
    for (int q = 0; q < ns; ++q) {
      rk4_tables(P, c.solves[q], t4.data());
      for (int m = 0; m < 4; ++m) c.htab.p[(size_t)m * ns + q] = t4[m];
      BatchStage b = t4[3];
      b.args.want_norm = 0;
      c.htab.p[(size_t)4 * ns + q] = b;
    }
    for (size_t r = 0; r < (size_t)5 * ns; ++r) set_f32_constants(c.htab.p[r].args);
    PCU(P, cudaMemcpyAsync(c.tab.p, c.htab.p, (size_t)5 * ns * sizeof(BatchStage), cudaMemcpyHostToDevice, c.st));
    const int kinds[4] = {K_RK4_1, K_RK4_2, K_RK4_3, K_RK4_4};
    int grids[4];
    for (int m = 0; m < 4; ++m) grids[m] = grid_for(cm, kinds[m], c.nitems, ns);
    PCU(P, cudaStreamSynchronize(c.st));
    if (int rc = capture_rk4_step(P, c, cm, ns, grids, false, &c.graph, &c.gexec)) return rc;
    if (int rc = capture_rk4_step(P, c, cm, ns, grids, true, &c.graph_n, &c.gexec_n)) return rc;
    c.dirty = false;
  }
  for (int64_t q = 0; q + 1 < chunk; ++q) PCU(P, cudaGraphLaunch(c.gexec, c.st));
  if (chunk > 0) PCU(P, cudaGraphLaunch(c.gexec_n, c.st));
  k_finalize_ranges<<<ns, 256, 0, c.st>>>(c.part.p, c.first.p, c.res.p);
  PCU(P, cudaGetLastError());
  PCU(P, cudaMemcpyAsync(c.hres.p, c.res.p, (size_t)ns * RED_SLOTS * sizeof(double), cudaMemcpyDeviceToHost, c.st));
  return GPE_OK;
}

// After rk4_enqueue's work completed: advance the solves' clocks.
int rk4_collect(gpe_pool* P, int cm, int64_t chunk) {
  Class& c = P->cls[cm][FAM_RK4];
  PCU(P, cudaStreamSynchronize(c.st));
  for (size_t q = 0; q < c.solves.size(); ++q) {
    Solve* s = c.solves[q];
    for (int64_t k = 0; k < chunk; ++k) {
      s->t = s->t + s->dr;
      s->im_t = s->im_t + fabs(s->di);
    }
    s->p_index += chunk;
    s->done += chunk;
    s->norm = ((c.hres.p[q * RED_SLOTS + 0] * s->d[0]) * s->d[1]) * s->d[2];
    if (!std::isfinite(s->norm)) s->status = GPE_ERR_NONFINITE;
  }
  return GPE_OK;
}

// One RKF45 attempt of every solve of an RK45 class that still has quota,
// enqueued on the class's stream.  *launched = number of solves attempted.
int rk45_enqueue(gpe_pool* P, int cm, std::vector<Solve*>& sv) {
  Class& c = P->cls[cm][FAM_RK45];
  sv.clear();
  for (Solve* s : c.solves)
    if (s->quota > 0 && s->status == GPE_OK) sv.push_back(s);
  if (sv.empty()) return GPE_OK;
  if (int rc = ensure_stream(P, c)) return rc;
  const int ns = (int)sv.size();
  if (c.dirty || sv != c.built_for) {
    if (int rc = build_items(P, c, sv)) return rc;
    c.dirty = false;
  }
  PCU(P, c.tab.ensure((size_t)6 * ns));
  PCU(P, c.htab.ensure((size_t)6 * ns));
  std::vector<BatchStage> t6(6);
  for (int q = 0; q < ns; ++q) {
    rk45_tables(P, sv[q], t6.data());
    for (int m = 0; m < 6; ++m) c.htab.p[(size_t)m * ns + q] = t6[m];
  }
  for (size_t r = 0; r < (size_t)6 * ns; ++r) set_f32_constants(c.htab.p[r].args);
  PCU(P, cudaMemcpyAsync(c.tab.p, c.htab.p, (size_t)6 * ns * sizeof(BatchStage), cudaMemcpyHostToDevice, c.st));
  PCU(P, cudaMemsetAsync(c.queue.p, 0, 6 * sizeof(int), c.st));
  for (int m = 0; m < 6; ++m)
    PCU(P, launch_batch(cm, K_CK_1 + m, grid_for(cm, K_CK_1 + m, c.nitems, ns), c.st,
                        BatchLaunch{c.tab.p + (size_t)m * ns, c.htab.p + (size_t)m * ns, ns, c.items.p, c.order.p,
                                    c.nitems, c.queue.p + m, m == 5 ? c.part.p : nullptr},
                        nullptr));
  k_finalize_ranges<<<ns, 256, 0, c.st>>>(c.part.p, c.first.p, c.res.p);
  PCU(P, cudaGetLastError());
  PCU(P, cudaMemcpyAsync(c.hres.p, c.res.p, (size_t)ns * RED_SLOTS * sizeof(double), cudaMemcpyDeviceToHost, c.st));
  // the status word comes back with the error norms: an attempt whose
  // bounded waits expired has no usable error norm to act on
  PCU(P, c.hstatus.ensure(1));
  PCU(P, cudaMemcpyAsync(c.hstatus.p, P->d_status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  return GPE_OK;
}

// rkqs step control (src/solve.f90:184-229) of each attempted solve.
int rk45_collect(gpe_pool* P, int cm, const std::vector<Solve*>& sv) {
  Class& c = P->cls[cm][FAM_RK45];
  PCU(P, cudaStreamSynchronize(c.st));
  if (c.hstatus.p[0] != 0) {
    // the attempt did not complete: these solves stop here (retired with
    // GPE_ERR_TIMEOUT by gpe_pool_step)
    for (Solve* s : sv) s->status = GPE_ERR_TIMEOUT;
    return GPE_OK;
  }
  for (size_t q = 0; q < sv.size(); ++q) {
    Solve* s = sv[q];
    const gpe_params& p = s->p;
    const double eps = p.eps != 0 ? p.eps : 1e-6, safety = p.safety != 0 ? p.safety : 0.9;
    const double dtdec = p.dt_decrease != 0 ? p.dt_decrease : -0.25;
    const double dtinc = p.dt_increase != 0 ? p.dt_increase : -0.2;
    const double errcon = pow(5.0 / safety, 1.0 / dtinc);
    const double errmax = c.hres.p[q * RED_SLOTS + 2] / eps;
    if (!std::isfinite(errmax)) {
      s->status = GPE_ERR_NONFINITE;
      continue;
    }
    if (errmax > 1.0) {  // reject: shrink and retry from the same psi
      s->rejected++;
      if (s->rejected > 100000) s->status = GPE_ERR_STATE;
      const double e = pow(errmax, dtdec);
      const double tr = (safety * s->dr) * e, ti = (safety * s->di) * e;
      const double mm = std::max(hypot(tr, ti), 0.1 * hypot(s->dr, s->di));
      if (!(s->di == 0.0)) { s->dr = 0.0; s->di = -mm; }  // imaginary time: dt on the negative imaginary axis
      else { s->dr = mm; s->di = 0.0; }
      continue;
    }
    double nr, ni;
    if (errmax > errcon) {
      const double e = pow(errmax, dtinc);
      nr = (safety * s->dr) * e;
      ni = (safety * s->di) * e;
    } else {
      nr = 5.0 * s->dr;
      ni = 5.0 * s->di;
    }
    s->t = s->t + s->dr;
    s->dr = nr;
    s->di = ni;
    s->im_t = s->im_t + fabs(ni);  // the new dt, as src/solve.f90:229
    s->errmax = errmax;
    s->cur = 1 - s->cur;
    s->p_index += 1;
    s->done += 1;
    s->quota -= 1;
    s->dte_r = s->dr;  // next step's psi_scal uses the dt at rkqs entry
    s->dte_i = s->di;
    s->norm = ((c.hres.p[q * RED_SLOTS + 0] * s->d[0]) * s->d[1]) * s->d[2];
  }
  return GPE_OK;
}

void release_solve(gpe_pool* P, Solve* s) {
  P->alloc.release(s->off, s->bytes);
  delete s;
}

}  // namespace

extern "C" {

int gpe_pool_create(int64_t budget_bytes, gpe_pool** out) {
  if (!out || budget_bytes <= 0) return GPE_ERR_BADARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GPE_ERR_CUDA;
  gpe_pool* P = new gpe_pool();
  cudaGetDevice(&P->dev);
  P->t0 = std::chrono::steady_clock::now();
  if (cudaStreamCreateWithFlags(&P->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&P->d_status, sizeof(int)) != cudaSuccess) {
    gpe_pool_destroy(P);
    return GPE_ERR_CUDA;
  }
  if (cudaMalloc(&P->arena, (size_t)budget_bytes) != cudaSuccess) {
    cudaGetLastError();
    gpe_pool_destroy(P);
    return GPE_ERR_NOMEM;
  }
  P->arena_bytes = (size_t)budget_bytes;
  P->alloc.init(P->arena_bytes);
  cudaMemset(P->d_status, 0, sizeof(int));
  *out = P;
  return GPE_OK;
}

int64_t gpe_pool_solve_bytes(const gpe_params* p) {
  std::string why;
  if (validate_params(p, why)) return -1;
  Geom g;
  int esz;
  param_layout(p, g, esz);
  const size_t fb = Arena::round((size_t)padded_elems(g) * esz);
  return (int64_t)(fb * scheme_fields(p->scheme) + Arena::round(tables_bytes(*p)));
}

static int pool_submit_impl(gpe_pool* P, const gpe_params* prm, const void* psi0, int32_t dtype,
                            const gpe_ic* icspec, int64_t nsteps, uint64_t tag, void* psi_out) {
  if (!P || !prm || !psi_out || nsteps < 0 || (!psi0 && !icspec)) return pfail(P, GPE_ERR_BADARG, "null argument");
  std::string why;
  if (int rc = validate_params(prm, why)) return pfail(P, rc, why);
  if (icspec)
    if (int rc = ic_validate(icspec, why)) return pfail(P, rc, why);
  if (prm->scheme != GPE_RK4 && prm->scheme != GPE_RK45)
    return pfail(P, GPE_ERR_BADARG, "the pool runs RK4 and RK45 solves");
  const int want = prm->storage == GPE_C128 ? GPE_C128 : GPE_C64;
  if (psi0 && dtype != want)
    return pfail(P, GPE_ERR_BADARG, "psi0/psi_out element type must match the solve's storage");
  PCU(P, cudaSetDevice(P->dev));
  Solve* s = new Solve();
  s->tag = tag;
  s->p = *prm;
  param_layout(prm, s->g, s->esz);
  s->R = prm->order / 2;
  s->cmode = cmode_of(*prm);
  s->fam = prm->scheme == GPE_RK45 ? FAM_RK45 : FAM_RK4;
  s->nf = scheme_fields(prm->scheme);
  // z planes per work item: the caller's (autotuned) choice, else a batch
  // default of up to 64 planes.  In a batch the other solves fill the GPU,
  // so items can be long (fewer z-halo re-reads and queue fills per plane)
  // instead of many: on the uneven 32^3-160^3 mix 64 beats 32, 48, 96 and
  // 128 (44.2 against 42.1-43.8 G site-updates/s).
  s->zc = prm->tile_zc > 0 ? std::min(prm->tile_zc, prm->nz) : std::min(prm->nz, 64);
  s->tile_h = batch_rows(s->cmode, s->fam);
  s->ntx = (prm->nx + 31) / 32;
  s->nty = (prm->ny + s->tile_h - 1) / s->tile_h;
  s->ntz = (prm->nz + s->zc - 1) / s->zc;
  s->field_bytes = Arena::round((size_t)padded_elems(s->g) * s->esz);
  s->bytes = s->field_bytes * s->nf + Arena::round(tables_bytes(*prm));
  if (!P->alloc.alloc(s->bytes, &s->off)) {
    const size_t need = s->bytes, have = P->alloc.free_bytes();
    delete s;
    return pfail(P, GPE_ERR_NOMEM_BUDGET, "pool budget: solve needs " + std::to_string(need) + " B, " +
                                               std::to_string(have) + " B free");
  }
  char* base = P->arena + s->off;
  for (int f = 0; f < s->nf; ++f) s->f[f] = base + (size_t)f * s->field_bytes;
  s->tables = (double*)(base + (size_t)s->nf * s->field_bytes);
  auto bail = [&](int rc, const std::string& m) {
    release_solve(P, s);
    return pfail(P, rc, m);
  };
  for (int f = 0; f < s->nf; ++f)
    if (!encode_maps(s->f[f], s->g, s->esz, s->R, &s->halo[f], &s->pw[f], s->tile_h))
      return bail(GPE_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  std::vector<double> tab;
  std::vector<double> xs, ys, zs;
  std::vector<double>* xyz[3] = {&xs, &ys, &zs};
  build_axis_tables(*prm, tab, xyz, s->d);
  if (cudaMemsetAsync(base, 0, (size_t)s->nf * s->field_bytes, P->st) != cudaSuccess ||
      cudaMemcpyAsync(s->tables, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, P->st) !=
          cudaSuccess)
    return bail(GPE_ERR_CUDA, "upload of tables failed");
  if (psi0) {
    if (int rc = upload_state(P, s, psi0, 0)) return bail(rc, P->err);
  } else {
    // the other fields are free until the first step: the generator's
    // scratch (spectrum + FFT) lives there
    const size_t wb = ic_work_bytes(*prm, *icspec);
    const size_t room = (size_t)(s->nf - 1) * s->field_bytes;
    if (wb > room) return bail(GPE_ERR_BADARG, "initial-condition scratch does not fit in the solve's fields");
    if (ic_generate(*prm, s->g, s->esz, s->R, *icspec, s->f[0], s->f[1], room, P->st) != cudaSuccess)
      return bail(GPE_ERR_CUDA, "device initial condition failed");
  }
  if (cudaStreamSynchronize(P->st) != cudaSuccess) return bail(GPE_ERR_CUDA, "state upload failed");
  if (prm->real_time) { s->dr = prm->tau; s->di = 0.0; }
  else { s->dr = 0.0; s->di = -prm->tau; }
  s->dte_r = s->dr;
  s->dte_i = s->di;
  s->nsteps = nsteps;
  s->out = psi_out;
  s->t_submit = now_s(P->t0);
  P->pending.push_back(s);
  return GPE_OK;
}

int gpe_pool_submit(gpe_pool* P, const gpe_params* prm, const void* psi0, int32_t dtype, int64_t nsteps,
                    uint64_t tag, void* psi_out) {
  if (!psi0) return pfail(P, GPE_ERR_BADARG, "null psi0");
  return pool_submit_impl(P, prm, psi0, dtype, nullptr, nsteps, tag, psi_out);
}

int gpe_pool_submit_ic(gpe_pool* P, const gpe_params* prm, const gpe_ic* ic, int64_t nsteps, uint64_t tag,
                       void* psi_out) {
  if (!ic) return pfail(P, GPE_ERR_BADARG, "null initial-condition spec");
  return pool_submit_impl(P, prm, nullptr, 0, ic, nsteps, tag, psi_out);
}

int gpe_pool_step(gpe_pool* P, int64_t max_steps, int32_t* n_active) {
  if (!P || max_steps < 0) return GPE_ERR_BADARG;
  PCU(P, cudaSetDevice(P->dev));
  // continuous batching: solves submitted since the last step join now
  for (Solve* s : P->pending) {
    s->t_start = now_s(P->t0);
    Class& c = P->cls[class_of(s->cmode, s->R)][s->fam];
    c.solves.push_back(s);
    c.dirty = true;
  }
  P->pending.clear();
  // RK4 classes: enqueue their chunk on their own streams and let them run
  // while the RKF45 classes go through their attempts
  int64_t chunks[NCLS] = {0};
  for (int cm = 0; cm < NCLS; ++cm) {
    Class& c = P->cls[cm][FAM_RK4];
    int64_t chunk = max_steps;
    for (Solve* s : c.solves) chunk = std::min(chunk, s->nsteps - s->done);
    if (!c.solves.empty() && chunk > 0) {
      if (int rc = rk4_enqueue(P, cm, chunk)) return rc;
      chunks[cm] = chunk;
    }
  }
  for (int cm = 0; cm < NCLS; ++cm)
    for (Solve* s : P->cls[cm][FAM_RK45].solves) {
      s->quota = std::min(max_steps, s->nsteps - s->done);
      s->dte_r = s->dr;
      s->dte_i = s->di;
    }
  for (int round = 0; round < 1000000; ++round) {
    std::vector<Solve*> sv[NCLS];
    bool any = false;
    for (int cm = 0; cm < NCLS; ++cm) {
      if (int rc = rk45_enqueue(P, cm, sv[cm])) return rc;
      any |= !sv[cm].empty();
    }
    if (!any) break;
    for (int cm = 0; cm < NCLS; ++cm)
      if (!sv[cm].empty())
        if (int rc = rk45_collect(P, cm, sv[cm])) return rc;
  }
  for (int cm = 0; cm < NCLS; ++cm)
    if (chunks[cm])
      if (int rc = rk4_collect(P, cm, chunks[cm])) return rc;
  // a stage kernel whose bounded waits expired left the status word set: the
  // solves of this step have states that cannot be trusted, so they are
  // retired with GPE_ERR_TIMEOUT (their results say so) and the call reports
  // the error; the pool itself stays usable
  const int timeout_rc = check_status(P);
  if (timeout_rc == GPE_ERR_TIMEOUT)
    for (int cm = 0; cm < NCLS; ++cm)
      for (int fam = 0; fam < NFAM; ++fam)
        for (Solve* s : P->cls[cm][fam].solves) s->status = GPE_ERR_TIMEOUT;
  else if (timeout_rc)
    return timeout_rc;
  // retire finished solves
  int active = 0;
  for (int cm = 0; cm < NCLS; ++cm)
    for (int fam = 0; fam < NFAM; ++fam) {
      Class& c = P->cls[cm][fam];
      std::vector<Solve*> keep, fin;
      bool retired = false;
      for (Solve* s : c.solves) {
        if (s->done < s->nsteps && s->status == GPE_OK) {
          keep.push_back(s);
          continue;
        }
        // all finished states go down back to back, one synchronisation
        if (int rc = download_state(P, s, s->fam == FAM_RK45 ? s->cur : 0)) return rc;
        fin.push_back(s);
      }
      if (!fin.empty()) PCU(P, cudaStreamSynchronize(P->st));
      for (Solve* s : fin) {
        gpe_result r;
        memset(&r, 0, sizeof(r));
        r.tag = s->tag;
        r.status = s->status;
        r.steps = s->done;
        r.rejected = s->rejected;
        r.t = s->t;
        r.im_t = s->im_t;
        r.dt_re = s->dr;
        r.dt_im = s->di;
        r.norm = s->norm;
        r.submit_s = s->t_submit;
        r.start_s = s->t_start;
        r.finish_s = now_s(P->t0);
        P->done.push_back(r);
        release_solve(P, s);
        retired = true;
      }
      if (retired) {
        c.solves.swap(keep);
        c.dirty = true;
      }
      active += (int)c.solves.size();
    }
  if (n_active) *n_active = active;
  return timeout_rc;
}

int gpe_pool_test_expire_waits(gpe_pool* P) {
  if (!P) return GPE_ERR_BADARG;
  PCU(P, cudaSetDevice(P->dev));
  PCU(P, cudaDeviceSynchronize());
  const int v = STATUS_EXPIRE_TEST;
  PCU(P, cudaMemcpy(P->d_status, &v, sizeof(int), cudaMemcpyHostToDevice));
  return GPE_OK;
}

int gpe_pool_poll(gpe_pool* P, gpe_result* out, int32_t max, int32_t* n_out) {
  if (!P || (!out && max > 0)) return GPE_ERR_BADARG;
  int n = 0;
  while (n < max && !P->done.empty()) {
    out[n++] = P->done.front();
    P->done.pop_front();
  }
  if (n_out) *n_out = n;
  return GPE_OK;
}

int64_t gpe_pool_free_bytes(const gpe_pool* P) { return P ? (int64_t)P->alloc.free_bytes() : -1; }

void* gpe_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0 || cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void gpe_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

const char* gpe_pool_last_error(const gpe_pool* P) { return P ? P->err.c_str() : ""; }

void gpe_pool_destroy(gpe_pool* P) {
  if (!P) return;
  cudaSetDevice(P->dev);
  if (P->st) cudaStreamSynchronize(P->st);
  for (Solve* s : P->pending) delete s;
  for (int cm = 0; cm < NCLS; ++cm)
    for (int fam = 0; fam < NFAM; ++fam) {
      Class& c = P->cls[cm][fam];
      for (Solve* s : c.solves) delete s;
      c.drop_graph();
      if (c.st) {
        cudaStreamSynchronize(c.st);
        cudaStreamDestroy(c.st);
      }
      c.tab.free();
      c.items.free();
      c.order.free();
      c.queue.free();
      c.first.free();
      c.part.free();
      c.res.free();
      c.htab.free();
      c.hres.free();
      c.hstatus.free();
    }
  if (P->arena) cudaFree(P->arena);
  if (P->d_status) cudaFree(P->d_status);
  if (P->st) cudaStreamDestroy(P->st);
  delete P;
}

}  // extern "C"

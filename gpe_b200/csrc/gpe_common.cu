// Host-side helpers shared by the single-solve handle (gpe_capi.cu) and the
// batched pool (gpe_pool.cu): parameter validation, HBM layout, per-axis
// tables, tensor-map encoding and the stage-argument template.
#include "gpe_common.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace gpe {

const double CK_B[5][5] = {
    {0.2, 0, 0, 0, 0},
    {0.075, 0.225, 0, 0, 0},
    {0.3, -0.9, 1.2, 0, 0},
    {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0},
};

int validate_params(const gpe_params* p, std::string& why) {
  if (!p) { why = "null parameters"; return GPE_ERR_BADARG; }
  if (p->nx < 6 || p->ny < 6 || p->nz < 6) { why = "nx, ny, nz must be >= 6"; return GPE_ERR_BADARG; }
  if (p->scheme < GPE_EULER || p->scheme > GPE_RK45) {
    why = "ERROR: Unrecognised time stepping scheme.";  // src/solve.f90:49
    return GPE_ERR_BADARG;
  }
  if (p->eqn < 1 || p->eqn > 4) { why = "eqn_to_solve must be 1..4"; return GPE_ERR_BADARG; }
  if (p->bcs != 1 && p->bcs != 2) { why = "bcs must be 1 (periodic) or 2 (reflective)"; return GPE_ERR_BADARG; }
  if (p->order != 2 && p->order != 4) { why = "order must be 2 or 4"; return GPE_ERR_BADARG; }
  if (p->storage != GPE_C128 && p->storage != GPE_C64) { why = "storage must be GPE_C128 or GPE_C64"; return GPE_ERR_BADARG; }
  if (!(p->xr > 0 && p->yr > 0 && p->zr > 0)) { why = "xr, yr, zr must be > 0"; return GPE_ERR_BADARG; }
  if (!(p->tau > 0) || !std::isfinite(p->tau)) { why = "tau must be > 0"; return GPE_ERR_BADARG; }
  if (p->tile_zc < 0) { why = "tile_zc must be >= 0"; return GPE_ERR_BADARG; }
  return GPE_OK;
}

void param_layout(const gpe_params* p, Geom& g, int& esz) {
  esz = p->storage == GPE_C128 ? 16 : 8;
  g.nx = p->nx;
  g.ny = p->ny;
  g.nz = p->nz;
  g.xoff = 128 / esz;
  const long long need = g.xoff + (long long)p->nx + 2;
  g.px = (need + g.xoff - 1) / g.xoff * g.xoff;
  g.pz = (long long)(p->ny + 4) * g.px;
}

long long padded_elems(const Geom& g) { return (long long)(g.nz + 4) * g.pz; }

int scheme_fields(int scheme) {
  switch (scheme) {
    case GPE_EULER: return 2;
    case GPE_RK2: return 2;
    case GPE_RK4: return 4;
    default: return 9;  // psi, psi_new, A, B, K1..K5
  }
}

// z planes per block: enough blocks for several waves on 148 SMs
int default_zc(const Geom& g, int tile_h, int esz) {
  if (const char* e = getenv("GPE_ZC")) {
    int v = atoi(e);
    if (v > 0) return std::min(v, g.nz);
  }
  // at most 24 planes per CTA for complex128 sites (32x8 tiles) and 20 for
  // complex64 (32x16 two-sites-per-thread tiles): at 256^3, sweeps of
  // 16..43 planes give these the best rates (complex128: 24 is +0.7 % over
  // 20 and 29, +3 % over 32; complex64: 20 is +1 % over 29, +2.4 % over 16,
  // +3.4 % over 24); small grids use fewer so that every SM gets several
  // CTAs.
  const long long bxy = (long long)((g.nx + 31) / 32) * ((g.ny + tile_h - 1) / tile_h);
  const long long target = 148LL * 8;
  const long long cap = esz >= 16 ? 24 : 20;
  long long zc = (g.nz * bxy + target - 1) / target;
  zc = std::max<long long>(4, std::min<long long>(zc, cap));
  return (int)std::min<long long>(zc, g.nz);
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// Tensor maps of one ghost-padded field: rank 3 over (x scalars, ny+4 rows,
// nz+4 planes); box = halo'd stencil tile or plain point-wise tile.  The x
// extent ends at the last column a box's consumer can use -- the ghost
// column x = nx+1 for the stencil, x = nx-1 for point-wise tiles -- so the
// TMA unit zero-fills the rest of a partial tile instead of reading the
// row padding from HBM (only lanes outside the grid see those zeros).  No
// L2 sector promotion: a box row is fetched as the sectors it covers.
bool encode_maps(void* base, const Geom& g, int esz, int R, CUtensorMap* halo, CUtensorMap* pw, int tile_h) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const CUtensorMapDataType dt = esz == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims_h[3] = {(cuuint64_t)(2 * (g.xoff + g.nx + 2)), (cuuint64_t)(g.ny + 4), (cuuint64_t)(g.nz + 4)};
  const cuuint64_t dims_p[3] = {(cuuint64_t)(2 * (g.xoff + g.nx)), (cuuint64_t)(g.ny + 4), (cuuint64_t)(g.nz + 4)};
  const cuuint64_t strides[2] = {(cuuint64_t)(g.px * esz), (cuuint64_t)(g.pz * esz)};
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t box_h[3] = {(cuuint32_t)(2 * tma_stencil_w()), (cuuint32_t)tma_stencil_h(tile_h, R), 1};
  const cuuint32_t box_p[3] = {(cuuint32_t)(2 * TMA_TX), (cuuint32_t)tile_h, 1};
  if (enc(halo, dt, 3, base, dims_h, strides, box_h, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  if (enc(pw, dt, 3, base, dims_p, strides, box_p, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  return true;
}

// algorithmic HBM traffic of one launch of a stage kind, in field elements
// per site: one read of every input field and one write of every output
// field (stencil neighbours come from on-chip reuse)
int kind_elems(int kind) {
  switch (kind) {
    case K_EULER: return 2;
    case K_RK2_1: return 2;
    case K_RK2_2: return 3;
    case K_RK4_1: return 2;
    case K_RK4_2: return 4;
    case K_RK4_3: return 3;
    case K_RK4_4: return 3;
    case K_CK_1: return 3;
    case K_CK_2: return 5;
    case K_CK_3: return 6;
    case K_CK_4: return 7;
    case K_CK_5: return 8;
    case K_CK_6: return 7;
    case K_ENERGY: return 1;
    default: return 0;
  }
}

// host tables and grid (src/ic.f90:32-69, solve.f90:397-409, ic.f90:713-731,
// variables.f90:49-51 + 730-840)
void build_axis_tables(const gpe_params& p, std::vector<double>& t, std::vector<double>* c[3], double d_out[3]) {
  const int n[3] = {p.nx, p.ny, p.nz};
  const double r[3] = {p.xr, p.yr, p.zr};
  const double om[3] = {p.omx, p.omy, p.omz};
  double dd[3];
  double* d[3] = {&dd[0], &dd[1], &dd[2]};
  const double QC1 = 3.0 / 8.0, QC2 = 7.0 / 6.0, QC3 = 23.0 / 24.0;
  const size_t ntot = (size_t)p.nx + p.ny + p.nz;
  t.assign(ntot * 4, 0.0);
  size_t off = 0;
  for (int ax = 0; ax < 3; ++ax) {
    const double lo = -r[ax];
    *d[ax] = (r[ax] - lo) / (n[ax] - 1);
    c[ax]->resize(n[ax]);
    for (int q = 0; q < n[ax]; ++q) (*c[ax])[q] = lo + (double)q * *d[ax];
    const double a = (*c[ax])[n[ax] - 3];
    for (int q = 0; q < n[ax]; ++q) {
      const double xq = (*c[ax])[q];
      t[0 * ntot + off + q] = (om[ax] * om[ax]) * (xq * xq);
      t[1 * ntot + off + q] = 1.0 + tanh(xq - a) * tanh(xq + a);
      double w = 1.0;
      if (q == 0) w = QC1;
      if (q == 1) w = QC2;
      if (q == 2) w = QC3;
      if (q == n[ax] - 3) w = QC3;
      if (q == n[ax] - 2) w = QC2;
      if (q == n[ax] - 1) w = QC1;
      t[2 * ntot + off + q] = w;
      t[3 * ntot + off + q] = xq;
    }
    off += n[ax];
  }
  for (int ax = 0; ax < 3; ++ax) d_out[ax] = dd[ax];
}

StageArgs make_base_args(const gpe_params& p, const Geom& g, int R, int zc, const double d[3], const double* tables) {
  StageArgs a;
  memset(&a, 0, sizeof(a));
  a.g = g;
  a.R = R;
  a.bcs = p.bcs;
  a.eqn = p.eqn;
  a.zc = zc;
  a.has_urhs = (p.Urhs != 0.0) && p.eqn != 4;
  a.has_diss = (p.diss_amp != 0.0) && (p.eqn == 1 || p.eqn == 3);
  a.eqn4_plain = p.eqn == 4 && p.omx == 0.0 && p.omy == 0.0 && p.omz == 0.0 && p.gamma == 0.0;
  const double dx2 = d[0] * d[0], dy2 = d[1] * d[1], dz2 = d[2] * d[2];
  if (p.order == 2) {
    a.ixx = 1.0 / dx2;
    a.iyy = 1.0 / dy2;
    a.izz = 1.0 / dz2;
    a.ix1 = 1.0 / (2.0 * d[0]);
  } else {
    a.ixx = 1.0 / (12.0 * dx2);
    a.iyy = 1.0 / (12.0 * dy2);
    a.izz = 1.0 / (12.0 * dz2);
    a.ix1 = 1.0 / (12.0 * d[0]);
  }
  a.zghost = 3;
  a.g_nl = p.g;
  a.mu = p.mu;
  a.gamma = p.eqn == 4 ? p.gamma : 0.0;
  a.urhs = p.Urhs;
  a.diss_amp = p.diss_amp;
  const size_t ntot = (size_t)p.nx + p.ny + p.nz;
  const double* T = tables;
  const double* blk[4] = {T, T + ntot, T + 2 * ntot, T + 3 * ntot};
  a.vx = blk[0];
  a.vy = blk[0] + p.nx;
  a.vz = blk[0] + p.nx + p.ny;
  a.sx = blk[1];
  a.sy = blk[1] + p.nx;
  a.sz = blk[1] + p.nx + p.ny;
  a.wx = blk[2];
  a.wy = blk[2] + p.nx;
  a.wz = blk[2] + p.nx + p.ny;
  a.cx = blk[3];
  a.cy = blk[3] + p.nx;
  a.cz = blk[3] + p.nx + p.ny;
  return a;
}

}  // namespace gpe

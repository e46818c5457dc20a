// Host-side helpers shared by the single-solve handle and the batched pool.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <string>
#include <vector>

#include "../../include/gpe_cuda.h"
#include "gpe_device.cuh"
#include "gpe_stage_tma.cuh"

namespace gpe {

// Cash-Karp tableau b_ij (src/solve.f90:255-269)
extern const double CK_B[5][5];

// argument checks of gpe_create (message in why)
int validate_params(const gpe_params* p, std::string& why);
// ghost-padded layout of one field; esz = bytes per complex element
void param_layout(const gpe_params* p, Geom& g, int& esz);
long long padded_elems(const Geom& g);
// fields a scheme keeps per solve
int scheme_fields(int scheme);
// z planes per CTA / work item
int default_zc(const Geom& g, int tile_h = 8, int esz = 16);
// tensor maps of one field: halo'd stencil box and point-wise box of a
// 32 x tile_h tile
bool encode_maps(void* base, const Geom& g, int esz, int R, CUtensorMap* halo, CUtensorMap* pw, int tile_h = 8);
// algorithmic field elements moved per site by one launch of a stage kind
int kind_elems(int kind);
// per-axis tables [vx|vy|vz, sx|sy|sz, wx|wy|wz, x|y|z] and grid spacings
void build_axis_tables(const gpe_params& p, std::vector<double>& t, std::vector<double>* xyz[3], double d[3]);
// stage arguments common to all stages of a solve (tables on the device)
StageArgs make_base_args(const gpe_params& p, const Geom& g, int R, int zc, const double d[3], const double* tables);

}  // namespace gpe

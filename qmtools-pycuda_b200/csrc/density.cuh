// Density path internals shared between the SIMT and tensor-core translation units.
#pragma once

#include "mol.cuh"

namespace qmt {

qmt_status make_point_map(int nx, int ny, int nz, float step, float ox, float oy, float oz,
                          int subgrid, int tile_rows, PointMap& pm, int64_t& ntiles);

qmt_status finish_density(qmt_mol* mol, int64_t nvox, int64_t ntiles, int rescale, float* qube,
                          double* sum_out, cudaStream_t s);

qmt_status density_tc(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                      float oz, int subgrid, int precision, int rescale, float* qube,
                      double* sum_out, cudaStream_t s);

}  // namespace qmt

// Shared definitions for libqmtools_b200: status handling, molecule layout on the
// device, and the basis-function evaluation used by every density kernel.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

#include "qmtools_b200.h"

namespace qmt {

// ---- status ------------------------------------------------------------------------
void set_error(const std::string& msg);
qmt_status fail(qmt_status code, const std::string& msg);
qmt_status cuda_fail(cudaError_t e, const char* what);

#define QMT_CUDA(call)                                              \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) return ::qmt::cuda_fail(e_, #call);      \
  } while (0)

// Every kernel launch of the library is followed by this check, which also counts it
// (qmt_launch_count); a call site that launches twice before one check adds the extra launch
// with note_launches.
#define QMT_CHECK_LAUNCH(what)                                      \
  do {                                                              \
    ::qmt::note_launches(1);                                        \
    cudaError_t e_ = cudaGetLastError();                            \
    if (e_ != cudaSuccess) return ::qmt::cuda_fail(e_, what);       \
  } while (0)

void note_launches(uint64_t n);
// Limit of the kernels' bounded waits on barriers (ns); qmt_set_wait_limit_ns changes it.
uint64_t wait_limit_ns();

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr double ANG2BOR = 1.8897259886;   // kernel_common.h:1
constexpr int MAXAOC = 20;                 // kernel_common.h:10
constexpr int MAX_L = 2;

// Real solid harmonics times r^l (the reference's constants, kernel_density.cu:17-28).
constexpr double YS = 0.28209479177387814;
constexpr double YP = 0.4886025119029199;
constexpr double YD1 = 1.0925484305920792;
constexpr double YD0 = 0.31539156525252005;
constexpr double YD2 = 0.5462742152960396;

// One contracted shell.  Functions of a shell are contiguous in the basis order and
// follow the reference's m order (qmtools/qmtools.py:52): p = (z, x, y),
// d = (2zz-xx-yy, xz, yz, xx-yy, xy).
struct Shell {
  int atom;
  int L;
  int nprim;
  int prim;    // offset into the primitive arrays
  int func;    // first basis function
  int same_exp;  // 1: same atom and the same exponents (at most 8) as the shell before it
  int pad[2];
};

// ---- device-side molecule view --------------------------------------------------------
struct MolView {
  int natoms;
  int nshells;
  int norbs;
  int npad;                  // norbs rounded up for GEMM operands
  const float* coords;       // [natoms*3] bohr
  const int* types;          // [natoms]
  const Shell* shells;       // [nshells]
  const int* atom_shell;     // [natoms+1]
  const float* alpha;        // [nprim_total]
  const float* coeff;        // [nprim_total]
  const double* alpha64;
  const double* coeff64;
};

// Primitive screening: a primitive with alpha r^2 above the cut contributes less than
// exp(-cut) of its contraction coefficient and is skipped -- 1.4e-11 for the FP32 paths
// (far below FP32 round-off), 4e-18 for FP64.  A warp skips the exponential when all of
// its points are beyond the cut.
constexpr float kExpCut = 25.0f;
constexpr double kExpCut64 = 40.0;

// Writes the values of the shell's functions at displacement (dx,dy,dz) from its atom
// into out[0..2L].  T = float or double.
template <typename T>
__device__ __forceinline__ int shell_values(const Shell& sh, const T* __restrict__ al,
                                            const T* __restrict__ co, T dx, T dy, T dz,
                                            T* out) {
  const T r2 = dx * dx + dy * dy + dz * dz;
  T rad = T(0);
  for (int k = 0; k < sh.nprim; ++k) {
    const T e = al[sh.prim + k] * r2;
    if (e < (sizeof(T) == 8 ? T(kExpCut64) : T(kExpCut))) rad += co[sh.prim + k] * exp(-e);
  }
  if (sh.L == 0) {
    out[0] = T(YS) * rad;
    return 1;
  }
  if (sh.L == 1) {
    const T c = T(YP) * rad;
    out[0] = c * dz;
    out[1] = c * dx;
    out[2] = c * dy;
    return 3;
  }
  const T c1 = T(YD1) * rad;
  out[0] = T(YD0) * rad * (T(2) * dz * dz - dx * dx - dy * dy);
  out[1] = c1 * dx * dz;
  out[2] = c1 * dz * dy;
  out[3] = T(YD2) * rad * (dx * dx - dy * dy);
  out[4] = c1 * dx * dy;
  return 5;
}

// Points of a density tile.  With subgrid 1 (128 voxels per tile) a tile is an 8 x 4 x 4 block
// of voxels (row v -> x + (v & 7), y + ((v >> 3) & 3), z + (v >> 5)), so that the rows of a work
// item are close together and primitive screening over them skips more; otherwise voxels are
// taken in flat x-fastest order, `vpt` per tile.  Each voxel has s^3 sub-points (sub-point index
// fastest within the voxel's rows).
struct PointMap {
  int nx, ny, nz;
  int s;          // subgrid
  int s3;
  int vpt;        // voxels per tile
  int64_t nvox;
  float h;
  float ox, oy, oz;
  double inv_s;   // 1 / s
  int blocked;    // 8 x 4 x 4 voxel blocks (vpt == 128)
  int nbx, nby;   // blocks along x and y
};

// Voxel v (< vpt) of `tile`: grid indices and flat x-fastest index; false outside the grid.
__device__ __forceinline__ bool tile_voxel(const PointMap& pm, int64_t tile, int v, int64_t& vox, int64_t& ix,
                                           int64_t& iy, int64_t& iz) {
  if (v >= pm.vpt) return false;
  if (pm.blocked) {
    const uint32_t tt = (uint32_t)tile;   // fewer than 2^31 tiles (checked on the host)
    const uint32_t q1 = tt / (uint32_t)pm.nbx, bz = q1 / (uint32_t)pm.nby;
    const uint32_t bx = tt - q1 * (uint32_t)pm.nbx, by = q1 - bz * (uint32_t)pm.nby;
    ix = (int64_t)(bx * 8 + (v & 7));
    iy = (int64_t)(by * 4 + ((v >> 3) & 3));
    iz = (int64_t)(bz * 4 + (v >> 5));
    if (ix >= pm.nx || iy >= pm.ny || iz >= pm.nz) return false;
    vox = ix + (int64_t)pm.nx * (iy + (int64_t)pm.ny * iz);
    return true;
  }
  vox = tile * pm.vpt + v;
  if (vox >= pm.nvox) return false;
  if (pm.nvox <= 0x7fffffffLL) {   // 32-bit index arithmetic (exact, several times cheaper)
    const uint32_t vv = (uint32_t)vox, nx = (uint32_t)pm.nx, ny = (uint32_t)pm.ny;
    const uint32_t qy = vv / nx, qz = qy / ny;
    ix = vv - qy * nx;
    iy = qy - qz * ny;
    iz = qz;
  } else {
    ix = vox % pm.nx;
    iy = (vox / pm.nx) % pm.ny;
    iz = vox / ((int64_t)pm.nx * pm.ny);
  }
  return true;
}

template <typename T>
__device__ __forceinline__ bool tile_point(const PointMap& pm, int64_t tile, int row,
                                           T& x, T& y, T& z, int64_t& vox) {
  int v = row, sub = 0;
  if (pm.s3 > 1) {
    v = row / pm.s3;
    sub = row - v * pm.s3;
  }
  int64_t ix, iy, iz;
  if (!tile_voxel(pm, tile, v, vox, ix, iy, iz)) return false;
  int sx = 0, sy = 0, sz = 0;
  if (pm.s > 1) {
    sx = sub % pm.s;
    sy = (sub / pm.s) % pm.s;
    sz = sub / (pm.s * pm.s);
  }
  const T inv = T(pm.inv_s);
  const T h = T(pm.h);
  x = T(pm.ox) + (T(ix) + (T(sx) + T(0.5)) * inv) * h;
  y = T(pm.oy) + (T(iy) + (T(sy) + T(0.5)) * inv) * h;
  z = T(pm.oz) + (T(iz) + (T(sz) + T(0.5)) * inv) * h;
  return true;
}

}  // namespace qmt

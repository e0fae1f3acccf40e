// Electron density on voxel grids: the SIMT contraction (FP32 plain path and FP64),
// the FP64 charge sum and the qtot rescale, and the qmt_density entry point that
// dispatches to the tensor-core path for the mixed precisions.
//
// Algorithm (replaces gpu_densityqube_shmem_subgrid, kernel_density.cu:34-155, which
// re-evaluates phi_p, phi_q for every DM pair at every voxel): a tile of TP sample points
// evaluates Phi[TP, N] once into shared memory, contracts T = Phi * P panel by panel with
// P staged through shared memory, and forms rho = rowsum(T o Phi).  Work per point drops
// from N^2/2 * 40 exponentials to sum_shells nprim exponentials plus 2 N^2 FMAs.
#include "density.cuh"
#include "reduce.cuh"

namespace qmt {

// ---------------------------------------------------------------------------------------
// Tile set-up shared by the SIMT and tensor-core paths.
// ---------------------------------------------------------------------------------------
qmt_status make_point_map(int nx, int ny, int nz, float step, float ox, float oy, float oz,
                          int subgrid, int tile_rows, PointMap& pm, int64_t& ntiles) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return fail(QMT_BAD_ARG, "grid dimensions must be positive");
  if (subgrid < 1 || subgrid > 8) return fail(QMT_BAD_ARG, "subgrid must be in 1..8");
  if (!(step > 0.f) || !std::isfinite(step)) return fail(QMT_BAD_ARG, "grid step must be positive");
  pm.nx = nx;
  pm.ny = ny;
  pm.nz = nz;
  pm.s = subgrid;
  pm.s3 = subgrid * subgrid * subgrid;
  if (pm.s3 > tile_rows) return fail(QMT_BAD_ARG, "subgrid^3 larger than a density tile");
  pm.vpt = tile_rows / pm.s3;
  pm.nvox = (int64_t)nx * ny * nz;
  pm.h = step;
  pm.ox = ox;
  pm.oy = oy;
  pm.oz = oz;
  pm.inv_s = 1.0 / subgrid;
  pm.blocked = pm.vpt == 128 ? 1 : 0;
  if (pm.blocked) {
    pm.nbx = (nx + 7) / 8;
    pm.nby = (ny + 3) / 4;
    ntiles = (int64_t)pm.nbx * pm.nby * ((nz + 3) / 4);
    if (ntiles >= (int64_t)1 << 31) return fail(QMT_BAD_ARG, "grid too large");
  } else {
    pm.nbx = pm.nby = 0;
    ntiles = (pm.nvox + pm.vpt - 1) / pm.vpt;
  }
  return QMT_OK;
}

// ---------------------------------------------------------------------------------------
// SIMT fused kernel.  256 threads = 16 point groups x 16 column groups; each thread owns
// PPT points x 16 columns of a 256-column panel of T.
// ---------------------------------------------------------------------------------------
template <typename T, int TP>
__global__ void __launch_bounds__(256) density_simt_kernel(MolView mol, PointMap pm,
                                                           const T* __restrict__ P,
                                                           int64_t ntiles, float* __restrict__ qube,
                                                           double* __restrict__ partials,
                                                           double outscale) {
  constexpr int PPT = TP / 16;
  constexpr int CPT = 16;
  constexpr int PANEL = 16 * CPT;
  constexpr int KC = 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ps = reinterpret_cast<T*>(smem_raw);   // [KC][PANEL]
  T* phi = Ps + KC * PANEL;                 // [TP][ldp]
  __shared__ T rho_s[TP];
  __shared__ double pts_s[TP][3];
  __shared__ double red[8];
  const int npad = mol.npad;
  const int ldp = npad + 16 / PPT;
  const int tid = threadIdx.x;
  const int cg = tid & 15;
  const int pg = tid >> 4;
  const T* al = nullptr;
  const T* co = nullptr;
  if constexpr (sizeof(T) == 8) {
    al = reinterpret_cast<const T*>(mol.alpha64);
    co = reinterpret_cast<const T*>(mol.coeff64);
  } else {
    al = reinterpret_cast<const T*>(mol.alpha);
    co = reinterpret_cast<const T*>(mol.coeff);
  }

  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    __syncthreads();  // previous tile fully consumed
    if (tid < TP) {
      double x, y, z;
      int64_t vox;
      if (!tile_point<double>(pm, tile, tid, x, y, z, vox)) x = y = z = 1e30;
      pts_s[tid][0] = x;
      pts_s[tid][1] = y;
      pts_s[tid][2] = z;
    }
    for (int i = tid; i < TP * (npad - mol.norbs); i += 256) {
      const int p = i / (npad - mol.norbs), j = i % (npad - mol.norbs);
      phi[p * ldp + mol.norbs + j] = T(0);
    }
    __syncthreads();
    // basis functions of every shell at every point of the tile
    for (int it = tid; it < TP * mol.nshells; it += 256) {
      const int p = it % TP;
      const Shell sh = mol.shells[it / TP];
      T v[5];
      const double px = pts_s[p][0];
      int n;
      if (px > 1e29) {
        n = 2 * sh.L + 1;
        for (int k = 0; k < n; ++k) v[k] = T(0);
      } else {
        // displacement from the nucleus in FP64, then rounded once: keeps steep core
        // exponents accurate near the nucleus
        const T dx = T(px - (double)mol.coords[3 * sh.atom + 0]);
        const T dy = T(pts_s[p][1] - (double)mol.coords[3 * sh.atom + 1]);
        const T dz = T(pts_s[p][2] - (double)mol.coords[3 * sh.atom + 2]);
        n = shell_values<T>(sh, al, co, dx, dy, dz, v);
      }
      for (int k = 0; k < n; ++k) phi[p * ldp + sh.func + k] = v[k];
    }

    T part[PPT];
#pragma unroll
    for (int i = 0; i < PPT; ++i) part[i] = T(0);

    for (int col0 = 0; col0 < npad; col0 += PANEL) {
      T acc[PPT][CPT];
#pragma unroll
      for (int i = 0; i < PPT; ++i)
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[i][c] = T(0);
      for (int k0 = 0; k0 < npad; k0 += KC) {
        __syncthreads();
        for (int i = tid; i < KC * PANEL; i += 256) {
          const int kk = i / PANEL, c = i % PANEL;
          const int col = col0 + c;
          Ps[i] = col < npad ? P[(int64_t)(k0 + kk) * npad + col] : T(0);
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
          T a[PPT], b[CPT];
#pragma unroll
          for (int i = 0; i < PPT; ++i) a[i] = phi[(pg * PPT + i) * ldp + k0 + kk];
#pragma unroll
          for (int c = 0; c < CPT; ++c) b[c] = Ps[kk * PANEL + cg + 16 * c];
#pragma unroll
          for (int i = 0; i < PPT; ++i)
#pragma unroll
            for (int c = 0; c < CPT; ++c) acc[i][c] = fma(a[i], b[c], acc[i][c]);
        }
      }
#pragma unroll
      for (int i = 0; i < PPT; ++i)
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const int col = col0 + cg + 16 * c;
          if (col < npad) part[i] = fma(acc[i][c], phi[(pg * PPT + i) * ldp + col], part[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      T v = part[i];
      for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (cg == 0) rho_s[pg * PPT + i] = v;
    }
    __syncthreads();
    double mysum = 0;
    if (tid < pm.vpt) {
      T acc = T(0);
      for (int s = 0; s < pm.s3; ++s) acc += rho_s[tid * pm.s3 + s];
      int64_t vox, ix, iy, iz;
      if (tile_voxel(pm, tile, tid, vox, ix, iy, iz)) {
        const float q = (float)((double)acc * outscale);
        qube[vox] = q;
        mysum = q;
      }
    }
    const double bs = block_sum<256>(mysum, red);
    if (tid == 0) partials[tile] = bs;
  }
}

template <typename T, int TP>
static size_t simt_smem(int npad) {
  return sizeof(T) * (32 * 256 + (size_t)TP * (npad + 16 / (TP / 16)));
}

template <typename T, int TP>
static qmt_status launch_simt(qmt_mol* mol, const PointMap& pm, int64_t ntiles, float* qube,
                              double* partials, double outscale, cudaStream_t s) {
  const size_t smem = simt_smem<T, TP>(mol->npad);
  auto kern = density_simt_kernel<T, TP>;
  QMT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  QMT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem));
  if (occ < 1) return fail(QMT_BAD_ARG, "density tile does not fit in shared memory");
  const int64_t grid = std::min<int64_t>(ntiles, (int64_t)sm_count() * occ);
  const T* P = sizeof(T) == 8 ? (const T*)mol->d_P64.ptr : (const T*)mol->d_P32.ptr;
  kern<<<(unsigned)grid, 256, smem, s>>>(mol->view(), pm, P, ntiles, qube, partials, outscale);
  QMT_CHECK_LAUNCH("density_simt_kernel");
  return QMT_OK;
}

static int max_smem() {
  static int v = 0;
  if (!v) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (v <= 0) v = 232448;
  }
  return v;
}

// Chooses the largest tile that fits; returns rows per tile (0 if none).
static int simt_tile_rows(bool fp64, int npad, int s3) {
  const size_t lim = (size_t)max_smem() - 4096;
  if (!fp64) {
    if (simt_smem<float, 64>(npad) <= lim) return 64;
    if (s3 <= 32 && simt_smem<float, 32>(npad) <= lim) return 32;
    if (s3 <= 16 && simt_smem<float, 16>(npad) <= lim) return 16;
  } else {
    if (simt_smem<double, 64>(npad) <= lim) return 64;
    if (s3 <= 32 && simt_smem<double, 32>(npad) <= lim) return 32;
    if (s3 <= 16 && simt_smem<double, 16>(npad) <= lim) return 16;
  }
  return 0;
}

__global__ void reduce_partials_kernel(const double* __restrict__ in, int64_t n, double* __restrict__ out,
                                       int nvals, int64_t stride) {
  __shared__ double sh[32];
  for (int v = 0; v < nvals; ++v) {
    double acc = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) acc += in[v * stride + i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
      out[v] = r;
    }
    __syncthreads();
  }
}

qmt_status reduce_partials(const double* in, int64_t n, double* out, int nvals, int64_t stride,
                           cudaStream_t s) {
  reduce_partials_kernel<<<1, 1024, 0, s>>>(in, n, out, nvals, stride);
  QMT_CHECK_LAUNCH("reduce_partials_kernel");
  return QMT_OK;
}

__global__ void rescale_to_total_kernel(float* __restrict__ q, int64_t n, const double* __restrict__ sum,
                                        double qtot) {
  const float f = (float)(qtot / *sum);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    q[i] = q[i] * f;
}

qmt_status finish_density(qmt_mol* mol, int64_t nvox, int64_t ntiles, int rescale, float* qube,
                          double* sum_out, cudaStream_t s) {
  double* d_sum = mol->d_scalars.as<double>();
  qmt_status st = reduce_partials(mol->d_partials.as<double>(), ntiles, d_sum, 1, 0, s);
  if (st) return st;
  if (rescale) {
    const int64_t blocks = std::min<int64_t>((nvox + 255) / 256, (int64_t)sm_count() * 8);
    rescale_to_total_kernel<<<(unsigned)blocks, 256, 0, s>>>(qube, nvox, d_sum, mol->qtot);
    QMT_CHECK_LAUNCH("rescale_to_total_kernel");
  }
  if (sum_out) {
    QMT_CUDA(cudaMemcpyAsync(sum_out, d_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
    QMT_CUDA(cudaStreamSynchronize(s));
    if (!std::isfinite(*sum_out)) return fail(QMT_NAN, "non-finite density sum");
  }
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_density(qmt_mol* mol, int nx, int ny, int nz, float step, float ox,
                                  float oy, float oz, int subgrid, int precision, int rescale,
                                  float* qube_dev, double* sum_out, void* stream) {
  if (!mol || !qube_dev) return fail(QMT_BAD_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  qmt_status st;
  if (st = mol->d_scalars.reserve(64 * sizeof(double))) return st;
  if (precision == QMT_PREC_FP32 || precision == QMT_PREC_FP64) {
    const bool fp64 = precision == QMT_PREC_FP64;
    const int s3 = subgrid * subgrid * subgrid;
    const int rows = simt_tile_rows(fp64, mol->npad, s3);
    if (!rows) return fail(QMT_BAD_ARG, "basis too large for the SIMT density tile");
    PointMap pm;
    int64_t ntiles;
    if ((st = make_point_map(nx, ny, nz, step, ox, oy, oz, subgrid, rows, pm, ntiles))) return st;
    if ((st = mol->d_partials.reserve(ntiles * sizeof(double)))) return st;
    const double outscale = 2.0 * (double)step * step * step / s3;
    double* part = mol->d_partials.as<double>();
    if (!fp64) {
      if (rows == 64) st = launch_simt<float, 64>(mol, pm, ntiles, qube_dev, part, outscale, s);
      else if (rows == 32) st = launch_simt<float, 32>(mol, pm, ntiles, qube_dev, part, outscale, s);
      else st = launch_simt<float, 16>(mol, pm, ntiles, qube_dev, part, outscale, s);
    } else {
      if (rows == 64) st = launch_simt<double, 64>(mol, pm, ntiles, qube_dev, part, outscale, s);
      else if (rows == 32) st = launch_simt<double, 32>(mol, pm, ntiles, qube_dev, part, outscale, s);
      else st = launch_simt<double, 16>(mol, pm, ntiles, qube_dev, part, outscale, s);
    }
    if (st) return st;
    return finish_density(mol, pm.nvox, ntiles, rescale, qube_dev, sum_out, s);
  }
  if (precision >= QMT_PREC_TF32 && precision <= QMT_PREC_FP16X3)
    return density_tc(mol, nx, ny, nz, step, ox, oy, oz, subgrid, precision, rescale, qube_dev,
                      sum_out, s);
  return fail(QMT_BAD_ARG, "unknown precision");
}

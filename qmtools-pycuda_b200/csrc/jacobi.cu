// Jacobi relaxation of the Poisson equation on the voxel grid.
//
// Reference mode (gpu_hartree_iteration, kernel_hartree.cu:85-171):
//     V'(interior) = (xm + xp + yp + ym + zp + zm - Q/h) / 6,  V' = 0 on the outer shell,
// summed in that order so FP32 results match the reference update.
// Dirichlet mode (new): V'(interior) = (sum of 6 neighbours + 4 pi h^2 rho) / 6 and the
// outer shell keeps its given values.
//
// Each CTA owns a 32 x 8 column of the x-y plane and marches along z holding the z-1, z,
// z+1 values in registers; the x-y halo of the current plane goes through shared memory,
// so every V value is read from memory about once per sweep.  The FP64 sum |V' - V| is
// formed only on sweeps that feed a convergence check.
#include "mol.cuh"
#include "reduce.cuh"

namespace qmt {

constexpr int JX = 32, JY = 8;

template <bool DIRICHLET>
__global__ void __launch_bounds__(JX* JY) jacobi_kernel(int nx, int ny, int nz, float h, float src_scale,
                                                        const float* __restrict__ Q, const float* __restrict__ V,
                                                        float* __restrict__ W, double* __restrict__ part) {
  __shared__ float tile[JY + 2][JX + 2];
  __shared__ double sh[8];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = blockIdx.x * JX + tx, y = blockIdx.y * JY + ty;
  const bool in = x < nx && y < ny;
  const int64_t plane = (int64_t)nx * ny;
  const int64_t col = (int64_t)y * nx + x;
  float vm = 0.f, vc = 0.f, vp = 0.f;
  if (in) {
    vc = V[col];
    vp = nz > 1 ? V[col + plane] : 0.f;
  }
  double dsum = 0.0;
  for (int z = 0; z < nz; ++z) {
    __syncthreads();
    tile[ty + 1][tx + 1] = vc;
    if (tx == 0) tile[ty + 1][0] = (in && x > 0) ? V[z * plane + col - 1] : 0.f;
    if (tx == JX - 1) tile[ty + 1][JX + 1] = (y < ny && x + 1 < nx) ? V[z * plane + col + 1] : 0.f;
    if (ty == 0) tile[0][tx + 1] = (x < nx && y > 0) ? V[z * plane + col - nx] : 0.f;
    if (ty == JY - 1) tile[JY + 1][tx + 1] = (x < nx && y + 1 < ny) ? V[z * plane + col + nx] : 0.f;
    __syncthreads();
    if (in) {
      const int64_t g = z * plane + col;
      const bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
      float out;
      if constexpr (!DIRICHLET) {
        float s = tile[ty + 1][tx] + tile[ty + 1][tx + 2];
        s = s + tile[ty + 2][tx + 1];
        s = s + tile[ty][tx + 1];
        s = s + vp;
        s = s + vm;
        s = s - Q[g] / h;
        out = edge ? 0.f : s / 6.0f;
      } else {
        const float s = tile[ty + 1][tx] + tile[ty + 1][tx + 2] + tile[ty + 2][tx + 1] + tile[ty][tx + 1] + vp + vm;
        out = edge ? vc : (s + src_scale * Q[g]) * (1.0f / 6.0f);
      }
      W[g] = out;
      if (part) dsum += fabs((double)out - (double)vc);
      vm = vc;
      vc = vp;
      vp = (z + 2 < nz) ? V[g + 2 * plane] : 0.f;
    }
  }
  if (part) {
    const int lin = ty * JX + tx;
    double v = dsum;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((lin & 31) == 0) sh[lin >> 5] = v;
    __syncthreads();
    if (lin == 0) {
      double r = 0;
      for (int w = 0; w < JX * JY / 32; ++w) r += sh[w];
      part[blockIdx.y * gridDim.x + blockIdx.x] = r;
    }
  }
}

template <bool DIRICHLET>
static qmt_status run_jacobi(int nx, int ny, int nz, float step, const float* rho, float* v, float* t,
                             int max_sweeps, int check_every, double tol, int* sweeps_out,
                             double* delta_out, cudaStream_t s) {
  if (nx < 1 || ny < 1 || nz < 1 || !(step > 0.f) || !rho || !v || !t || max_sweeps < 0 || check_every < 1)
    return fail(QMT_BAD_ARG, "bad Jacobi arguments");
  const dim3 blk(JX, JY), grd((nx + JX - 1) / JX, (ny + JY - 1) / JY);
  const int64_t nblk = (int64_t)grd.x * grd.y;
  static thread_local DevBuf scratch;
  qmt_status st = scratch.reserve((nblk + 8) * sizeof(double));
  if (st) return st;
  double* part = scratch.as<double>();
  double* res = part + nblk;
  const float src = DIRICHLET ? (float)(4.0 * 3.14159265358979323846 * (double)step * step) : 0.f;
  double delta = INFINITY;
  int sweeps = 0, pairs = 0;
  bool converged = false;
  while (sweeps + 2 <= max_sweeps) {
    ++pairs;
    const bool check = pairs % check_every == 0 || sweeps + 4 > max_sweeps;
    if constexpr (DIRICHLET) {
      jacobi_kernel<true><<<grd, blk, 0, s>>>(nx, ny, nz, 0.f, src, rho, v, t, nullptr);
      jacobi_kernel<true><<<grd, blk, 0, s>>>(nx, ny, nz, 0.f, src, rho, t, v, check ? part : nullptr);
    } else {
      jacobi_kernel<false><<<grd, blk, 0, s>>>(nx, ny, nz, step, 0.f, rho, v, t, nullptr);
      jacobi_kernel<false><<<grd, blk, 0, s>>>(nx, ny, nz, step, 0.f, rho, t, v, check ? part : nullptr);
    }
    QMT_CHECK_LAUNCH("jacobi_kernel");
    sweeps += 2;
    if (check) {
      if ((st = reduce_partials(part, nblk, res, 1, 0, s))) return st;
      QMT_CUDA(cudaMemcpyAsync(&delta, res, sizeof(double), cudaMemcpyDeviceToHost, s));
      QMT_CUDA(cudaStreamSynchronize(s));
      if (!std::isfinite(delta)) {
        if (sweeps_out) *sweeps_out = sweeps;
        if (delta_out) *delta_out = delta;
        return fail(QMT_NAN, "Jacobi residual is not finite");
      }
      if (delta <= tol) {
        converged = true;
        break;
      }
    }
  }
  if (sweeps_out) *sweeps_out = sweeps;
  if (delta_out) *delta_out = delta;
  if (!converged && tol > 0) return fail(QMT_NOT_CONVERGED, "Jacobi stopped at its sweep cap");
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_jacobi(int nx, int ny, int nz, float step, const float* rho_dev, float* v_dev,
                                 float* t_dev, int max_sweeps, int check_every, double tol, int* sweeps_out,
                                 double* delta_out, void* stream) {
  return run_jacobi<false>(nx, ny, nz, step, rho_dev, v_dev, t_dev, max_sweeps, check_every, tol, sweeps_out,
                           delta_out, as_stream(stream));
}

extern "C" qmt_status qmt_jacobi_dirichlet(int nx, int ny, int nz, float step, const float* rho_dev, float* v_dev,
                                           float* t_dev, int max_sweeps, int check_every, double tol,
                                           int* sweeps_out, double* delta_out, void* stream) {
  return run_jacobi<true>(nx, ny, nz, step, rho_dev, v_dev, t_dev, max_sweeps, check_every, tol, sweeps_out,
                          delta_out, as_stream(stream));
}

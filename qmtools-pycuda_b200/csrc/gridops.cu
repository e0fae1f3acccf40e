// Grid reductions (deterministic FP64), rescale, nuclear seed, Vne fields and the FP64
// overlap trace Tr(PS).
#include "mol.cuh"
#include "reduce.cuh"

namespace qmt {

// ---- reductions ---------------------------------------------------------------------------
// op 0: sum a; op 1: sum |a-b|; op 2: sum |a-b|/b; op 3: error report (5 values:
// max|a-b|, sum (a-b)^2, sum b^2, sum a, sum b).
template <int OP>
__global__ void __launch_bounds__(RED_THREADS) grid_reduce_kernel(const float* __restrict__ a,
                                                                  const float* __restrict__ b, int64_t n,
                                                                  double* __restrict__ part, int64_t nblk) {
  __shared__ double sh[RED_THREADS / 32];
  const int64_t base = (int64_t)blockIdx.x * RED_CHUNK;
  const int64_t end = min(n, base + RED_CHUNK);
  constexpr int NV = OP == 3 ? 5 : 1;
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int64_t i = base + threadIdx.x; i < end; i += RED_THREADS) {
    const double x = a[i];
    if constexpr (OP == 0) v[0] += x;
    if constexpr (OP == 1) v[0] += fabs(x - (double)b[i]);
    if constexpr (OP == 2) v[0] += (double)(fabsf(a[i] - b[i]) / b[i]);
    if constexpr (OP == 3) {
      const double y = b[i], d = x - y;
      v[0] = fmax(v[0], fabs(d));
      v[1] += d * d;
      v[2] += y * y;
      v[3] += x;
      v[4] += y;
    }
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double r;
    if (OP == 3 && k == 0) {
      double m = v[0];
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
      __syncthreads();
      r = 0;
      if (threadIdx.x == 0)
        for (int w = 0; w < RED_THREADS / 32; ++w) r = fmax(r, sh[w]);
      __syncthreads();
    } else {
      r = block_sum<RED_THREADS>(v[k], sh);
    }
    if (threadIdx.x == 0) part[k * nblk + blockIdx.x] = r;
  }
}

__global__ void max_partials_kernel(const double* __restrict__ in, int64_t n, double* __restrict__ out) {
  __shared__ double sh[32];
  double m = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, in[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    *out = r;
  }
}

struct Scratch {
  double* part = nullptr;
  double* res = nullptr;
  size_t cap = 0;
};

// Per-thread scratch for the stateless grid utilities (grows, never freed before exit).
static thread_local DevBuf tl_scratch;

static qmt_status run_reduce(int op, const float* a, const float* b, int64_t n, double* out, cudaStream_t s) {
  if (!a || n <= 0 || (op != 0 && !b) || !out) return fail(QMT_BAD_ARG, "bad reduction arguments");
  const int64_t nblk = (n + RED_CHUNK - 1) / RED_CHUNK;
  const int nv = op == 3 ? 5 : 1;
  qmt_status st = tl_scratch.reserve((nblk * nv + 8) * sizeof(double));
  if (st) return st;
  double* part = tl_scratch.as<double>();
  double* res = part + nblk * nv;
  switch (op) {
    case 0: grid_reduce_kernel<0><<<(unsigned)nblk, RED_THREADS, 0, s>>>(a, b, n, part, nblk); break;
    case 1: grid_reduce_kernel<1><<<(unsigned)nblk, RED_THREADS, 0, s>>>(a, b, n, part, nblk); break;
    case 2: grid_reduce_kernel<2><<<(unsigned)nblk, RED_THREADS, 0, s>>>(a, b, n, part, nblk); break;
    default: grid_reduce_kernel<3><<<(unsigned)nblk, RED_THREADS, 0, s>>>(a, b, n, part, nblk); break;
  }
  QMT_CHECK_LAUNCH("grid_reduce_kernel");
  if (op == 3) {
    max_partials_kernel<<<1, 1024, 0, s>>>(part, nblk, res);
    QMT_CHECK_LAUNCH("max_partials_kernel");
    if ((st = reduce_partials(part + nblk, nblk, res + 1, 4, nblk, s))) return st;
  } else {
    if ((st = reduce_partials(part, nblk, res, 1, 0, s))) return st;
  }
  double h[5];
  QMT_CUDA(cudaMemcpyAsync(h, res, nv * sizeof(double), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  if (op == 3) {
    out[0] = h[0];
    out[1] = h[2] > 0 ? std::sqrt(h[1] / h[2]) : std::sqrt(h[1]);
    out[2] = h[3];
    out[3] = h[4];
  } else {
    out[0] = op == 2 ? h[0] * 100.0 : h[0];
  }
  return QMT_OK;
}

__global__ void scale_kernel(float* __restrict__ q, int64_t n, float f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    q[i] = q[i] * f;
}

// ---- nuclear seed (kernel_utils.cu:5-50), one thread per node, atoms in order -------------
__global__ void density_seed_kernel(MolView mol, int nx, int ny, int nz, float h, float ox, float oy,
                                    float oz, float* __restrict__ q) {
  const int t = threadIdx.x;  // 8 nodes
  const int tx = t & 1, ty = (t >> 1) & 1, tz = t >> 2;
  for (int a = 0; a < mol.natoms; ++a) {
    const float x = mol.coords[3 * a] - ox, y = mol.coords[3 * a + 1] - oy, z = mol.coords[3 * a + 2] - oz;
    const long ix = (long)floorf(x / h) + tx, iy = (long)floorf(y / h) + ty, iz = (long)floorf(z / h) + tz;
    float p = (float)mol.types[a];
    p *= fabsf(x - (float)ix * h) / h;
    p *= fabsf(y - (float)iy * h) / h;
    p *= fabsf(z - (float)iz * h) / h;
    if (ix >= 0 && iy >= 0 && iz >= 0 && ix < nx && iy < ny && iz < nz)
      q[ix + iy * (int64_t)nx + iz * (int64_t)nx * ny] = p;
    __syncwarp(0xffu);
  }
}

// ---- sum Z/r at voxel centres (kernel_hartree.cu:209-251) ----------------------------------
__global__ void vne_point_kernel(MolView mol, int nx, int ny, int nz, float h, float ox, float oy, float oz,
                                 int accumulate, float* __restrict__ v) {
  extern __shared__ float sa[];  // natoms * 4
  for (int i = threadIdx.x; i < mol.natoms; i += blockDim.x) {
    sa[4 * i] = mol.coords[3 * i];
    sa[4 * i + 1] = mol.coords[3 * i + 1];
    sa[4 * i + 2] = mol.coords[3 * i + 2];
    sa[4 * i + 3] = (float)mol.types[i];
  }
  __syncthreads();
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = idx % nx, y = (idx / nx) % ny, z = idx / ((int64_t)nx * ny);
    const float px = ox + x * h + 0.5f * h, py = oy + y * h + 0.5f * h, pz = oz + z * h + 0.5f * h;
    float acc = 0.f;
    for (int a = 0; a < mol.natoms; ++a) {
      const float cx = px - sa[4 * a], cy = py - sa[4 * a + 1], cz = pz - sa[4 * a + 2];
      acc += sa[4 * a + 3] / sqrtf(cx * cx + cy * cy + cz * cz);
    }
    v[idx] = accumulate ? v[idx] + acc : acc;
  }
}

// ---- classic Vne (kernel_vne_classic.cu:13-84) ---------------------------------------------
__global__ void vne_classic_kernel(MolView mol, int nx, int ny, int nz, float h, float ox, float oy, float oz,
                                   int ndiv, float* __restrict__ v) {
  extern __shared__ float sa[];
  for (int i = threadIdx.x; i < mol.natoms; i += blockDim.x) {
    sa[4 * i] = mol.coords[3 * i] - ox;
    sa[4 * i + 1] = mol.coords[3 * i + 1] - oy;
    sa[4 * i + 2] = mol.coords[3 * i + 2] - oz;
    sa[4 * i + 3] = (float)mol.types[i];
  }
  __syncthreads();
  const int64_t n = (int64_t)nx * ny * nz;
  const double dx = (double)h / ndiv;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = idx % nx, y = (idx / nx) % ny, z = idx / ((int64_t)nx * ny);
    const float x0 = x * h, y0 = y * h, z0 = z * h;
    float acc = 0.f;
    int cnt = 0;
    for (int ii = 0; ii < ndiv; ++ii)
      for (int jj = 0; jj < ndiv; ++jj)
        for (int kk = 0; kk < ndiv; ++kk) {
          const float px = (float)(x0 + (ii + 0.5) * dx);
          const float py = (float)(y0 + (jj + 0.5) * dx);
          const float pz = (float)(z0 + (kk + 0.5) * dx);
          for (int a = 0; a < mol.natoms; ++a) {
            const float cx = px - sa[4 * a], cy = py - sa[4 * a + 1], cz = pz - sa[4 * a + 2];
            const float d = cx * cx + cy * cy + cz * cz;
            if (d != 0.f) {
              acc += sa[4 * a + 3] * rsqrtf(d);
              ++cnt;
            }
          }
        }
    float r = cnt ? acc / (float)cnt : 0.f;
    v[idx] = (float)((double)r / ((double)h * h * h));
  }
}

// ---- pseudo-field Vne step (kernel_vne.cu:13-128) ------------------------------------------
__global__ void __launch_bounds__(256) vne_pseudo_kernel(MolView mol, int nx, int ny, int nz, float h,
                                                         float ox, float oy, float oz, float ads, float dif,
                                                         const float* __restrict__ q, float* __restrict__ out,
                                                         double* __restrict__ part) {
  __shared__ float sa[4 * 256];
  __shared__ double sh[8];
  const int na = min(mol.natoms, 256);
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    sa[4 * i] = mol.coords[3 * i] - ox;
    sa[4 * i + 1] = mol.coords[3 * i + 1] - oy;
    sa[4 * i + 2] = mol.coords[3 * i + 2] - oz;
    sa[4 * i + 3] = (float)mol.types[i];
  }
  __syncthreads();
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t base = (int64_t)blockIdx.x * RED_CHUNK;
  const int64_t end = min(n, base + RED_CHUNK);
  const float w1 = dif, w2 = dif * 0.70710678118654752f, w3 = dif * 0.57735026918962576f;
  const float self = 1.0f - dif * 16.794682450997072f;
  const float cut = 1.7320508075688772f * h;
  double dsum = 0.0;
  for (int64_t idx = base + threadIdx.x; idx < end; idx += blockDim.x) {
    const int x = (int)(idx % nx), y = (int)((idx / nx) % ny), z = (int)(idx / ((int64_t)nx * ny));
    const float vnn = q[idx];
    float acc = 0.f;
    for (int dz = -1; dz <= 1; ++dz) {
      const int zz = (z + dz + nz) % nz;
      for (int dy = -1; dy <= 1; ++dy) {
        const int yy = (y + dy + ny) % ny;
        for (int dxx = -1; dxx <= 1; ++dxx) {
          const int d = abs(dxx) + abs(dy) + abs(dz);
          if (d == 0) continue;
          const int xx = (x + dxx + nx) % nx;
          const float w = d == 1 ? w1 : (d == 2 ? w2 : w3);
          acc += w * q[xx + (int64_t)yy * nx + (int64_t)zz * nx * ny];
        }
      }
    }
    acc += self * vnn;
    acc -= vnn * ads;
    const float px = x * h + 0.5f * h, py = y * h + 0.5f * h, pz = z * h + 0.5f * h;
    for (int a = 0; a < na; ++a) {
      const float cx = px - sa[4 * a], cy = py - sa[4 * a + 1], cz = pz - sa[4 * a + 2];
      const float d = sqrtf(cx * cx + cy * cy + cz * cz);
      if (d < cut) acc += sa[4 * a + 3] * expf(-d);
    }
    if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) acc = 0.f;
    out[idx] = acc;
    dsum += fabs((double)vnn - (double)acc);
  }
  const double bs = block_sum<256>(dsum, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
}

// ---- FP64 overlap trace ---------------------------------------------------------------------
// 1D Hermite E^{ij}_0 for i, j <= 2 (McMurchie-Davidson), including no exponential prefactor.
__device__ void overlap_e0(double a, double b, double xa, double xb, double E0[3][3]) {
  const double p = a + b, xp = (a * xa + b * xb) / p;
  const double pa = xp - xa, pb = xp - xb, i2p = 0.5 / p;
  double E[3][3][5];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int t = 0; t < 5; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = 1.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i > 0) {
          v = pa * E[i - 1][j][t] + (t + 1 < 5 ? (t + 1) * E[i - 1][j][t + 1] : 0.0);
          if (t > 0) v += i2p * E[i - 1][j][t - 1];
        } else {
          v = pb * E[i][j - 1][t] + (t + 1 < 5 ? (t + 1) * E[i][j - 1][t + 1] : 0.0);
          if (t > 0) v += i2p * E[i][j - 1][t - 1];
        }
        E[i][j][t] = v;
      }
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) E0[i][j] = E[i][j][0];
}

// Cartesian expansion of the shell's m-ordered functions: up to 3 terms (coef, i, j, k).
__device__ int cart_terms(int L, int k, double* c, int (*e)[3]) {
  if (L == 0) { c[0] = YS; e[0][0] = e[0][1] = e[0][2] = 0; return 1; }
  if (L == 1) {
    c[0] = YP; e[0][0] = e[0][1] = e[0][2] = 0;
    e[0][k == 0 ? 2 : (k == 1 ? 0 : 1)] = 1;
    return 1;
  }
  switch (k) {
    case 0:
      c[0] = 2 * YD0; e[0][0] = 0; e[0][1] = 0; e[0][2] = 2;
      c[1] = -YD0; e[1][0] = 2; e[1][1] = 0; e[1][2] = 0;
      c[2] = -YD0; e[2][0] = 0; e[2][1] = 2; e[2][2] = 0;
      return 3;
    case 1: c[0] = YD1; e[0][0] = 1; e[0][1] = 0; e[0][2] = 1; return 1;
    case 2: c[0] = YD1; e[0][0] = 0; e[0][1] = 1; e[0][2] = 1; return 1;
    case 3:
      c[0] = YD2; e[0][0] = 2; e[0][1] = 0; e[0][2] = 0;
      c[1] = -YD2; e[1][0] = 0; e[1][1] = 2; e[1][2] = 0;
      return 2;
    default: c[0] = YD1; e[0][0] = 1; e[0][1] = 1; e[0][2] = 0; return 1;
  }
}

// One block per shell pair (A, B); thread-strided over primitive pairs; FP64 sum of
// P_ab S_ab over the pair's functions.
__global__ void trace_ps_kernel(MolView mol, const double* __restrict__ P, double* __restrict__ part) {
  __shared__ double sh[8];
  const int sA = blockIdx.x % mol.nshells, sB = blockIdx.x / mol.nshells;
  const Shell A = mol.shells[sA], B = mol.shells[sB];
  const double Ax = mol.coords[3 * A.atom], Ay = mol.coords[3 * A.atom + 1], Az = mol.coords[3 * A.atom + 2];
  const double Bx = mol.coords[3 * B.atom], By = mol.coords[3 * B.atom + 1], Bz = mol.coords[3 * B.atom + 2];
  const double AB2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
  double acc = 0.0;
  for (int pp = threadIdx.x; pp < A.nprim * B.nprim; pp += blockDim.x) {
    const double a = mol.alpha64[A.prim + pp % A.nprim], ca = mol.coeff64[A.prim + pp % A.nprim];
    const double b = mol.alpha64[B.prim + pp / A.nprim], cb = mol.coeff64[B.prim + pp / A.nprim];
    const double p = a + b;
    const double K = exp(-a * b / p * AB2) * pow(3.14159265358979323846 / p, 1.5) * ca * cb;
    double Ex[3][3], Ey[3][3], Ez[3][3];
    overlap_e0(a, b, Ax, Bx, Ex);
    overlap_e0(a, b, Ay, By, Ey);
    overlap_e0(a, b, Az, Bz, Ez);
    for (int k1 = 0; k1 < 2 * A.L + 1; ++k1) {
      double c1[3];
      int e1[3][3];
      const int n1 = cart_terms(A.L, k1, c1, e1);
      for (int k2 = 0; k2 < 2 * B.L + 1; ++k2) {
        double c2[3];
        int e2[3][3];
        const int n2 = cart_terms(B.L, k2, c2, e2);
        double s = 0.0;
        for (int u = 0; u < n1; ++u)
          for (int w = 0; w < n2; ++w)
            s += c1[u] * c2[w] * Ex[e1[u][0]][e2[w][0]] * Ey[e1[u][1]][e2[w][1]] * Ez[e1[u][2]][e2[w][2]];
        acc += K * s * P[(int64_t)(A.func + k1) * mol.npad + B.func + k2];
      }
    }
  }
  const double bs = block_sum<128>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
}

}  // namespace qmt

using namespace qmt;

static bool grid_ok(int nx, int ny, int nz, float step) {
  return nx > 0 && ny > 0 && nz > 0 && step > 0.f && std::isfinite(step);
}

extern "C" {

qmt_status qmt_grid_total(const float* q_dev, int64_t n, double* out, void* stream) {
  return run_reduce(0, q_dev, nullptr, n, out, as_stream(stream));
}

qmt_status qmt_grid_scale(float* q_dev, int64_t n, float factor, void* stream) {
  if (!q_dev || n <= 0) return fail(QMT_BAD_ARG, "bad scale arguments");
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
  scale_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(q_dev, n, factor);
  QMT_CHECK_LAUNCH("scale_kernel");
  return QMT_OK;
}

qmt_status qmt_grid_diff(const float* a_dev, const float* b_dev, int64_t n, int rel, double* out, void* stream) {
  return run_reduce(rel ? 2 : 1, a_dev, b_dev, n, out, as_stream(stream));
}

qmt_status qmt_grid_errors(const float* a_dev, const float* b_dev, int64_t n, double* out4, void* stream) {
  return run_reduce(3, a_dev, b_dev, n, out4, as_stream(stream));
}

qmt_status qmt_density_seed(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                            float* q_dev, void* stream) {
  if (!mol || !q_dev || !grid_ok(nx, ny, nz, step)) return fail(QMT_BAD_ARG, "bad seed arguments");
  density_seed_kernel<<<1, 8, 0, as_stream(stream)>>>(mol->view(), nx, ny, nz, step, ox, oy, oz, q_dev);
  QMT_CHECK_LAUNCH("density_seed_kernel");
  return QMT_OK;
}

qmt_status qmt_vne_point(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                         int accumulate, float* v_dev, void* stream) {
  if (!mol || !v_dev || !grid_ok(nx, ny, nz, step)) return fail(QMT_BAD_ARG, "bad vne arguments");
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16);
  vne_point_kernel<<<(unsigned)blocks, 256, 16 * mol->natoms, as_stream(stream)>>>(mol->view(), nx, ny, nz, step,
                                                                                    ox, oy, oz, accumulate, v_dev);
  QMT_CHECK_LAUNCH("vne_point_kernel");
  return QMT_OK;
}

qmt_status qmt_vne_classic(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                           int divisions, float* v_dev, void* stream) {
  if (!mol || !v_dev || !grid_ok(nx, ny, nz, step) || divisions < 1 || divisions > 64)
    return fail(QMT_BAD_ARG, "bad vne_classic arguments");
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16);
  vne_classic_kernel<<<(unsigned)blocks, 256, 16 * mol->natoms, as_stream(stream)>>>(
      mol->view(), nx, ny, nz, step, ox, oy, oz, divisions, v_dev);
  QMT_CHECK_LAUNCH("vne_classic_kernel");
  return QMT_OK;
}

qmt_status qmt_vne_pseudo(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                          float ads, float dif, double tol, int maxiters, float* res_dev, float* out_dev,
                          int* iters_out, void* stream) {
  if (!mol || !res_dev || !out_dev || !grid_ok(nx, ny, nz, step) || maxiters < 0)
    return fail(QMT_BAD_ARG, "bad vne_pseudo arguments");
  if (mol->natoms > 256) return fail(QMT_BAD_ARG, "vne_pseudo supports up to 256 atoms");
  cudaStream_t s = as_stream(stream);
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t nblk = (n + RED_CHUNK - 1) / RED_CHUNK;
  qmt_status st = mol->d_work.reserve((nblk + 8) * sizeof(double));
  if (st) return st;
  double* part = mol->d_work.as<double>();
  double* res = part + nblk;
  QMT_CUDA(cudaMemsetAsync(res_dev, 0, n * sizeof(float), s));
  QMT_CUDA(cudaMemsetAsync(out_dev, 0, n * sizeof(float), s));
  double delta = 1.0;
  int it = 0;
  while (delta > tol) {
    vne_pseudo_kernel<<<(unsigned)nblk, 256, 0, s>>>(mol->view(), nx, ny, nz, step, ox, oy, oz, ads, dif,
                                                     res_dev, out_dev, part);
    vne_pseudo_kernel<<<(unsigned)nblk, 256, 0, s>>>(mol->view(), nx, ny, nz, step, ox, oy, oz, ads, dif,
                                                     out_dev, res_dev, part);
    note_launches(1);   // the first of the two ping-pong launches
    QMT_CHECK_LAUNCH("vne_pseudo_kernel");
    if ((st = reduce_partials(part, nblk, res, 1, 0, s))) return st;
    double h = 0;
    QMT_CUDA(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, s));
    QMT_CUDA(cudaStreamSynchronize(s));
    delta = h / (double)n;
    ++it;
    if (it > maxiters) break;
  }
  if (iters_out) *iters_out = it;
  return QMT_OK;
}

qmt_status qmt_mol_trace_ps(qmt_mol* mol, double* trace_out, void* stream) {
  if (!mol || !trace_out) return fail(QMT_BAD_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  const int64_t npairs = (int64_t)mol->nshells * mol->nshells;
  qmt_status st = mol->d_work.reserve((npairs + 8) * sizeof(double));
  if (st) return st;
  double* part = mol->d_work.as<double>();
  trace_ps_kernel<<<(unsigned)npairs, 128, 0, s>>>(mol->view(), mol->d_P64.as<double>(), part);
  QMT_CHECK_LAUNCH("trace_ps_kernel");
  if ((st = reduce_partials(part, npairs, part + npairs, 1, 0, s))) return st;
  QMT_CUDA(cudaMemcpyAsync(trace_out, part + npairs, sizeof(double), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  return QMT_OK;
}

}  // extern "C"

// ---- grid total without allocation ----------------------------------------------------------
// Same reduction as qmt_grid_total, but its partial sums live in a fixed array compiled into
// the library instead of in memory obtained from cudaMalloc.  The array is part of the module
// image: every GPU that loads the library holds its 32 KiB until the process exits.
#include <mutex>

namespace qmt {

constexpr int64_t NOALLOC_MAX_BLOCKS = 4096;                          // first-pass partial sums
constexpr int64_t NOALLOC_MAX_POINTS = NOALLOC_MAX_BLOCKS * RED_CHUNK;  // 33,554,432 grid points
constexpr int NOALLOC_MAX_DEVICES = 64;

// [0, NOALLOC_MAX_BLOCKS): one partial sum per first-pass block; [NOALLOC_MAX_BLOCKS]: the total.
static __device__ __align__(256) double g_total_scratch[NOALLOC_MAX_BLOCKS + 32];

static std::mutex g_total_scratch_mu;
static double* g_total_scratch_dev[NOALLOC_MAX_DEVICES] = {};

// Device address of g_total_scratch on the current device.  On the host the symbol only names
// a host-side stand-in, so the address is looked up once per device with that device current.
static qmt_status total_scratch(double** out) {
  int dev = -1;
  QMT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(QMT_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_total_scratch_mu);
  if (!g_total_scratch_dev[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_total_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_total_scratch)");
    g_total_scratch_dev[dev] = static_cast<double*>(p);
  }
  *out = g_total_scratch_dev[dev];
  return QMT_OK;
}

}  // namespace qmt

extern "C" qmt_status qmt_grid_total_noalloc(const float* q_dev, int64_t n, double* out, void* stream) {
  using namespace qmt;
  if (!q_dev || n <= 0 || !out) return fail(QMT_BAD_ARG, "bad reduction arguments");
  if (n > NOALLOC_MAX_POINTS)
    return fail(QMT_BAD_ARG, "qmt_grid_total_noalloc: " + std::to_string(n) +
                                 " points exceed its fixed scratch limit of " +
                                 std::to_string(NOALLOC_MAX_POINTS) + " points; use qmt_grid_total");
  double* part = nullptr;
  qmt_status st = total_scratch(&part);
  if (st) return st;
  double* res = part + NOALLOC_MAX_BLOCKS;
  cudaStream_t s = as_stream(stream);
  const int64_t nblk = (n + RED_CHUNK - 1) / RED_CHUNK;
  // every slot read below is written earlier in this call, so nothing needs clearing
  grid_reduce_kernel<0><<<(unsigned)nblk, RED_THREADS, 0, s>>>(q_dev, nullptr, n, part, nblk);
  QMT_CHECK_LAUNCH("grid_reduce_kernel");
  reduce_partials_kernel<<<1, 1024, 0, s>>>(part, nblk, res, 1, 0);
  QMT_CHECK_LAUNCH("reduce_partials_kernel");
  double h = 0.0;
  QMT_CUDA(cudaMemcpyAsync(&h, res, sizeof(double), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  *out = h;
  return QMT_OK;
}

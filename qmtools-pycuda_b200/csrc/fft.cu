// FFT Poisson solves with an in-house FFT.
//
// Reference semantics (QMTools.Compute_hartree_fft, qmtools/qmtools.py:2578-2639):
//   gpu_add_nuclear_charge (kernel_fft.cu:23-79) builds, in Angstrom units,
//       RHS = -( -q/h^3 + sum_A Z_A g_sigma(r - R_A) [r^2 <= (cutoff sigma)^2] ) / EPS0,
//   a periodic FFT, V_hat = -RHS_hat / (4 pi^2 |k|^2) with V_hat(0) = 0
//   (gpu_poisson_frequency_solve, kernel_fft.cu:82-107), an inverse FFT scaled by 1/N and the
//   real part returned in C order (i*NY*NZ + j*NZ + k) in volts.  The reference called cuFFT
//   through scikit-cuda, whose import is commented out (qmtools/qmtools.py:16).
// Free-space variant (new): the same charge density, convolved with the Hockney Green's
//   function 1/(4 pi EPS0 |r|) on a zero-padded grid of at least 2n per axis (sizes with
//   factors 2, 3, 5, 7), G(0) = voxel-cube average of 1/|r|; G_hat is cached per (M, h).
//
// The 1D transforms are mixed-radix Stockham (self-sorting) FFTs on batches of lines held
// in shared memory; the 3D transform is three axis passes over an x-fastest complex grid,
// each CTA reading whole lines (x pass) or B consecutive x-columns (y and z passes) so that
// global accesses are contiguous.
#include <algorithm>
#include <map>
#include <tuple>

#include "mol.cuh"

namespace qmt {

constexpr double EPS0 = 0.0055263494;       // e/(V*Ang), kernel_fft.cu:18
constexpr double R_BOHR = 0.529177211;      // kernel_fft.cu:17
constexpr double CUBE_INV_R = 2.3800772417; // h * <1/|r|> over a voxel cube
constexpr int FFT_MAXFAC = 16;

struct Plan1D {
  int L;
  int nfac;
  int fac[FFT_MAXFAC];
};

static bool factorize(int L, Plan1D& p) {
  p.L = L;
  p.nfac = 0;
  int n = L;
  const int pref[] = {4, 2, 3, 5, 7};
  for (int r : pref)
    while (n % r == 0) {
      if (p.nfac >= FFT_MAXFAC) return false;
      p.fac[p.nfac++] = r;
      n /= r;
    }
  for (int r = 11; n > 1; r += 2)
    while (n % r == 0) {
      if (p.nfac >= FFT_MAXFAC) return false;
      p.fac[p.nfac++] = r;
      n /= r;
    }
  return true;
}

static bool nice(int n) {
  for (int r : {2, 3, 5, 7})
    while (n % r == 0) n /= r;
  return n == 1;
}

static int nice_at_least(int n) {
  while (!nice(n)) ++n;
  return n;
}

// Lines: line l has elements at base(l) + e*se, base(l) = (l % n1)*s1 + (l / n1)*s2.
struct Lines {
  int64_t n1, s1, s2, se;
  int64_t nlines;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(sign * 2 pi i * num / den), num reduced mod den
__device__ __forceinline__ float2 root(int64_t num, int den, float sign) {
  const int64_t m = num % den;
  float s, c;
  sincospif(2.0f * (float)m / (float)den, &s, &c);
  return make_float2(c, sign * s);
}

// One radix-R butterfly of a Stockham stage: twiddle by exp(sign 2 pi i k q/(Ns R)), DFT_R,
// scatter to the self-sorted position.
template <int R>
__device__ __forceinline__ void radix_stage(const float2* __restrict__ s, float2* __restrict__ d, int j, int k,
                                            int idxD, int nbf, int Ns, float sign) {
  float2 v[R], w[R];
#pragma unroll
  for (int m = 0; m < R; ++m) w[m] = root(m, R, sign);
  const float2 t1 = root(k, Ns * R, sign);
  float2 tw = make_float2(1.f, 0.f);
#pragma unroll
  for (int q = 0; q < R; ++q) {
    v[q] = q ? cmul(s[j + q * nbf], tw) : s[j];
    tw = cmul(tw, t1);
  }
#pragma unroll
  for (int q = 0; q < R; ++q) {
    float2 acc = v[0];
#pragma unroll
    for (int p = 1; p < R; ++p) {
      const float2 w2 = w[(p * q) % R];
      acc.x += v[p].x * w2.x - v[p].y * w2.y;
      acc.y += v[p].x * w2.y + v[p].y * w2.x;
    }
    d[idxD + q * Ns] = acc;
  }
}

__global__ void __launch_bounds__(256) fft_lines_kernel(float2* __restrict__ data, Plan1D plan, Lines ln, int B,
                                                        float sign, float scale) {
  extern __shared__ float2 fsm[];
  const int L = plan.L;
  float2* b0 = fsm;
  float2* b1 = fsm + (size_t)B * L;
  const int64_t l0 = (int64_t)blockIdx.x * B;
  const int64_t rem = ln.nlines - l0;
  const int nb = rem < B ? (int)rem : B;
  const bool xfirst = ln.s1 == 1;   // consecutive lines are adjacent in memory
  // load
  for (int i = threadIdx.x; i < nb * L; i += blockDim.x) {
    int b, e;
    if (xfirst) { b = i % nb; e = i / nb; } else { e = i % L; b = i / L; }
    const int64_t l = l0 + b;
    b0[b * L + e] = data[(l % ln.n1) * ln.s1 + (l / ln.n1) * ln.s2 + e * ln.se];
  }
  __syncthreads();
  float2* src = b0;
  float2* dst = b1;
  int Ns = 1;
  for (int st = 0; st < plan.nfac; ++st) {
    const int R = plan.fac[st];
    const int nbf = L / R;
    for (int w = threadIdx.x; w < nb * nbf; w += blockDim.x) {
      const int b = w / nbf, j = w % nbf;
      const float2* s = src + b * L;
      float2* d = dst + b * L;
      const int k = j % Ns;
      const int idxD = (j / Ns) * Ns * R + k;
      switch (R) {
        case 2: radix_stage<2>(s, d, j, k, idxD, nbf, Ns, sign); break;
        case 3: radix_stage<3>(s, d, j, k, idxD, nbf, Ns, sign); break;
        case 4: radix_stage<4>(s, d, j, k, idxD, nbf, Ns, sign); break;
        case 5: radix_stage<5>(s, d, j, k, idxD, nbf, Ns, sign); break;
        case 7: radix_stage<7>(s, d, j, k, idxD, nbf, Ns, sign); break;
        default:
          for (int q = 0; q < R; ++q) {
            float2 acc = make_float2(0.f, 0.f);
            for (int p = 0; p < R; ++p) {
              float2 x = s[j + p * nbf];
              if (p) x = cmul(x, root((int64_t)k * p, Ns * R, sign));
              const float2 w2 = root((int64_t)p * q, R, sign);
              acc.x += x.x * w2.x - x.y * w2.y;
              acc.y += x.x * w2.y + x.y * w2.x;
            }
            d[idxD + q * Ns] = acc;
          }
      }
    }
    __syncthreads();
    float2* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  for (int i = threadIdx.x; i < nb * L; i += blockDim.x) {
    int b, e;
    if (xfirst) { b = i % nb; e = i / nb; } else { e = i % L; b = i / L; }
    const int64_t l = l0 + b;
    float2 v = src[b * L + e];
    v.x *= scale;
    v.y *= scale;
    data[(l % ln.n1) * ln.s1 + (l / ln.n1) * ln.s2 + e * ln.se] = v;
  }
}

struct Fft3D {
  int nx, ny, nz;
  Plan1D px, py, pz;
};

static qmt_status fft_axis(float2* d, const Plan1D& p, const Lines& ln, float sign, float scale, cudaStream_t s) {
  int B = std::max(1, std::min(16, 12288 / p.L));
  const size_t smem = 2 * (size_t)B * p.L * sizeof(float2);
  QMT_CUDA(cudaFuncSetAttribute(fft_lines_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t blocks = (ln.nlines + B - 1) / B;
  fft_lines_kernel<<<(unsigned)blocks, 256, smem, s>>>(d, p, ln, B, sign, scale);
  QMT_CHECK_LAUNCH("fft_lines_kernel");
  return QMT_OK;
}

// In-place 3D transform of an x-fastest nx*ny*nz complex grid; inverse includes 1/N.
static qmt_status fft3d(float2* d, const Fft3D& f, bool inverse, cudaStream_t s) {
  const float sign = inverse ? 1.f : -1.f;
  const int64_t nx = f.nx, ny = f.ny, nz = f.nz;
  const float sc = inverse ? (float)(1.0 / ((double)nx * ny * nz)) : 1.f;
  Lines lx{ny, nx, nx * ny, 1, ny * nz};
  Lines ly{nx, 1, nx * ny, nx, nx * nz};
  Lines lz{nx, 1, nx, nx * ny, nx * ny};
  qmt_status st;
  if ((st = fft_axis(d, f.px, lx, sign, 1.f, s))) return st;
  if ((st = fft_axis(d, f.py, ly, sign, 1.f, s))) return st;
  return fft_axis(d, f.pz, lz, sign, sc, s);
}

// ---- RHS assembly (kernel_fft.cu:23-79, Angstrom units) ---------------------------------------
// Writes the complex grid (x-fastest, dims M) with the value at voxel (x,y,z) < (nx,ny,nz);
// mode 0: RHS = -rho_tot/EPS0 (periodic); mode 1: rho_tot * h^3 (charge per voxel, free space).
__global__ void fft_rhs_kernel(MolView mol, const float* __restrict__ q, int nx, int ny, int nz, float h_ang,
                               float ox, float oy, float oz, float sigma, float cut2, int mode, int Mx, int My,
                               int Mz, float2* __restrict__ out) {
  extern __shared__ float sat[];
  for (int i = threadIdx.x; i < mol.natoms; i += blockDim.x) {
    sat[4 * i] = mol.coords[3 * i] * (float)R_BOHR;
    sat[4 * i + 1] = mol.coords[3 * i + 1] * (float)R_BOHR;
    sat[4 * i + 2] = mol.coords[3 * i + 2] * (float)R_BOHR;
    sat[4 * i + 3] = (float)mol.types[i];
  }
  __syncthreads();
  const int64_t n = (int64_t)Mx * My * Mz;
  const float norm = 1.0f / (sigma * sigma * sigma * 2.0f * 3.14159265358979f * sqrtf(2.0f * 3.14159265358979f));
  const float i2s2 = 1.0f / (2.0f * sigma * sigma);
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(idx % Mx), y = (int)((idx / Mx) % My), z = (int)(idx / ((int64_t)Mx * My));
    float v = 0.f;
    if (x < nx && y < ny && z < nz) {
      const float px = ox + (x + 0.5f) * h_ang, py = oy + (y + 0.5f) * h_ang, pz = oz + (z + 0.5f) * h_ang;
      float rho = q[x + (int64_t)y * nx + (int64_t)z * nx * ny] / (-h_ang * h_ang * h_ang);
      for (int a = 0; a < mol.natoms; ++a) {
        const float cx = px - sat[4 * a], cy = py - sat[4 * a + 1], cz = pz - sat[4 * a + 2];
        const float r2 = cx * cx + cy * cy + cz * cz;
        if (r2 <= cut2) rho += sat[4 * a + 3] * norm * expf(-r2 * i2s2);
      }
      v = mode == 0 ? (float)(-(double)rho / EPS0) : rho * h_ang * h_ang * h_ang;
    }
    out[idx] = make_float2(v, 0.f);
  }
}

// V_hat = -RHS_hat / (4 pi^2 |k|^2), k in cycles/Ang; k = 0 -> 0  (kernel_fft.cu:82-107)
__global__ void periodic_scale_kernel(float2* __restrict__ c, int nx, int ny, int nz, float h_ang) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((int64_t)nx * ny));
    if (idx == 0) {
      c[0] = make_float2(0.f, 0.f);
      continue;
    }
    const float kx = (i > nx / 2 - 1 ? (float)(i - nx) : (float)i) / (nx * h_ang);
    const float ky = (j > ny / 2 - 1 ? (float)(j - ny) : (float)j) / (ny * h_ang);
    const float kz = (k > nz / 2 - 1 ? (float)(k - nz) : (float)k) / (nz * h_ang);
    const float sc = (float)(-1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846 *
                                     (double)(kx * kx + ky * ky + kz * kz)));
    float2 v = c[idx];
    v.x *= sc;
    v.y *= sc;
    c[idx] = v;
  }
}

// Green's function on the padded grid (minimum image), real part only.
__global__ void green_kernel(float2* __restrict__ g, int Mx, int My, int Mz, float h_ang) {
  const int64_t n = (int64_t)Mx * My * Mz;
  const double pref = 1.0 / (4.0 * 3.14159265358979323846 * EPS0);
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % Mx, j = (idx / Mx) % My, k = idx / ((int64_t)Mx * My);
    const double x = (double)min(i, Mx - i) * h_ang, y = (double)min(j, My - j) * h_ang,
                 z = (double)min(k, Mz - k) * h_ang;
    const double r = sqrt(x * x + y * y + z * z);
    const double v = r > 0 ? pref / r : pref * CUBE_INV_R / h_ang;
    g[idx] = make_float2((float)v, 0.f);
  }
}

__global__ void take_real_kernel(const float2* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i].x;
}

__global__ void mul_real_kernel(float2* __restrict__ c, const float* __restrict__ g, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float2 v = c[i];
    const float s = g[i];
    c[i] = make_float2(v.x * s, v.y * s);
  }
}

// out[i*ny*nz + j*nz + k] = Re c[x=i, y=j, z=k] for the first (nx,ny,nz) of an Mx-by-My-by-Mz grid.
__global__ void to_corder_kernel(const float2* __restrict__ c, int Mx, int My, int nx, int ny, int nz,
                                 float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int y = blockIdx.z;
  const int x0 = blockIdx.x * 32, z0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int z = z0 + r, x = x0 + threadIdx.x;
    if (z < nz && x < nx) tile[r][threadIdx.x] = c[x + (int64_t)y * Mx + (int64_t)z * Mx * My].x;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int x = x0 + r, z = z0 + threadIdx.x;
    if (z < nz && x < nx) out[(int64_t)x * ny * nz + (int64_t)y * nz + z] = tile[threadIdx.x][r];
  }
}

// ---- host ------------------------------------------------------------------------------------
struct GreenCache {
  DevBuf g;
};
static std::map<std::tuple<int, int, int, float, int>, DevBuf*>& green_cache() {
  static std::map<std::tuple<int, int, int, float, int>, DevBuf*> m;
  return m;
}

static qmt_status make_plan(int nx, int ny, int nz, Fft3D& f) {
  f.nx = nx;
  f.ny = ny;
  f.nz = nz;
  if (!factorize(nx, f.px) || !factorize(ny, f.py) || !factorize(nz, f.pz))
    return fail(QMT_BAD_ARG, "FFT size has too many factors");
  for (const Plan1D* p : {&f.px, &f.py, &f.pz})
    for (int i = 0; i < p->nfac; ++i)
      if (p->fac[i] > 127) return fail(QMT_BAD_ARG, "FFT size has a prime factor above 127");
  if (std::max(nx, std::max(ny, nz)) > 4096) return fail(QMT_BAD_ARG, "FFT line longer than 4096");
  return QMT_OK;
}

static unsigned grid_blocks(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16); }

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                                      float oz, float sigma, float cutoff, int padded, const float* q_dev,
                                      float* out_dev, void* stream) {
  if (!mol || !q_dev || !out_dev || nx < 2 || ny < 2 || nz < 2 || !(step > 0.f) || !(sigma > 0.f) || cutoff < 0)
    return fail(QMT_BAD_ARG, "bad FFT Poisson arguments");
  if (mol->natoms > 8192) return fail(QMT_BAD_ARG, "too many atoms");
  cudaStream_t s = as_stream(stream);
  const float h_ang = (float)(step / ANG2BOR);
  const float oxa = (float)(ox / ANG2BOR), oya = (float)(oy / ANG2BOR), oza = (float)(oz / ANG2BOR);
  const float cut2 = (cutoff * sigma) * (cutoff * sigma);
  int Mx = nx, My = ny, Mz = nz;
  if (padded) {
    Mx = nice_at_least(2 * nx);
    My = nice_at_least(2 * ny);
    Mz = nice_at_least(2 * nz);
  }
  Fft3D plan;
  qmt_status st = make_plan(Mx, My, Mz, plan);
  if (st) return st;
  const int64_t M = (int64_t)Mx * My * Mz;
  if ((st = mol->d_work.reserve(M * sizeof(float2)))) return st;
  float2* c = mol->d_work.as<float2>();
  const size_t ash = 16 * (size_t)mol->natoms;
  fft_rhs_kernel<<<grid_blocks(M), 256, ash, s>>>(mol->view(), q_dev, nx, ny, nz, h_ang, oxa, oya, oza, sigma, cut2,
                                                  padded ? 1 : 0, Mx, My, Mz, c);
  QMT_CHECK_LAUNCH("fft_rhs_kernel");
  if ((st = fft3d(c, plan, false, s))) return st;
  if (!padded) {
    periodic_scale_kernel<<<grid_blocks(M), 256, 0, s>>>(c, Mx, My, Mz, h_ang);
    QMT_CHECK_LAUNCH("periodic_scale_kernel");
  } else {
    int dev = 0;
    cudaGetDevice(&dev);
    auto key = std::make_tuple(Mx, My, Mz, h_ang, dev);
    auto& cache = green_cache();
    DevBuf*& gb = cache[key];
    if (!gb) {
      gb = new DevBuf();
      DevBuf tmp;
      if ((st = gb->reserve(M * sizeof(float))) || (st = tmp.reserve(M * sizeof(float2)))) {
        delete gb;
        gb = nullptr;
        cache.erase(key);
        return st;
      }
      green_kernel<<<grid_blocks(M), 256, 0, s>>>(tmp.as<float2>(), Mx, My, Mz, h_ang);
      QMT_CHECK_LAUNCH("green_kernel");
      if ((st = fft3d(tmp.as<float2>(), plan, false, s))) return st;
      take_real_kernel<<<grid_blocks(M), 256, 0, s>>>(tmp.as<float2>(), gb->as<float>(), M);
      QMT_CHECK_LAUNCH("take_real_kernel");
      QMT_CUDA(cudaStreamSynchronize(s));
      tmp.release();
    }
    mul_real_kernel<<<grid_blocks(M), 256, 0, s>>>(c, gb->as<float>(), M);
    QMT_CHECK_LAUNCH("mul_real_kernel");
  }
  if ((st = fft3d(c, plan, true, s))) return st;
  dim3 tb(32, 8), tg((nx + 31) / 32, (nz + 31) / 32, ny);
  to_corder_kernel<<<tg, tb, 0, s>>>(c, Mx, My, nx, ny, nz, out_dev);
  QMT_CHECK_LAUNCH("to_corder_kernel");
  return QMT_OK;
}

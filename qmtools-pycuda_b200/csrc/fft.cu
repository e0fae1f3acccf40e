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
//   factors 2, 3, 5, 7), G(0) = voxel-cube average of 1/|r|; G_hat is real and even, so only
//   its octant [0, M/2]^3 is stored, cached per (M, h, device).
//
// 1D transforms are mixed-radix Stockham (self-sorting) FFTs of batches of lines in shared
// memory, twiddles from a per-length table computed in FP64 on the host; 256- and 128-point
// lines (the padded axes of 128- and 64-voxel boxes) take register kernels instead (16 x 16 and
// 16 x 8 four-step, one shared-memory exchange per transform).  A solve is five passes over an
// x-fastest complex work grid:
//   1. x forward, with the RHS assembled on the fly from q and the nuclei (only lines and
//      elements inside the physical box are non-zero: y < ny, z < nz, x < nx);
//   2. y forward on the z < nz planes (elements y >= ny are zero and not read);
//   3. z forward, multiply by G_hat (or the periodic k-space factor), z inverse, store z < nz;
//   4. y inverse on the z < nz planes, store y < ny;
//   5. x inverse, 1/M^3, real part written straight into the C-order output (x < nx).
// Zero padding therefore costs about 2.5 full-grid passes instead of 6.
#include <algorithm>
#include <map>
#include <tuple>

#include <mutex>

#include "mol.cuh"

namespace qmt {

constexpr double EPS0 = 0.0055263494;       // e/(V*Ang), kernel_fft.cu:18
constexpr double R_BOHR = 0.529177211;      // kernel_fft.cu:17
constexpr double CUBE_INV_R = 2.3800772417; // h * <1/|r|> over a voxel cube
constexpr double PI = 3.14159265358979323846;
constexpr int FFT_MAXFAC = 16;
constexpr int FFT_MAXLEN = 2048;

struct Plan1D {
  int L;
  int nfac;
  int fac[FFT_MAXFAC];
  // per stage: Ns (product of the earlier radices) and exact multiply-high divisors
  // ceil(2^32 / d) for d = L / R and d = Ns (dividends stay below 2^16, divisors <= 2048;
  // d == 1 does not fit in 32 bits and is handled without the multiply)
  int ns[FFT_MAXFAC];
  unsigned m_nbf[FFT_MAXFAC], m_ns[FFT_MAXFAC];
  unsigned m_len;   // ceil(2^32 / L)
};

constexpr int FFT_CAND = 24;   // nuclei listed per x line for the right-hand side

__device__ __forceinline__ unsigned fdiv(unsigned n, unsigned m) { return __umulhi(n, m); }

static bool factorize(int L, Plan1D& p) {
  p.L = L;
  p.nfac = 0;
  int n = L;
  for (int r : {4, 2, 3, 5, 7})
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

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// table entry m: exp(-2 pi i m / L); conjugated for the inverse direction
__device__ __forceinline__ float2 twid(const float2* tw, int m, bool inv) {
  const float2 t = tw[m];
  return inv ? make_float2(t.x, -t.y) : t;
}

// One radix-R butterfly of a Stockham stage (twiddle, DFT_R, scatter to sorted position).
template <int R>
__device__ __forceinline__ void radix_stage(const float2* __restrict__ s, float2* __restrict__ d, int j, int k,
                                            int idxD, int nbf, int Ns, const float2* tw, int L, bool inv) {
  const int step = L / (Ns * R);
  float2 v[R];
  v[0] = s[j];
#pragma unroll
  for (int q = 1; q < R; ++q) v[q] = cmul(s[j + q * nbf], twid(tw, k * q * step, inv));
  if constexpr (R == 2) {
    d[idxD] = cadd(v[0], v[1]);
    d[idxD + Ns] = csub(v[0], v[1]);
  } else if constexpr (R == 4) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    // b1 times exp(-+ i pi/2): forward -i, inverse +i
    const float2 b1r = inv ? make_float2(-b1.y, b1.x) : make_float2(b1.y, -b1.x);
    d[idxD] = cadd(a0, b0);
    d[idxD + Ns] = cadd(a1, b1r);
    d[idxD + 2 * Ns] = csub(a0, b0);
    d[idxD + 3 * Ns] = csub(a1, b1r);
  } else {
    float2 w[R];
#pragma unroll
    for (int m = 0; m < R; ++m) w[m] = twid(tw, m * (L / R), inv);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float2 acc = v[0];
#pragma unroll
      for (int p = 1; p < R; ++p) acc = cadd(acc, cmul(v[p], w[(p * q) % R]));
      d[idxD + q * Ns] = acc;
    }
  }
}

// Transforms nb lines of length plan.L held in `src` (ping-pong with `dst`); the pointer
// holding the result is returned in *result.
__device__ void fft_lines_smem(float2* src, float2* dst, const Plan1D& plan, int nb, const float2* tw, bool inv,
                               float2** result) {
  const int L = plan.L;
  for (int st = 0; st < plan.nfac; ++st) {
    const int R = plan.fac[st];
    const int nbf = L / R;
    const int Ns = plan.ns[st];
    const unsigned mnbf = plan.m_nbf[st], mns = plan.m_ns[st];
    for (int w = threadIdx.x; w < nb * nbf; w += blockDim.x) {
      const int b = nbf == 1 ? w : (int)fdiv((unsigned)w, mnbf), j = w - b * nbf;
      const float2* s = src + b * L;
      float2* d = dst + b * L;
      const int jq = Ns == 1 ? j : (int)fdiv((unsigned)j, mns);
      const int k = j - jq * Ns;
      const int idxD = jq * Ns * R + k;
      switch (R) {
        case 2: radix_stage<2>(s, d, j, k, idxD, nbf, Ns, tw, L, inv); break;
        case 3: radix_stage<3>(s, d, j, k, idxD, nbf, Ns, tw, L, inv); break;
        case 4: radix_stage<4>(s, d, j, k, idxD, nbf, Ns, tw, L, inv); break;
        case 5: radix_stage<5>(s, d, j, k, idxD, nbf, Ns, tw, L, inv); break;
        case 7: radix_stage<7>(s, d, j, k, idxD, nbf, Ns, tw, L, inv); break;
        default: {
          const int step = L / (Ns * R);
          for (int q = 0; q < R; ++q) {
            float2 acc = make_float2(0.f, 0.f);
            for (int p = 0; p < R; ++p) {
              float2 x = s[j + p * nbf];
              if (p) x = cmul(x, twid(tw, k * p * step, inv));
              acc = cadd(acc, cmul(x, twid(tw, ((p * q) % R) * (L / R), inv)));
            }
            d[idxD + q * Ns] = acc;
          }
        }
      }
    }
    __syncthreads();
    float2* t = src;
    src = dst;
    dst = t;
  }
  *result = src;
}

enum { PASS_PLAIN = 0, PASS_X_RHS = 1, PASS_Z_MUL = 2, PASS_X_OUT = 3 };

struct PassArgs {
  Plan1D plan;
  int64_t n1, s1, s2, se, nlines;   // line l: base (l % n1)*s1 + (l / n1)*s2, element e at + e*se
  int lload, lstore;                // elements >= lload are zero; only e < lstore are stored
  int B;                            // lines per CTA
  int inv;                          // direction of the (first) transform
  float scale;
  const float2* tw;
  float2* data;
  // RHS assembly (PASS_X_RHS): lines are (y, z) with n1 = ny
  MolView mol;
  const float* q;
  int nx, ny, nz;
  float h_ang, ox, oy, oz, norm, i2s2, cut2;
  int periodic;
  // multiply (PASS_Z_MUL): lines are (x, y) with n1 = Mx
  const float* gsym;
  int Mx, My, Mz;
  // C-order real output (PASS_X_OUT): lines are (z, y) with n1 = nz
  float* out;
};

template <int MODE>
__global__ void __launch_bounds__(256) fft_pass_kernel(const PassArgs a) {
  extern __shared__ float2 fsm[];
  const int L = a.plan.L;
  float2* tw = fsm;
  float2* b0 = fsm + L;
  float2* b1 = b0 + (size_t)a.B * L;
  float* sat = reinterpret_cast<float*>(b1 + (size_t)a.B * L);   // atoms (PASS_X_RHS)
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = a.tw[i];
  if constexpr (MODE == PASS_X_RHS) {
    for (int i = threadIdx.x; i < a.mol.natoms; i += blockDim.x) {
      sat[4 * i] = a.mol.coords[3 * i] * (float)R_BOHR;
      sat[4 * i + 1] = a.mol.coords[3 * i + 1] * (float)R_BOHR;
      sat[4 * i + 2] = a.mol.coords[3 * i + 2] * (float)R_BOHR;
      sat[4 * i + 3] = (float)a.mol.types[i];
    }
  }
  const int64_t l0 = (int64_t)blockIdx.x * a.B;
  const int64_t rem = a.nlines - l0;
  const int nb = rem < a.B ? (int)rem : a.B;
  const bool lines_adjacent = a.s1 == 1;
  // per-line data, computed once per CTA (B <= 16 lines)
  __shared__ int64_t lbase[16];          // element 0 of the line in the work grid / output
  __shared__ int lx[16], ly[16];         // the line's two grid coordinates (RHS, multiply, output)
  __shared__ int ncand[16];              // RHS: nuclei within the cut-off of the line, or -1 for all
  __shared__ int cand[16][FFT_CAND];
  __syncthreads();   // twiddles and nuclei are in shared memory
  if (threadIdx.x < nb) {
    const int b = threadIdx.x;
    const int64_t l = l0 + b;
    const int c0 = (int)(l % a.n1), c1 = (int)(l / a.n1);
    lx[b] = c0;
    ly[b] = c1;
    lbase[b] = (int64_t)c0 * a.s1 + (int64_t)c1 * a.s2;
    if constexpr (MODE == PASS_X_RHS) {
      // line (y = c0, z = c1) along x: keep the nuclei whose (y, z) distance passes the cut-off
      const float py = a.oy + (c0 + 0.5f) * a.h_ang, pz = a.oz + (c1 + 0.5f) * a.h_ang;
      int cnt = 0;
      for (int at = 0; at < a.mol.natoms; ++at) {
        const float cy = py - sat[4 * at + 1], cz = pz - sat[4 * at + 2];
        if (cy * cy + cz * cz <= a.cut2 * 1.0001f) {   // superset of the per-point test below
          if (cnt < FFT_CAND) cand[b][cnt] = at;
          ++cnt;
        }
      }
      ncand[b] = cnt <= FFT_CAND ? cnt : -1;
    }
  }
  __syncthreads();
  // ---- load ----
  auto load_one = [&](int b, int e) {
    float2 v = make_float2(0.f, 0.f);
    if (e < a.lload) {
      if constexpr (MODE == PASS_X_RHS) {
        const int y = lx[b], z = ly[b], x = e;
        const float px = a.ox + (x + 0.5f) * a.h_ang, py = a.oy + (y + 0.5f) * a.h_ang,
                    pz = a.oz + (z + 0.5f) * a.h_ang;
        float rho = a.q[x + (int64_t)y * a.nx + (int64_t)z * a.nx * a.ny] / (-a.h_ang * a.h_ang * a.h_ang);
        const int nc = ncand[b];
        const int cnt = nc < 0 ? a.mol.natoms : nc;
        for (int c = 0; c < cnt; ++c) {
          const int at = nc < 0 ? c : cand[b][c];
          const float cx = px - sat[4 * at], cy = py - sat[4 * at + 1], cz = pz - sat[4 * at + 2];
          const float r2 = cx * cx + cy * cy + cz * cz;
          if (r2 <= a.cut2) rho += sat[4 * at + 3] * a.norm * expf(-r2 * a.i2s2);
        }
        v.x = a.periodic ? (float)(-(double)rho / EPS0) : rho * a.h_ang * a.h_ang * a.h_ang;
      } else {
        v = a.data[lbase[b] + (int64_t)e * a.se];
      }
    }
    b0[b * L + e] = v;
  };
  if (lines_adjacent) {
    // 16 adjacent lines side by side: one 128-byte row of the grid per element index
    const int b = threadIdx.x & 15;
    for (int e = threadIdx.x >> 4; e < L; e += 16)
      if (b < nb) load_one(b, e);
  } else {
    for (int b = 0; b < nb; ++b)
      for (int e = threadIdx.x; e < L; e += blockDim.x) load_one(b, e);
  }
  __syncthreads();
  float2* res;
  fft_lines_smem(b0, b1, a.plan, nb, tw, a.inv != 0, &res);
  if constexpr (MODE == PASS_Z_MUL) {
    const int hx = a.Mx / 2 + 1, hy = a.My / 2 + 1;
    for (int i = threadIdx.x; i < nb * L; i += blockDim.x) {
      const int b = (int)fdiv((unsigned)i, a.plan.m_len), kz = i - b * L;
      const int x = lx[b], y = ly[b];
      float f;
      if (a.periodic) {
        // kernel_fft.cu:90-104: k in cycles/Ang, negative frequencies above N/2 - 1, k = 0 -> 0
        const float kx = (x > a.Mx / 2 - 1 ? (float)(x - a.Mx) : (float)x) / (a.Mx * a.h_ang);
        const float ky = (y > a.My / 2 - 1 ? (float)(y - a.My) : (float)y) / (a.My * a.h_ang);
        const float kk = (kz > a.Mz / 2 - 1 ? (float)(kz - a.Mz) : (float)kz) / (a.Mz * a.h_ang);
        const double k2 = (double)(kx * kx + ky * ky + kk * kk);
        f = (x == 0 && y == 0 && kz == 0) ? 0.f : (float)(-1.0 / (4.0 * PI * PI * k2));
      } else {
        const int gx = min(x, a.Mx - x), gy = min(y, a.My - y), gz = min(kz, a.Mz - kz);
        f = __ldg(a.gsym + gx + (int64_t)hx * (gy + (int64_t)hy * gz));
      }
      float2 v = res[b * L + kz];
      res[b * L + kz] = make_float2(v.x * f, v.y * f);
    }
    __syncthreads();
    float2* other = res == b0 ? b1 : b0;
    fft_lines_smem(res, other, a.plan, nb, tw, a.inv == 0, &res);
  }
  // ---- store ----
  auto store_one = [&](int b, int e) {
    const float2 v = res[b * L + e];
    if constexpr (MODE == PASS_X_OUT) {
      // line (z = lx, y = ly) along x into the C-order output
      a.out[(int64_t)e * a.ny * a.nz + (int64_t)ly[b] * a.nz + lx[b]] = v.x * a.scale;
    } else {
      a.data[lbase[b] + (int64_t)e * a.se] = make_float2(v.x * a.scale, v.y * a.scale);
    }
  };
  if (lines_adjacent || MODE == PASS_X_OUT) {
    const int b = threadIdx.x & 15;
    for (int e = threadIdx.x >> 4; e < a.lstore; e += 16)
      if (b < nb) store_one(b, e);
  } else {
    for (int b = 0; b < nb; ++b)
      for (int e = threadIdx.x; e < a.lstore; e += blockDim.x) store_one(b, e);
  }
}

// ---- 256- and 128-point lines in registers -----------------------------------------------
// Four-step transforms with every thread holding 16 elements e = t + TPL m (m = 0..15) of its
// line, TPL = L / 16 threads per line, 256 / TPL lines per CTA: the 16-point DFT over m, the
// twiddle W_L^(t k1), one exchange through shared memory, then the DFTs over t.  L = 256: thread
// t forms the 16-point DFT of k1 = t (16 values); L = 128: the two 8-point DFTs of k1 = t and
// t + 8.  Either way the thread then holds X[t + TPL m'] in register m', the same element pattern
// as its input, so global loads and stores are issued 16 per thread back to back.
struct Tw16 {
  float2 w1, w2, w3, w6, w9;   // W16^p = table entry (L/16) p (conjugated for the inverse)
};

template <int L>
__device__ __forceinline__ Tw16 tw16(const float2* tw, bool inv) {
  constexpr int st = L / 16;
  return Tw16{twid(tw, st, inv), twid(tw, 2 * st, inv), twid(tw, 3 * st, inv), twid(tw, 6 * st, inv),
              twid(tw, 9 * st, inv)};
}

// In-place 4-point DFT (forward: W4 = -i; inverse: +i).
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3, bool inv) {
  const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
  const float2 t3r = inv ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3r);
  a3 = csub(t1, t3r);
}

// 16-point DFT of x[0..15] (4 x 4), result in natural order.
__device__ __forceinline__ void dft16(float2 (&x)[16], const Tw16& w, bool inv) {
#pragma unroll
  for (int m2 = 0; m2 < 4; ++m2) dft4(x[m2], x[4 + m2], x[8 + m2], x[12 + m2], inv);
  // x[m2 + 4 k1] holds the m2-th partial DFT at k1: twiddle W16^(m2 k1)
  x[5] = cmul(x[5], w.w1);
  x[9] = cmul(x[9], w.w2);
  x[13] = cmul(x[13], w.w3);
  x[6] = cmul(x[6], w.w2);
  x[10] = inv ? make_float2(-x[10].y, x[10].x) : make_float2(x[10].y, -x[10].x);   // W16^4 = -+i
  x[14] = cmul(x[14], w.w6);
  x[7] = cmul(x[7], w.w3);
  x[11] = cmul(x[11], w.w6);
  x[15] = cmul(x[15], w.w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3], inv);
  // x[4 k1 + k2] holds X[k1 + 4 k2]
  float2 y[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) y[k1 + 4 * k2] = x[4 * k1 + k2];
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = y[k];
}

// 8-point DFT of y[0..7] (even/odd 4-point DFTs), result in natural order; w1, w3 = W8^1, W8^3.
__device__ __forceinline__ void dft8(float2 (&y)[8], float2 w1, float2 w3, bool inv) {
  float2 a0 = y[0], a1 = y[2], a2 = y[4], a3 = y[6];
  float2 b0 = y[1], b1 = y[3], b2 = y[5], b3 = y[7];
  dft4(a0, a1, a2, a3, inv);
  dft4(b0, b1, b2, b3, inv);
  b1 = cmul(b1, w1);
  b2 = inv ? make_float2(-b2.y, b2.x) : make_float2(b2.y, -b2.x);   // W8^2 = -+i
  b3 = cmul(b3, w3);
  y[0] = cadd(a0, b0);
  y[1] = cadd(a1, b1);
  y[2] = cadd(a2, b2);
  y[3] = cadd(a3, b3);
  y[4] = csub(a0, b0);
  y[5] = csub(a1, b1);
  y[6] = csub(a2, b2);
  y[7] = csub(a3, b3);
}

// Exchange-buffer geometry per length: element (k1, t) of line b at b S + k1 R + t.  R and S are
// chosen so that neither thread mapping (lines or elements fastest) has bank conflicts.
template <int L> struct RegFft;
template <> struct RegFft<256> {
  static constexpr int TPL = 16, LINES = 16, R = 17, S_MAX = 273;
  static __device__ __forceinline__ int S(bool) { return 273; }
};
template <> struct RegFft<128> {
  static constexpr int TPL = 8, LINES = 32, R = 9, S_MAX = 152;
  static __device__ __forceinline__ int S(bool bfast) { return bfast ? 143 : 152; }
};

// One transform of the thread's line b (thread t of it); `buf` is the CTA's exchange buffer,
// free on entry (the barrier below orders it after earlier readers).
template <int L>
__device__ __forceinline__ void fft_regs(float2 (&x)[16], const float2* tw, float2* buf, int b, int t, int S,
                                         bool inv) {
  constexpr int R = RegFft<L>::R;
  const Tw16 w = tw16<L>(tw, inv);
  dft16(x, w, inv);
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1) x[k1] = cmul(x[k1], twid(tw, (t * k1) & (L - 1), inv));
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) buf[b * S + k1 * R + t] = x[k1];
  __syncthreads();
  if constexpr (L == 256) {
#pragma unroll
    for (int u = 0; u < 16; ++u) x[u] = buf[b * S + t * R + u];
    dft16(x, w, inv);
  } else {
    const float2 w1 = twid(tw, L / 8, inv), w3 = twid(tw, 3 * L / 8, inv);
    float2 ya[8], yb[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      ya[u] = buf[b * S + t * R + u];
      yb[u] = buf[b * S + (t + 8) * R + u];
    }
    dft8(ya, w1, w3, inv);
    dft8(yb, w1, w3, inv);
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
      x[2 * k2] = ya[k2];       // X[t + 16 k2]     = element t + 8 (2 k2)
      x[2 * k2 + 1] = yb[k2];   // X[t + 8 + 16 k2] = element t + 8 (2 k2 + 1)
    }
  }
}

template <int MODE, int L>
__global__ void __launch_bounds__(256) fft_reg_pass_kernel(const PassArgs a) {
  constexpr int TPL = RegFft<L>::TPL, LINES = RegFft<L>::LINES;
  extern __shared__ float2 fsm[];
  float2* tw = fsm;
  float2* buf = fsm + L;
  float* sat = reinterpret_cast<float*>(buf + LINES * RegFft<L>::S_MAX);   // atoms (PASS_X_RHS)
  for (int i = threadIdx.x; i < L; i += blockDim.x) tw[i] = a.tw[i];
  if constexpr (MODE == PASS_X_RHS) {
    for (int i = threadIdx.x; i < a.mol.natoms; i += blockDim.x) {
      sat[4 * i] = a.mol.coords[3 * i] * (float)R_BOHR;
      sat[4 * i + 1] = a.mol.coords[3 * i + 1] * (float)R_BOHR;
      sat[4 * i + 2] = a.mol.coords[3 * i + 2] * (float)R_BOHR;
      sat[4 * i + 3] = (float)a.mol.types[i];
    }
  }
  const int64_t l0 = (int64_t)blockIdx.x * LINES;
  const int64_t rem = a.nlines - l0;
  const int nb = rem < LINES ? (int)rem : LINES;
  __shared__ int64_t lbase[LINES];
  __shared__ int lx[LINES], ly[LINES];
  __shared__ int ncand[LINES];
  __shared__ int cand[LINES][FFT_CAND];
  __syncthreads();
  if (threadIdx.x < nb) {
    const int bb = threadIdx.x;
    const int64_t l = l0 + bb;
    const int c0 = (int)(l % a.n1), c1 = (int)(l / a.n1);
    lx[bb] = c0;
    ly[bb] = c1;
    lbase[bb] = (int64_t)c0 * a.s1 + (int64_t)c1 * a.s2;
    if constexpr (MODE == PASS_X_RHS) {
      const float py = a.oy + (c0 + 0.5f) * a.h_ang, pz = a.oz + (c1 + 0.5f) * a.h_ang;
      int cnt = 0;
      for (int at = 0; at < a.mol.natoms; ++at) {
        const float cy = py - sat[4 * at + 1], cz = pz - sat[4 * at + 2];
        if (cy * cy + cz * cz <= a.cut2 * 1.0001f) {
          if (cnt < FFT_CAND) cand[bb][cnt] = at;
          ++cnt;
        }
      }
      ncand[bb] = cnt <= FFT_CAND ? cnt : -1;
    }
  }
  __syncthreads();
  // lines adjacent in memory: a half-warp spans 16 lines at one element; lines contiguous: it
  // spans consecutive elements of one (L = 256) or two (L = 128) lines
  const bool bfast = a.s1 == 1;
  const int b = bfast ? (int)(threadIdx.x % LINES) : (int)(threadIdx.x / TPL);
  const int t = bfast ? (int)(threadIdx.x / LINES) : (int)(threadIdx.x % TPL);
  const int S = RegFft<L>::S(bfast);
  const bool live = b < nb;
  float2 x[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int e = t + TPL * m;
    float2 v = make_float2(0.f, 0.f);
    if (live && e < a.lload) {
      if constexpr (MODE == PASS_X_RHS) {
        const int y = lx[b], z = ly[b], xx = e;
        const float px = a.ox + (xx + 0.5f) * a.h_ang, py = a.oy + (y + 0.5f) * a.h_ang,
                    pz = a.oz + (z + 0.5f) * a.h_ang;
        float rho = a.q[xx + (int64_t)y * a.nx + (int64_t)z * a.nx * a.ny] / (-a.h_ang * a.h_ang * a.h_ang);
        const int nc = ncand[b];
        const int cnt = nc < 0 ? a.mol.natoms : nc;
        for (int c = 0; c < cnt; ++c) {
          const int at = nc < 0 ? c : cand[b][c];
          const float cx = px - sat[4 * at], cy = py - sat[4 * at + 1], cz = pz - sat[4 * at + 2];
          const float r2 = cx * cx + cy * cy + cz * cz;
          if (r2 <= a.cut2) rho += sat[4 * at + 3] * a.norm * expf(-r2 * a.i2s2);
        }
        v.x = a.periodic ? (float)(-(double)rho / EPS0) : rho * a.h_ang * a.h_ang * a.h_ang;
      } else {
        v = a.data[lbase[b] + (int64_t)e * a.se];
      }
    }
    x[m] = v;
  }
  fft_regs<L>(x, tw, buf, b, t, S, a.inv != 0);
  if constexpr (MODE == PASS_Z_MUL) {
    const int hx = a.Mx / 2 + 1, hy = a.My / 2 + 1;
    const int xg = lx[b], yg = ly[b];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int kz = t + TPL * m;
      float f;
      if (a.periodic) {
        // kernel_fft.cu:90-104: k in cycles/Ang, negative frequencies above N/2 - 1, k = 0 -> 0
        const float kx = (xg > a.Mx / 2 - 1 ? (float)(xg - a.Mx) : (float)xg) / (a.Mx * a.h_ang);
        const float ky = (yg > a.My / 2 - 1 ? (float)(yg - a.My) : (float)yg) / (a.My * a.h_ang);
        const float kk = (kz > a.Mz / 2 - 1 ? (float)(kz - a.Mz) : (float)kz) / (a.Mz * a.h_ang);
        const double k2d = (double)(kx * kx + ky * ky + kk * kk);
        f = (xg == 0 && yg == 0 && kz == 0) ? 0.f : (float)(-1.0 / (4.0 * PI * PI * k2d));
      } else {
        const int gx = min(xg, a.Mx - xg), gy = min(yg, a.My - yg), gz = min(kz, a.Mz - kz);
        f = live ? __ldg(a.gsym + gx + (int64_t)hx * (gy + (int64_t)hy * gz)) : 0.f;
      }
      x[m] = make_float2(x[m].x * f, x[m].y * f);
    }
    fft_regs<L>(x, tw, buf, b, t, S, a.inv == 0);
  }
  if constexpr (MODE == PASS_X_OUT) {
    // line (z = lx, y = ly) along x into the C-order output: regroup through shared memory so
    // that a warp writes consecutive z of one x
    constexpr int S2 = L + 1;
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 16; ++m) buf[b * S2 + t + TPL * m] = x[m];
    __syncthreads();
    const int bo = (int)(threadIdx.x % LINES);
    if (bo < nb)
      for (int e = (int)(threadIdx.x / LINES); e < a.lstore; e += TPL)
        a.out[(int64_t)e * a.ny * a.nz + (int64_t)ly[bo] * a.nz + lx[bo]] = buf[bo * S2 + e].x * a.scale;
  } else {
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int e = t + TPL * m;
      if (live && e < a.lstore)
        a.data[lbase[b] + (int64_t)e * a.se] = make_float2(x[m].x * a.scale, x[m].y * a.scale);
    }
  }
}

// ---- Green's function ----------------------------------------------------------------
__global__ void green_kernel(float2* __restrict__ g, int Mx, int My, int Mz, float h_ang) {
  const int64_t n = (int64_t)Mx * My * Mz;
  const double pref = 1.0 / (4.0 * PI * EPS0);
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % Mx, j = (idx / Mx) % My, k = idx / ((int64_t)Mx * My);
    const double x = (double)min(i, Mx - i) * h_ang, y = (double)min(j, My - j) * h_ang,
                 z = (double)min(k, Mz - k) * h_ang;
    const double r = sqrt(x * x + y * y + z * z);
    const double v = r > 0 ? pref / r : pref * CUBE_INV_R / h_ang;
    g[idx] = make_float2((float)v, 0.f);
  }
}

__global__ void green_octant_kernel(const float2* __restrict__ g, int Mx, int My, int Mz, float* __restrict__ out) {
  const int ox = Mx / 2 + 1, oy = My / 2 + 1, oz = Mz / 2 + 1;
  const int64_t n = (int64_t)ox * oy * oz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx % ox, j = (idx / ox) % oy, k = idx / ((int64_t)ox * oy);
    out[idx] = g[i + j * Mx + k * (int64_t)Mx * My].x;
  }
}

// ---- host ------------------------------------------------------------------------------------
static unsigned grid_blocks(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 16); }

struct GreenEntry {
  DevBuf* buf;
  uint64_t used;        // last use, for least-recently-used eviction
  size_t bytes;
  cudaEvent_t ready;    // recorded after the build, on the stream that built it
  bool built;           // `ready` seen complete: later solves need no wait (and, inside a CUDA-graph
                        // capture, make no event call)
};

// Device-side caches shared by all calls: twiddle tables per (length, device), transformed
// Green's functions per (padded shape, step, device) up to GREEN_CACHE_BYTES of octants, and one
// growing scratch grid per device for building them.  `tw_mu` guards the twiddles and `green_mu`
// the rest; building a Green's function takes green_mu and then (through its FFT passes) tw_mu,
// never the other way round.  No host synchronisation in steady state: a solve on another
// stream waits for a cached octant's `ready` event on the device, and a build waits for the
// previous build's use of the scratch grid (`tmp_done`) the same way.  (Growing the scratch and
// evicting an entry past GREEN_CACHE_BYTES free device memory with cudaFree, which does
// synchronise the device: a workload of many new shapes pays that per new shape.)
constexpr size_t GREEN_CACHE_BYTES = (size_t)4 << 30;
struct DevCache {
  std::mutex tw_mu, green_mu;
  std::map<std::tuple<int, int>, DevBuf*> tw;                         // (L, device)
  std::map<std::tuple<int, int, int, float, int>, GreenEntry> green;  // (Mx, My, Mz, h, device)
  std::map<int, DevBuf*> green_tmp;                                   // device -> scratch
  std::map<int, cudaEvent_t> tmp_done;                                // device -> last build's end
  size_t green_bytes = 0;
  uint64_t clock = 0;
};
static DevCache& cache() {
  static DevCache c;
  return c;
}

static qmt_status twiddles(int L, const float2** out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(cache().tw_mu);
  DevBuf*& b = cache().tw[std::make_tuple(L, dev)];
  if (!b) {
    std::vector<float2> h(L);
    for (int m = 0; m < L; ++m) {
      const double a = -2.0 * PI * (double)m / (double)L;
      h[m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    b = new DevBuf();
    qmt_status st = b->reserve(L * sizeof(float2));
    if (st) {
      delete b;
      b = nullptr;
      return st;
    }
    // synchronous: the table is shared by every stream (built once per length and device)
    QMT_CUDA(cudaMemcpy(b->ptr, h.data(), L * sizeof(float2), cudaMemcpyHostToDevice));
  }
  *out = b->as<float2>();
  return QMT_OK;
}

template <int MODE>
static qmt_status launch_mode(const PassArgs& a, unsigned blocks, size_t smem, cudaStream_t s) {
  QMT_CUDA(cudaFuncSetAttribute(fft_pass_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fft_pass_kernel<MODE><<<blocks, 256, smem, s>>>(a);
  QMT_CHECK_LAUNCH("fft_pass_kernel");
  return QMT_OK;
}

template <int MODE, int L>
static qmt_status launch_mode_reg(const PassArgs& a, unsigned blocks, size_t smem, cudaStream_t s) {
  QMT_CUDA(cudaFuncSetAttribute(fft_reg_pass_kernel<MODE, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fft_reg_pass_kernel<MODE, L><<<blocks, 256, smem, s>>>(a);
  QMT_CHECK_LAUNCH("fft_reg_pass_kernel");
  return QMT_OK;
}

template <int L>
static qmt_status launch_pass_reg(int mode, PassArgs a, cudaStream_t s) {
  constexpr int LINES = RegFft<L>::LINES;
  a.B = LINES;
  size_t smem = ((size_t)L + (size_t)LINES * RegFft<L>::S_MAX) * sizeof(float2);
  if (mode == PASS_X_RHS) smem += 16 * (size_t)a.mol.natoms;
  const unsigned blocks = (unsigned)((a.nlines + LINES - 1) / LINES);
  if (blocks == 0) return QMT_OK;
  switch (mode) {
    case PASS_PLAIN: return launch_mode_reg<PASS_PLAIN, L>(a, blocks, smem, s);
    case PASS_X_RHS: return launch_mode_reg<PASS_X_RHS, L>(a, blocks, smem, s);
    case PASS_Z_MUL: return launch_mode_reg<PASS_Z_MUL, L>(a, blocks, smem, s);
    default: return launch_mode_reg<PASS_X_OUT, L>(a, blocks, smem, s);
  }
}

static qmt_status launch_pass(int mode, PassArgs a, cudaStream_t s) {
  a.B = std::max(1, std::min(16, 12288 / a.plan.L));
  const float2* tw;
  qmt_status st = twiddles(a.plan.L, &tw);
  if (st) return st;
  a.tw = tw;
  if (a.plan.L == 256) return launch_pass_reg<256>(mode, a, s);   // register kernels
  if (a.plan.L == 128) return launch_pass_reg<128>(mode, a, s);
  size_t smem = ((size_t)a.plan.L * (1 + 2 * a.B)) * sizeof(float2);
  if (mode == PASS_X_RHS) smem += 16 * (size_t)a.mol.natoms;
  const unsigned blocks = (unsigned)((a.nlines + a.B - 1) / a.B);
  if (blocks == 0) return QMT_OK;
  switch (mode) {
    case PASS_PLAIN: return launch_mode<PASS_PLAIN>(a, blocks, smem, s);
    case PASS_X_RHS: return launch_mode<PASS_X_RHS>(a, blocks, smem, s);
    case PASS_Z_MUL: return launch_mode<PASS_Z_MUL>(a, blocks, smem, s);
    default: return launch_mode<PASS_X_OUT>(a, blocks, smem, s);
  }
}

static qmt_status plan_of(int L, Plan1D& p) {
  if (L < 2 || L > FFT_MAXLEN) return fail(QMT_BAD_ARG, "FFT line length out of range");
  if (!factorize(L, p)) return fail(QMT_BAD_ARG, "FFT size has too many factors");
  p.m_len = (unsigned)(((1ull << 32) + (uint64_t)L - 1) / (uint64_t)L);
  int ns = 1;
  for (int i = 0; i < p.nfac; ++i) {
    if (p.fac[i] > 127) return fail(QMT_BAD_ARG, "FFT size has a prime factor above 127");
    const uint64_t nbf = (uint64_t)(L / p.fac[i]);
    p.ns[i] = ns;
    p.m_nbf[i] = nbf > 1 ? (unsigned)(((1ull << 32) + nbf - 1) / nbf) : 0u;
    p.m_ns[i] = ns > 1 ? (unsigned)(((1ull << 32) + (uint64_t)ns - 1) / (uint64_t)ns) : 0u;
    ns *= p.fac[i];
  }
  return QMT_OK;
}

// Hockney G_hat octant for (Mx, My, Mz, h): one unpruned forward 3D transform, cached.
static qmt_status green_hat(int Mx, int My, int Mz, float h_ang, const Plan1D& px, const Plan1D& py,
                            const Plan1D& pz, const float** out, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  auto key = std::make_tuple(Mx, My, Mz, h_ang, dev);
  DevCache& c = cache();
  std::lock_guard<std::mutex> lock(c.green_mu);
  auto it = c.green.find(key);
  if (it != c.green.end()) {
    GreenEntry& e = it->second;
    e.used = ++c.clock;
    if (!e.built) {
      if (cudaEventQuery(e.ready) == cudaSuccess) e.built = true;
      else QMT_CUDA(cudaStreamWaitEvent(s, e.ready, 0));   // still being built on another stream, maybe
    }
    *out = e.buf->as<float>();
    return QMT_OK;
  }
  const int64_t M = (int64_t)Mx * My * Mz;
  DevBuf*& tmp = c.green_tmp[dev];
  if (!tmp) tmp = new DevBuf();
  cudaEvent_t& tmp_done = c.tmp_done[dev];
  if (!tmp_done) QMT_CUDA(cudaEventCreateWithFlags(&tmp_done, cudaEventDisableTiming));
  // growing the scratch frees the old one (cudaFree waits for its users); otherwise the previous
  // build's use of it is ordered before this one on the device
  qmt_status st = tmp->reserve(M * sizeof(float2));   // grows only: no allocation in steady state
  if (st) return st;
  QMT_CUDA(cudaStreamWaitEvent(s, tmp_done, 0));
  float2* g = tmp->as<float2>();
  green_kernel<<<grid_blocks(M), 256, 0, s>>>(g, Mx, My, Mz, h_ang);
  QMT_CHECK_LAUNCH("green_kernel");
  PassArgs a{};
  a.data = g;
  a.scale = 1.f;
  a.inv = 0;
  a.plan = px; a.n1 = My; a.s1 = Mx; a.s2 = (int64_t)Mx * My; a.se = 1; a.nlines = (int64_t)My * Mz;
  a.lload = a.lstore = Mx;
  if ((st = launch_pass(PASS_PLAIN, a, s))) return st;
  a.plan = py; a.n1 = Mx; a.s1 = 1; a.s2 = (int64_t)Mx * My; a.se = Mx; a.nlines = (int64_t)Mx * Mz;
  a.lload = a.lstore = My;
  if ((st = launch_pass(PASS_PLAIN, a, s))) return st;
  a.plan = pz; a.n1 = Mx; a.s1 = 1; a.s2 = Mx; a.se = (int64_t)Mx * My; a.nlines = (int64_t)Mx * My;
  a.lload = a.lstore = Mz;
  if ((st = launch_pass(PASS_PLAIN, a, s))) return st;
  auto* gb = new DevBuf();
  const int64_t no = (int64_t)(Mx / 2 + 1) * (My / 2 + 1) * (Mz / 2 + 1);
  if ((st = gb->reserve(no * sizeof(float)))) {
    delete gb;
    return st;
  }
  green_octant_kernel<<<grid_blocks(no), 256, 0, s>>>(g, Mx, My, Mz, gb->as<float>());
  QMT_CHECK_LAUNCH("green_octant_kernel");
  QMT_CUDA(cudaEventRecord(tmp_done, s));
  cudaEvent_t ready;
  QMT_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  QMT_CUDA(cudaEventRecord(ready, s));
  const size_t nbytes = (size_t)no * sizeof(float);
  while (!c.green.empty() && c.green_bytes + nbytes > GREEN_CACHE_BYTES) {
    auto lru = c.green.begin();
    for (auto e = c.green.begin(); e != c.green.end(); ++e)
      if (e->second.used < lru->second.used) lru = e;
    lru->second.buf->release();   // cudaFree waits for kernels still reading it
    delete lru->second.buf;
    cudaEventDestroy(lru->second.ready);
    c.green_bytes -= lru->second.bytes;
    c.green.erase(lru);
  }
  c.green[key] = GreenEntry{gb, ++c.clock, nbytes, ready, false};
  c.green_bytes += nbytes;
  *out = gb->as<float>();
  return QMT_OK;
}

static qmt_status fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                              float sigma, float cutoff, int padded, int Mx, int My, int Mz, const float* q_dev,
                              float* out_dev, cudaStream_t s);

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                                      float oz, float sigma, float cutoff, int padded, const float* q_dev,
                                      float* out_dev, void* stream) {
  if (nx < 2 || ny < 2 || nz < 2) return fail(QMT_BAD_ARG, "bad FFT Poisson arguments");
  const int Mx = padded ? nice_at_least(2 * nx) : nx;
  const int My = padded ? nice_at_least(2 * ny) : ny;
  const int Mz = padded ? nice_at_least(2 * nz) : nz;
  return fft_poisson(mol, nx, ny, nz, step, ox, oy, oz, sigma, cutoff, padded ? 1 : 0, Mx, My, Mz, q_dev, out_dev,
                     as_stream(stream));
}

extern "C" qmt_status qmt_fft_poisson_padded(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                                             float oz, float sigma, float cutoff, int mx, int my, int mz,
                                             const float* q_dev, float* out_dev, void* stream) {
  if (nx < 2 || ny < 2 || nz < 2 || mx < 2 * nx || my < 2 * ny || mz < 2 * nz)
    return fail(QMT_BAD_ARG, "padded FFT lengths must be at least twice the grid");
  return fft_poisson(mol, nx, ny, nz, step, ox, oy, oz, sigma, cutoff, 1, mx, my, mz, q_dev, out_dev,
                     as_stream(stream));
}

namespace qmt {

static qmt_status fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                              float sigma, float cutoff, int padded, int Mx, int My, int Mz, const float* q_dev,
                              float* out_dev, cudaStream_t s) {
  if (!mol || !q_dev || !out_dev || nx < 2 || ny < 2 || nz < 2 || !(step > 0.f) || !(sigma > 0.f) || cutoff < 0)
    return fail(QMT_BAD_ARG, "bad FFT Poisson arguments");
  if (mol->natoms > 4096) return fail(QMT_BAD_ARG, "too many atoms");
  Plan1D px, py, pz;
  qmt_status st;
  if ((st = plan_of(Mx, px)) || (st = plan_of(My, py)) || (st = plan_of(Mz, pz))) return st;
  const int64_t M = (int64_t)Mx * My * Mz;
  // work grid: x-fastest, only the planes z < nz are ever touched
  if ((st = mol->d_work.reserve((int64_t)Mx * My * nz * sizeof(float2)))) return st;
  float2* c = mol->d_work.as<float2>();
  const float h_ang = (float)(step / ANG2BOR);
  const float* gsym = nullptr;
  if (padded && (st = green_hat(Mx, My, Mz, h_ang, px, py, pz, &gsym, s))) return st;

  PassArgs a{};
  a.data = c;
  a.mol = mol->view();
  a.q = q_dev;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.h_ang = h_ang;
  a.ox = (float)(ox / ANG2BOR);
  a.oy = (float)(oy / ANG2BOR);
  a.oz = (float)(oz / ANG2BOR);
  a.norm = 1.0f / (sigma * sigma * sigma * 2.0f * (float)PI * sqrtf(2.0f * (float)PI));
  a.i2s2 = 1.0f / (2.0f * sigma * sigma);
  a.cut2 = (cutoff * sigma) * (cutoff * sigma);
  a.periodic = padded ? 0 : 1;
  a.gsym = gsym;
  a.Mx = Mx;
  a.My = My;
  a.Mz = Mz;
  a.out = out_dev;
  a.scale = 1.f;
  // 1. x forward with the RHS: lines (y < ny, z < nz), elements x < nx non-zero
  a.plan = px; a.n1 = ny; a.s1 = Mx; a.s2 = (int64_t)Mx * My; a.se = 1; a.nlines = (int64_t)ny * nz;
  a.lload = nx; a.lstore = Mx; a.inv = 0;
  if ((st = launch_pass(PASS_X_RHS, a, s))) return st;
  // 2. y forward on the planes z < nz: lines (x < Mx, z < nz), elements y < ny non-zero
  a.plan = py; a.n1 = Mx; a.s1 = 1; a.s2 = (int64_t)Mx * My; a.se = Mx; a.nlines = (int64_t)Mx * nz;
  a.lload = ny; a.lstore = My;
  if ((st = launch_pass(PASS_PLAIN, a, s))) return st;
  // 3. z forward, kernel multiply, z inverse: lines (x < Mx, y < My), store z < nz
  a.plan = pz; a.n1 = Mx; a.s1 = 1; a.s2 = Mx; a.se = (int64_t)Mx * My; a.nlines = (int64_t)Mx * My;
  a.lload = nz; a.lstore = nz;
  if ((st = launch_pass(PASS_Z_MUL, a, s))) return st;
  // 4. y inverse on the planes z < nz, store y < ny
  a.plan = py; a.n1 = Mx; a.s1 = 1; a.s2 = (int64_t)Mx * My; a.se = Mx; a.nlines = (int64_t)Mx * nz;
  a.lload = My; a.lstore = ny; a.inv = 1;
  if ((st = launch_pass(PASS_PLAIN, a, s))) return st;
  // 5. x inverse, 1/M^3, real part into the C-order output: lines (z < nz, y < ny)
  a.plan = px; a.n1 = nz; a.s1 = (int64_t)Mx * My; a.s2 = Mx; a.se = 1; a.nlines = (int64_t)ny * nz;
  a.lload = Mx; a.lstore = nx; a.inv = 1; a.scale = (float)(1.0 / (double)M);
  return launch_pass(PASS_X_OUT, a, s);
}

}  // namespace qmt

// Analytic electrostatic potential of the GTO density plus the nuclei.
//
// Replaces gpu_hartree_GTO (kernel_hartree.cu:288-869), which loops over DM pairs p >= q and
// then primitive pairs with per-(L,m) closed forms, serialising the block on thread 0.
// Here the density is first written as a sum over merged primitive pairs of Hermite
// Gaussians (McMurchie-Davidson):
//     rho(r) = 2 sum_pq P_pq phi_p phi_q = sum_pairs sum_tuv D_tuv Lambda_tuv(r; p, P)
// with D_tuv already contracted with the density matrix (host, FP64).  The potential at a
// point C is then
//     V(C) = -sum_pairs (2 pi / p) sum_tuv D_tuv R_tuv(p, P - C) + sum_A Z_A / |C - R_A|,
// with R_tuv from Boys functions F_0..F_L (table + Taylor, downward recursion).
//
// Two evaluations.  The default (gto32_pairs_kernel, gto64_pairs_kernel, gto32_atoms_kernel) is
// mixed precision:
//  * pairs of two different atoms are ranked by size (their far-field multipoles); the largest,
//    which together hold 95% of the total (a few percent of the pairs), are evaluated in FP64
//    throughout from FP64 coefficients and centres (gto64_pairs_kernel): an FP32 term's error
//    (rounded coefficients and arithmetic) is proportional to its size, and the potential at a
//    grid boundary is the small difference of large electronic and nuclear parts;
//  * the rest (gto32_pairs_kernel), less those below 1e-11 of the total size (kFp32Screen): where
//    T = p |P - C|^2 >= 30 (99.5% of the point-pair terms on the boundary of the medium
//    molecule's grid) the Boys functions take their asymptotic form
//        (-2p)^n F_n(T) = sqrt(pi) / (2 sqrt(p)) * (-1)^n (2n-1)!! / r^(2n+1)
//    (relative error below e^-T T^(L-1/2) < 2e-9 for L <= 4): one reciprocal square root and the
//    Hermite recursion in FP32, summed in FP32 in groups of four and the groups in FP64; nearer
//    terms in FP64 (a function kept out of line, so the FP32 loop keeps its register count);
//  * both pair lists are cut into slices over several CTAs whose FP64 partial sums are added in
//    order (deterministic);
//  * pairs centred on one atom: kept per atom in descending exponent order with cumulative FP64
//    moments, so that the far-field ones at a point are one FP64 multipole evaluation about the
//    nucleus (an FP32 1/r common to an atom's electrons and missing from its nucleus would leave
//    Z_A * 1e-7 / r of error), the near-field ones in FP64 from FP64 coefficients;
//  * point and pair centres relative to the molecule's centroid (FP32 for the FP32 terms, FP64
//    for the others), the density matrix and prefactor folded into the Hermite coefficients; the
//    nuclear term in FP64.
// gto_kernel keeps every operation in FP64 (qmt_set_gto_precision selects it; the checker).
#include <algorithm>
#include <cstdio>
#include <string>
#include <unordered_map>

#include "mol.cuh"

namespace qmt {

__host__ __device__ constexpr int ncoef(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
constexpr int BOYS_NT = 401;     // T = 0, 0.1, ..., 40
constexpr int BOYS_NM = 11;      // m = 0..10
constexpr double BOYS_DT = 0.1;

struct GPair {
  double px, py, pz, p;
  double pref;   // -(2 pi / p) * spin/triangle factors * K * ca * cb (D carries P)
  int L;
  int doff;      // offset of the D coefficients
};

// (t,u,v) triples ordered by t+u+v; recursion parents for R^{(j)}_{tuv} from R^{(j+1)}.
struct HermIdx {
  int t, u, v, dir, p1, p2, mult;
};

__host__ __device__ constexpr int herm_index(int t, int u, int v) {
  // position in the list ordered by total order, then t descending, then u descending
  int s = t + u + v, base = 0;
  for (int k = 0; k < s; ++k) base += (k + 1) * (k + 2) / 2;
  int pos = 0;
  for (int tt = s; tt > t; --tt) pos += s - tt + 1;
  pos += (s - t) - u;
  return base + pos;
}

struct HermTable {
  HermIdx e[35];
};

__host__ __device__ constexpr HermTable make_herm_table() {
  HermTable h{};
  int k = 0;
  for (int s = 0; s <= 4; ++s)
    for (int t = s; t >= 0; --t)
      for (int u = s - t; u >= 0; --u) {
        const int v = s - t - u;
        HermIdx x{t, u, v, -1, -1, -1, 0};
        if (t > 0) {
          x.dir = 0;
          x.p1 = herm_index(t - 1, u, v);
          x.mult = t - 1;
          x.p2 = t > 1 ? herm_index(t - 2, u, v) : 0;
        } else if (u > 0) {
          x.dir = 1;
          x.p1 = herm_index(t, u - 1, v);
          x.mult = u - 1;
          x.p2 = u > 1 ? herm_index(t, u - 2, v) : 0;
        } else if (v > 0) {
          x.dir = 2;
          x.p1 = herm_index(t, u, v - 1);
          x.mult = v - 1;
          x.p2 = v > 1 ? herm_index(t, u, v - 2) : 0;
        }
        h.e[k++] = x;
      }
  return h;
}

// F_m(T) for m = 0..L into F[], FP64.
template <int L>
__device__ __forceinline__ void boys_fn(double T, const double* __restrict__ tab, double* F) {
  if (T < 40.0) {
    const int i = (int)(T * (1.0 / BOYS_DT) + 0.5);
    const double d = T - i * BOYS_DT;
    const double* row = tab + (size_t)i * BOYS_NM;
    // Taylor: F_L(T) = sum_k F_{L+k}(T_i) (-d)^k / k!
    double f = 0.0, c = 1.0;
#pragma unroll
    for (int k = 0; k <= 6; ++k) {
      f += row[L + k] * c;
      c *= -d / (k + 1);
    }
    F[L] = f;
    const double et = exp(-T);
#pragma unroll
    for (int m = L - 1; m >= 0; --m) F[m] = (2.0 * T * F[m + 1] + et) / (2 * m + 1);
  } else {
    const double it = 1.0 / T;
    F[0] = 0.88622692545275801365 * sqrt(it);  // sqrt(pi)/2 / sqrt(T)
#pragma unroll
    for (int m = 0; m < L; ++m) F[m + 1] = F[m] * (2 * m + 1) * 0.5 * it;
  }
}

template <int L>
__device__ __forceinline__ double pair_potential(const GPair& g, const double* __restrict__ D, double cx, double cy,
                                                 double cz, const double* __restrict__ tab) {
  const double X = g.px - cx, Y = g.py - cy, Z = g.pz - cz;
  const double T = g.p * (X * X + Y * Y + Z * Z);
  double F[L + 1];
  boys_fn<L>(T, tab, F);
  constexpr int NC = ncoef(L);
  constexpr HermTable H = make_herm_table();
  double cur[NC], nxt[NC];
  const double m2p = -2.0 * g.p;
  double pw = 1.0;
#pragma unroll
  for (int j = 0; j < L; ++j) pw *= m2p;
  cur[0] = pw * F[L];
#pragma unroll
  for (int j = L - 1; j >= 0; --j) {
    pw = 1.0;
#pragma unroll
    for (int q = 0; q < j; ++q) pw *= m2p;
    nxt[0] = pw * F[j];
    const int n = ncoef(L - j);
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      if (k < n) {
        const HermIdx h = H.e[k];
        const double c = h.dir == 0 ? X : (h.dir == 1 ? Y : Z);
        double r = c * cur[h.p1];
        if (h.mult > 0) r += h.mult * cur[h.p2];
        nxt[k] = r;
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) cur[k] = nxt[k];
  }
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < NC; ++k) acc += D[k] * cur[k];
  return g.pref * acc;
}

constexpr int GTO_THREADS = 128;
constexpr int GTO_CHUNK = 64;

// mode 0: grid corners origin + i h (x-fastest);  mode 1: grid centres;  mode 2: point list;
// mode 3: outer shell of the grid at centres (boundary), written into the full grid.
struct GtoPoints {
  int mode;
  int nx, ny, nz;
  double h, ox, oy, oz;
  const float* pts;
  int64_t npts;
};

__device__ __forceinline__ bool gto_point(const GtoPoints& gp, int64_t i, double& x, double& y, double& z,
                                          int64_t& out) {
  if (gp.mode == 2) {
    x = gp.pts[3 * i];
    y = gp.pts[3 * i + 1];
    z = gp.pts[3 * i + 2];
    out = i;
    return true;
  }
  int64_t ix, iy, iz;
  if (gp.mode == 3) {
    // enumerate the outer shell: z = 0 and z = nz-1 planes, then the y faces, then x faces
    const int64_t nx = gp.nx, ny = gp.ny, nz = gp.nz;
    const int64_t pl = nx * ny;
    if (i < 2 * pl) {
      iz = i < pl ? 0 : nz - 1;
      const int64_t r = i % pl;
      ix = r % nx;
      iy = r / nx;
    } else {
      int64_t r = i - 2 * pl;
      const int64_t inner = nz - 2;
      const int64_t yf = nx * inner;
      if (r < 2 * yf) {
        iy = r < yf ? 0 : ny - 1;
        r %= yf;
        ix = r % nx;
        iz = 1 + r / nx;
      } else {
        r -= 2 * yf;
        const int64_t xf = (ny - 2) * inner;
        ix = r < xf ? 0 : nx - 1;
        r %= xf;
        iy = 1 + r % (ny - 2);
        iz = 1 + r / (ny - 2);
      }
    }
  } else {
    ix = i % gp.nx;
    iy = (i / gp.nx) % gp.ny;
    iz = i / ((int64_t)gp.nx * gp.ny);
  }
  const double off = gp.mode == 0 ? 0.0 : 0.5;
  x = gp.ox + (ix + off) * gp.h;
  y = gp.oy + (iy + off) * gp.h;
  z = gp.oz + (iz + off) * gp.h;
  out = ix + iy * (int64_t)gp.nx + iz * (int64_t)gp.nx * gp.ny;
  return true;
}

__global__ void __launch_bounds__(GTO_THREADS) gto_kernel(const GPair* __restrict__ pairs, int npairs,
                                                          const double* __restrict__ dco,
                                                          const double* __restrict__ tab, MolView mol,
                                                          GtoPoints gp, float* __restrict__ out) {
  __shared__ GPair sp[GTO_CHUNK];
  __shared__ double sd[GTO_CHUNK * 35];
  __shared__ int soff[GTO_CHUNK];
  const int64_t i = blockIdx.x * (int64_t)GTO_THREADS + threadIdx.x;
  double cx = 0, cy = 0, cz = 0;
  int64_t o = -1;
  const bool valid = i < gp.npts && gto_point(gp, i, cx, cy, cz, o);
  double V = 0.0;
  for (int c0 = 0; c0 < npairs; c0 += GTO_CHUNK) {
    const int nc = min(GTO_CHUNK, npairs - c0);
    __syncthreads();
    if (threadIdx.x < nc) sp[threadIdx.x] = pairs[c0 + threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int k = 0; k < nc; ++k) {
        soff[k] = acc;
        acc += ncoef(sp[k].L);
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nc * 35; k += GTO_THREADS) {
      const int pk = k / 35, j = k % 35;
      if (j < ncoef(sp[pk].L)) sd[soff[pk] + j] = dco[sp[pk].doff + j];
    }
    __syncthreads();
    if (valid) {
      for (int k = 0; k < nc; ++k) {
        const GPair g = sp[k];
        const double* D = sd + soff[k];
        switch (g.L) {
          case 0: V += pair_potential<0>(g, D, cx, cy, cz, tab); break;
          case 1: V += pair_potential<1>(g, D, cx, cy, cz, tab); break;
          case 2: V += pair_potential<2>(g, D, cx, cy, cz, tab); break;
          case 3: V += pair_potential<3>(g, D, cx, cy, cz, tab); break;
          default: V += pair_potential<4>(g, D, cx, cy, cz, tab); break;
        }
      }
    }
  }
  if (!valid) return;
  for (int a = 0; a < mol.natoms; ++a) {
    const double dx = cx - mol.coords[3 * a], dy = cy - mol.coords[3 * a + 1], dz = cz - mol.coords[3 * a + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r > 1e-8) V += mol.types[a] / r;
  }
  out[o] = (float)V;
}

// ---- FP32 kernel with FP64 accumulation -----------------------------------------------------
constexpr float T_FAR = 30.0f;

// R_tuv (t+u+v <= L) from h_j = (-2p)^j F_j, j = 0..L, dotted with D.
template <int L>
__device__ __forceinline__ float hermite_dot32(const float (&D)[ncoef(L)], float X, float Y, float Z,
                                               const float (&h)[L + 1]) {
  constexpr int NC = ncoef(L);
  constexpr HermTable H = make_herm_table();
  float cur[NC], nxt[NC];
  cur[0] = h[L];
#pragma unroll
  for (int j = L - 1; j >= 0; --j) {
    nxt[0] = h[j];
    const int n = ncoef(L - j);
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      if (k < n) {
        const HermIdx e = H.e[k];
        const float c = e.dir == 0 ? X : (e.dir == 1 ? Y : Z);
        float r = c * cur[e.p1];
        if (e.mult > 0) r = fmaf((float)e.mult, cur[e.p2], r);
        nxt[k] = r;
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) cur[k] = nxt[k];
  }
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < NC; ++k) acc = fmaf(D[k], cur[k], acc);
  return acc;
}

// FP64 R_tuv (t+u+v <= L) from h_j, dotted with the coefficients D (float or double).
template <int L, typename DT>
__device__ __forceinline__ double hermite_dot64(const DT (&D)[ncoef(L)], double X, double Y, double Z,
                                                const double (&h)[L + 1]) {
  constexpr int NC = ncoef(L);
  constexpr HermTable H = make_herm_table();
  double cur[NC], nxt[NC];
  cur[0] = h[L];
#pragma unroll
  for (int j = L - 1; j >= 0; --j) {
    nxt[0] = h[j];
    const int n = ncoef(L - j);
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      if (k < n) {
        const HermIdx e = H.e[k];
        const double c = e.dir == 0 ? X : (e.dir == 1 ? Y : Z);
        double r = c * cur[e.p1];
        if (e.mult > 0) r = fma((double)e.mult, cur[e.p2], r);
        nxt[k] = r;
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) cur[k] = nxt[k];
  }
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < NC; ++k) acc = fma((double)D[k], cur[k], acc);
  return acc;
}

// F_m(T), m = 0..L <= 4, T < 40: each from its own Taylor step about the nearest table point,
// F_m(T) = sum_k F_{m+k}(T_i) (-d)^k / k!, |d| <= 0.05, k <= 6 (truncation ~1e-13 relative):
// no exponential and no division, unlike the downward recursion of boys_fn.
template <int L>
__device__ __forceinline__ void boys_taylor(double T, const double* __restrict__ tab, double* F) {
  const int i = (int)(T * (1.0 / BOYS_DT) + 0.5);
  const double d = T - i * BOYS_DT;
  const double* row = tab + (size_t)i * BOYS_NM;
  double c[7];
  c[0] = 1.0;
#pragma unroll
  for (int k = 1; k < 7; ++k) c[k] = c[k - 1] * (-d * (1.0 / k));
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    double f = 0.0;
#pragma unroll
    for (int k = 6; k >= 0; --k) f = fma(row[m + k], c[k], f);
    F[m] = f;
  }
}

// The near-field term of an FP32 pair (T < 30) in FP64: Boys functions from the FP64 table
// (boys_taylor), FP64 recursion, the FP32 coefficients read from `d`.  Not inlined, so the few
// near terms do not raise the register count of the FP32 loop around them.
template <int L>
__device__ __noinline__ double near_term(float px, float py, float pz, float p, const float* __restrict__ d, float cx,
                                         float cy, float cz, const double* __restrict__ tab64) {
  const double Xd = (double)(px - cx), Yd = (double)(py - cy), Zd = (double)(pz - cz);
  const double pd = p;
  const double Td = pd * (Xd * Xd + Yd * Yd + Zd * Zd);   // < 30.001: inside the FP64 table
  double F[L + 1], h[L + 1];
  boys_taylor<L>(Td, tab64, F);
  double pw = 1.0;
#pragma unroll
  for (int j = 0; j <= L; ++j) {
    h[j] = pw * F[j];
    pw *= -2.0 * pd;
  }
  float D[ncoef(L)];
#pragma unroll
  for (int c = 0; c < ncoef(L); ++c) D[c] = d[c];
  return hermite_dot64<L>(D, Xd, Yd, Zd, h);
}

// One FP32 pair's term at a point.  Far field (T = p r^2 >= 30): FP32, returned (the caller sums
// these in FP32 groups).  Near field: the diffuse pairs at short range in FP64 (near_term), added to
// `vnear`; 0 is returned.  The near / far test is the FP32 one, the same everywhere.
template <int L>
__device__ __forceinline__ float pair_term32(const GPair32& g, const float (&D)[ncoef(L)], const float* d, float cx,
                                             float cy, float cz, const double* __restrict__ tab64, double& vnear) {
  const float X = g.px - cx, Y = g.py - cy, Z = g.pz - cz;
  const float r2 = fmaf(X, X, fmaf(Y, Y, Z * Z));
  const float T = g.p * r2;
  if (!(T < T_FAR)) {   // (a non-finite T takes this branch too: the table is never indexed by it)
    // asymptotic Boys functions: h_j = (-1)^j (2j-1)!! r^-(2j+1), the factor sqrt(pi)/(2 sqrt p)
    // applied to the sum; one Newton step makes the reciprocal square root correctly rounded
    float h[L + 1];
    float ri = rsqrtf(r2);
    ri = ri * fmaf(-0.5f * r2 * ri, ri, 1.5f);
    const float ri2 = ri * ri;
    h[0] = ri;
#pragma unroll
    for (int j = 0; j < L; ++j) h[j + 1] = -(float)(2 * j + 1) * h[j] * ri2;
    return g.fscale * hermite_dot32<L>(D, X, Y, Z, h);
  }
  vnear += near_term<L>(g.px, g.py, g.pz, g.p, d, cx, cy, cz, tab64);
  return 0.f;
}

// One pair's term at a point in FP64 throughout (FP64 coefficients): the far field from the
// asymptotic Boys functions, the near field from the FP64 table (boys_taylor).
template <int L>
__device__ __forceinline__ double pair_term64(double px, double py, double pz, double p, double fscale,
                                              const double (&D)[ncoef(L)], double cx, double cy, double cz,
                                              const double* __restrict__ tab64) {
  const double X = px - cx, Y = py - cy, Z = pz - cz;
  const double r2 = X * X + Y * Y + Z * Z;
  const double T = p * r2;
  double h[L + 1];
  if (!(T < 30.0)) {
    const double ri = rsqrt(r2), ri2 = ri * ri;
    h[0] = fscale * ri;
#pragma unroll
    for (int j = 0; j < L; ++j) h[j + 1] = -(double)(2 * j + 1) * h[j] * ri2;
  } else {
    double F[L + 1];
    boys_taylor<L>(T, tab64, F);
    double pw = 1.0;
#pragma unroll
    for (int j = 0; j <= L; ++j) {
      h[j] = pw * F[j];
      pw *= -2.0 * p;
    }
  }
  return hermite_dot64<L>(D, X, Y, Z, h);
}

constexpr int GTO32_THREADS = 128;
constexpr int GTO32_PPT = 2;                          // points per thread
constexpr int GTO32_POINTS = GTO32_THREADS * GTO32_PPT;
constexpr int GTO32_CHUNK = 128;
constexpr int GTO64_CHUNK = 64;

// The terms of `nc` pairs of one angular momentum L (all in shared memory) at the thread's two
// points, summed in FP32 in groups of four, the groups in FP64.  One L per loop (no dispatch per
// pair); a pair's header and coefficients are read once into registers for both points, whose
// independent dependency chains overlap.
template <int L>
__device__ __forceinline__ void chunk_terms(const GPair32* sp, const float* sd, const int* soff, int nc,
                                            const float (&x)[GTO32_PPT], const float (&y)[GTO32_PPT],
                                            const float (&z)[GTO32_PPT], const double* __restrict__ tab64,
                                            double (&V)[GTO32_PPT]) {
  constexpr int NC = ncoef(L);
  float acc[GTO32_PPT];
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q) acc[q] = 0.f;
#pragma unroll 2
  for (int k = 0; k < nc; ++k) {
    const GPair32 g = sp[k];
    float D[NC];
    const float* d = sd + soff[k];
#pragma unroll
    for (int c = 0; c < NC; ++c) D[c] = d[c];
#pragma unroll
    for (int q = 0; q < GTO32_PPT; ++q) acc[q] += pair_term32<L>(g, D, d, x[q], y[q], z[q], tab64, V[q]);
    if ((k & 3) == 3) {
#pragma unroll
      for (int q = 0; q < GTO32_PPT; ++q) {
        V[q] += (double)acc[q];
        acc[q] = 0.f;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q) V[q] += (double)acc[q];
}

// The terms of `nc` FP64 pairs of one angular momentum L (in shared memory) at the thread's points.
template <int L>
__device__ __forceinline__ void chunk_terms64(const GPair64* sp, const double* sd, const int* soff, int nc,
                                              const double (&x)[GTO32_PPT], const double (&y)[GTO32_PPT],
                                              const double (&z)[GTO32_PPT], const double* __restrict__ tab64,
                                              double (&V)[GTO32_PPT]) {
  constexpr int NC = ncoef(L);
#pragma unroll 1
  for (int k = 0; k < nc; ++k) {
    const GPair64 g = sp[k];
    double D[NC];
    const double* d = sd + soff[k];
#pragma unroll
    for (int c = 0; c < NC; ++c) D[c] = d[c];
#pragma unroll
    for (int q = 0; q < GTO32_PPT; ++q) V[q] += pair_term64<L>(g.px, g.py, g.pz, g.p, g.fscale, D, x[q], y[q], z[q], tab64);
  }
}

// The point relative to the centroid in FP64 (the FP64 terms and the nuclei) and rounded once to
// FP32 (the FP32 terms).
__device__ __forceinline__ void point32(const GtoPoints& gp, const Gto32Tables& t, int64_t i, double& xd,
                                        double& yd, double& zd, float& x, float& y, float& z, int64_t& o,
                                        bool& valid) {
  double cx = 0, cy = 0, cz = 0;
  o = -1;
  valid = i < gp.npts && gto_point(gp, i, cx, cy, cz, o);
  xd = cx - t.rx;
  yd = cy - t.ry;
  zd = cz - t.rz;
  x = (float)xd;
  y = (float)yd;
  z = (float)zd;
}

// The block's points: FP64 and FP32 coordinates relative to the centroid; invalid stand-ins copy
// the first point (finite arithmetic, nothing written).
__device__ __forceinline__ void block_points(const GtoPoints& gp, const Gto32Tables& t, double (&xd)[GTO32_PPT],
                                             double (&yd)[GTO32_PPT], double (&zd)[GTO32_PPT],
                                             float (&x)[GTO32_PPT], float (&y)[GTO32_PPT], float (&z)[GTO32_PPT],
                                             int64_t (&idx)[GTO32_PPT], bool (&valid)[GTO32_PPT]) {
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q) {
    int64_t o;
    idx[q] = blockIdx.x * (int64_t)GTO32_POINTS + q * GTO32_THREADS + threadIdx.x;
    point32(gp, t, idx[q], xd[q], yd[q], zd[q], x[q], y[q], z[q], o, valid[q]);
    if (!valid[q] && q > 0) {
      x[q] = x[0];
      y[q] = y[0];
      z[q] = z[0];
      xd[q] = xd[0];
      yd[q] = yd[0];
      zd[q] = zd[0];
    }
  }
}

// FP32 off-site pairs of slice blockIdx.y at the block's points; FP64 partial sums into
// part[blockIdx.y * npts + i].
__global__ void __launch_bounds__(GTO32_THREADS, 8) gto32_pairs_kernel(Gto32Tables t, const double* __restrict__ tab64,
                                                                    GtoPoints gp, double* __restrict__ part) {
  __shared__ GPair32 sp[GTO32_CHUNK];
  __shared__ float sd[GTO32_CHUNK * 35];
  __shared__ int soff[GTO32_CHUNK];
  float x[GTO32_PPT], y[GTO32_PPT], z[GTO32_PPT];
  double xd[GTO32_PPT], yd[GTO32_PPT], zd[GTO32_PPT];
  int64_t idx[GTO32_PPT];
  bool valid[GTO32_PPT];
  block_points(gp, t, xd, yd, zd, x, y, z, idx, valid);
  double V[GTO32_PPT];
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q) V[q] = 0.0;
  const int s0 = t.slice[blockIdx.y], s1 = t.slice[blockIdx.y + 1];
#pragma unroll 1
  for (int L = 0; L <= 4; ++L) {
    const int p0 = max(s0, t.lstart[L]), p1 = min(s1, t.lstart[L + 1]);
    for (int c0 = p0; c0 < p1; c0 += GTO32_CHUNK) {
      const int nc = min(GTO32_CHUNK, p1 - c0);
      __syncthreads();   // the previous chunk's readers are done
      const int dbase = t.pairs[c0].doff;
      if (threadIdx.x < nc) {
        const GPair32 g = t.pairs[c0 + threadIdx.x];
        sp[threadIdx.x] = g;
        soff[threadIdx.x] = g.doff - dbase;   // coefficients of a chunk are contiguous
      }
      const int dn = nc * ncoef(L);
      for (int k = threadIdx.x; k < dn; k += GTO32_THREADS) sd[k] = t.dco[dbase + k];
      __syncthreads();
      if (valid[0]) {
        switch (L) {
          case 0: chunk_terms<0>(sp, sd, soff, nc, x, y, z, tab64, V); break;
          case 1: chunk_terms<1>(sp, sd, soff, nc, x, y, z, tab64, V); break;
          case 2: chunk_terms<2>(sp, sd, soff, nc, x, y, z, tab64, V); break;
          case 3: chunk_terms<3>(sp, sd, soff, nc, x, y, z, tab64, V); break;
          default: chunk_terms<4>(sp, sd, soff, nc, x, y, z, tab64, V); break;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q)
    if (valid[q]) part[blockIdx.y * gp.npts + idx[q]] = V[q];
}

// FP64 off-site pairs of slice blockIdx.y at the block's points; FP64 partial sums into
// part[(nslice + blockIdx.y) * npts + i].
__global__ void __launch_bounds__(GTO32_THREADS) gto64_pairs_kernel(Gto32Tables t, const double* __restrict__ tab64,
                                                                    GtoPoints gp, double* __restrict__ part) {
  __shared__ GPair64 sp[GTO64_CHUNK];
  __shared__ double sd[GTO64_CHUNK * 35];
  __shared__ int soff[GTO64_CHUNK];
  float x[GTO32_PPT], y[GTO32_PPT], z[GTO32_PPT];
  double xd[GTO32_PPT], yd[GTO32_PPT], zd[GTO32_PPT];
  int64_t idx[GTO32_PPT];
  bool valid[GTO32_PPT];
  block_points(gp, t, xd, yd, zd, x, y, z, idx, valid);
  double V[GTO32_PPT];
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q) V[q] = 0.0;
  const int s0 = t.slice64[blockIdx.y], s1 = t.slice64[blockIdx.y + 1];
#pragma unroll 1
  for (int L = 0; L <= 4; ++L) {
    const int p0 = max(s0, t.lstart64[L]), p1 = min(s1, t.lstart64[L + 1]);
    for (int c0 = p0; c0 < p1; c0 += GTO64_CHUNK) {
      const int nc = min(GTO64_CHUNK, p1 - c0);
      __syncthreads();
      const int dbase = t.pairs64[c0].doff;
      if (threadIdx.x < nc) {
        const GPair64 g = t.pairs64[c0 + threadIdx.x];
        sp[threadIdx.x] = g;
        soff[threadIdx.x] = g.doff - dbase;
      }
      const int dn = nc * ncoef(L);
      for (int k = threadIdx.x; k < dn; k += GTO32_THREADS) sd[k] = t.dco64[dbase + k];
      __syncthreads();
      if (valid[0]) {
        switch (L) {
          case 0: chunk_terms64<0>(sp, sd, soff, nc, xd, yd, zd, tab64, V); break;
          case 1: chunk_terms64<1>(sp, sd, soff, nc, xd, yd, zd, tab64, V); break;
          case 2: chunk_terms64<2>(sp, sd, soff, nc, xd, yd, zd, tab64, V); break;
          case 3: chunk_terms64<3>(sp, sd, soff, nc, xd, yd, zd, tab64, V); break;
          default: chunk_terms64<4>(sp, sd, soff, nc, xd, yd, zd, tab64, V); break;
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < GTO32_PPT; ++q)
    if (valid[q]) part[(t.nslice + blockIdx.y) * gp.npts + idx[q]] = V[q];
}

// FP64 R_tuv (t+u+v <= 4) from h_j, dotted with the 35 moments M.
__device__ __forceinline__ double moments_dot64(const double* __restrict__ M, double X, double Y, double Z,
                                                const double (&h)[5]) {
  constexpr int NC = ncoef(4);
  constexpr HermTable H = make_herm_table();
  double cur[NC], nxt[NC];
  cur[0] = h[4];
#pragma unroll
  for (int j = 3; j >= 0; --j) {
    nxt[0] = h[j];
    const int n = ncoef(4 - j);
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      if (k < n) {
        const HermIdx e = H.e[k];
        const double c = e.dir == 0 ? X : (e.dir == 1 ? Y : Z);
        double r = c * cur[e.p1];
        if (e.mult > 0) r = fma((double)e.mult, cur[e.p2], r);
        nxt[k] = r;
      }
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) cur[k] = nxt[k];
  }
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < NC; ++k) acc = fma(__ldg(M + k), cur[k], acc);
  return acc;
}

// Per point: the slices' partial sums in order, then atom by atom the far-field on-site pairs as
// one FP64 multipole, the near-field on-site pairs and the nucleus, all in FP64 about the FP64
// nucleus.
__global__ void __launch_bounds__(GTO32_THREADS) gto32_atoms_kernel(Gto32Tables t, const double* __restrict__ tab64,
                                                                    MolView mol, GtoPoints gp,
                                                                    const double* __restrict__ part,
                                                                    float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)GTO32_THREADS + threadIdx.x;
  float x, y, z;
  double xd, yd, zd;
  int64_t o;
  bool valid;
  point32(gp, t, i, xd, yd, zd, x, y, z, o, valid);
  if (!valid) return;
  double V = 0.0;
  for (int sl = 0; sl < t.nslice + t.nslice64; ++sl) V += part[sl * gp.npts + i];
  for (int a = 0; a < mol.natoms; ++a) {
    // far / near split of the atom's pairs by the FP32 test p r^2 >= 30 (any consistent split is
    // exact up to the asymptotic form's error)
    const float X = t.nuc[3 * a] - x, Y = t.nuc[3 * a + 1] - y, Z = t.nuc[3 * a + 2] - z;
    const float r2 = fmaf(X, X, fmaf(Y, Y, Z * Z));
    const int b0 = t.onsite_off[a], b1 = t.onsite_off[a + 1];
    int lo = b0, hi = b1;   // first pair that is not far (exponents descend, so far ones lead)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (!(__ldg(t.onsite_p + mid) * r2 < T_FAR)) lo = mid + 1;
      else hi = mid;
    }
    const double ax = t.nuc64[3 * a], ay = t.nuc64[3 * a + 1], az = t.nuc64[3 * a + 2];
    const double Xd = ax - xd, Yd = ay - yd, Zd = az - zd;
    const double r2d = Xd * Xd + Yd * Yd + Zd * Zd;
    if (lo > b0) {
      const double ri = rsqrt(r2d), ri2 = ri * ri;
      double h[5];
      h[0] = ri;
#pragma unroll
      for (int j = 0; j < 4; ++j) h[j + 1] = -(double)(2 * j + 1) * h[j] * ri2;
      V += moments_dot64(t.cum + (size_t)(t.cum_off[a] + (lo - b0)) * 35, Xd, Yd, Zd, h);
    }
    for (int k = lo; k < b1; ++k) {
      const GPair32 g = t.onsite[k];
      const double* d = t.dco_on + g.pad;   // p, sqrt(pi) / (2 sqrt(p)), pref * D_tuv
      const double pk = d[0], fs = d[1];
      d += 2;
      switch (g.L) {
        case 0: { double D[1]; D[0] = d[0]; V += pair_term64<0>(ax, ay, az, pk, fs, D, xd, yd, zd, tab64); break; }
        case 1: { double D[4]; for (int c = 0; c < 4; ++c) D[c] = d[c]; V += pair_term64<1>(ax, ay, az, pk, fs, D, xd, yd, zd, tab64); break; }
        case 2: { double D[10]; for (int c = 0; c < 10; ++c) D[c] = d[c]; V += pair_term64<2>(ax, ay, az, pk, fs, D, xd, yd, zd, tab64); break; }
        case 3: { double D[20]; for (int c = 0; c < 20; ++c) D[c] = d[c]; V += pair_term64<3>(ax, ay, az, pk, fs, D, xd, yd, zd, tab64); break; }
        default: { double D[35]; for (int c = 0; c < 35; ++c) D[c] = d[c]; V += pair_term64<4>(ax, ay, az, pk, fs, D, xd, yd, zd, tab64); break; }
      }
    }
    const double r = sqrt(r2d);
    if (r > 1e-8) V += mol.types[a] / r;
  }
  out[o] = (float)V;
}

// ---- host: Boys table ------------------------------------------------------------------------
static qmt_status boys_table(const double** out) {
  static thread_local DevBuf tab;  // one copy per host thread (per device in practice)
  static thread_local bool ready = false;
  if (!ready) {
    std::vector<double> h((size_t)BOYS_NT * BOYS_NM);
    for (int i = 0; i < BOYS_NT; ++i) {
      const double T = i * BOYS_DT;
      for (int m = 0; m < BOYS_NM; ++m) {
        double term = 1.0 / (2 * m + 1), acc = term;
        for (int k = 1; k < 400; ++k) {
          term *= 2 * T / (2 * m + 2 * k + 1);
          acc += term;
          if (term < 1e-18 * acc) break;
        }
        h[(size_t)i * BOYS_NM + m] = std::exp(-T) * acc;
      }
    }
    qmt_status st = tab.reserve(h.size() * sizeof(double));
    if (st) return st;
    QMT_CUDA(cudaMemcpy(tab.ptr, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    ready = true;
  }
  *out = tab.as<double>();
  return QMT_OK;
}

static int g_gto_prec = QMT_PREC_FP32;   // FP32 with FP64 accumulation, or FP64 throughout
// Share of the off-site pairs' total size (far-field multipoles) left to FP32 terms; the largest
// pairs, holding the rest, take FP64 terms.
constexpr double kFp32Share = 0.05;
// Off-site pairs whose size is below this fraction of the total are left out of the FP32 terms.
// On the medium molecule (30 atoms, cc-pVDZ) the FP32 pairs' sizes spread evenly over the decades
// from 1e-4 to 1e-20 of the total; the half below 1e-11 (together 7e-8 of the total) moves the
// potential on its grid boundary by 1e-7 of its norm against the FP64 kernel (6e-8 with every
// pair; 1e-6 with the cut at 1e-10) and took a third of the FP32 kernel's time.  The FP64 kernel
// keeps every pair.
constexpr double kFp32Screen = 1e-11;

// ---- host: pair table --------------------------------------------------------------------------
static void hermite_e_host(int la, int lb, double a, double b, double xa, double xb, double E[3][3][5]) {
  const double p = a + b, xp = (a * xa + b * xb) / p, pa = xp - xa, pb = xp - xb, i2p = 0.5 / p;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int t = 0; t < 5; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = 1.0;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
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
}

static int cart_host(int L, int k, double* c, int (*e)[3]) {
  for (int q = 0; q < 3; ++q) e[q][0] = e[q][1] = e[q][2] = 0;
  if (L == 0) { c[0] = YS; return 1; }
  if (L == 1) { c[0] = YP; e[0][k == 0 ? 2 : (k == 1 ? 0 : 1)] = 1; return 1; }
  switch (k) {
    case 0: c[0] = 2 * YD0; e[0][2] = 2; c[1] = -YD0; e[1][0] = 2; c[2] = -YD0; e[2][1] = 2; return 3;
    case 1: c[0] = YD1; e[0][0] = 1; e[0][2] = 1; return 1;
    case 2: c[0] = YD1; e[0][1] = 1; e[0][2] = 1; return 1;
    case 3: c[0] = YD2; e[0][0] = 2; c[1] = -YD2; e[1][1] = 2; return 2;
    default: c[0] = YD1; e[0][0] = 1; e[0][1] = 1; return 1;
  }
}

static qmt_status build_pairs(qmt_mol* m, cudaStream_t s) {
  if (m->gto_ready) return QMT_OK;
  struct Acc {
    double px, py, pz, p, pref;
    int L;
    int atom_a, atom_b;
    double D[35];
  };
  std::vector<Acc> acc;
  std::unordered_map<std::string, int> index;
  const int ns = m->nshells, np = m->npad;
  const std::vector<double>& P64 = m->host_P64();
  for (int iA = 0; iA < ns; ++iA) {
    const Shell& A = m->shells[iA];
    const double Ax = m->coords[3 * A.atom], Ay = m->coords[3 * A.atom + 1], Az = m->coords[3 * A.atom + 2];
    for (int iB = iA; iB < ns; ++iB) {
      const Shell& B = m->shells[iB];
      const double Bx = m->coords[3 * B.atom], By = m->coords[3 * B.atom + 1], Bz = m->coords[3 * B.atom + 2];
      const double AB2 = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
      const double fac = iA == iB ? 1.0 : 2.0;
      double pmax = 0;
      for (int k1 = 0; k1 < 2 * A.L + 1; ++k1)
        for (int k2 = 0; k2 < 2 * B.L + 1; ++k2)
          pmax = std::max(pmax, std::fabs(P64[(size_t)(A.func + k1) * np + B.func + k2]));
      if (pmax == 0) continue;
      for (int ia = 0; ia < A.nprim; ++ia)
        for (int ib = 0; ib < B.nprim; ++ib) {
          const double a = m->alpha64[A.prim + ia], ca = m->coeff64[A.prim + ia];
          const double b = m->alpha64[B.prim + ib], cb = m->coeff64[B.prim + ib];
          const double p = a + b;
          const double K = std::exp(-a * b / p * AB2);
          // -2 (electron charge x spin) * triangle factor * (2 pi / p) * K * ca * cb
          const double pref = -2.0 * fac * 2.0 * 3.14159265358979323846 / p * K * ca * cb;
          const double chg = std::fabs(pref) * pmax * std::pow(std::max(1.0, 2 * p), 0.5 * (A.L + B.L));
          if (chg < 1e-15) continue;
          double Ex[3][3][5], Ey[3][3][5], Ez[3][3][5];
          hermite_e_host(A.L, B.L, a, b, Ax, Bx, Ex);
          hermite_e_host(A.L, B.L, a, b, Ay, By, Ey);
          hermite_e_host(A.L, B.L, a, b, Az, Bz, Ez);
          double D[35] = {0};
          const int L = A.L + B.L;
          for (int k1 = 0; k1 < 2 * A.L + 1; ++k1) {
            double c1[3];
            int e1[3][3];
            const int n1 = cart_host(A.L, k1, c1, e1);
            for (int k2 = 0; k2 < 2 * B.L + 1; ++k2) {
              const double w = P64[(size_t)(A.func + k1) * np + B.func + k2];
              if (w == 0) continue;
              double c2[3];
              int e2[3][3];
              const int n2 = cart_host(B.L, k2, c2, e2);
              for (int u1 = 0; u1 < n1; ++u1)
                for (int u2 = 0; u2 < n2; ++u2) {
                  const int i = e1[u1][0], k = e1[u1][1], mm = e1[u1][2];
                  const int j = e2[u2][0], l = e2[u2][1], n = e2[u2][2];
                  const double cc = w * c1[u1] * c2[u2];
                  for (int t = 0; t <= i + j; ++t)
                    for (int u = 0; u <= k + l; ++u)
                      for (int v = 0; v <= mm + n; ++v)
                        D[herm_index(t, u, v)] += cc * Ex[i][j][t] * Ey[k][l][u] * Ez[mm][n][v];
                }
            }
          }
          // merge products with the same centres and exponents (general contractions)
          int ka = A.atom, kb = B.atom;
          double xa = a, xb = b;
          if (ka > kb || (ka == kb && xa > xb)) {
            std::swap(ka, kb);
            std::swap(xa, xb);
          }
          char key[64];
          std::snprintf(key, sizeof(key), "%d:%a:%d:%a", ka, xa, kb, xb);
          auto it = index.find(key);
          if (it == index.end()) {
            Acc g{};
            g.px = A.atom == B.atom ? Ax : (a * Ax + b * Bx) / p;   // on-site pairs sit on the nucleus
            g.py = A.atom == B.atom ? Ay : (a * Ay + b * By) / p;
            g.pz = A.atom == B.atom ? Az : (a * Az + b * Bz) / p;
            g.p = p;
            g.pref = pref;
            g.L = L;
            g.atom_a = ka;
            g.atom_b = kb;
            for (int q = 0; q < ncoef(L); ++q) g.D[q] = D[q];
            index.emplace(key, (int)acc.size());
            acc.push_back(g);
          } else {
            Acc& g = acc[it->second];
            const double r = pref / g.pref;
            g.L = std::max(g.L, L);
            for (int q = 0; q < ncoef(L); ++q) g.D[q] += r * D[q];
          }
        }
    }
  }
  // sort by L so that warps see uniform work, pack D
  std::vector<int> order(acc.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return acc[x].L < acc[y].L; });
  std::vector<GPair> pairs;
  std::vector<double> dco;
  for (int idx : order) {
    const Acc& g = acc[idx];
    GPair q;
    q.px = g.px;
    q.py = g.py;
    q.pz = g.pz;
    q.p = g.p;
    q.pref = g.pref;
    q.L = g.L;
    q.doff = (int)dco.size();
    for (int k = 0; k < ncoef(g.L); ++k) dco.push_back(g.D[k]);
    pairs.push_back(q);
  }
  if (pairs.empty()) {
    GPair z{};
    pairs.push_back(z);
    dco.push_back(0.0);
  }
  const size_t pb = pairs.size() * sizeof(GPair), db = dco.size() * sizeof(double);
  qmt_status st = m->d_pairs.reserve(pb + db + 256);
  if (st) return st;
  QMT_CUDA(cudaMemcpyAsync(m->d_pairs.ptr, pairs.data(), pb, cudaMemcpyHostToDevice, s));
  QMT_CUDA(cudaMemcpyAsync(m->d_pairs.as<uint8_t>() + ((pb + 255) / 256) * 256, dco.data(), db,
                           cudaMemcpyHostToDevice, s));
  // FP32 tables (Gto32Tables): centres relative to the centroid, pref * D_tuv as the coefficients.
  double ref[3] = {0, 0, 0};
  for (int a = 0; a < m->natoms; ++a)
    for (int d = 0; d < 3; ++d) ref[d] += m->coords[3 * a + d] / m->natoms;
  auto to32 = [&](const Acc& g, std::vector<float>& d32) {
    GPair32 q;
    q.px = (float)(g.px - ref[0]);
    q.py = (float)(g.py - ref[1]);
    q.pz = (float)(g.pz - ref[2]);
    q.p = (float)g.p;
    q.fscale = (float)(0.88622692545275801365 / std::sqrt(g.p));
    q.L = g.L;
    q.doff = (int)d32.size();
    q.pad = 0;
    for (int c = 0; c < ncoef(g.L); ++c) d32.push_back((float)(g.pref * g.D[c]));
    return q;
  };
  auto to64 = [&](const Acc& g, std::vector<double>& d64) {
    GPair64 q;
    q.px = g.px - ref[0];
    q.py = g.py - ref[1];
    q.pz = g.pz - ref[2];
    q.p = g.p;
    q.fscale = 0.88622692545275801365 / std::sqrt(g.p);
    q.L = g.L;
    q.doff = (int)d64.size();
    for (int c = 0; c < ncoef(g.L); ++c) d64.push_back(g.pref * g.D[c]);
    return q;
  };
  std::vector<GPair32> off32, on32;
  std::vector<GPair64> off64;
  std::vector<float> d32, onp;
  std::vector<double> d64, don;
  std::vector<int> on_off(m->natoms + 1, 0), cum_off(m->natoms + 1, 0);
  std::vector<double> cum;
  // The off-site pairs that carry most of the charge are evaluated in FP64: the error of an FP32
  // term (its rounded coefficients and arithmetic) is proportional to its size, and a few percent
  // of the pairs hold nearly all of it.  Size of a pair at a distance: its far-field multipoles,
  // order n weighted 10^-n.
  std::vector<int> offs;
  for (int idx : order)
    if (acc[idx].atom_a != acc[idx].atom_b) offs.push_back(idx);
  std::vector<double> size(acc.size(), 0.0);
  double total = 0.0;
  for (int idx : offs) {
    const Acc& g = acc[idx];
    double w = 0.0;
    for (int c = 0, n = 0; n <= g.L; ++n) {
      double sn = 0.0;
      for (; c < ncoef(n); ++c) sn += std::fabs(g.D[c]);
      w += sn * std::pow(0.1, n);
    }
    size[idx] = w * std::fabs(g.pref) / std::sqrt(g.p);
    total += size[idx];
  }
  std::vector<int> by_size(offs);
  std::stable_sort(by_size.begin(), by_size.end(), [&](int x, int y) { return size[x] > size[y]; });
  std::vector<char> heavy(acc.size(), 0);
  double rest = total;
  for (int idx : by_size) {
    if (rest <= kFp32Share * total) break;
    heavy[idx] = 1;
    rest -= size[idx];
  }
  for (int idx : offs)    // both lists keep the order by L
    if (heavy[idx]) off64.push_back(to64(acc[idx], d64));
    else if (size[idx] >= kFp32Screen * total) off32.push_back(to32(acc[idx], d32));
  if (off32.empty()) {    // one zero pair keeps the tables well formed
    Acc z{};
    z.p = 1.0;
    off32.push_back(to32(z, d32));
  }
  if (off64.empty()) {
    Acc z{};
    z.p = 1.0;
    off64.push_back(to64(z, d64));
  }
  std::vector<std::vector<int>> by_atom(m->natoms);
  for (size_t i = 0; i < acc.size(); ++i)
    if (acc[i].atom_a == acc[i].atom_b) by_atom[acc[i].atom_a].push_back((int)i);
  for (int a = 0; a < m->natoms; ++a) {
    std::vector<int>& v = by_atom[a];
    // descending exponent: for every point the far-field pairs (p r^2 >= 30) come first
    std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return (float)acc[x].p > (float)acc[y].p; });
    on_off[a] = (int)on32.size();
    cum_off[a] = (int)(cum.size() / 35);
    std::vector<double> run(35, 0.0);
    cum.insert(cum.end(), run.begin(), run.end());
    for (int idx : v) {
      const Acc& g = acc[idx];
      GPair32 q = to32(g, d32);
      q.pad = (int)don.size();   // the FP64 record: p, sqrt(pi) / (2 sqrt(p)), pref * D_tuv
      don.push_back(g.p);
      don.push_back(0.88622692545275801365 / std::sqrt(g.p));
      for (int c = 0; c < ncoef(g.L); ++c) don.push_back(g.pref * g.D[c]);
      on32.push_back(q);
      onp.push_back((float)g.p);
      const double f = 0.88622692545275801365 / std::sqrt(g.p) * g.pref;
      for (int c = 0; c < ncoef(g.L); ++c) run[c] += f * g.D[c];
      cum.insert(cum.end(), run.begin(), run.end());
    }
  }
  on_off[m->natoms] = (int)on32.size();
  cum_off[m->natoms] = (int)(cum.size() / 35);
  std::vector<float> nuc(3 * m->natoms);
  std::vector<double> nuc64(3 * m->natoms);
  for (int a = 0; a < m->natoms; ++a)
    for (int d = 0; d < 3; ++d) {
      nuc64[3 * a + d] = (double)m->coords[3 * a + d] - ref[d];
      nuc[3 * a + d] = (float)nuc64[3 * a + d];
    }
  if (on32.empty()) {     // keep the device arrays non-empty
    on32.push_back(GPair32{});
    onp.push_back(0.f);
    don.push_back(0.0);
  }
  // one device buffer: off-site pairs (FP32, FP64) | on-site pairs | doubles (cum, FP64
  // coefficients, on-site records, nuclei) | floats (dco, on-site p, nuclei) | ints
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_off = al(off32.size() * sizeof(GPair32)), b_on = al(on32.size() * sizeof(GPair32));
  const size_t b_o64 = al(off64.size() * sizeof(GPair64)), b_d64 = al(d64.size() * sizeof(double));
  const size_t b_don = al(don.size() * sizeof(double)), b_n64 = al(nuc64.size() * sizeof(double));
  const size_t b_cum = al(cum.size() * sizeof(double)), b_d = al(d32.size() * sizeof(float));
  const size_t b_p = al(onp.size() * sizeof(float)), b_nuc = al(nuc.size() * sizeof(float));
  const size_t b_i = al((on_off.size() + cum_off.size()) * sizeof(int));
  if ((st = m->d_pairs32.reserve(b_off + b_o64 + b_on + b_cum + b_d64 + b_don + b_n64 + b_d + b_p + b_nuc + b_i)))
    return st;
  uint8_t* base = m->d_pairs32.as<uint8_t>();
  std::vector<int> ints(on_off);
  ints.insert(ints.end(), cum_off.begin(), cum_off.end());
  size_t o = 0;
  auto put = [&](const void* src, size_t bytes, size_t span) -> uint8_t* {
    uint8_t* dst = base + o;
    o += span;
    if (bytes && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return nullptr;
    return dst;
  };
  Gto32Tables& T = m->gto32;
  T = Gto32Tables{};
  T.pairs = reinterpret_cast<const GPair32*>(put(off32.data(), off32.size() * sizeof(GPair32), b_off));
  T.pairs64 = reinterpret_cast<const GPair64*>(put(off64.data(), off64.size() * sizeof(GPair64), b_o64));
  T.onsite = reinterpret_cast<const GPair32*>(put(on32.data(), on32.size() * sizeof(GPair32), b_on));
  T.cum = reinterpret_cast<const double*>(put(cum.data(), cum.size() * sizeof(double), b_cum));
  T.dco64 = reinterpret_cast<const double*>(put(d64.data(), d64.size() * sizeof(double), b_d64));
  T.dco_on = reinterpret_cast<const double*>(put(don.data(), don.size() * sizeof(double), b_don));
  T.nuc64 = reinterpret_cast<const double*>(put(nuc64.data(), nuc64.size() * sizeof(double), b_n64));
  T.dco = reinterpret_cast<const float*>(put(d32.data(), d32.size() * sizeof(float), b_d));
  T.onsite_p = reinterpret_cast<const float*>(put(onp.data(), onp.size() * sizeof(float), b_p));
  T.nuc = reinterpret_cast<const float*>(put(nuc.data(), nuc.size() * sizeof(float), b_nuc));
  const int* ip = reinterpret_cast<const int*>(put(ints.data(), ints.size() * sizeof(int), b_i));
  if (!T.pairs || !T.pairs64 || !T.onsite || !T.cum || !T.dco64 || !T.dco_on || !T.nuc64 || !T.dco || !T.onsite_p ||
      !T.nuc || !ip)
    return fail(QMT_CUDA_ERR, "upload of the analytic-potential tables failed");
  T.onsite_off = ip;
  T.cum_off = ip + on_off.size();
  T.rx = ref[0];
  T.ry = ref[1];
  T.rz = ref[2];
  for (int L = 0; L <= 5; ++L) {   // off-site pairs are sorted by L
    int k = 0;
    while (k < (int)off32.size() && off32[k].L < L) ++k;
    T.lstart[L] = k;
    k = 0;
    while (k < (int)off64.size() && off64[k].L < L) ++k;
    T.lstart64[L] = k;
  }
  // cumulative estimated work for the slices (a term costs about 12 + 2 ncoef(L) operations)
  auto work = [](const auto& v) {
    std::vector<double> w(v.size() + 1, 0.0);
    for (size_t k = 0; k < v.size(); ++k) w[k + 1] = w[k] + 12.0 + 2.0 * ncoef(v[k].L);
    return w;
  };
  m->gto32_work = work(off32);
  m->gto64_work = work(off64);
  QMT_CUDA(cudaStreamSynchronize(s));
  m->gto_npairs = (int)pairs.size();
  m->gto_doff_bytes = ((pb + 255) / 256) * 256;
  m->gto_ready = true;
  return QMT_OK;
}

static qmt_status run_gto(qmt_mol* m, const GtoPoints& gp, float* out, cudaStream_t s) {
  qmt_status st;
  if ((st = build_pairs(m, s))) return st;
  if (gp.npts <= 0) return QMT_OK;
  if (g_gto_prec == QMT_PREC_FP32) {
    const double* tab64 = nullptr;
    if ((st = boys_table(&tab64))) return st;
    // enough CTAs to fill the device: each list of off-site pairs is split into slices whose FP64
    // partial sums the last kernel adds in slice order (deterministic)
    const int64_t pblocks = (gp.npts + GTO32_POINTS - 1) / GTO32_POINTS;
    const int64_t want = (int64_t)sm_count() * 12;
    const int nslice = (int)std::max<int64_t>(1, std::min<int64_t>(16, (want + pblocks - 1) / pblocks));
    Gto32Tables T = m->gto32;
    auto cut = [](const std::vector<double>& w, int n, int* slice) {
      const int np = (int)w.size() - 1;
      for (int k = 0, j = 0; k <= n; ++k) {   // slice k starts at the first pair past k/n of the work
        const double target = w.back() * k / n;
        while (j < np && w[j] < target) ++j;
        slice[k] = k == n ? np : j;
      }
    };
    T.nslice = nslice;
    T.nslice64 = nslice;
    cut(m->gto32_work, T.nslice, T.slice);
    cut(m->gto64_work, T.nslice64, T.slice64);
    if ((st = m->d_gto_part.reserve((size_t)(T.nslice + T.nslice64) * gp.npts * sizeof(double)))) return st;
    double* part = m->d_gto_part.as<double>();
    gto32_pairs_kernel<<<dim3((unsigned)pblocks, (unsigned)T.nslice), GTO32_THREADS, 0, s>>>(T, tab64, gp, part);
    QMT_CHECK_LAUNCH("gto32_pairs_kernel");
    gto64_pairs_kernel<<<dim3((unsigned)pblocks, (unsigned)T.nslice64), GTO32_THREADS, 0, s>>>(T, tab64, gp, part);
    QMT_CHECK_LAUNCH("gto64_pairs_kernel");
    const int64_t ablocks = (gp.npts + GTO32_THREADS - 1) / GTO32_THREADS;
    gto32_atoms_kernel<<<(unsigned)ablocks, GTO32_THREADS, 0, s>>>(T, tab64, m->view(), gp, part, out);
    QMT_CHECK_LAUNCH("gto32_atoms_kernel");
    return QMT_OK;
  }
  const double* tab = nullptr;
  if ((st = boys_table(&tab))) return st;
  const GPair* pairs = m->d_pairs.as<GPair>();
  const double* dco = reinterpret_cast<const double*>(m->d_pairs.as<uint8_t>() + m->gto_doff_bytes);
  const int64_t blocks = (gp.npts + GTO_THREADS - 1) / GTO_THREADS;
  gto_kernel<<<(unsigned)blocks, GTO_THREADS, 0, s>>>(pairs, m->gto_npairs, dco, tab, m->view(), gp, out);
  QMT_CHECK_LAUNCH("gto_kernel");
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" {

qmt_status qmt_hartree_gto(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                           float* v_dev, void* stream) {
  if (!mol || !v_dev || nx < 1 || ny < 1 || nz < 1 || !(step > 0.f)) return fail(QMT_BAD_ARG, "bad GTO arguments");
  GtoPoints gp{0, nx, ny, nz, step, ox, oy, oz, nullptr, (int64_t)nx * ny * nz};
  return run_gto(mol, gp, v_dev, as_stream(stream));
}

qmt_status qmt_hartree_gto_points(qmt_mol* mol, int npts, const float* pts_dev, float* v_dev, void* stream) {
  if (!mol || npts < 0 || (npts > 0 && (!pts_dev || !v_dev))) return fail(QMT_BAD_ARG, "bad GTO arguments");
  GtoPoints gp{2, 0, 0, 0, 0, 0, 0, 0, pts_dev, npts};
  return run_gto(mol, gp, v_dev, as_stream(stream));
}

qmt_status qmt_set_gto_precision(int precision) {
  if (precision != QMT_PREC_FP32 && precision != QMT_PREC_FP64)
    return fail(QMT_BAD_ARG, "analytic potential precision must be QMT_PREC_FP32 or QMT_PREC_FP64");
  g_gto_prec = precision;
  return QMT_OK;
}

qmt_status qmt_hartree_gto_boundary(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                                    float oz, float* v_dev, void* stream) {
  if (!mol || !v_dev || nx < 3 || ny < 3 || nz < 3 || !(step > 0.f))
    return fail(QMT_BAD_ARG, "bad GTO boundary arguments");
  const int64_t n = 2 * (int64_t)nx * ny + 2 * (int64_t)nx * (nz - 2) + 2 * (int64_t)(ny - 2) * (nz - 2);
  GtoPoints gp{3, nx, ny, nz, step, ox, oy, oz, nullptr, n};
  return run_gto(mol, gp, v_dev, as_stream(stream));
}

}  // extern "C"

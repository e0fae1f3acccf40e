// Tensor-core density path (sm_100a, tcgen05 + TMA).
//
//   stage:  basis_stage_kernel evaluates Phi' = Phi * 2^s_j (power-of-two column scales)
//           for 128-row tiles of sample points and writes it as operand pieces
//           hi = fmt(Phi'), lo = fmt(Phi' - hi) to HBM, row-major [row][kpad].
//   mma:    density_mma_kernel, one CTA per SM, warp-specialised:
//             warp 0      TMA producer: A (Phi' pieces, 128 x 64B..128B K-chunks) and
//                         B (scaled density-matrix pieces) into a shared-memory ring;
//             warp 1      tcgen05.mma issuer (one thread); T' = Phi' * Ptilde accumulated
//                         in TMEM, two 256-column accumulator buffers;
//             warps 2..5  epilogue: tcgen05.ld of T' rows, row-dot with Phi' (FP64
//                         accumulation), sub-point average, grid write, FP64 tile sums.
//   With Ptilde_jk = P_jk 2^(g - s_j - s_k):  rho_i = 2^-g sum_j Phi'_ij T'_ij.
//   Split products (3 terms) hi*hi + hi*lo + lo*hi recover ~22 significant bits for fp16
//   pieces (scaled to stay in the normal range) and tf32, ~16 bits for bf16.
//
// Replaces the per-voxel pair loop of gpu_densityqube_shmem_subgrid (kernel_density.cu:74-140).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>

#include "density.cuh"
#include "reduce.cuh"
#include "sm100.cuh"

namespace qmt {
using namespace sm100;

enum { FMT_F16 = 0, FMT_BF16 = 1, FMT_TF32 = 2 };

struct TcShape {
  int fmt, nsplit, esize, ke, kpad, npanels, pw, nrows_b;
};

static TcShape tc_shape(int prec, int norbs) {
  TcShape t{};
  switch (prec) {
    case QMT_PREC_TF32: t.fmt = FMT_TF32; t.nsplit = 1; break;
    case QMT_PREC_TF32X3: t.fmt = FMT_TF32; t.nsplit = 2; break;
    case QMT_PREC_BF16: t.fmt = FMT_BF16; t.nsplit = 1; break;
    case QMT_PREC_BF16X3: t.fmt = FMT_BF16; t.nsplit = 2; break;
    default: t.fmt = FMT_F16; t.nsplit = 2; break;
  }
  t.esize = t.fmt == FMT_TF32 ? 4 : 2;
  t.ke = 128 / t.esize;
  t.kpad = (norbs + 63) / 64 * 64;
  t.npanels = (t.kpad + 255) / 256;
  t.pw = ((t.kpad + t.npanels - 1) / t.npanels + 15) / 16 * 16;
  t.nrows_b = t.npanels * t.pw;
  return t;
}

// ---- element conversions (host and device) ------------------------------------------
__host__ __device__ inline uint32_t tf32_round_bits(float x) {
  uint32_t u;
#ifdef __CUDA_ARCH__
  u = __float_as_uint(x);
#else
  std::memcpy(&u, &x, 4);
#endif
  if ((u & 0x7f800000u) == 0x7f800000u) return u;
  u += 0xfffu + ((u >> 13) & 1u);
  return u & 0xffffe000u;
}
__host__ __device__ inline float bits_f32(uint32_t u) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  std::memcpy(&f, &u, 4);
  return f;
#endif
}

// ---------------------------------------------------------------------------------------
// Stage 2: tcgen05 contraction with the fused row-dot epilogue.
// ---------------------------------------------------------------------------------------
struct TcParams {
  PointMap pm;
  int64_t tile0;
  int ntiles;
  int kpad, kchunks, npanels, pw, stages, nsplit, esize;
  uint32_t a_bytes, b_bytes, stage_bytes, tx_bytes;
  uint32_t idesc;
  const void* phi_hi;
  const void* phi_lo;
  float* qube;
  double* partials;
  double outscale;
  const double* gsc;   // device {max, 2^g, 2^-g} of the split density matrix (factored: the
                       // column scales 2^-2h_k of the squares)
  int* err;
  uint64_t wait_ns;    // limit of every bounded wait (a test shortens it)
  int nb;              // factored: rank rounded up to 16 (B holds its hi rows, then its lo rows)
  const int* gate;     // when set, the launch runs only if *gate == gate_want (device-side check
  int gate_want;       // of the factor picks the factored or the unfactored launch)
};

constexpr int MAX_STAGES = 8;

__device__ __forceinline__ void load_phi32(const TcParams& p, int64_t row, int col, float* out) {
  if (p.esize == 4) {
    const float4* h = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(p.phi_hi) + row * p.kpad + col);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float4 a = h[i];
      out[4 * i] = a.x;
      out[4 * i + 1] = a.y;
      out[4 * i + 2] = a.z;
      out[4 * i + 3] = a.w;
    }
    if (p.nsplit == 2) {
      const float4* l = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(p.phi_lo) + row * p.kpad + col);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const float4 a = l[i];
        out[4 * i] += a.x;
        out[4 * i + 1] += a.y;
        out[4 * i + 2] += a.z;
        out[4 * i + 3] += a.w;
      }
    }
  }
}

template <int FMT>
__device__ __forceinline__ void load_phi16(const TcParams& p, int64_t row, int col, float* out) {
  const uint4* h = reinterpret_cast<const uint4*>(reinterpret_cast<const uint16_t*>(p.phi_hi) + row * p.kpad + col);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint4 a = h[i];
    const uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if constexpr (FMT == FMT_F16) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[j]));
        out[8 * i + 2 * j] = f.x;
        out[8 * i + 2 * j + 1] = f.y;
      } else {
        out[8 * i + 2 * j] = __uint_as_float(w[j] << 16);
        out[8 * i + 2 * j + 1] = __uint_as_float(w[j] & 0xffff0000u);
      }
    }
  }
  if (p.nsplit == 2) {
    const uint4* l = reinterpret_cast<const uint4*>(reinterpret_cast<const uint16_t*>(p.phi_lo) + row * p.kpad + col);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint4 a = l[i];
      const uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if constexpr (FMT == FMT_F16) {
          const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[j]));
          out[8 * i + 2 * j] += f.x;
          out[8 * i + 2 * j + 1] += f.y;
        } else {
          out[8 * i + 2 * j] += __uint_as_float(w[j] << 16);
          out[8 * i + 2 * j + 1] += __uint_as_float(w[j] & 0xffff0000u);
        }
      }
    }
  }
}

// FACT: B is the factored density matrix (one box of nb hi rows then nb lo rows per K-chunk, one
// output panel); per K-step one MMA [A_hi B_hi | A_hi B_lo] into the buffer's first accumulator and
// one [A_lo B_hi | A_lo B_lo] into its second; the epilogue adds the four column groups and sums
// the squares with the column scales (no re-read of Phi').  TMEM buffers of 2 x N columns, two of
// them when they fit in 512.
template <int FMT, bool FACT>
__global__ void __launch_bounds__(192, 1)
    density_mma_kernel(const __grid_constant__ CUtensorMap tmA_hi, const __grid_constant__ CUtensorMap tmA_lo,
                       const __grid_constant__ CUtensorMap tmB_hi, const __grid_constant__ CUtensorMap tmB_lo,
                       const TcParams p) {
  extern __shared__ uint8_t smem_dyn[];
  if (p.gate && *p.gate != p.gate_want) return;   // the other launch of the pair does the work
  __shared__ __align__(8) uint64_t full_bar[MAX_STAGES], empty_bar[MAX_STAGES];
  __shared__ __align__(8) uint64_t tfull[2], tempty[2], drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ double rho_s[128];
  __shared__ double red[4];
  __shared__ volatile int abort_flag;

  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 128);
    }
    mbar_init(&drain_bar, 1);
    fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    prefetch_tmap(&tmA_hi);
    prefetch_tmap(&tmB_hi);
    if (p.nsplit == 2) {
      prefetch_tmap(&tmA_lo);
      prefetch_tmap(&tmB_lo);
    }
  }
  if (warp == 1) {
    tmem_alloc(&tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  auto stage_ptr = [&](int s) { return smem + (size_t)s * p.stage_bytes; };

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      int last_par[MAX_STAGES];
      for (int s = 0; s < MAX_STAGES; ++s) last_par[s] = -1;
      bool ok = true;
      for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
        for (int pn = 0; pn < p.npanels && ok; ++pn) {
          for (int kc = 0; kc < p.kchunks; ++kc, ++it) {
            const int s = it % p.stages;
            const uint32_t ph = (it / p.stages) & 1u;
            if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_flag, p.wait_ns)) {
              ok = false;
              break;
            }
            uint8_t* st = stage_ptr(s);
            mbar_expect_tx(&full_bar[s], p.tx_bytes);
            const int x = kc * (128 / p.esize);
            tma_load_2d(st, &tmA_hi, &full_bar[s], x, t * 128);
            if (p.nsplit == 2) tma_load_2d(st + p.a_bytes, &tmA_lo, &full_bar[s], x, t * 128);
            uint8_t* bst = st + p.nsplit * p.a_bytes;
            tma_load_2d(bst, &tmB_hi, &full_bar[s], x, pn * p.pw);
            if (p.nsplit == 2 && !FACT) tma_load_2d(bst + p.b_bytes, &tmB_lo, &full_bar[s], x, pn * p.pw);
            last_par[s] = (int)ph;
          }
        }
      }
      if (!ok) {  // drain copies still in flight before the CTA exits
        for (int s = 0; s < p.stages; ++s)
          if (last_par[s] >= 0) mbar_wait_drain(&full_bar[s], (uint32_t)last_par[s], 100000000ull);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, acc_it = 0;
      bool ok = true;
      const int ksteps = 128 / (p.esize * (p.esize == 4 ? 8 : 16));  // 4 steps of 32 bytes
      // factored: N = the factor's hi and lo rows, a buffer holds two accumulators of N
      const uint32_t nfac = (uint32_t)(p.nsplit * p.nb), fbuf = (uint32_t)p.nsplit * nfac;
      const uint32_t nbuf = FACT ? (fbuf <= 256u ? 2u : 1u) : 2u;
      for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
        for (int pn = 0; pn < p.npanels && ok; ++pn, ++acc_it) {
          const uint32_t buf = nbuf == 2u ? (acc_it & 1u) : 0u, aph = ((nbuf == 2u ? acc_it >> 1 : acc_it)) & 1u;
          if (!mbar_wait(&tempty[buf], aph ^ 1u, &abort_flag, p.wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + buf * (FACT ? 256u * (2u / nbuf) : 256u);
          for (int kc = 0; kc < p.kchunks; ++kc, ++it) {
            const int s = it % p.stages;
            const uint32_t ph = (it / p.stages) & 1u;
            if (!mbar_wait(&full_bar[s], ph, &abort_flag, p.wait_ns)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(stage_ptr(s));
            const uint32_t a1 = a0 + p.a_bytes;
            const uint32_t b0 = a0 + p.nsplit * p.a_bytes;
            const uint32_t b1 = b0 + p.b_bytes;
            for (int ks = 0; ks < ksteps; ++ks) {
              const uint32_t off = ks * 32u;
              const uint32_t acc = (kc | ks) != 0;
              if constexpr (FMT == FMT_TF32) {
                mma_tf32(d, sw128_kmajor_desc(a0 + off), sw128_kmajor_desc(b0 + off), p.idesc, acc);
                if (p.nsplit == 2) {
                  mma_tf32(d, sw128_kmajor_desc(a0 + off), sw128_kmajor_desc(b1 + off), p.idesc, 1u);
                  mma_tf32(d, sw128_kmajor_desc(a1 + off), sw128_kmajor_desc(b0 + off), p.idesc, 1u);
                }
              } else if (FACT) {
                mma_f16(d, sw128_kmajor_desc(a0 + off), sw128_kmajor_desc(b0 + off), p.idesc, acc);
                if (p.nsplit == 2) mma_f16(d + nfac, sw128_kmajor_desc(a1 + off), sw128_kmajor_desc(b0 + off), p.idesc, acc);
              } else {
                mma_f16(d, sw128_kmajor_desc(a0 + off), sw128_kmajor_desc(b0 + off), p.idesc, acc);
                if (p.nsplit == 2) {
                  mma_f16(d, sw128_kmajor_desc(a0 + off), sw128_kmajor_desc(b1 + off), p.idesc, 1u);
                  mma_f16(d, sw128_kmajor_desc(a1 + off), sw128_kmajor_desc(b0 + off), p.idesc, 1u);
                }
              }
            }
            tc_commit(&empty_bar[s]);
          }
          if (ok) tc_commit(&tfull[buf]);
        }
      }
      // every MMA issued by this thread has completed once drain_bar flips
      tc_commit(&drain_bar);
      mbar_wait_drain(&drain_bar, 0u, 500000000ull);
    }
  } else {
    // epilogue: warps 2..5 -> TMEM lane quadrants 2,3,0,1
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const int et = threadIdx.x - 64;
    uint32_t acc_it = 0;
    bool ok = true;
    const uint32_t nfac = (uint32_t)(p.nsplit * p.nb), fbuf = (uint32_t)p.nsplit * nfac;
    const uint32_t nbuf = FACT ? (fbuf <= 256u ? 2u : 1u) : 2u;
    for (int t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
      double acc = 0.0;
      const int64_t grow = (int64_t)t * 128 + row;
      for (int pn = 0; pn < p.npanels; ++pn, ++acc_it) {
        const uint32_t buf = nbuf == 2u ? (acc_it & 1u) : 0u, aph = ((nbuf == 2u ? acc_it >> 1 : acc_it)) & 1u;
        // the four epilogue warps leave together: one of them giving up while the others go on
        // would leave those waiting at the next named barrier
        const bool got = mbar_wait(&tfull[buf], aph, &abort_flag, p.wait_ns);
        if (barrier_any(1, 128, !got)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (FACT) {
          // T_k = the sum of the column groups (hi x hi, hi x lo, lo x hi, lo x lo), then
          // rho = sum_k 2^-2h_k T_k^2
          const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + buf * 256u * (2u / nbuf);
          const int ng = p.nsplit == 2 ? 4 : 1;
          for (int c = 0; c * 16 < p.nb; ++c) {
            float tsum[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) tsum[e] = 0.f;
            for (int gi = 0; gi < ng; ++gi) {
              uint32_t tv[16];
              tmem_ld16_issue(tb + (uint32_t)(gi * p.nb + c * 16), tv);
              tmem_ld16_wait(tv);
#pragma unroll
              for (int e = 0; e < 16; ++e) tsum[e] += __uint_as_float(tv[e]);
            }
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const double v = (double)tsum[e];
              acc = fma(__ldg(p.gsc + c * 16 + e) * v, v, acc);
            }
          }
        } else {
          for (int c = 0; c < p.pw / 32; ++c) {
            const int col = pn * p.pw + 32 * c;
            if (col >= p.kpad) break;
            float v[32], ph[32];
            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * 256u + 32u * c, v);
            if constexpr (FMT == FMT_TF32) load_phi32(p, grow, col, ph);
            else load_phi16<FMT>(p, grow, col, ph);
#pragma unroll
            for (int k = 0; k < 32; ++k) acc = fma((double)ph[k], (double)v[k], acc);
          }
        }
        tc_fence_before();
        mbar_arrive(&tempty[buf]);
      }
      if (!ok) break;
      rho_s[row] = FACT ? acc : acc * p.gsc[2];
      named_barrier(1, 128);
      double mysum = 0.0;
      if (et < p.pm.vpt) {
        double r = 0.0;
        for (int s = 0; s < p.pm.s3; ++s) r += rho_s[et * p.pm.s3 + s];
        int64_t vox, ix, iy, iz;
        if (tile_voxel(p.pm, p.tile0 + t, et, vox, ix, iy, iz)) {
          const float qv = (float)(r * p.outscale);
          p.qube[vox] = qv;
          mysum = qv;
        }
      }
      for (int o = 16; o > 0; o >>= 1) mysum += __shfl_xor_sync(0xffffffffu, mysum, o);
      if (lane == 0) red[q] = mysum;
      named_barrier(1, 128);
      if (et == 0) p.partials[p.tile0 + t] = red[0] + red[1] + red[2] + red[3];
    }
  }

  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicExch(p.err, 1);
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

static qmt_status make_map(CUtensorMap* m, const void* base, int esize, uint64_t inner, uint64_t outer,
                           uint32_t box_inner, uint32_t box_outer) {
  auto fn = encode_fn();
  if (!fn) return fail(QMT_CUDA_ERR, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * (uint64_t)esize};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
  CUresult r = fn(m, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(QMT_CUDA_ERR, "cuTensorMapEncodeTiled failed");
  return QMT_OK;
}

__host__ __device__ inline void split_host(double x, int fmt, void* hi, void* lo, size_t idx) {
  if (fmt == FMT_TF32) {
    const uint32_t h = tf32_round_bits((float)x);
    const uint32_t l = tf32_round_bits((float)(x - (double)bits_f32(h)));
    reinterpret_cast<uint32_t*>(hi)[idx] = h;
    reinterpret_cast<uint32_t*>(lo)[idx] = l;
  } else if (fmt == FMT_F16) {
    const __half h = __float2half_rn((float)x);
    const __half l = __float2half_rn((float)(x - (double)__half2float(h)));
    reinterpret_cast<__half*>(hi)[idx] = h;
    reinterpret_cast<__half*>(lo)[idx] = l;
  } else {
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    reinterpret_cast<__nv_bfloat16*>(hi)[idx] = h;
    reinterpret_cast<__nv_bfloat16*>(lo)[idx] = l;
  }
}

// Scaled, split density matrix on the device: element (r, c), r, c < n, at r * K + c holds
// P_rc 2^(g - s_r - s_c) split into hi + lo (inv_s = 2^-s, exact powers of two, so this equals
// ldexp of the same exponents).  The pieces must be cleared beforehand (padding stays zero).
// Element (r, c) goes to r * K + c (row-major), or, with blk_rows > 0, to the K-step blocks of
// the fused path: block c / 16 holds blk_rows rows of 32 bytes (the 16 columns of one K-step),
// each row's two 16-byte units exchanged when bit 2 of the row is set -- the 32-byte swizzled
// K-major image that the MMA reads from shared memory, so that a stage is one contiguous copy.
__global__ void split_P_kernel(const double* __restrict__ P, int np, int n, int K, const double* __restrict__ inv_s,
                               const double* __restrict__ gsc, int fmt, int blk_rows, uint8_t* hi, uint8_t* lo) {
  const int64_t tot = (int64_t)n * n;
  const double two_g = gsc[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i % n);
    const double v = P[(size_t)c * np + r] * two_g * inv_s[r] * inv_s[c];
    const int e = c & 15, pe = ((((e >> 3) ^ (r >> 2)) & 1) << 3) | (e & 7);   // swizzled position in the row
    const size_t idx = blk_rows > 0 ? ((size_t)(c >> 4) * blk_rows + r) * 16 + pe : (size_t)r * K + c;
    split_host(v, fmt, hi, lo, idx);
  }
}

// max_jk |P_jk| 2^(-s_j - s_k) over the n x n block, as the bits of a non-negative double
// (ordered like the values), into gsc[0].
__global__ void split_max_kernel(const double* __restrict__ P, int np, int n, const double* __restrict__ inv_s,
                                 unsigned long long* gsc_bits) {
  __shared__ double red[32];
  double mx = 0.0;
  const int64_t tot = (int64_t)n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(i / n), k = (int)(i - (int64_t)j * n);
    mx = fmax(mx, fabs(P[(size_t)j * np + k]) * inv_s[k] * inv_s[j]);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    mx = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (threadIdx.x == 0) atomicMax(gsc_bits, (unsigned long long)__double_as_longlong(mx));
  }
}

// The exponent g that puts that maximum near 2^14 (g in [-100, 100], 0 for a zero matrix):
// gsc[1] = 2^g, gsc[2] = 2^-g.
__global__ void split_exp_kernel(double* gsc) {
  const double mx = __longlong_as_double((long long)reinterpret_cast<const unsigned long long*>(gsc)[0]);
  int g = mx > 0 ? (int)floor(log2(16000.0 / mx)) : 0;
  g = max(-100, min(100, g));
  gsc[1] = ldexp(1.0, g);
  gsc[2] = ldexp(1.0, -g);
}

// Column scales 2^s_j (fs, folded into the producer tables) and 2^-s_j (device, for the split)
// and the producer tables: they depend on the basis only, so they are built once per molecule.
static qmt_status ensure_mol_tables(qmt_mol* m, const std::vector<float>& fs, int K, cudaStream_t s);
static qmt_status ensure_basis_operands(qmt_mol* m, int K, cudaStream_t s) {
  if (m->basis_ops_ready) return QMT_OK;
  const int n = m->norbs;
  std::vector<float> fs(K, 0.f);
  std::vector<double> inv(K, 1.0);
  for (int j = 0; j < n; ++j) {
    const double b = std::max(m->fbound[j], 1e-30);
    const int sj = std::max(-60, std::min(60, (int)std::floor(std::log2(16000.0 / b))));
    fs[j] = (float)std::ldexp(1.0, sj);
    inv[j] = std::ldexp(1.0, -sj);
  }
  qmt_status st = m->d_split_scale.reserve(K * sizeof(double));
  if (st) return st;
  m->split_inv = inv;
  // pageable uploads return once the data is staged, so `inv` may go
  QMT_CUDA(cudaMemcpyAsync(m->d_split_scale.ptr, inv.data(), K * sizeof(double), cudaMemcpyHostToDevice, s));
  if ((st = ensure_mol_tables(m, fs, K, s))) return st;
  m->basis_ops_ready = true;
  return QMT_OK;
}

// Exponent of the scaled density matrix, on the device (no host round trip).
static qmt_status split_exponent(qmt_mol* m, cudaStream_t s) {
  qmt_status st = m->d_gscale.reserve(4 * sizeof(double));
  if (st) return st;
  QMT_CUDA(cudaMemsetAsync(m->d_gscale.ptr, 0, sizeof(double), s));
  const int64_t tot = (int64_t)m->norbs * m->norbs;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 2);
  split_max_kernel<<<std::max(blocks, 1), 256, 0, s>>>(m->d_P64.as<double>(), m->npad, m->norbs,
                                                       m->d_split_scale.as<double>(),
                                                       reinterpret_cast<unsigned long long*>(m->d_gscale.ptr));
  QMT_CHECK_LAUNCH("split_max_kernel");
  split_exp_kernel<<<1, 1, 0, s>>>(m->d_gscale.as<double>());
  QMT_CHECK_LAUNCH("split_exp_kernel");
  return QMT_OK;
}

static qmt_status launch_split(qmt_mol* m, int K, int fmt, int blk_rows, void* hi, void* lo,
                               size_t piece_bytes, cudaStream_t s) {
  QMT_CUDA(cudaMemsetAsync(hi, 0, piece_bytes, s));
  QMT_CUDA(cudaMemsetAsync(lo, 0, piece_bytes, s));
  const int64_t tot = (int64_t)m->norbs * m->norbs;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 8);
  split_P_kernel<<<std::max(blocks, 1), 256, 0, s>>>(m->d_P64.as<double>(), m->npad, m->norbs, K,
                                                     m->d_split_scale.as<double>(), m->d_gscale.as<double>(), fmt, blk_rows,
                                                     reinterpret_cast<uint8_t*>(hi), reinterpret_cast<uint8_t*>(lo));
  QMT_CHECK_LAUNCH("split_P_kernel");
  return QMT_OK;
}

// ---------------------------------------------------------------------------------------
// Fused path (kind::f16 formats, K <= 320): Phi' never leaves shared memory.
//
//   rho = sum_k Phi_k (Phi P)_k over the full symmetric P.  (Streaming only the upper triangle,
//   rho = 2 sum_k Phi_k (Phi U)_k with U = triu(P, 1) + diag(P)/2, halves the tensor work but
//   doubles the FP32 accumulation error, and measured 4% slower: the K-step loop is not bound
//   by tensor work.)
//
// CTA layout (one per SM, persistent over 128-row tiles), 10 warps:
//   warp 0     producer of U: one bulk copy per stage and piece of a K-step block that HBM
//              already holds in the 32-byte swizzled layout (tensor-map boxes of 32-byte rows
//              ran the copy engine at ~40 GB/s per SM; contiguous copies do not);
//              U is the same for every tile, so it streams ahead across tiles;
//   warp 1     TMEM allocation and the single MMA-issuing thread;
//   warps 2-9  evaluate Phi' for the tile straight into the 128-byte swizzled K-major
//              A layout (hi and lo pieces), then run the epilogue: T' rows from TMEM
//              (warp w reads lane quadrant w%4, column chunks of parity (w-2)/4), Phi'
//              from shared memory, FP64 row-dot, sub-point average, grid write, FP64 sums.
// Per tile the phases are serial (A is resident and single-buffered); the U stream and
// the MMA run asynchronously to the compute warps' work.
// ---------------------------------------------------------------------------------------
constexpr int MAX_FUSED_CHUNKS = 5;   // fused path: kpad <= 320

// One molecule of a fused launch.  A launch covers the tiles of one or more molecules; global tile
// t belongs to the molecule with tile0 <= t < tile0 + ntiles.
struct FusedMol {
  PointMap pm;
  int64_t tile0, ntiles;
  int natoms, norbs;
  int n16;                 // functions rounded up to 16: K of the MMAs; the K-steps beyond it
                           // only hold zero padding and are skipped
  int nb;                  // N of the MMAs (rows of a K-step block of B): n16 for the density
                           // matrix, the rank rounded up to 16 for its factor
  int ksteps, nchunks;     // n16 / 16 K-steps; ceil(n16 / 64) column chunks of A
  int tail0;               // n16 & ~63: first column of A's 32-byte swizzled tail blocks
  int u_rows;              // rows of one K-step block of U in HBM (kpad + 64)
  const uint8_t* u_hi;     // U pieces in K-step blocks (split_P_kernel with blk_rows = u_rows)
  const uint8_t* u_lo;
  int chunk_need[MAX_FUSED_CHUNKS];  // production items (atom halves) writing each chunk
  const int4* tab;         // molecule tables (ensure_mol_tables)
  int tab_words;           // 16-byte words of tab
  int off_prim;            // byte offsets inside the staged tables: primitive pairs,
  int off_ashell;          //   first shell of each atom,
  int off_coords;          //   nuclear coordinates (float x, y, z)
  const float* coords;
  float* qube;
  double* partials;        // per tile of this molecule
  double outscale;
  const double* gsc;       // device {max, 2^g, 2^-g} of the split density matrix
};

struct FusedParams {
  FusedMol one;            // the molecule of a single-molecule launch (nmol == 1)
  const FusedMol* mols;    // device array of nmol molecules (nmol > 1)
  int nmol;
  int64_t ntiles;          // tiles of all molecules
  int nsplit, stages;
  uint32_t a_bytes;        // one A piece: 128 rows x (largest n16) x 2 B
  uint32_t b_slot;         // one U piece slot in a stage: (largest n16) rows x 32 B
  uint32_t stage_bytes;
  uint32_t fmt;
  int* err;
  uint64_t wait_ns;        // limit of every bounded wait (a test shortens it)
  const int* gate;         // when set, the launch runs only if *gate == gate_want (the device-side
  int gate_want;           // check of the factored matrix picks one of two launches)
};

// Factored path: a stage holds the factor's hi rows followed by its lo rows, so one MMA of
// N = 2 nb gives [A_hi B_hi | A_hi B_lo] and, with two pieces, one more [A_lo B_hi | A_lo B_lo].
// The first kind of the K-steps of the nchunks column chunks goes to fact_nacc(nchunks, nb, two)
// TMEM accumulators of 2 nb columns (chunk c to accumulator c * na / nchunks), the second kind to
// one more, and the epilogue adds them.  The accumulators' FP32 additions round with a bias
// toward zero, which the squares of T would double into rho; few additions of large terms per
// accumulator keep it small.  Two different accumulators alternate, so no MMA waits on the one
// before it.
__host__ __device__ __forceinline__ int fact_nacc(int nchunks, int nb, bool two) {
  const int fit = 512 / (two ? 2 * nb : nb) - (two ? 1 : 0);
  return nchunks < fit ? nchunks : fit;
}

// Arrival count of a column-chunk barrier: each tile pre-arrives CHUNK_COUNT - need, the
// production items the rest, so that molecules with different atom counts share the barriers.
constexpr uint32_t CHUNK_COUNT = 1024;

// The molecule of global tile t: p.one in a single-molecule launch (MULTI false: read from the
// parameter space), else a binary search over the launch's molecules.
template <bool MULTI>
__device__ __forceinline__ const FusedMol& fused_mol(const FusedParams& p, int64_t t, int& m) {
  if (!MULTI) {
    m = 0;
    return p.one;
  }
  int lo = 0, hi = p.nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&p.mols[mid].tile0) <= t) lo = mid;
    else hi = mid - 1;
  }
  m = lo;
  return p.mols[lo];
}

// Byte offset of element (row, j) in the K-major A tile of a molecule with n16 columns: columns
// below tail0 = n16 & ~63 in 128-byte swizzled 64-column chunks (8-row atoms of 1024 B, 16-byte
// unit u of a row at u ^ (row & 7)); the last n16 - tail0 columns in 32-byte swizzled 16-column
// blocks (rows of 32 B, the two 16-byte units exchanged when bit 2 of the row is set), so the tile
// holds exactly n16 columns.  Row r + 64 of a column sits a_row64 bytes after row r.
__device__ __forceinline__ uint32_t a_offset(int row, int j, int tail0) {
  if (j < tail0) {
    const int kc = j >> 6, e = j & 63;
    const int u = (e >> 3) ^ (row & 7);
    return (uint32_t)(kc * 16384 + (row >> 3) * 1024 + (row & 7) * 128 + u * 16 + (e & 7) * 2);
  }
  const int e = j & 15;
  return (uint32_t)(tail0 * 256 + ((j - tail0) >> 4) * 4096 + row * 32 + ((((e >> 3) ^ (row >> 2)) & 1) << 4) +
                    (e & 7) * 2);
}
__device__ __forceinline__ uint32_t a_row64(int j, int tail0) { return j < tail0 ? 8192u : 2048u; }

__device__ __forceinline__ uint64_t sw32_kmajor_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;             // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(256u >> 4) << 32;    // stride byte offset: 8 rows x 32 B
  d |= (uint64_t)1u << 46;             // descriptor version for sm_100
  d |= (uint64_t)6u << 61;             // 32-byte swizzle
  return d;
}

template <int FMT>
__device__ __forceinline__ void store_split16(uint8_t* hi, uint8_t* lo, uint32_t off, float x, bool two) {
  if constexpr (FMT == FMT_F16) {
    const __half h = __float2half_rn(x);
    *reinterpret_cast<__half*>(hi + off) = h;
    if (two) *reinterpret_cast<__half*>(lo + off) = __float2half_rn(x - __half2float(h));
  } else {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    *reinterpret_cast<__nv_bfloat16*>(hi + off) = h;
    if (two) *reinterpret_cast<__nv_bfloat16*>(lo + off) = __float2bfloat16_rn(x - __bfloat162float(h));
  }
}

template <int FMT>
__device__ __forceinline__ void store_pair16(uint8_t* hi, uint8_t* lo, uint32_t off, float x0, float x1, bool two) {
  if constexpr (FMT == FMT_F16) {
    const __half2 h = __floats2half2_rn(x0, x1);
    *reinterpret_cast<__half2*>(hi + off) = h;
    if (two) {
      const float2 hf = __half22float2(h);
      *reinterpret_cast<__half2*>(lo + off) = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    }
  } else {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    *reinterpret_cast<__nv_bfloat162*>(hi + off) = h;
    if (two) {
      const float2 hf = __bfloat1622float2(h);
      *reinterpret_cast<__nv_bfloat162*>(lo + off) = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
    }
  }
}

template <int FMT>
__device__ __forceinline__ void unpack8(uint4 a, float* out) {
  const uint32_t w[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if constexpr (FMT == FMT_F16) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[j]));
      out[2 * j] = f.x;
      out[2 * j + 1] = f.y;
    } else {
      out[2 * j] = __uint_as_float(w[j] << 16);
      out[2 * j + 1] = __uint_as_float(w[j] & 0xffff0000u);
    }
  }
}

// Primitive exponentials exp(-alpha q), zero at and beyond the cut-off.  FAST producers (the fused
// kernel with the factored density matrix) take 2^(-beta q), beta = alpha log2(e) formed once per
// primitive, with a single ex2.approx in place of the longer expf sequence: Phi' about a sixth
// faster, at a larger error (fp16x3 density against the FP64 path, relative L2: 4.1e-7 -> 5.4e-7
// on a 24^3 grid at 0.8 bohr around the 30-atom molecule, 4.2e-7 -> 4.5e-7 on its 128^3 grid at
// 0.15 bohr).  The unfactored contraction sits nearer its 1e-6 budget (9.7e-7 on the coarse grid)
// and keeps expf.
constexpr float kLog2e = 1.44269504f;
constexpr float kExpCut2 = kExpCut * kLog2e;   // the cut-off in the base-2 scale

template <bool FAST>
__device__ __forceinline__ float exp_scale(float alpha) {
  if constexpr (FAST) return alpha * kLog2e;
  else return alpha;
}

template <bool FAST>
__device__ __forceinline__ float exp_cut(float x) {   // x = exp_scale<FAST>(alpha) * q
  if constexpr (FAST) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(-x));
    return x < kExpCut2 ? r : 0.f;
  } else {
    return x < kExpCut ? expf(-x) : 0.f;
  }
}

// Contracted radial parts sum_k c_k exp(-alpha_k r^2) (zero beyond the cut-off) of NP primitives
// (alpha, c) at two points, in primitive order.  When the next shell of the atom has the same
// exponents (pn != nullptr) its radial parts are formed from the same exponentials.
template <int NP, bool FAST>
__device__ __forceinline__ void radial_np(const float2* pa, const float2* pn, float q0, float q1, float& r0,
                                          float& r1, float& n0, float& n1) {
  float2 ac[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) ac[k] = pa[k];
  float e0[NP], e1[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const float b = exp_scale<FAST>(ac[k].x);
    e0[k] = exp_cut<FAST>(b * q0);
    e1[k] = exp_cut<FAST>(b * q1);
  }
  r0 = 0.f;
  r1 = 0.f;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    r0 = fmaf(ac[k].y, e0[k], r0);
    r1 = fmaf(ac[k].y, e1[k], r1);
  }
  if (pn) {
    n0 = 0.f;
    n1 = 0.f;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const float d = pn[k].y;
      n0 = fmaf(d, e0[k], n0);
      n1 = fmaf(d, e1[k], n1);
    }
  }
}

// ---- fixed atom layouts ----------------------------------------------------------------------
// Atoms whose shells follow a known layout are produced by fully unrolled code (one dispatch per
// atom, every table load independent); others take the generic shell loop.  Per-primitive
// screening skips exponentials that vanish on all rows of the item; the terms are summed in the
// same order as the generic loop, so the values are identical.
enum { SHAPE_GENERIC = 0, SHAPE_S3S1P1 = 1, SHAPE_S8S8S1P3P1D1 = 2 };

template <int NP, bool FAST>
__device__ __forceinline__ void exps2(const float2* pa, float q0, float q1, float qmin, float (&e0)[NP],
                                      float (&e1)[NP], float (&c)[NP]) {
  float2 ac[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) ac[k] = pa[k];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    c[k] = ac[k].y;
    e0[k] = 0.f;
    e1[k] = 0.f;
    if (ac[k].x * qmin < kExpCut) {   // uniform over the warp: qmin is the item's minimum
      const float b = exp_scale<FAST>(ac[k].x);
      e0[k] = exp_cut<FAST>(b * q0);
      e1[k] = exp_cut<FAST>(b * q1);
    }
  }
}

template <int NP>
__device__ __forceinline__ void contract2(const float (&c)[NP], const float (&e0)[NP], const float (&e1)[NP],
                                          float& r0, float& r1) {
  r0 = 0.f;
  r1 = 0.f;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    r0 = fmaf(c[k], e0[k], r0);
    r1 = fmaf(c[k], e1[k], r1);
  }
}

// Real solid-harmonic values of one shell at the two rows, from the radial parts and the
// displacements: L = 0, 1, 2 fixed, or L = -1 for the runtime angular momentum `lrt` (<= 2).
__device__ __forceinline__ void sh_s_vals(float rad, float* v) { v[0] = (float)YS * rad; }
__device__ __forceinline__ void sh_p_vals(float rad, float x, float y, float z, float* v) {
  const float c = (float)YP * rad;
  v[0] = c * z; v[1] = c * x; v[2] = c * y;
}
__device__ __forceinline__ void sh_d_vals(float rad, float x, float y, float z, float* v) {
  const float c = (float)YD1 * rad;
  v[0] = (float)YD0 * rad * (2.f * z * z - x * x - y * y);
  v[1] = c * x * z; v[2] = c * z * y;
  v[3] = (float)YD2 * rad * (x * x - y * y); v[4] = c * x * y;
}

template <int L>
__device__ __forceinline__ void shell_vals(int lrt, float rad0, float rad1, float x0, float y0, float z0, float x1,
                                           float y1, float z1, float (&v0)[L < 0 ? 5 : 2 * L + 1],
                                           float (&v1)[L < 0 ? 5 : 2 * L + 1]) {
  if constexpr (L == 0) {
    sh_s_vals(rad0, v0);
    sh_s_vals(rad1, v1);
  } else if constexpr (L == 1) {
    sh_p_vals(rad0, x0, y0, z0, v0);
    sh_p_vals(rad1, x1, y1, z1, v1);
  } else if constexpr (L == 2) {
    sh_d_vals(rad0, x0, y0, z0, v0);
    sh_d_vals(rad1, x1, y1, z1, v1);
  } else if (lrt == 0) {
    sh_s_vals(rad0, v0);
    sh_s_vals(rad1, v1);
  } else if (lrt == 1) {
    sh_p_vals(rad0, x0, y0, z0, v0);
    sh_p_vals(rad1, x1, y1, z1, v1);
  } else {
    sh_d_vals(rad0, x0, y0, z0, v0);
    sh_d_vals(rad1, x1, y1, z1, v1);
  }
}

// Output of the fused kernel's production: rows r0 and r0 + 64 of the 128-byte swizzled K-major
// A tile (hi and lo pieces).  put() takes the nf (<= NF) values of one shell at functions j0..
template <int FMT>
struct SwizzledRowsOut {
  uint8_t* hi;
  uint8_t* lo;
  int r0;
  bool two;
  int tail0;
  // functions K0, K0 + 2, ... of a whole group (nf == NF) inside the swizzled chunks, from an even
  // column j0 + K0 on: pairs, the last one alone when the count is odd
  template <int K0, int NF>
  __device__ __forceinline__ void put_pairs(int j0, const float (&v0)[NF], const float (&v1)[NF]) const {
#pragma unroll
    for (int k = K0; k < NF; k += 2) {
      const uint32_t off = a_offset(r0, j0 + k, 1 << 30);
      if (k + 1 < NF) {
        store_pair16<FMT>(hi, lo, off, v0[k], v0[k + 1], two);
        store_pair16<FMT>(hi, lo, off + 8192u, v1[k], v1[k + 1], two);
      } else {
        store_split16<FMT>(hi, lo, off, v0[k], two);
        store_split16<FMT>(hi, lo, off + 8192u, v1[k], two);
      }
    }
  }
  template <int NF>
  __device__ __forceinline__ void put(int j0, int nf, const float (&v0)[NF], const float (&v1)[NF]) const {
    if (NF >= 5 && nf == NF && j0 + NF <= tail0) {
      // a whole atom's group inside the swizzled chunks (uniform over the warp): the pairing is
      // fixed by the parity of j0, with no per-function test
      if (j0 & 1) {
        const uint32_t off = a_offset(r0, j0, 1 << 30);
        store_split16<FMT>(hi, lo, off, v0[0], two);
        store_split16<FMT>(hi, lo, off + 8192u, v1[0], two);
        put_pairs<1>(j0, v0, v1);
      } else {
        put_pairs<0>(j0, v0, v1);
      }
      return;
    }
    bool skip = false;   // the function was stored with its predecessor
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      if (k >= nf) break;
      if (skip) {
        skip = false;
        continue;
      }
      const int j = j0 + k;
      const uint32_t off = a_offset(r0, j, tail0);
      const uint32_t off1 = off + a_row64(j, tail0);   // row r0 + 64
      // two consecutive functions in the same 16-byte unit: one 4-byte store per piece
      if (k + 1 < nf && (j & 1) == 0) {
        store_pair16<FMT>(hi, lo, off, v0[k], v0[k + 1], two);
        store_pair16<FMT>(hi, lo, off1, v1[k], v1[k + 1], two);
        skip = true;
      } else {
        store_split16<FMT>(hi, lo, off, v0[k], two);
        store_split16<FMT>(hi, lo, off1, v1[k], two);
      }
    }
  }
};

// Output of the staging kernel's production: FP32 rows r0 and r0 + 64 of a shared-memory window
// of STAGE_W columns starting at function c0 (functions outside the window are dropped; rows
// without a sample point get zeros).
constexpr int STAGE_W = 128;        // columns of one staging window
constexpr int STAGE_LD = STAGE_W + 1;  // row stride (odd: lanes on consecutive rows hit distinct banks)

struct WindowRowsOut {
  float* b0;   // row r0 of the window buffer
  float* b1;   // row r0 + 64
  int c0;
  bool ok0, ok1;
  template <int NF>
  __device__ __forceinline__ void put(int j0, int nf, const float (&v0)[NF], const float (&v1)[NF]) const {
#pragma unroll
    for (int k = 0; k < NF; ++k) {
      if (k >= nf) break;
      const int j = j0 + k - c0;
      if ((unsigned)j < (unsigned)STAGE_W) {
        b0[j] = ok0 ? v0[k] : 0.f;
        b1[j] = ok1 ? v1[k] : 0.f;
      }
    }
  }
};

// Values of every function of atom `a` at rows r0 and r0 + 64 of a 128-row tile (FP64 positions
// in `pos`, 1e30 for rows without a point), handed to `out` shell by shell.  Tables as staged
// by the kernels: shell records, (alpha, scaled coefficient) pairs in descending alpha order,
// per-atom words (first shell | layout << 24), float nuclear coordinates.  The whole warp works
// on the atom (lanes r0 = half * 32 + lane); FAST selects the exponentials of exp_cut.  Returns
// the atom's last function.
template <bool FAST, class Out>
__device__ __forceinline__ int atom_rows(const int4* sh_s, const float2* pr_s, const int* ash_s, const float* crd_s,
                                         int a, const double (*pos)[3], int r0, const Out& out) {
  const int as0 = ash_s[a];
  const int s0 = as0 & 0xffffff, s1 = ash_s[a + 1] & 0xffffff, shape = as0 >> 24;
  const int r1 = r0 + 64;
  const double ax = crd_s[3 * a], ay = crd_s[3 * a + 1], az = crd_s[3 * a + 2];
  const bool ok0 = pos[r0][0] < 1e29, ok1 = pos[r1][0] < 1e29;
  // FP64 displacement from the nucleus, rounded once (accuracy of steep exponents)
  const float x0 = (float)(pos[r0][0] - ax), y0 = (float)(pos[r0][1] - ay), z0 = (float)(pos[r0][2] - az);
  const float x1 = (float)(pos[r1][0] - ax), y1 = (float)(pos[r1][1] - ay), z1 = (float)(pos[r1][2] - az);
  const float q0 = x0 * x0 + y0 * y0 + z0 * z0, q1 = x1 * x1 + y1 * y1 + z1 * z1;
  // primitives with alpha * min_rows(r^2) >= the cut-off are zero at every row of the item:
  // with exponents in descending order they are the leading ones of a shell and are skipped
  // (the remaining terms are summed in the same order, so the result is unchanged)
  float qmin = fminf(q0, q1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) qmin = fminf(qmin, __shfl_xor_sync(0xffffffffu, qmin, o));
  float nx0 = 0.f, nx1 = 0.f;   // radial parts of the next shell when it shares the exponents
  int flast = 0;
  if (shape != SHAPE_GENERIC) {
    const int4 rec0 = sh_s[s0];
    const float2* pa = pr_s + rec0.x;
    const int f0 = rec0.y;
    float rA0, rA1;
    float s_0[1], s_1[1], p_0[3], p_1[3];
    if (shape == SHAPE_S3S1P1) {
      {
        float e0[3], e1[3], c[3];
        exps2<3, FAST>(pa, q0, q1, qmin, e0, e1, c);
        contract2<3>(c, e0, e1, rA0, rA1);
      }
      float rB0, rB1, rC0, rC1;
      {
        float e0[1], e1[1], c[1];
        exps2<1, FAST>(pa + 3, q0, q1, qmin, e0, e1, c);
        contract2<1>(c, e0, e1, rB0, rB1);
        exps2<1, FAST>(pa + 4, q0, q1, qmin, e0, e1, c);
        contract2<1>(c, e0, e1, rC0, rC1);
      }
      if (!ok0) rA0 = rB0 = rC0 = 0.f;
      if (!ok1) rA1 = rB1 = rC1 = 0.f;
      // the atom's five functions stored as one group (pairs across the shells' boundaries)
      float g0[5], g1[5];
      shell_vals<0>(0, rA0, rA1, x0, y0, z0, x1, y1, z1, s_0, s_1);
      g0[0] = s_0[0];
      g1[0] = s_1[0];
      shell_vals<0>(0, rB0, rB1, x0, y0, z0, x1, y1, z1, s_0, s_1);
      g0[1] = s_0[0];
      g1[1] = s_1[0];
      shell_vals<1>(1, rC0, rC1, x0, y0, z0, x1, y1, z1, p_0, p_1);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        g0[2 + k] = p_0[k];
        g1[2 + k] = p_1[k];
      }
      out.put(f0, 5, g0, g1);
      flast = f0 + 4;
    } else {
      float rB0, rB1;
      {
        float e0[8], e1[8], c[8], d[8];
        exps2<8, FAST>(pa, q0, q1, qmin, e0, e1, c);
        contract2<8>(c, e0, e1, rA0, rA1);
#pragma unroll
        for (int k = 0; k < 8; ++k) d[k] = pa[8 + k].y;   // second s shell: same exponents
        contract2<8>(d, e0, e1, rB0, rB1);
      }
      float rC0, rC1, rD0, rD1, rE0, rE1, rF0, rF1;
      {
        float e0[1], e1[1], c[1];
        exps2<1, FAST>(pa + 16, q0, q1, qmin, e0, e1, c);
        contract2<1>(c, e0, e1, rC0, rC1);
      }
      {
        float e0[3], e1[3], c[3];
        exps2<3, FAST>(pa + 17, q0, q1, qmin, e0, e1, c);
        contract2<3>(c, e0, e1, rD0, rD1);
      }
      {
        float e0[1], e1[1], c[1];
        exps2<1, FAST>(pa + 20, q0, q1, qmin, e0, e1, c);
        contract2<1>(c, e0, e1, rE0, rE1);
        exps2<1, FAST>(pa + 21, q0, q1, qmin, e0, e1, c);
        contract2<1>(c, e0, e1, rF0, rF1);
      }
      if (!ok0) rA0 = rB0 = rC0 = rD0 = rE0 = rF0 = 0.f;
      if (!ok1) rA1 = rB1 = rC1 = rD1 = rE1 = rF1 = 0.f;
      // the atom's fourteen functions stored as one group (pairs across the shells' boundaries)
      float g0[14], g1[14];
      shell_vals<0>(0, rA0, rA1, x0, y0, z0, x1, y1, z1, s_0, s_1);
      g0[0] = s_0[0];
      g1[0] = s_1[0];
      shell_vals<0>(0, rB0, rB1, x0, y0, z0, x1, y1, z1, s_0, s_1);
      g0[1] = s_0[0];
      g1[1] = s_1[0];
      shell_vals<0>(0, rC0, rC1, x0, y0, z0, x1, y1, z1, s_0, s_1);
      g0[2] = s_0[0];
      g1[2] = s_1[0];
      shell_vals<1>(1, rD0, rD1, x0, y0, z0, x1, y1, z1, p_0, p_1);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        g0[3 + k] = p_0[k];
        g1[3 + k] = p_1[k];
      }
      shell_vals<1>(1, rE0, rE1, x0, y0, z0, x1, y1, z1, p_0, p_1);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        g0[6 + k] = p_0[k];
        g1[6 + k] = p_1[k];
      }
      float d_0[5], d_1[5];
      shell_vals<2>(2, rF0, rF1, x0, y0, z0, x1, y1, z1, d_0, d_1);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        g0[9 + k] = d_0[k];
        g1[9 + k] = d_1[k];
      }
      out.put(f0, 14, g0, g1);
      flast = f0 + 13;
    }
  }
  for (int sidx = shape != SHAPE_GENERIC ? s1 : s0; sidx < s1; ++sidx) {
    const int4 rec = sh_s[sidx];   // prim, func, L | nprim << 8 | same_exp << 16 | next_same << 24, next prim
    const int L = rec.z & 0xff, np_ = (rec.z >> 8) & 0xff, f0 = rec.y;
    float rad0, rad1;
    if (rec.z & 0x10000) {
      rad0 = nx0;
      rad1 = nx1;
    } else {
      int sk = 0;
      while (sk < np_ && pr_s[rec.x + sk].x * qmin >= kExpCut) ++sk;
      const float2* pa = pr_s + rec.x + sk;
      const float2* pn = (rec.z >> 24) ? pr_s + rec.w + sk : nullptr;
      switch (np_ - sk) {
        case 0:
          rad0 = rad1 = 0.f;
          nx0 = nx1 = 0.f;
          break;
        case 1: radial_np<1, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 2: radial_np<2, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 3: radial_np<3, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 4: radial_np<4, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 5: radial_np<5, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 6: radial_np<6, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 7: radial_np<7, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        case 8: radial_np<8, FAST>(pa, pn, q0, q1, rad0, rad1, nx0, nx1); break;
        default:
          rad0 = 0.f;
          rad1 = 0.f;
          for (int k = 0; k < np_ - sk; ++k) {
            const float2 ac = pa[k];
            const float b = exp_scale<FAST>(ac.x);
            rad0 = fmaf(ac.y, exp_cut<FAST>(b * q0), rad0);
            rad1 = fmaf(ac.y, exp_cut<FAST>(b * q1), rad1);
          }
      }
    }
    if (!ok0) rad0 = 0.f;
    if (!ok1) rad1 = 0.f;
    float v0[5], v1[5];
    shell_vals<-1>(L, rad0, rad1, x0, y0, z0, x1, y1, z1, v0, v1);
    const int nf = 2 * L + 1;
    flast = f0 + nf - 1;
    out.put(f0, nf, v0, v1);
  }
  return flast;
}

// ---------------------------------------------------------------------------------------
// Staged path, stage 1: Phi' of 128-row tiles into operand pieces in HBM.
//
// Persistent CTAs take whole tiles; a tile is produced in windows of STAGE_W columns.  Per
// window the warps take (atom, row half) items of the atoms with functions in the window from
// a shared counter and write FP32 values into the window buffer (atom_rows, the producer of
// the fused kernel); then the CTA converts the window to hi = fmt(Phi'), lo = fmt(Phi' - hi)
// and writes it with coalesced stores to the row-major [row][kpad] pieces.  Padding columns
// (>= norbs) and rows without a point are zero.
// ---------------------------------------------------------------------------------------
struct StageParams {
  PointMap pm;
  int64_t tile0;           // first tile of this chunk
  int ntiles;              // tiles of this chunk
  int kpad, norbs, nwin;   // nwin = ceil(kpad / STAGE_W)
  const int4* tab;         // molecule tables (ensure_mol_tables)
  const float* coords;     // nuclear coordinates, 3 per atom
  int ncoords;             // 3 * natoms
  const int2* win;         // atoms [x, y) with functions in each window
  int tab_words;           // 16-byte words of shell records, primitive pairs and atom words
  int off_prim, off_ashell, off_coords;   // byte offsets of the tables
  int tab_bytes;           // shared-memory bytes of the staged tables (0: read from global memory)
  void* out_hi;
  void* out_lo;
  int two;
};

constexpr int STAGE_THREADS = 256;

template <int FMT>
__device__ __forceinline__ void split_store2(float x0, float x1, void* hi, void* lo, int64_t idx, bool two) {
  if constexpr (FMT == FMT_TF32) {
    const uint32_t h0 = tf32_round_bits(x0), h1 = tf32_round_bits(x1);
    reinterpret_cast<uint2*>(reinterpret_cast<uint32_t*>(hi) + idx)[0] = make_uint2(h0, h1);
    if (two)
      reinterpret_cast<uint2*>(reinterpret_cast<uint32_t*>(lo) + idx)[0] =
          make_uint2(tf32_round_bits(x0 - bits_f32(h0)), tf32_round_bits(x1 - bits_f32(h1)));
  } else if constexpr (FMT == FMT_F16) {
    const __half2 h = __floats2half2_rn(x0, x1);
    reinterpret_cast<__half2*>(reinterpret_cast<__half*>(hi) + idx)[0] = h;
    if (two) {
      const float2 hf = __half22float2(h);
      reinterpret_cast<__half2*>(reinterpret_cast<__half*>(lo) + idx)[0] = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    }
  } else {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(hi) + idx)[0] = h;
    if (two) {
      const float2 hf = __bfloat1622float2(h);
      reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(lo) + idx)[0] =
          __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
    }
  }
}

template <int FMT>
__global__ void __launch_bounds__(STAGE_THREADS, 2) basis_window_kernel(const StageParams p) {
  extern __shared__ __align__(16) uint8_t smem_dyn[];
  __shared__ double pos[128][3];
  __shared__ int item_ctr;
  const int lane = threadIdx.x & 31;
  const bool two = p.two != 0;
  float* buf = reinterpret_cast<float*>(smem_dyn + p.tab_bytes);   // [128][STAGE_LD]
  const int4* sh_s;
  const float2* pr_s;
  const int* ash_s;
  const float* crd_s;
  if (p.tab_bytes > 0) {
    for (int i = threadIdx.x; i < p.tab_words; i += blockDim.x) reinterpret_cast<int4*>(smem_dyn)[i] = __ldg(p.tab + i);
    for (int i = threadIdx.x; i < p.ncoords; i += blockDim.x)
      reinterpret_cast<float*>(smem_dyn + p.off_coords)[i] = __ldg(p.coords + i);
    sh_s = reinterpret_cast<const int4*>(smem_dyn);
    pr_s = reinterpret_cast<const float2*>(smem_dyn + p.off_prim);
    ash_s = reinterpret_cast<const int*>(smem_dyn + p.off_ashell);
    crd_s = reinterpret_cast<const float*>(smem_dyn + p.off_coords);
  } else {
    const uint8_t* g = reinterpret_cast<const uint8_t*>(p.tab);
    sh_s = p.tab;
    pr_s = reinterpret_cast<const float2*>(g + p.off_prim);
    ash_s = reinterpret_cast<const int*>(g + p.off_ashell);
    crd_s = p.coords;
  }
  for (int t = blockIdx.x; t < p.ntiles; t += gridDim.x) {
    // positions: every reader of the previous tile's positions passed the barrier that ends
    // the last window's production
    if (threadIdx.x < 128) {
      double x, y, z;
      int64_t vox;
      if (!tile_point<double>(p.pm, p.tile0 + t, threadIdx.x, x, y, z, vox)) x = y = z = 1e30;
      pos[threadIdx.x][0] = x;
      pos[threadIdx.x][1] = y;
      pos[threadIdx.x][2] = z;
    }
    for (int w = 0; w < p.nwin; ++w) {
      if (threadIdx.x == 0) item_ctr = 0;
      __syncthreads();   // positions and tables ready, window buffer free, counter reset
      const int2 ar = __ldg(p.win + w);
      const int c0 = w * STAGE_W;
      const int nitems = 2 * (ar.y - ar.x);
      for (;;) {
        int itm = 0;
        if (lane == 0) itm = atomicAdd(&item_ctr, 1);
        itm = __shfl_sync(0xffffffffu, itm, 0);
        if (itm >= nitems) break;
        const int a = ar.x + (itm >> 1);
        if ((ash_s[a + 1] & 0xffffff) <= (ash_s[a] & 0xffffff)) continue;
        const int r0 = (itm & 1) * 32 + lane;
        atom_rows<false>(sh_s, pr_s, ash_s, crd_s, a, pos, r0,
                  WindowRowsOut{buf + r0 * STAGE_LD, buf + (r0 + 64) * STAGE_LD, c0, pos[r0][0] < 1e29,
                                pos[r0 + 64][0] < 1e29});
      }
      __syncthreads();
      // write-out: a warp covers 64 consecutive columns of a row (two per lane)
      const int ncol = min(STAGE_W, p.kpad - c0);   // 128 or 64
      const int nval = p.norbs - c0;                // columns beyond hold padding zeros
      const int lp = ncol == STAGE_W ? 6 : 5;       // log2(column pairs per row)
      const int64_t rowbase = (int64_t)t * 128;
      for (int i = threadIdx.x; i < (128 << lp); i += blockDim.x) {
        const int r = i >> lp, c = (i & ((1 << lp) - 1)) * 2;
        const float v0 = c < nval ? buf[r * STAGE_LD + c] : 0.f;
        const float v1 = c + 1 < nval ? buf[r * STAGE_LD + c + 1] : 0.f;
        split_store2<FMT>(v0, v1, p.out_hi, p.out_lo, (rowbase + r) * p.kpad + c0 + c, two);
      }
    }
  }
}

constexpr int FUSED_NCW = 16;                 // compute warps (Phi production and epilogue)
constexpr int FUSED_NCT = FUSED_NCW * 32;
constexpr int FUSED_THREADS = 64 + FUSED_NCT;  // + U-producer warp + MMA warp

// The single-thread roles of the fused kernel (warp 0 lane 0 and warp 1 lane 0).

// U producer: streams the K-step blocks of U into the stage ring (one bulk copy per stage and
// piece, already in the 32-byte swizzled layout; stage slots and r0 are multiples of 256 bytes
// and 16 rows).  On an abort it waits (bounded) for its copies in flight before returning.
template <bool MULTI>
__device__ __forceinline__ void fused_produce_u(const FusedParams* pp, uint8_t* stages, uint64_t* full_bar,
                                             uint64_t* empty_bar, volatile int* abort_flag) {
  const FusedParams& p = *pp;
  const bool two = p.nsplit == 2;
  uint32_t it = 0, issued = 0, par = 0;   // bit s: stage s has a copy in flight / its phase parity
  bool ok = true;
  for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
    int m;
    const FusedMol& M = fused_mol<MULTI>(p, t, m);
    // the molecule's values in registers for the tile: read through a reference, they would be
    // reloaded after every barrier operation (each an asm statement that clobbers memory)
    const int ksteps = M.ksteps, u_rows = M.u_rows;
    const uint32_t bytes = (uint32_t)M.nb * 32u;
    const uint8_t* const u_hi = M.u_hi;
    const uint8_t* const u_lo = M.u_lo;
    for (int ks = 0; ks < ksteps; ++ks, ++it) {
      const int s = it % p.stages;
      const uint32_t ph = (it / p.stages) & 1u;
      if (!mbar_wait(&empty_bar[s], ph ^ 1u, abort_flag, p.wait_ns)) {
        ok = false;
        break;
      }
      const size_t src = (size_t)ks * u_rows * 32u;
      uint8_t* st = stages + (size_t)s * p.stage_bytes;
      mbar_expect_tx(&full_bar[s], bytes * (uint32_t)p.nsplit);
      bulk_load(st, u_hi + src, bytes, &full_bar[s]);
      if (two) bulk_load(st + p.b_slot, u_lo + src, bytes, &full_bar[s]);
      issued |= 1u << s;
      par = (par & ~(1u << s)) | (ph << s);
    }
  }
  if (!ok)
    for (int s = 0; s < p.stages; ++s)
      if ((issued >> s) & 1u) mbar_wait_drain(&full_bar[s], (par >> s) & 1u, 100000000ull);
}

// MMA issuer: per tile, per K-step (after its column chunk of A is complete and its U stage has
// landed) the split products T' += A_hi U_hi + A_hi U_lo + A_lo U_hi into TMEM; frees the stage
// with a commit, and signals t_full after the tile's last K-step.
template <bool MULTI>
__device__ __forceinline__ void fused_issue_mma(const FusedParams* pp, uint32_t abase, uint32_t lbase, uint8_t* stages,
                                             uint32_t tmem, uint64_t* full_bar, uint64_t* empty_bar,
                                             uint64_t* chunk_bar, uint64_t* t_full, uint64_t* drain_bar,
                                             volatile int* abort_flag) {
  const FusedParams& p = *pp;
  const bool two = p.nsplit == 2;
  uint32_t it = 0, cpar = 0;   // bit c: phase parity of chunk barrier c
  bool ok = true;
  for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
    int m;
    const FusedMol& M = fused_mol<MULTI>(p, t, m);
    // the molecule's values in registers for the tile (see the producer)
    const int ksteps = M.ksteps, nb = M.nb, tail0 = M.tail0;
    uint32_t need = 0;
#pragma unroll
    for (int c = 0; c < MAX_FUSED_CHUNKS; ++c)
      if (M.chunk_need[c] > 0) need |= 1u << c;
    for (int ks = 0; ks < ksteps; ++ks, ++it) {
      // columns 64c .. 64c+63 of A are complete once every item writing them arrived
      const int c = ks >> 2;
      if ((ks & 3) == 0 && ((need >> c) & 1u)) {
        if (!mbar_wait(&chunk_bar[c], (cpar >> c) & 1u, abort_flag, p.wait_ns)) {
          ok = false;
          break;
        }
        cpar ^= 1u << c;
        tc_fence_after();
      }
      const int s = it % p.stages;
      const uint32_t ph = (it / p.stages) & 1u;
      if (!mbar_wait(&full_bar[s], ph, abort_flag, p.wait_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int j0 = ks * 16;
      // A K-step: 32 bytes inside a 128-byte swizzled chunk, or one 32-byte swizzled tail block
      uint64_t ahi, alo;
      if (j0 < tail0) {
        const uint32_t aoff = (uint32_t)((j0 >> 6) * 16384 + ((j0 & 63) >> 4) * 32);
        ahi = sw128_kmajor_desc(abase + aoff);
        alo = sw128_kmajor_desc(lbase + aoff);
      } else {
        const uint32_t aoff = (uint32_t)(tail0 * 256 + ((j0 - tail0) >> 4) * 4096);
        ahi = sw32_kmajor_desc(abase + aoff);
        alo = sw32_kmajor_desc(lbase + aoff);
      }
      const uint32_t bst = smem_u32(stages + (size_t)s * p.stage_bytes);
      for (int c0 = 0; c0 < nb; c0 += 256) {
        const int n = min(256, nb - c0);
        const uint32_t idesc = make_idesc(p.fmt, 128, (uint32_t)n);
        const uint32_t boff = (uint32_t)c0 * 32u;
        const uint32_t d = tmem + (uint32_t)c0;
        mma_f16(d, ahi, sw32_kmajor_desc(bst + boff), idesc, ks > 0 ? 1u : 0u);
        if (two) {
          mma_f16(d, ahi, sw32_kmajor_desc(bst + p.b_slot + boff), idesc, 1u);
          mma_f16(d, alo, sw32_kmajor_desc(bst + boff), idesc, 1u);
        }
      }
      tc_commit(&empty_bar[s]);
    }
    if (ok) tc_commit(t_full);
  }
  tc_commit(drain_bar);
  mbar_wait_drain(drain_bar, 0u, 500000000ull);
}

// Factored path: a stage is one column chunk of the factor, its K-steps each [hi rows | lo rows]
// (nb rows of 32 bytes apiece), one contiguous copy from HBM (ensure_factor's layout).
__device__ __forceinline__ uint32_t fact_chunk_ksteps(int c, int ksteps) { return (uint32_t)min(4, ksteps - 4 * c); }

template <bool MULTI>
__device__ __forceinline__ void fact_produce(const FusedParams& p, uint8_t* stages, uint64_t* full_bar,
                                             uint64_t* empty_bar, volatile int* abort_flag) {
  int s = 0;
  uint32_t ph = 0, issued = 0, par = 0;
  bool ok = true;
  for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
    int m;
    const FusedMol& M = fused_mol<MULTI>(p, t, m);
    const int ksteps = M.ksteps, nchunks = M.nchunks;
    const uint32_t kbytes = (uint32_t)p.nsplit * (uint32_t)M.nb * 32u;   // one K-step of the factor
    const uint8_t* const src0 = M.u_hi;
    for (int c = 0; c < nchunks; ++c) {
      if (!mbar_wait(&empty_bar[s], ph ^ 1u, abort_flag, p.wait_ns)) {
        ok = false;
        break;
      }
      const uint32_t bytes = fact_chunk_ksteps(c, ksteps) * kbytes;
      mbar_expect_tx(&full_bar[s], bytes);
      bulk_load(stages + (size_t)s * p.stage_bytes, src0 + (size_t)c * 4 * kbytes, bytes, &full_bar[s]);
      issued |= 1u << s;
      par = (par & ~(1u << s)) | (ph << s);
      if (++s == p.stages) {
        s = 0;
        ph ^= 1u;
      }
    }
  }
  if (!ok)
    for (int q = 0; q < p.stages; ++q)
      if ((issued >> q) & 1u) mbar_wait_drain(&full_bar[q], (par >> q) & 1u, 100000000ull);
}

// Per chunk: wait for its columns of A and its stage, then per K-step one MMA of N = 2 nb
// [A_hi B_hi | A_hi B_lo] into the chunk's accumulator and, with two pieces, [A_lo B_hi | A_lo B_lo]
// into the last (fact_nacc); the stage is freed by one commit per chunk.
template <bool MULTI>
__device__ __forceinline__ void fact_issue(const FusedParams& p, uint32_t abase, uint32_t lbase, uint8_t* stages,
                                           uint32_t tmem, uint64_t* full_bar, uint64_t* empty_bar, uint64_t* chunk_bar,
                                           uint64_t* t_full, uint64_t* drain_bar, volatile int* abort_flag) {
  const bool two = p.nsplit == 2;
  int s = 0, cur_m = -1;
  uint32_t ph = 0, cpar = 0;
  int ksteps = 0, nb = 0, tail0 = 0, nchunks = 0;
  uint32_t idesc = 0, kbytes = 0, dsmall = 0, firstmask = 0, need = 0;
  uint32_t dmain[MAX_FUSED_CHUNKS];
  bool ok = true;
  for (int64_t t = blockIdx.x; t < p.ntiles && ok; t += gridDim.x) {
    int m;
    const FusedMol& M = fused_mol<MULTI>(p, t, m);
    if (m != cur_m) {   // the molecule's shape of the contraction (once for a single molecule)
      ksteps = M.ksteps;
      nb = M.nb;
      tail0 = M.tail0;
      nchunks = M.nchunks;
      const int nfull = two ? 2 * nb : nb;
      const int na = fact_nacc(nchunks, nb, two);
      idesc = make_idesc(p.fmt, 128, (uint32_t)nfull);
      kbytes = (uint32_t)nfull * 32u;
      dsmall = tmem + (uint32_t)(na * nfull);
      firstmask = need = 0;
#pragma unroll
      for (int c = 0; c < MAX_FUSED_CHUNKS; ++c) {
        const int a = c < nchunks ? c * na / nchunks : 0;
        dmain[c] = tmem + (uint32_t)(a * nfull);
        if (c < nchunks && (c == 0 || (c - 1) * na / nchunks != a)) firstmask |= 1u << c;
        if (M.chunk_need[c] > 0) need |= 1u << c;
      }
      cur_m = m;
    }
#pragma unroll 1
    for (int c = 0; c < nchunks; ++c) {
      if ((need >> c) & 1u) {
        if (!mbar_wait(&chunk_bar[c], (cpar >> c) & 1u, abort_flag, p.wait_ns)) {
          ok = false;
          break;
        }
        cpar ^= 1u << c;
      }
      if (!mbar_wait(&full_bar[s], ph, abort_flag, p.wait_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t bst = smem_u32(stages + (size_t)s * p.stage_bytes);
      const uint32_t kc = fact_chunk_ksteps(c, ksteps);
      const uint32_t dm = dmain[c];
      const bool first = (firstmask >> c) & 1u;
      for (uint32_t kk = 0; kk < kc; ++kk) {
        const int j0 = (4 * c + (int)kk) * 16;
        uint64_t ahi, alo;
        if (j0 < tail0) {
          const uint32_t aoff = (uint32_t)(c * 16384 + kk * 32);
          ahi = sw128_kmajor_desc(abase + aoff);
          alo = sw128_kmajor_desc(lbase + aoff);
        } else {
          const uint32_t aoff = (uint32_t)(tail0 * 256 + ((j0 - tail0) >> 4) * 4096);
          ahi = sw32_kmajor_desc(abase + aoff);
          alo = sw32_kmajor_desc(lbase + aoff);
        }
        const uint64_t bd = sw32_kmajor_desc(bst + kk * kbytes);
        mma_f16(dm, ahi, bd, idesc, (first && kk == 0) ? 0u : 1u);
        if (two) mma_f16(dsmall, alo, bd, idesc, (c == 0 && kk == 0) ? 0u : 1u);
      }
      tc_commit(&empty_bar[s]);
      if (++s == p.stages) {
        s = 0;
        ph ^= 1u;
      }
    }
    if (ok) tc_commit(t_full);
  }
  tc_commit(drain_bar);
  mbar_wait_drain(drain_bar, 0u, 500000000ull);
}

template <int FMT, bool MULTI, bool FACT>
__global__ void __launch_bounds__(FUSED_THREADS, 1)
    density_fused_kernel(const __grid_constant__ FusedParams p) {
  extern __shared__ uint8_t smem_dyn[];
  if (p.gate && *p.gate != p.gate_want) return;   // the other launch of the pair does the work
  __shared__ __align__(8) uint64_t full_bar[MAX_STAGES], empty_bar[MAX_STAGES];
  __shared__ __align__(8) uint64_t chunk_bar[MAX_FUSED_CHUNKS], t_full, drain_bar;
  __shared__ int item_ctr;
  __shared__ uint32_t tmem_slot;
  // tile positions (production) and the epilogue's row partials share their storage: every
  // reader of the one is past a barrier of all compute warps before the other is written
  __shared__ union {
    double pos[128][3];
    double rho_part[FUSED_NCW / 4][128];
  } ps;
  double(*pos)[3] = ps.pos;
  double(*rho_part)[128] = ps.rho_part;
  // per-warp sums of the tile (written after the next tile's first epilogue barrier, read by
  // compute thread 0 before it reaches that barrier: no barrier needed after the read)
  __shared__ double red[FUSED_NCW];
  __shared__ volatile int abort_flag;

  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~uintptr_t(1023));
  uint8_t* A_hi = smem;
  uint8_t* A_lo = smem + p.a_bytes;
  uint8_t* stages = smem + p.nsplit * p.a_bytes;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool two = p.nsplit == 2;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    // a single molecule's barriers count its own production items; a batch's count CHUNK_COUNT,
    // the difference pre-arrived per tile
    for (int c = 0; c < MAX_FUSED_CHUNKS; ++c)
      mbar_init(&chunk_bar[c], MULTI ? CHUNK_COUNT : (uint32_t)max(1, p.one.chunk_need[c]));
    mbar_init(&t_full, 1);
    mbar_init(&drain_bar, 1);
    fence_mbar_init();
  }
  // zero A once: padding rows are rewritten with zeros by every tile, padding columns when a
  // CTA moves to another molecule
  for (uint32_t i = threadIdx.x; i < p.nsplit * p.a_bytes / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  // molecule tables in shared memory (loaded per molecule): the production loop reads them in
  // dependent chains
  uint8_t* tabs = stages + (size_t)p.stages * p.stage_bytes;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 1) {
    tmem_alloc(&tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      if (FACT) fact_produce<MULTI>(p, stages, full_bar, empty_bar, &abort_flag);
      else fused_produce_u<MULTI>(&p, stages, full_bar, empty_bar, &abort_flag);
    }
  } else if (warp == 1) {
    if (lane == 0 && FACT)
      fact_issue<MULTI>(p, smem_u32(A_hi), smem_u32(A_lo), stages, tmem, full_bar, empty_bar, chunk_bar, &t_full,
                        &drain_bar, &abort_flag);
    else if (lane == 0)
      fused_issue_mma<MULTI>(&p, smem_u32(A_hi), smem_u32(A_lo), stages, tmem, full_bar, empty_bar, chunk_bar, &t_full,
                      &drain_bar, &abort_flag);
  } else {
    const int ct = threadIdx.x - 64;           // compute thread 0 .. FUSED_NCT-1
    const int4* sh_s = reinterpret_cast<const int4*>(tabs);
    const int cw = ct >> 5;                    // compute warp 0 .. FUSED_NCW-1
    const int q = warp & 3;                    // TMEM lane quadrant of this warp
    const int hh = cw >> 2;                    // epilogue column-chunk class 0 .. FUSED_NCW/4-1
    const int row = q * 32 + lane;
    uint32_t tile_it = 0;
    int cur_m = -1;
    // table pointers, derived from the shared-memory base (a single molecule's never change)
    const float2* pr_s = reinterpret_cast<const float2*>(tabs + (MULTI ? 0 : p.one.off_prim));
    const int* ash_s = reinterpret_cast<const int*>(tabs + (MULTI ? 0 : p.one.off_ashell));
    const float* crd_s = reinterpret_cast<const float*>(tabs + (MULTI ? 0 : p.one.off_coords));
    for (int64_t t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++tile_it) {
      int m;
      const FusedMol& M = fused_mol<MULTI>(p, t, m);
      const int64_t lt = t - M.tile0;          // tile within the molecule
      const int natoms = M.natoms, n16 = M.n16, tail0 = M.tail0;   // (in registers, see the producer)
      if (m != cur_m) {
        // another molecule: its tables into shared memory and its padding columns of A cleared
        // (the previous tile's epilogue, the last reader of both, ended with a named barrier)
        for (int i = ct; i < M.tab_words; i += FUSED_NCT) reinterpret_cast<int4*>(tabs)[i] = __ldg(M.tab + i);
        for (int i = ct; i < 3 * M.natoms; i += FUSED_NCT)
          reinterpret_cast<float*>(tabs + M.off_coords)[i] = __ldg(M.coords + i);
        const int npadc = M.n16 - M.norbs;
        for (int i = ct; i < 128 * npadc; i += FUSED_NCT) {
          const uint32_t off = a_offset(i / npadc, M.norbs + i % npadc, M.tail0);
          *reinterpret_cast<uint16_t*>(A_hi + off) = 0;
          if (two) *reinterpret_cast<uint16_t*>(A_lo + off) = 0;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (MULTI) {
          pr_s = reinterpret_cast<const float2*>(tabs + M.off_prim);
          ash_s = reinterpret_cast<const int*>(tabs + M.off_ashell);
          crd_s = reinterpret_cast<const float*>(tabs + M.off_coords);
        }
        cur_m = m;
      }
      // ---- Phi' for the tile into A -------------------------------------------------------
      if (ct < 128) {
        double x, y, z;
        int64_t vox;
        if (!tile_point<double>(M.pm, lt, ct, x, y, z, vox)) x = y = z = 1e30;
        pos[ct][0] = x;
        pos[ct][1] = y;
        pos[ct][2] = z;
      }
      if (ct == 0) {
        item_ctr = 0;
        // the arrivals that this molecule's production does not make
        if (MULTI)
          for (int c = 0; c < M.nchunks; ++c)
            if (M.chunk_need[c] > 0) mbar_arrive_count(&chunk_bar[c], CHUNK_COUNT - (uint32_t)M.chunk_need[c]);
      }
      named_barrier(1, FUSED_NCT);
      // work item = (atom, half of the rows), taken in atom order from a shared counter so that
      // column chunks complete roughly in order and the warps stay balanced; two rows per thread
      // (lane and lane + 64 of its half) for independent exponential chains
      for (;;) {
        int itm = 0;
        if (lane == 0) itm = atomicAdd(&item_ctr, 1);
        itm = __shfl_sync(0xffffffffu, itm, 0);
        if (itm >= 2 * natoms) break;
        const int a = itm >> 1;
        const int s0 = ash_s[a] & 0xffffff;
        if ((ash_s[a + 1] & 0xffffff) <= s0) continue;
        const int flast = atom_rows<FACT>(sh_s, pr_s, ash_s, crd_s, a, pos, (itm & 1) * 32 + lane,
                                    SwizzledRowsOut<FMT>{A_hi, A_lo, (itm & 1) * 32 + lane, two, tail0});
        // publish: generic-proxy writes of A become visible to the tensor core, then one arrival
        // per column chunk this atom wrote
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          const int cfirst = sh_s[s0].y >> 6, clast = flast >> 6;
          for (int c = cfirst; c <= clast; ++c) mbar_arrive(&chunk_bar[c]);
        }
      }
      // ---- epilogue -----------------------------------------------------------------------
      // the compute warps leave together: one of them giving up while the others go on would
      // leave those waiting at the next named barrier
      const bool got = mbar_wait(&t_full, tile_it & 1u, &abort_flag, p.wait_ns);
      if (barrier_any(1, FUSED_NCT, !got)) break;
      tc_fence_after();
      double acc[2] = {0.0, 0.0};
      const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
      if (FACT) {
        // T = the accumulators' sum (FP32, rounded), rho = sum_k (2^-h_k T_ik)^2 over this warp's
        // column chunks; M.gsc holds the column scales (layout of ensure_factor)
        // (each accumulator: nb columns of A_x B_hi, then with two pieces nb of A_x B_lo)
        const int nb = M.nb, nfull = two ? 2 * nb : nb;
        const int ngrp = (fact_nacc(M.nchunks, nb, two) + (two ? 1 : 0)) * (two ? 2 : 1);
        for (int c = hh; c * 16 < nb; c += FUSED_NCW / 4) {
          float tsum[16];
#pragma unroll
          for (int k = 0; k < 16; ++k) tsum[k] = 0.f;
          for (int gi = 0; gi < ngrp; gi += 2) {   // column group gi: accumulator gi / 2, half gi % 2
            uint32_t t0[16], t1[16];
            const uint32_t c0 = (uint32_t)((two ? (gi >> 1) * nfull + (gi & 1) * nb : gi * nb) + c * 16);
            const uint32_t c1 = (uint32_t)((two ? ((gi + 1) >> 1) * nfull + ((gi + 1) & 1) * nb : (gi + 1) * nb) + c * 16);
            tmem_ld16_issue(trow + c0, t0);
            if (gi + 1 < ngrp) tmem_ld16_issue(trow + c1, t1);
            tmem_ld16_wait(t0);
            if (gi + 1 < ngrp) {
              tmem_ld16_wait(t1);
#pragma unroll
              for (int k = 0; k < 16; ++k) tsum[k] += __uint_as_float(t0[k]) + __uint_as_float(t1[k]);
            } else {
#pragma unroll
              for (int k = 0; k < 16; ++k) tsum[k] += __uint_as_float(t0[k]);
            }
          }
          // (2^-h_k T_k)^2 with the FP32 scales after the FP64 ones: eight squares per FP32
          // partial, the partials summed in FP64, as in the unfactored epilogue
          const float4* hs = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(M.gsc + 2 * nb) + c * 16);
          float a32[2] = {0.f, 0.f};
#pragma unroll
          for (int k4 = 0; k4 < 4; ++k4) {
            const float4 h4 = __ldg(hs + k4);
            const float hk[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float u = tsum[4 * k4 + e] * hk[e];
              a32[e & 1] = fmaf(u, u, a32[e & 1]);
            }
          }
          acc[0] += (double)a32[0];
          acc[1] += (double)a32[1];
        }
      } else {
        for (int c = hh; c * 16 < n16; c += FUSED_NCW / 4) {
          const int col = c * 16;
          // the TMEM load of T' is in flight while the row's Phi' units are read from shared memory
          uint32_t tv[16];
          tmem_ld16_issue(trow + (uint32_t)col, tv);
          float ph[16];
          // the row's two 16-byte units of columns col .. col + 15 (layout of a_offset)
          uint32_t rbase, uo[2];
          if (col < tail0) {
            const int u0 = (col & 63) >> 3;
            rbase = (uint32_t)((col >> 6) * 16384 + (row >> 3) * 1024 + (row & 7) * 128);
            uo[0] = (uint32_t)((u0 ^ (row & 7)) * 16);
            uo[1] = (uint32_t)(((u0 + 1) ^ (row & 7)) * 16);
          } else {
            rbase = (uint32_t)(tail0 * 256 + ((col - tail0) >> 4) * 4096 + row * 32);
            uo[0] = (uint32_t)(((row >> 2) & 1) << 4);
            uo[1] = 16u - uo[0];
          }
          const uint8_t* rb = A_hi + rbase;
#pragma unroll
          for (int u = 0; u < 2; ++u) unpack8<FMT>(*reinterpret_cast<const uint4*>(rb + uo[u]), ph + 8 * u);
          if (two) {
            const uint8_t* rl = A_lo + rbase;
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              float lo8[8];
              unpack8<FMT>(*reinterpret_cast<const uint4*>(rl + uo[u]), lo8);
#pragma unroll
              for (int e = 0; e < 8; ++e) ph[8 * u + e] += lo8[e];
            }
          }
          tmem_ld16_wait(tv);
          // eight products per FP32 partial, partials summed in FP64 (the FP32 partials add
          // ~3e-8 relative error; converting every product to FP64 ties up the conversion pipe)
          float a32[2] = {0.f, 0.f};
#pragma unroll
          for (int k = 0; k < 16; ++k) a32[k & 1] = fmaf(ph[k], __uint_as_float(tv[k]), a32[k & 1]);
          acc[0] += (double)a32[0];
          acc[1] += (double)a32[1];
        }
      }
      tc_fence_before();
      rho_part[hh][row] = acc[0] + acc[1];
      named_barrier(1, FUSED_NCT);
      double mysum = 0.0;
      if (ct < M.pm.vpt) {
        double r = 0.0;
        for (int sub = 0; sub < M.pm.s3; ++sub) {
          const int rr = ct * M.pm.s3 + sub;
#pragma unroll
          for (int h3 = 0; h3 < FUSED_NCW / 4; ++h3) r += rho_part[h3][rr];
        }
        int64_t vox, ix, iy, iz;
        if (tile_voxel(M.pm, lt, ct, vox, ix, iy, iz)) {
          const float qv = (float)(r * (FACT ? 1.0 : M.gsc[2]) * M.outscale);
          M.qube[vox] = qv;
          mysum = qv;
        }
      }
      for (int o = 16; o > 0; o >>= 1) mysum += __shfl_xor_sync(0xffffffffu, mysum, o);
      if (lane == 0) red[cw] = mysum;
      named_barrier(1, FUSED_NCT);
      if (ct == 0) {   // the other warps go on to the next tile meanwhile
        double tot = 0;
        for (int w = 0; w < FUSED_NCW; ++w) tot += red[w];
        M.partials[lt] = tot;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicExch(p.err, 1);
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Molecule tables of the producers (fused and staging kernels), in 16-byte words:
//   shell records {prim, func, L | nprim << 8 | same_exp << 16 | next_same << 24, next shell's
//   prim}; (alpha, coefficient x column scale) pairs, descending alpha within a shell; per-atom
//   words (first shell | layout << 24), natoms + 1 of them; then, per STAGE_W-column window of
//   the kpad columns, the atoms [first, end) with a function in the window (int2).
struct MolTabLayout {
  int off_prim, off_ashell;   // byte offsets
  int words;                  // words up to and including the atom words
  int off_win;                // word index of the window ranges
  int nwin, total_words;
};

static MolTabLayout mol_tab_layout(const qmt_mol* m, int K) {
  MolTabLayout l{};
  const int nsh = (int)m->shells.size(), npr = (int)m->alpha.size();
  l.off_prim = nsh * 16;
  l.off_ashell = (nsh + (npr + 1) / 2) * 16;
  l.words = l.off_ashell / 16 + (m->natoms + 1 + 3) / 4;
  l.off_win = l.words;
  l.nwin = (K + STAGE_W - 1) / STAGE_W;
  l.total_words = l.off_win + (l.nwin + 1) / 2;
  return l;
}

static qmt_status ensure_mol_tables(qmt_mol* m, const std::vector<float>& fs, int K, cudaStream_t s) {
  const MolTabLayout lay = mol_tab_layout(m, K);
  const size_t nsh = m->shells.size();
  std::vector<int4> tab(lay.total_words, make_int4(0, 0, 0, 0));
  for (size_t i = 0; i < nsh; ++i) {
    const Shell& a = m->shells[i];
    if (a.nprim > 255 || a.L > 255) return fail(QMT_BAD_ARG, "shell too large for the density tables");
    const bool nxt = i + 1 < nsh && m->shells[i + 1].same_exp;
    tab[i] = make_int4(a.prim, a.func, a.L | (a.nprim << 8) | (a.same_exp << 16) | ((int)nxt << 24),
                       nxt ? m->shells[i + 1].prim : 0);
  }
  // every function of a shell shares the shell's bound, hence its scale: fold it into the
  // contraction coefficients (exact, powers of two).  Primitives of a shell in descending
  // exponent order (the kernels skip the leading ones that vanish on a whole work item);
  // basis files normally list them that way already.
  float2* pt = reinterpret_cast<float2*>(tab.data() + nsh);
  for (const Shell& shl : m->shells) {
    for (int k = 0; k < shl.nprim; ++k)
      pt[shl.prim + k] = make_float2(m->alpha[shl.prim + k], m->coeff[shl.prim + k] * fs[shl.func]);
    std::stable_sort(pt + shl.prim, pt + shl.prim + shl.nprim,
                     [](const float2& u, const float2& v) { return u.x > v.x; });
  }
  // per-atom words: first shell, and the atom's layout when it is one of the unrolled ones
  int* aw = reinterpret_cast<int*>(tab.data() + lay.off_ashell / 16);
  auto is = [&](int sidx, int L, int np, int same) {
    const Shell& x = m->shells[sidx];
    return x.L == L && x.nprim == np && x.same_exp == same;
  };
  for (int a = 0; a <= m->natoms; ++a) {
    const int sa = m->atom_shell[a];
    int shape = SHAPE_GENERIC;
    if (a < m->natoms) {
      const int ns = m->atom_shell[a + 1] - sa;
      if (ns == 3 && is(sa, 0, 3, 0) && is(sa + 1, 0, 1, 0) && is(sa + 2, 1, 1, 0)) shape = SHAPE_S3S1P1;
      if (ns == 6 && is(sa, 0, 8, 0) && is(sa + 1, 0, 8, 1) && is(sa + 2, 0, 1, 0) && is(sa + 3, 1, 3, 0) &&
          is(sa + 4, 1, 1, 0) && is(sa + 5, 2, 1, 0))
        shape = SHAPE_S8S8S1P3P1D1;
    }
    if (sa >= (1 << 24)) return fail(QMT_BAD_ARG, "too many shells for the density tables");
    aw[a] = sa | (shape << 24);
  }
  // staging windows: atoms whose functions [first, last] meet [c0, c0 + STAGE_W)
  int2* wr = reinterpret_cast<int2*>(tab.data() + lay.off_win);
  for (int w = 0; w < lay.nwin; ++w) {
    const int c0 = w * STAGE_W, c1 = c0 + STAGE_W;
    int first = m->natoms, end = 0;
    for (int a = 0; a < m->natoms; ++a) {
      const int sa = m->atom_shell[a], sb = m->atom_shell[a + 1];
      if (sb <= sa) continue;
      const Shell& last = m->shells[sb - 1];
      const int f0 = m->shells[sa].func, f1 = last.func + 2 * last.L;
      if (f1 >= c0 && f0 < c1) {
        first = std::min(first, a);
        end = a + 1;
      }
    }
    wr[w] = first < end ? make_int2(first, end) : make_int2(0, 0);
  }
  qmt_status st;
  if ((st = m->d_fused_tab.reserve(tab.size() * sizeof(int4)))) return st;
  // pageable uploads return once the data is staged, so the host vectors may go
  QMT_CUDA(cudaMemcpyAsync(m->d_fused_tab.ptr, tab.data(), tab.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  return QMT_OK;
}

// Scaled density matrix of the fused path, stored as K-step blocks of kpad + 64 rows x 16 columns
// in the 32-byte swizzled image of a stage (split_P_kernel), read by one contiguous copy per
// stage and piece.

static qmt_status ensure_fused_operands(qmt_mol* m, int prec, const TcShape& sh, cudaStream_t s) {
  const int key = prec;
  if (m->fused_prec == key) return QMT_OK;
  const int K = sh.kpad;
  qmt_status st;
  if ((st = ensure_basis_operands(m, K, s)) || (st = split_exponent(m, s))) return st;
  const int rows = K + 64;
  const size_t piece = (size_t)rows * K * 2;
  if ((st = m->d_fused_B.reserve(2 * piece))) return st;
  if ((st = launch_split(m, K, sh.fmt, K + 64, m->d_fused_B.ptr, m->d_fused_B.as<uint8_t>() + piece,
                         piece, s)))
    return st;
  m->fused_prec = key;
  return QMT_OK;
}

// ---- factored density matrix -----------------------------------------------------------------
// A density matrix of rank r (r = occupied orbitals for an SCF density, P = 2 C_occ C_occ^T) is
// P = L L^T with L n x r, and then rho_i = sum_jk Phi_ij P_jk Phi_ik = sum_k (Phi L)_ik^2: the
// contraction needs N = r columns instead of n.  L comes from a pivoted Cholesky factorisation in
// FP64 (largest remaining diagonal first), stopped once every remaining diagonal element is at
// most kFactorTol of the largest one; the factor is used when the matrix it leaves out is at most
// kFactorResid of max |P| (float32 input rounding is ~6e-8) and the rank is at most half of n.
// A matrix that is not positive semi-definite, or of high rank, takes the unfactored path.
// Raises *bad when some |P_ij - sum_q L_iq L_jq| (i >= j) exceeds tol; L row i at L[i * ld].
__global__ void fact_residual_kernel(const double* __restrict__ P, int np, const double* __restrict__ L, int n, int ld,
                                     int r, double tol, int* bad) {
  const int64_t tot = (int64_t)n * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < tot; idx += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx - (int64_t)i * n);
    if (j > i) continue;
    double v = P[(size_t)i * np + j];
    const double* li = L + (size_t)i * ld;
    const double* lj = L + (size_t)j * ld;
    for (int q = 0; q < r; ++q) v -= li[q] * lj[q];
    if (fabs(v) > tol) *bad = 1;
  }
}

// The factor's stage layout (ensure_factor): element (j, q), j < n16, q < r16, of W = L_jq 2^-s_j
// 2^h_q (zero outside j < n, q < r) split into hi + lo (fp16 or bf16, as split_host); K-step block j / 16 holds nsplit x r16 rows
// of 32 bytes (hi rows, then lo rows), the two 16-byte units of a row exchanged when bit 2 of the
// row is set.
__global__ void fact_split_kernel(const double* __restrict__ L, int n, int ld, int r, int n16, int r16,
                                  const double* __restrict__ inv_s, const double* __restrict__ two_h, int fmt,
                                  int nsplit, uint8_t* __restrict__ out) {
  const int64_t tot = (int64_t)n16 * r16;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(i / r16), q = (int)(i - (int64_t)j * r16);
    const double w = (j < n && q < r) ? L[(size_t)j * ld + q] * inv_s[j] * two_h[q] : 0.0;
    const int e = j & 15, pe = ((((e >> 3) ^ (q >> 2)) & 1) << 3) | (e & 7);
    const size_t idx = (size_t)(j >> 4) * nsplit * r16 * 16 + (size_t)q * 16 + pe;
    uint16_t hi, lo;
    if (fmt == FMT_F16) {
      const __half h = __float2half_rn((float)w);
      hi = __half_as_ushort(h);
      lo = __half_as_ushort(__float2half_rn((float)(w - (double)__half2float(h))));
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn((float)w);
      hi = __bfloat16_as_ushort(h);
      lo = __bfloat16_as_ushort(__float2bfloat16_rn((float)(w - (double)__bfloat162float(h))));
    }
    reinterpret_cast<uint16_t*>(out)[idx] = hi;
    if (nsplit == 2) reinterpret_cast<uint16_t*>(out)[idx + (size_t)r16 * 16] = lo;
  }
}

// The factor as the staged path's B operand: row q < r16 holds the hi piece of factor column q,
// row r16 + q its lo piece (two pieces), each kpad elements of W_jq = L_jq 2^-s_j 2^h_q (zero
// outside j < n, q < r), row-major; the tensor map gives the 128-byte swizzle.
__global__ void fact_rows_kernel(const double* __restrict__ L, int n, int ld, int r, int kpad, int r16,
                                 const double* __restrict__ inv_s, const double* __restrict__ two_h, int fmt,
                                 int nsplit, uint16_t* __restrict__ out) {
  const int64_t tot = (int64_t)r16 * kpad;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(i / kpad), j = (int)(i - (int64_t)q * kpad);
    const double w = (j < n && q < r) ? L[(size_t)j * ld + q] * inv_s[j] * two_h[q] : 0.0;
    uint16_t hi, lo;
    if (fmt == FMT_F16) {
      const __half h = __float2half_rn((float)w);
      hi = __half_as_ushort(h);
      lo = __half_as_ushort(__float2half_rn((float)(w - (double)__half2float(h))));
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn((float)w);
      hi = __bfloat16_as_ushort(h);
      lo = __bfloat16_as_ushort(__float2bfloat16_rn((float)(w - (double)__bfloat162float(h))));
    }
    out[(size_t)q * kpad + j] = hi;
    if (nsplit == 2) out[(size_t)(r16 + q) * kpad + j] = lo;
  }
}

constexpr double kFactorTol = 1e-7;
constexpr double kFactorResid = 2e-7;
constexpr int kFactorMaxRank = 128;   // N = 2 x 128 per MMA of the staged path's factored kernel
constexpr int kFusedFactorMaxR16 = 64; // the fused factored kernel: N = 2 x 64, three main accumulators

// The scaled factor W_jk = L_jk 2^(h_k - s_j) (so Phi' W = 2^h_k (Phi L)_k, each column scaled
// to a maximum near 2^14) split into hi + lo pieces, as the fused kernel streams it: K-step block
// j / 16 holds the r16 hi rows, then (two pieces) the r16 lo rows, one row per factor column k of
// 32 bytes (functions j .. j + 15 of that column, the two 16-byte units exchanged when bit 2 of the
// row is set), so that one MMA of N = 2 r16 takes both and four consecutive blocks are one
// stage.  The column scales 2^-2h_k of the squares go to d_fact_scale.  Sets fact_rank = 0 when
// the matrix is not factored.
static qmt_status ensure_factor(qmt_mol* m, int prec, const TcShape& sh, cudaStream_t s) {
  if (m->fact_prec == prec) return QMT_OK;
  qmt_status st;
  if ((st = ensure_basis_operands(m, sh.kpad, s))) return st;
  const int n = m->norbs, np = m->npad, n16 = (n + 15) / 16 * 16;
  m->fact_prec = prec;
  m->fact_rank = 0;
  const int rmax = std::min(kFactorMaxRank, n16 / 2);
  // a density matrix of N_e electrons whose occupations are at most 2 has rank >= N_e / 2: with
  // the nuclear charge for N_e (ions of up to 16 charges allowed for) a rank above rmax is known
  // without the factorisation's host work (tens of milliseconds at a thousand functions)
  if (0.5 * m->qtot > rmax + 8) return QMT_OK;
  // P_ij from the lower triangle of the matrix as given (no symmetric host copy is built)
  const float* dm = m->dm_host.data();
  auto Pij = [&](int i, int j) -> double { return i >= j ? dm[(size_t)i * n + j] : dm[(size_t)j * n + i]; };
  // the scale of the device check's tolerance: max |P_jk| <= max_j P_jj for a positive
  // semi-definite P (for any other matrix the check is only the stricter and falls back to the
  // unfactored one)
  double dmax = 0.0;
  for (int j = 0; j < n; ++j) dmax = std::max(dmax, Pij(j, j));
  const double pmax = dmax;
  // L row by row (row i at Lr[i * rmax]), so that the dot products run over contiguous memory;
  // the host buffers are the handle's, reused (no fresh pages per density-matrix change)
  std::vector<double>& Lr = m->fact_Lr_host;
  std::vector<double>& d = m->fact_d_host;
  Lr.assign((size_t)n * rmax, 0.0);
  d.assign(n, 0.0);
  for (int j = 0; j < n; ++j) d[j] = Pij(j, j);
  int r = 0;
  for (;;) {
    int jp = 0;
    for (int j = 1; j < n; ++j)
      if (d[j] > d[jp]) jp = j;
    if (!(d[jp] > kFactorTol * dmax)) break;
    if (r == rmax) return QMT_OK;   // rank too high for the factored path to pay
    const double piv = std::sqrt(d[jp]), ipiv = 1.0 / piv;
    const double* lj = Lr.data() + (size_t)jp * rmax;
    for (int i = 0; i < n; ++i) {
      const double* li = Lr.data() + (size_t)i * rmax;
      double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
      int q = 0;
      for (; q + 4 <= r; q += 4) {
        a0 += li[q] * lj[q];
        a1 += li[q + 1] * lj[q + 1];
        a2 += li[q + 2] * lj[q + 2];
        a3 += li[q + 3] * lj[q + 3];
      }
      for (; q < r; ++q) a0 += li[q] * lj[q];
      Lr[(size_t)i * rmax + r] = (Pij(i, jp) - ((a0 + a1) + (a2 + a3))) * ipiv;
    }
    Lr[(size_t)jp * rmax + r] = piv;
    for (int i = 0; i < n; ++i) d[i] -= Lr[(size_t)i * rmax + r] * Lr[(size_t)i * rmax + r];
    d[jp] = 0.0;
    ++r;
  }
  // an indefinite matrix leaves clearly negative diagonal elements behind
  for (int i = 0; i < n; ++i)
    if (d[i] < -10.0 * kFactorTol * dmax) return QMT_OK;
  // what the factor leaves out, max |P - L L^T|, is checked on the device (n^2 r products) into
  // the gate flag, without a round trip: the factored launch runs when it is 0, the unfactored
  // one when it is 1 (density_tc)
  {
    const size_t lbytes = (size_t)n * rmax * sizeof(double);
    if ((st = m->d_fact_L.reserve(lbytes + 16))) return st;
    int* flag = reinterpret_cast<int*>(m->d_fact_L.as<uint8_t>() + lbytes);
    QMT_CUDA(cudaMemcpyAsync(m->d_fact_L.ptr, Lr.data(), lbytes, cudaMemcpyHostToDevice, s));
    QMT_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    const int64_t tot = (int64_t)n * n;
    const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 4);
    fact_residual_kernel<<<std::max(blocks, 1), 256, 0, s>>>(m->d_P64.as<double>(), np, m->d_fact_L.as<double>(), n,
                                                             rmax, r, kFactorResid * pmax, flag);
    QMT_CHECK_LAUNCH("fact_residual_kernel");
    m->fact_gate = flag;
  }
  // column scales on the host -- 2^-2h_k (FP64, the staged path's squares), 2^h_k (FP64, the
  // split), then 2^-h_k (FP32, the fused path's squares (2^-h_k T_k)^2: an exact scaling) -- and
  // the scaled, split factor in its stage layout on the device
  const int r16 = std::max(16, (r + 15) / 16 * 16);
  std::vector<double> sc(2 * r16 + r16 / 2, 0.0);
  float* scf = reinterpret_cast<float*>(sc.data() + 2 * r16);
  for (int q = 0; q < r; ++q) {
    double wmax = 0.0;
    for (int j = 0; j < n; ++j) wmax = std::max(wmax, std::fabs(Lr[(size_t)j * rmax + q] * m->split_inv[j]));
    int h = wmax > 0 ? (int)std::floor(std::log2(16000.0 / wmax)) : 0;
    h = std::max(-100, std::min(100, h));
    sc[q] = std::ldexp(1.0, -2 * h);
    sc[r16 + q] = std::ldexp(1.0, h);
    scf[q] = std::ldexp(1.0f, -h);
  }
  const size_t sc_bytes = sc.size() * sizeof(double);
  const size_t total = (size_t)(n16 / 16) * sh.nsplit * r16 * 32;   // bytes
  if ((st = m->d_fact_B.reserve(total)) || (st = m->d_fact_scale.reserve(sc_bytes))) return st;
  QMT_CUDA(cudaMemcpyAsync(m->d_fact_scale.ptr, sc.data(), sc_bytes, cudaMemcpyHostToDevice, s));
  const int64_t tot = (int64_t)n16 * r16;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 4);
  fact_split_kernel<<<std::max(blocks, 1), 256, 0, s>>>(m->d_fact_L.as<double>(), n, rmax, r, n16, r16,
                                                         m->d_split_scale.as<double>(),
                                                         m->d_fact_scale.as<double>() + r16, sh.fmt, sh.nsplit,
                                                         m->d_fact_B.as<uint8_t>());
  QMT_CHECK_LAUNCH("fact_split_kernel");
  m->fact_rank = r;
  m->fact_r16 = r16;
  m->fact_rows_prec = -1;
  return QMT_OK;
}

// The factor in the staged path's B layout (fact_rows_kernel), once per factor.
static qmt_status ensure_factor_rows(qmt_mol* m, int prec, const TcShape& sh, cudaStream_t s) {
  if (m->fact_rows_prec == prec) return QMT_OK;
  const int r16 = m->fact_r16, n16 = (m->norbs + 15) / 16 * 16;
  const int rmax = std::min(kFactorMaxRank, n16 / 2);
  qmt_status st = m->d_fact_Bs.reserve((size_t)sh.nsplit * r16 * sh.kpad * 2);
  if (st) return st;
  const int64_t tot = (int64_t)r16 * sh.kpad;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 4);
  fact_rows_kernel<<<std::max(blocks, 1), 256, 0, s>>>(m->d_fact_L.as<double>(), m->norbs, rmax, m->fact_rank,
                                                        sh.kpad, r16, m->d_split_scale.as<double>(),
                                                        m->d_fact_scale.as<double>() + r16, sh.fmt, sh.nsplit,
                                                        m->d_fact_Bs.as<uint16_t>());
  QMT_CHECK_LAUNCH("fact_rows_kernel");
  m->fact_rows_prec = prec;
  return QMT_OK;
}

// Shared-memory bytes of the molecule tables staged by the fused kernel.
static int fused_tab_bytes(const qmt_mol* m) {
  const int words = (int)(m->shells.size() + (m->alpha.size() + 1) / 2);
  return words * 16 + (m->natoms + 1 + 3) / 4 * 16 + (3 * m->natoms + 3) / 4 * 16;
}

// Functions rounded up to 16 (K-steps of the fused MMAs), bytes of one A piece (n16 columns)
// and of one U piece slot in a stage.
static int fused_n16(const qmt_mol* m) { return (m->norbs + 15) / 16 * 16; }
static uint32_t fused_a_bytes(int n16) { return 128u * (uint32_t)n16 * 2u; }
static uint32_t fused_b_slot(int nb) { return (uint32_t)nb * 32u; }

// U pipeline stages that fit beside A and the tables (below 2: the fused path does not fit).
// Bytes of one stage: a K-step of B (nb rows per piece), or four for the factor.
static long fused_stage_bytes(const TcShape& sh, int nb, bool fact) {
  return (long)(fact ? 4 : 1) * sh.nsplit * fused_b_slot(nb);
}

template <int FMT>
static int fused_stages(const TcShape& sh, int n16, int nb, int tab_bytes, bool fact = false) {
  int maxsm = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, density_fused_kernel<FMT, true, false>) != cudaSuccess) return 0;
  const long a_bytes = fused_a_bytes(n16), stage_bytes = fused_stage_bytes(sh, nb, fact);
  const long avail = (long)maxsm - (long)fa.sharedSizeBytes - 1024 - sh.nsplit * a_bytes - tab_bytes;
  return (int)std::max<long>(0, std::min<long>(MAX_STAGES, avail / stage_bytes));
}

// The descriptor of one molecule in a fused launch, its tiles starting at global tile `tile0`; B
// is the scaled density matrix, or its factor (`fact`, built by ensure_factor).
static qmt_status fused_mol_desc(qmt_mol* m, const TcShape& sh, const PointMap& pm, int64_t tile0, int64_t ntiles,
                                 float* qube, double outscale, FusedMol& d, int& tab_bytes, bool fact = false) {
  const int K = sh.kpad, n16 = fused_n16(m);
  const size_t piece = fact ? 0 : (size_t)(K + 64) * K * 2;   // (the factor's pieces are interleaved)
  const uint8_t* B = fact ? m->d_fact_B.as<uint8_t>() : m->d_fused_B.as<uint8_t>();
  d = FusedMol{};
  d.pm = pm;
  d.tile0 = tile0;
  d.ntiles = ntiles;
  d.natoms = m->natoms;
  d.norbs = m->norbs;
  d.n16 = n16;
  d.ksteps = n16 / 16;
  d.nchunks = (n16 + 63) / 64;
  d.tail0 = n16 & ~63;
  d.nb = fact ? m->fact_r16 : n16;
  d.u_rows = fact ? m->fact_r16 : K + 64;
  d.u_hi = B;
  d.u_lo = B + piece;
  if (d.nchunks > MAX_FUSED_CHUNKS) return fail(QMT_BAD_ARG, "fused density path supports kpad <= 320");
  if (2 * m->natoms >= (int)CHUNK_COUNT) return fail(QMT_BAD_ARG, "too many atoms for the fused density path");
  for (int a = 0; a < m->natoms; ++a) {
    const int sa = m->atom_shell[a], sb = m->atom_shell[a + 1];
    if (sb <= sa) continue;
    const Shell& last = m->shells[sb - 1];
    const int cfirst = m->shells[sa].func >> 6, clast = (last.func + 2 * last.L) >> 6;
    for (int c = cfirst; c <= clast; ++c) d.chunk_need[c] += 2;   // two row halves per atom
  }
  d.tab = m->d_fused_tab.as<int4>();
  d.off_prim = (int)m->shells.size() * 16;
  d.off_ashell = (int)(m->shells.size() + (m->alpha.size() + 1) / 2) * 16;
  d.tab_words = d.off_ashell / 16 + (m->natoms + 1 + 3) / 4;
  d.off_coords = d.tab_words * 16;
  d.coords = m->d_coords.as<float>();
  tab_bytes = d.off_coords + (3 * m->natoms + 3) / 4 * 16;
  d.qube = qube;
  d.partials = m->d_partials.as<double>();
  d.outscale = outscale;
  d.gsc = fact ? m->d_fact_scale.as<double>() : m->d_gscale.as<double>();
  return QMT_OK;
}

// One persistent launch over every tile of the molecules in `p` (p.one, or the device array
// p.mols); shared memory is sized for the largest operand, stage and table of the set.
template <int FMT>
static qmt_status launch_fused(FusedParams& p, const TcShape& sh_max, int n16_max, int nb_max, int tab_bytes_max,
                               cudaStream_t s, bool fact = false) {
  p.nsplit = sh_max.nsplit;
  p.a_bytes = fused_a_bytes(n16_max);
  p.b_slot = fused_b_slot(nb_max);
  p.stage_bytes = (uint32_t)fused_stage_bytes(sh_max, nb_max, fact);
  p.fmt = (uint32_t)sh_max.fmt;
  p.wait_ns = wait_limit_ns();
  auto kern = p.nmol > 1 ? (fact ? density_fused_kernel<FMT, true, true> : density_fused_kernel<FMT, true, false>)
                         : (fact ? density_fused_kernel<FMT, false, true> : density_fused_kernel<FMT, false, false>);
  const int stages = fused_stages<FMT>(sh_max, n16_max, nb_max, tab_bytes_max, fact);
  if (stages < 2) return fail(QMT_BAD_ARG, "fused density tile does not fit in shared memory");
  p.stages = stages;
  const size_t dyn = (size_t)p.nsplit * p.a_bytes + (size_t)stages * p.stage_bytes + tab_bytes_max + 1024;
  QMT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  const int grid = (int)std::min<int64_t>(p.ntiles, sm_count());
  if (grid <= 0) return QMT_OK;
  kern<<<grid, FUSED_THREADS, dyn, s>>>(p);
  QMT_CHECK_LAUNCH("density_fused_kernel");
  return QMT_OK;
}

template <int FMT>
static qmt_status run_fused(qmt_mol* m, const TcShape& sh, const PointMap& pm, int64_t ntiles, float* qube,
                            double outscale, cudaStream_t s, bool fact = false, const int* gate = nullptr,
                            int gate_want = 0) {
  FusedParams p{};
  int tab_bytes = 0;
  qmt_status st = fused_mol_desc(m, sh, pm, 0, ntiles, qube, outscale, p.one, tab_bytes, fact);
  if (st) return st;
  p.gate = gate;
  p.gate_want = gate_want;
  p.nmol = 1;
  p.ntiles = ntiles;
  p.err = reinterpret_cast<int*>(m->d_scalars.as<double>() + 8);
  return launch_fused<FMT>(p, sh, p.one.n16, p.one.nb, tab_bytes, s, fact);
}

// Builds the scaled, split density matrix and the Phi column scales for `prec`.
static qmt_status ensure_tc_operands(qmt_mol* m, int prec, const TcShape& sh, cudaStream_t s) {
  if (m->tc_prec == prec) return QMT_OK;
  const int K = sh.kpad;
  qmt_status st;
  if ((st = ensure_basis_operands(m, K, s)) || (st = split_exponent(m, s))) return st;
  const size_t piece = (size_t)sh.nrows_b * K * sh.esize;
  if ((st = m->d_tc_P.reserve(2 * piece))) return st;
  if ((st = launch_split(m, K, sh.fmt, 0, m->d_tc_P.ptr, m->d_tc_P.as<uint8_t>() + piece, piece, s))) return st;
  m->tc_prec = prec;
  return QMT_OK;
}

// Staged path.  Basis values go through `phi_hi` / `phi_lo` (the molecule's own buffers, or a
// batch's shared ones) in chunks of tiles of at most `stage_bytes` in all.
template <int FMT>
static qmt_status run_tc(qmt_mol* m, const TcShape& sh, const PointMap& pm, int64_t ntiles, int prec,
                         float* qube, double outscale, cudaStream_t s, DevBuf* phi_hi = nullptr,
                         DevBuf* phi_lo = nullptr, size_t stage_bytes = (size_t)2 << 30, int fact = 0) {
  // fact: 0 unfactored; 1 factored only; 2 both launches, gated by the device check of the factor
  qmt_status st;
  if (!phi_hi) {
    phi_hi = &m->d_Phi_hi;
    phi_lo = &m->d_Phi_lo;
  }
  const size_t tile_bytes = (size_t)128 * sh.kpad * sh.esize;
  const int nsm = sm_count();
  // staging chunk: bounded by stage_bytes, a multiple of the SM count when larger than one wave
  int64_t chunk = std::max<int64_t>(1, stage_bytes / (tile_bytes * sh.nsplit));
  if (chunk > nsm) chunk = chunk / nsm * nsm;
  chunk = std::min<int64_t>(chunk, ntiles);
  if ((st = phi_hi->reserve(chunk * tile_bytes))) return st;
  if (sh.nsplit == 2 && (st = phi_lo->reserve(chunk * tile_bytes))) return st;
  void* lo_ptr = sh.nsplit == 2 ? phi_lo->ptr : phi_hi->ptr;

  CUtensorMap tA_hi, tA_lo, tB_hi, tB_lo, tF;
  const uint8_t* Pb = m->d_tc_P.as<uint8_t>();
  const size_t piece = (size_t)sh.nrows_b * sh.kpad * sh.esize;
  if ((st = make_map(&tA_hi, phi_hi->ptr, sh.esize, sh.kpad, (uint64_t)chunk * 128, sh.ke, 128)) ||
      (st = make_map(&tA_lo, lo_ptr, sh.esize, sh.kpad, (uint64_t)chunk * 128, sh.ke, 128)))
    return st;
  if (fact != 1 && ((st = make_map(&tB_hi, Pb, sh.esize, sh.kpad, sh.nrows_b, sh.ke, sh.pw)) ||
                    (st = make_map(&tB_lo, Pb + piece, sh.esize, sh.kpad, sh.nrows_b, sh.ke, sh.pw))))
    return st;
  const int nfac = sh.nsplit * m->fact_r16;   // the factored launch's N: hi rows, then lo rows
  if (fact && (st = make_map(&tF, m->d_fact_Bs.ptr, sh.esize, sh.kpad, (uint64_t)nfac, sh.ke, (uint32_t)nfac)))
    return st;

  TcParams p{};
  p.pm = pm;
  p.kpad = sh.kpad;
  p.kchunks = sh.kpad / sh.ke;
  p.npanels = sh.npanels;
  p.pw = sh.pw;
  p.nsplit = sh.nsplit;
  p.esize = sh.esize;
  p.a_bytes = 128u * 128u;
  p.b_bytes = (uint32_t)sh.pw * 128u;
  p.stage_bytes = sh.nsplit * (p.a_bytes + p.b_bytes);
  p.tx_bytes = p.stage_bytes;
  p.idesc = make_idesc((uint32_t)sh.fmt, 128, (uint32_t)sh.pw);
  p.phi_hi = phi_hi->ptr;
  p.phi_lo = lo_ptr;
  p.qube = qube;
  p.partials = m->d_partials.as<double>();
  p.outscale = outscale;
  p.gsc = m->d_gscale.as<double>();
  p.err = reinterpret_cast<int*>(m->d_scalars.as<double>() + 8);
  p.wait_ns = wait_limit_ns();
  if (fact == 2) {
    p.gate = m->fact_gate;
    p.gate_want = 1;
  }
  // the factored launch: one panel of N = nfac (the factor's hi and lo rows in one box)
  TcParams pf = p;
  pf.npanels = 1;
  pf.pw = nfac;
  pf.b_bytes = (uint32_t)nfac * 128u;
  pf.stage_bytes = sh.nsplit * pf.a_bytes + pf.b_bytes;
  pf.tx_bytes = pf.stage_bytes;
  pf.idesc = make_idesc((uint32_t)sh.fmt, 128, (uint32_t)nfac);
  pf.gsc = m->d_fact_scale.as<double>();
  pf.nb = m->fact_r16;
  pf.gate = fact == 2 ? m->fact_gate : nullptr;
  pf.gate_want = 0;

  int maxsm = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int static_bytes = 4096;
  auto plan = [&](TcParams& q) -> size_t {
    q.stages = std::min((int)((maxsm - static_bytes - 1024) / q.stage_bytes), MAX_STAGES);
    return (size_t)q.stages * q.stage_bytes + 1024;
  };
  const size_t dyn = plan(p), dynf = plan(pf);
  if ((fact != 1 && p.stages < 2) || (fact && pf.stages < 2))
    return fail(QMT_BAD_ARG, "tensor-core stage does not fit in shared memory");
  constexpr int FF = FMT == FMT_TF32 ? FMT_F16 : FMT;   // (the factored kernel takes fp16 / bf16)
  auto kern = density_mma_kernel<FMT, false>;
  auto kernf = density_mma_kernel<FF, true>;
  if (fact != 1) QMT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  if (fact) QMT_CUDA(cudaFuncSetAttribute(kernf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynf));

  // staging kernel: molecule tables in shared memory unless they would keep two CTAs off an SM
  const MolTabLayout lay = mol_tab_layout(m, sh.kpad);
  StageParams sp{};
  sp.pm = pm;
  sp.kpad = sh.kpad;
  sp.norbs = m->norbs;
  sp.nwin = lay.nwin;
  sp.tab = m->d_fused_tab.as<int4>();
  sp.coords = m->d_coords.as<float>();
  sp.ncoords = 3 * m->natoms;
  sp.win = reinterpret_cast<const int2*>(sp.tab + lay.off_win);
  sp.tab_words = lay.words;
  sp.off_prim = lay.off_prim;
  sp.off_ashell = lay.off_ashell;
  sp.off_coords = lay.words * 16;
  sp.tab_bytes = sp.off_coords + (3 * m->natoms + 3) / 4 * 16;
  sp.out_hi = phi_hi->ptr;
  sp.out_lo = lo_ptr;
  sp.two = sh.nsplit == 2;
  const int buf_bytes = 128 * STAGE_LD * 4;
  if (sp.tab_bytes + buf_bytes > (maxsm - 8192) / 2) sp.tab_bytes = 0;
  const size_t sdyn = (size_t)sp.tab_bytes + buf_bytes;
  auto skern = basis_window_kernel<FMT>;
  QMT_CUDA(cudaFuncSetAttribute(skern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sdyn));
  int stage_ctas = 0;
  QMT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&stage_ctas, skern, STAGE_THREADS, sdyn));
  stage_ctas = std::max(1, stage_ctas);

  for (int64_t t0 = 0; t0 < ntiles; t0 += chunk) {
    const int nt = (int)std::min<int64_t>(chunk, ntiles - t0);
    sp.tile0 = t0;
    sp.ntiles = nt;
    const int gb = (int)std::min<int64_t>(nt, (int64_t)nsm * stage_ctas);
    skern<<<gb, STAGE_THREADS, sdyn, s>>>(sp);
    QMT_CHECK_LAUNCH("basis_window_kernel");
    p.tile0 = pf.tile0 = t0;
    p.ntiles = pf.ntiles = nt;
    const int gm = (int)std::min<int64_t>(nt, nsm);
    if (fact) {
      kernf<<<gm, 192, dynf, s>>>(tA_hi, tA_lo, tF, tF, pf);
      QMT_CHECK_LAUNCH("density_mma_kernel");
    }
    if (fact != 1) {
      kern<<<gm, 192, dyn, s>>>(tA_hi, tA_lo, tB_hi, tB_lo, p);
      QMT_CHECK_LAUNCH("density_mma_kernel");
    }
  }
  (void)prec;
  return QMT_OK;
}

static int g_density_path = 0;   // 0 auto, 1 staged, 2 fused, 3 fused with the factored matrix

// The fused path takes fp16/bf16 contractions of up to 320 functions whose tile, stages and tables
// fit in shared memory.
static bool fused_fits(const qmt_mol* mol, const TcShape& sh) {
  if (sh.fmt == FMT_TF32 || sh.kpad > 320 || 2 * mol->natoms >= (int)CHUNK_COUNT) return false;
  const int tb = fused_tab_bytes(mol);
  const int n16 = fused_n16(mol);
  return (sh.fmt == FMT_F16 ? fused_stages<FMT_F16>(sh, n16, n16, tb) : fused_stages<FMT_BF16>(sh, n16, n16, tb)) >= 2;
}

qmt_status density_tc(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy, float oz,
                      int subgrid, int precision, int rescale, float* qube, double* sum_out,
                      cudaStream_t s) {
  const TcShape sh = tc_shape(precision, mol->norbs);
  qmt_status st;
  PointMap pm;
  int64_t ntiles;
  if ((st = make_point_map(nx, ny, nz, step, ox, oy, oz, subgrid, 128, pm, ntiles))) return st;
  if ((st = mol->d_partials.reserve(ntiles * sizeof(double)))) return st;
  const double outscale = 2.0 * (double)step * step * step / pm.s3;
  const bool fusable = fused_fits(mol, sh);
  const bool fused = g_density_path == 1 ? false : fusable;
  if (g_density_path == 2 && !fusable)
    return fail(QMT_BAD_ARG, "fused density path needs fp16/bf16, N <= 320 and molecule tables that fit in shared memory");
  // the factored matrix when there is one (automatic, or asked for): fused (rank <= 64) or staged
  // (rank <= 128, fp16 / bf16)
  bool fact = false;
  if (sh.fmt != FMT_TF32 && g_density_path != 1 && g_density_path != 2) {
    if ((st = ensure_factor(mol, precision, sh, s))) return st;
    fact = mol->fact_rank > 0 && (!fused || mol->fact_r16 <= kFusedFactorMaxR16);
    if (g_density_path == 3 && !fact)
      return fail(QMT_BAD_ARG, "factored density path needs a positive semi-definite density matrix of low rank");
  }
  if (fused) {
    // with a factor, the device check of what it leaves out picks the launch (no host round trip)
    if ((st = ensure_fused_operands(mol, precision, sh, s))) return st;
    const int* gate = fact ? mol->fact_gate : nullptr;
    if (sh.fmt == FMT_F16) {
      if (fact) st = run_fused<FMT_F16>(mol, sh, pm, ntiles, qube, outscale, s, true, gate, 0);
      if (!st) st = run_fused<FMT_F16>(mol, sh, pm, ntiles, qube, outscale, s, false, gate, 1);
    } else {
      if (fact) st = run_fused<FMT_BF16>(mol, sh, pm, ntiles, qube, outscale, s, true, gate, 0);
      if (!st) st = run_fused<FMT_BF16>(mol, sh, pm, ntiles, qube, outscale, s, false, gate, 1);
    }
  } else {
    if ((st = ensure_tc_operands(mol, precision, sh, s))) return st;
    if (fact && (st = ensure_factor_rows(mol, precision, sh, s))) return st;
    const int fmode = fact ? 2 : 0;   // with a factor, the device check picks the launch
    if (sh.fmt == FMT_TF32) st = run_tc<FMT_TF32>(mol, sh, pm, ntiles, precision, qube, outscale, s);
    else if (sh.fmt == FMT_F16)
      st = run_tc<FMT_F16>(mol, sh, pm, ntiles, precision, qube, outscale, s, nullptr, nullptr, (size_t)2 << 30, fmode);
    else
      st = run_tc<FMT_BF16>(mol, sh, pm, ntiles, precision, qube, outscale, s, nullptr, nullptr, (size_t)2 << 30, fmode);
  }
  if (st) return st;
  st = finish_density(mol, pm.nvox, ntiles, rescale, qube, sum_out, s);
  if (st) return st;
  // The kernels' barrier-timeout flag is sticky: a call that returns a host sum (and so
  // synchronises anyway) reads and clears it; fully asynchronous calls leave it for the next
  // synchronous call on this molecule.
  if (sum_out) {
    int err = 0;
    QMT_CUDA(cudaMemcpyAsync(&err, mol->d_scalars.as<double>() + 8, sizeof(int), cudaMemcpyDeviceToHost, s));
    QMT_CUDA(cudaStreamSynchronize(s));
    if (err) {
      QMT_CUDA(cudaMemsetAsync(mol->d_scalars.as<double>() + 8, 0, sizeof(int), s));
      return fail(QMT_CUDA_ERR, "tensor-core density kernel gave up waiting on a barrier");
    }
  }
  return QMT_OK;
}

// ---- batches ---------------------------------------------------------------------------------
// Staged-path molecules of a batch run one after another on one stream and share one basis-value
// buffer of this size (both pieces), instead of each holding its own.
constexpr size_t BATCH_STAGE_BYTES = (size_t)1 << 30;

struct BatchItem {
  qmt_mol* mol;
  TcShape sh;
  PointMap pm;
  int64_t ntiles;
  float* qube;
  double outscale;
  bool fused;
  bool fact;   // fused, with the factored density matrix
};

}  // namespace qmt

// One persistent fused launch of a batch: its molecules' descriptors, tiles numbered across them.
struct qmt_batch_group {
  std::vector<qmt::FusedMol> fdesc;
  qmt::TcShape sh_max{};
  int n16_max = 0, nb_max = 0, tab_bytes_max = 0;
  int64_t tiles = 0;
  qmt::DevBuf d_fdesc;
};

struct qmt_batch {
  int precision = 0, fmt = 0;
  std::vector<qmt::BatchItem> items;
  qmt_batch_group fused, fact;        // unfactored and factored fused launches
  qmt::DevBuf d_err;
  qmt::DevBuf phi_hi, phi_lo;         // staged-path basis values, shared by the batch's molecules
};

namespace qmt {

// Re-derives (refresh) or checks the molecule's contraction operands for its path (a factored
// molecule's factor comes from the host matrix at batch creation and is not re-derived).
static qmt_status batch_operands(const BatchItem& it, int prec, bool refresh, cudaStream_t s) {
  if (it.fact) {
    if (refresh) return fail(QMT_BAD_ARG, "a batch with factored molecules cannot re-derive their operands");
    return it.fused ? QMT_OK : ensure_factor_rows(it.mol, prec, it.sh, s);
  }
  if (refresh) {
    it.mol->fused_prec = -1;
    it.mol->tc_prec = -1;
  }
  return it.fused ? ensure_fused_operands(it.mol, prec, it.sh, s) : ensure_tc_operands(it.mol, prec, it.sh, s);
}

// Descriptors of the fused molecules of one kind (factored or not) and the shared-memory plan of
// their launch; `stages` < 2 when the plan does not fit, `largest` the molecule to move out then.
static qmt_status batch_group(qmt_batch* b, qmt_batch_group& g, bool fact, int& stages, int& largest) {
  g.fdesc.clear();
  g.sh_max = TcShape{};
  g.n16_max = g.nb_max = g.tab_bytes_max = 0;
  g.tiles = 0;
  largest = -1;
  stages = MAX_STAGES;
  for (size_t i = 0; i < b->items.size(); ++i) {
    BatchItem& it = b->items[i];
    if (!it.fused || it.fact != fact) continue;
    FusedMol d;
    int tb = 0;
    qmt_status st = fused_mol_desc(it.mol, it.sh, it.pm, g.tiles, it.ntiles, it.qube, it.outscale, d, tb, fact);
    if (st) return st;
    g.tiles += it.ntiles;
    g.fdesc.push_back(d);
    if (it.sh.kpad > g.sh_max.kpad) g.sh_max = it.sh;
    g.n16_max = std::max(g.n16_max, d.n16);
    g.nb_max = std::max(g.nb_max, d.nb);
    g.tab_bytes_max = std::max(g.tab_bytes_max, tb);
    if (largest < 0 || it.sh.kpad + tb / 1024 > b->items[largest].sh.kpad + fused_tab_bytes(b->items[largest].mol) / 1024)
      largest = (int)i;
  }
  if (!g.fdesc.empty())
    stages = b->fmt == FMT_F16 ? fused_stages<FMT_F16>(g.sh_max, g.n16_max, g.nb_max, g.tab_bytes_max, fact)
                               : fused_stages<FMT_BF16>(g.sh_max, g.n16_max, g.nb_max, g.tab_bytes_max, fact);
  return QMT_OK;
}

template <int FMT>
static qmt_status batch_launch(qmt_batch* b, const qmt_batch_group& g, bool fact, cudaStream_t s) {
  if (g.fdesc.empty()) return QMT_OK;
  FusedParams p{};
  p.nmol = (int)g.fdesc.size();
  if (p.nmol == 1) p.one = g.fdesc[0];
  p.mols = g.d_fdesc.as<FusedMol>();
  p.ntiles = g.tiles;
  p.err = b->d_err.as<int>();
  return launch_fused<FMT>(p, g.sh_max, g.n16_max, g.nb_max, g.tab_bytes_max, s, fact);
}

template <int FMT>
static qmt_status batch_run(qmt_batch* b, int rescale, bool refresh, cudaStream_t s) {
  qmt_status st;
  for (const BatchItem& it : b->items)
    if ((st = batch_operands(it, b->precision, refresh, s))) return st;
  if (FMT != FMT_TF32) {
    constexpr int F = FMT == FMT_TF32 ? FMT_F16 : FMT;
    if ((st = batch_launch<F>(b, b->fact, true, s)) || (st = batch_launch<F>(b, b->fused, false, s))) return st;
  }
  for (const BatchItem& it : b->items)
    if (!it.fused && (st = run_tc<FMT>(it.mol, it.sh, it.pm, it.ntiles, b->precision, it.qube, it.outscale, s,
                                       &b->phi_hi, &b->phi_lo, BATCH_STAGE_BYTES, it.fact ? 1 : 0)))
      return st;
  for (const BatchItem& it : b->items)
    if ((st = finish_density(it.mol, it.pm.nvox, it.ntiles, rescale, it.qube, nullptr, s))) return st;
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" {

qmt_status qmt_batch_create(int nmol, qmt_mol* const* mols, const int32_t* shapes, const float* geoms,
                            int subgrid, int precision, const int32_t* paths, float* const* qube_devs,
                            void* stream, qmt_batch** out) {
  if (!out || nmol <= 0 || !mols || !shapes || !geoms || !qube_devs)
    return fail(QMT_BAD_ARG, "bad batch arguments");
  *out = nullptr;
  if (precision < QMT_PREC_TF32 || precision > QMT_PREC_FP16X3)
    return fail(QMT_BAD_ARG, "batches take the tensor-core precisions");
  cudaStream_t s = as_stream(stream);
  auto* b = new qmt_batch();
  b->precision = precision;
  qmt_status st = QMT_OK;
  for (int i = 0; i < nmol && !st; ++i) {
    qmt_mol* m = mols[i];
    if (!m || !qube_devs[i]) {
      st = fail(QMT_BAD_ARG, "null molecule or grid in a batch");
      break;
    }
    BatchItem it{};
    it.mol = m;
    it.qube = qube_devs[i];
    it.sh = tc_shape(precision, m->norbs);
    const float step = geoms[4 * i];
    if ((st = make_point_map(shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2], step, geoms[4 * i + 1],
                             geoms[4 * i + 2], geoms[4 * i + 3], subgrid, 128, it.pm, it.ntiles)))
      break;
    it.outscale = 2.0 * (double)step * step * step / it.pm.s3;
    const int path = paths ? paths[i] : 0;
    if (path < 0 || path > 3) {
      st = fail(QMT_BAD_ARG, "batch path must be 0 (automatic), 1 (staged), 2 (fused) or 3 (fused, factored)");
      break;
    }
    const bool fits = fused_fits(m, it.sh);
    if (path == 2 && !fits) {
      st = fail(QMT_BAD_ARG, "fused density path requested for a molecule it does not take");
      break;
    }
    it.fused = path == 2 || ((path == 0 || path == 3) && fits);
    it.fact = false;
    if (path == 3 && it.sh.fmt != FMT_TF32) {   // factored when the matrix has a factor that passes the check
      int gate = 1;
      if ((st = ensure_factor(m, precision, it.sh, s))) break;
      if (m->fact_rank > 0) {
        const cudaError_t e1 = cudaMemcpyAsync(&gate, m->fact_gate, sizeof(int), cudaMemcpyDeviceToHost, s);
        const cudaError_t e2 = cudaStreamSynchronize(s);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
          st = cuda_fail(e1 != cudaSuccess ? e1 : e2, "factor check");
          break;
        }
      }
      it.fact = m->fact_rank > 0 && gate == 0 && (!it.fused || m->fact_r16 <= kFusedFactorMaxR16);
    }
    if ((st = m->d_partials.reserve(it.ntiles * sizeof(double))) || (st = m->d_scalars.reserve(64 * sizeof(double))))
      break;
    if ((st = batch_operands(it, precision, false, s))) break;
    b->items.push_back(it);
  }
  b->fmt = tc_shape(precision, 1).fmt;
  // fused molecules of each kind: one launch sized for the largest of them; drop the largest to
  // the staged path until the shared-memory plan of the set fits
  for (int kind = 0; kind < 2 && !st; ++kind) {
    qmt_batch_group& g = kind ? b->fact : b->fused;
    for (;;) {
      int stg = 0, largest = -1;
      if ((st = batch_group(b, g, kind == 1, stg, largest))) break;
      if (g.fdesc.empty() || stg >= 2) break;
      b->items[largest].fused = false;   // (a factored molecule stays factored on the staged path)
      if ((st = batch_operands(b->items[largest], precision, false, s))) break;
    }
  }
  if (!st) st = b->d_err.reserve(256);
  for (qmt_batch_group* g : {&b->fused, &b->fact}) {
    if (st || g->fdesc.empty()) continue;
    const size_t bytes = g->fdesc.size() * sizeof(FusedMol);
    st = g->d_fdesc.reserve(bytes);
    if (!st) {
      const cudaError_t e1 = cudaMemcpyAsync(g->d_fdesc.ptr, g->fdesc.data(), bytes, cudaMemcpyHostToDevice, s);
      if (e1 != cudaSuccess) st = cuda_fail(e1, "batch descriptors");
    }
  }
  if (!st) {
    const cudaError_t e2 = cudaMemsetAsync(b->d_err.ptr, 0, 256, s);
    const cudaError_t e3 = cudaStreamSynchronize(s);
    if (e2 != cudaSuccess || e3 != cudaSuccess) st = cuda_fail(e2 != cudaSuccess ? e2 : e3, "batch descriptors");
  }
  if (st) {
    delete b;
    return st;
  }
  *out = b;
  return QMT_OK;
}

qmt_status qmt_batch_density(qmt_batch* b, int rescale, int refresh, void* stream) {
  if (!b) return fail(QMT_BAD_ARG, "null batch");
  cudaStream_t s = as_stream(stream);
  if (b->fmt == FMT_TF32) return batch_run<FMT_TF32>(b, rescale, refresh != 0, s);
  if (b->fmt == FMT_F16) return batch_run<FMT_F16>(b, rescale, refresh != 0, s);
  return batch_run<FMT_BF16>(b, rescale, refresh != 0, s);
}

qmt_status qmt_batch_sums(qmt_batch* b, double* sums, void* stream) {
  if (!b || !sums) return fail(QMT_BAD_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  std::vector<int> errs(b->items.size() + 1, 0);
  for (size_t i = 0; i < b->items.size(); ++i) {
    qmt_mol* m = b->items[i].mol;
    QMT_CUDA(cudaMemcpyAsync(sums + i, m->d_scalars.as<double>(), sizeof(double), cudaMemcpyDeviceToHost, s));
    QMT_CUDA(cudaMemcpyAsync(&errs[i], m->d_scalars.as<double>() + 8, sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  if (b->d_err.ptr)
    QMT_CUDA(cudaMemcpyAsync(&errs.back(), b->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  bool bad = false;
  for (size_t i = 0; i < b->items.size(); ++i)
    if (errs[i]) {
      bad = true;
      QMT_CUDA(cudaMemsetAsync(b->items[i].mol->d_scalars.as<double>() + 8, 0, sizeof(int), s));
    }
  if (errs.back()) {
    bad = true;
    QMT_CUDA(cudaMemsetAsync(b->d_err.ptr, 0, sizeof(int), s));
  }
  if (bad) return fail(QMT_CUDA_ERR, "tensor-core density kernel gave up waiting on a barrier");
  for (size_t i = 0; i < b->items.size(); ++i)
    if (!std::isfinite(sums[i])) return fail(QMT_NAN, "non-finite density sum");
  return QMT_OK;
}

int qmt_batch_fused_count(const qmt_batch* b) {
  if (!b) return -1;
  return (int)(b->fused.fdesc.size() + b->fact.fdesc.size());
}

int qmt_batch_factored_count(const qmt_batch* b) {
  if (!b) return -1;
  int n = 0;
  for (const BatchItem& it : b->items) n += it.fact ? 1 : 0;
  return n;
}

qmt_status qmt_batch_destroy(qmt_batch* b) {
  if (!b) return QMT_OK;
  cudaDeviceSynchronize();
  b->fused.d_fdesc.release();
  b->fact.d_fdesc.release();
  b->d_err.release();
  b->phi_hi.release();
  b->phi_lo.release();
  delete b;
  return QMT_OK;
}

}  // extern "C"

extern "C" qmt_status qmt_density_factor_rank(qmt_mol* mol, int* rank_out, void* stream) {
  if (!mol || !rank_out) return qmt::fail(QMT_BAD_ARG, "null argument");
  *rank_out = 0;
  if (mol->fact_prec < 0 || mol->fact_rank <= 0 || !mol->fact_gate) return QMT_OK;
  int gate = 1;
  cudaStream_t s = qmt::as_stream(stream);
  QMT_CUDA(cudaMemcpyAsync(&gate, mol->fact_gate, sizeof(int), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  if (gate == 0) *rank_out = mol->fact_rank;
  return QMT_OK;
}

extern "C" qmt_status qmt_set_density_path(int mode) {
  if (mode < 0 || mode > 3)
    return qmt::fail(QMT_BAD_ARG, "density path must be 0 (auto), 1 (staged), 2 (fused) or 3 (fused, factored)");
  qmt::g_density_path = mode;
  return QMT_OK;
}

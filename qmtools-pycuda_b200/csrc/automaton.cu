// Single-shot neural-network automaton (the GA training path of the reference):
// gpu_automaton_nn_singleshot, kernel_nn_ss.cu:33-178, driven by
// AutomatonSingleShot.Evaluate (qmtools/automaton_nn_singleshot.py:78-183).
//
// For every voxel v and each of its 26 neighbours u (periodic wrap at the grid edge), a small
// multilayer perceptron maps 16 inputs -- the pseudo-field (field 1 of the input grid) at v and
// at u, then parameters 0..13 -- through NL layers of 16 tanh neurons (16 weights + bias each,
// parameters from index 14 on) to one linear output t; the voxel's result is
//     q(v) = field1(v) * sum_u t(v,u)^2 rsqrt(|du|_1) / h * 0.0523448...
// with the neighbours visited in the reference's order and its rounding (float, with the
// grid step and the last factor applied in double as the reference's literals are).  The
// output neuron reads two parameters past the reference's parameter array (indices DNASIZE and
// DNASIZE + 1, 272 NL + 29 and 272 NL + 30); here they are zero, which is what the reference
// kernel reads there.
//
// Design: the parameters travel in the launch itself (a __grid_constant__ block of up to
// 272 * 8 + 32 floats), and the layer count is a template argument, so every weight index is a
// compile-time constant and each FMA takes its weight straight from the constant bank: no
// device allocation, no copy before the launch and no state shared between calls.
#include "mol.cuh"

namespace qmt {

constexpr int NNSS_MAX_LAYERS = 8;
constexpr int NNSS_MAXP = 272 * NNSS_MAX_LAYERS + 32;

struct NNSSParams {
  float w[NNSS_MAXP];
};

// neighbour offsets (dx, dy, dz, |d|_1) in the order of the reference's `deltas` loop
// (kernel_nn_ss.cu:57-60 skip the encodings of a zero step with a sign)
__constant__ int8_t c_nnss_nb[26][4] = {
    {1, 0, 0, 1},   {-1, 0, 0, 1},   {0, 1, 0, 1},   {1, 1, 0, 2},   {-1, 1, 0, 2},   {0, -1, 0, 1},
    {1, -1, 0, 2},  {-1, -1, 0, 2},  {0, 0, 1, 1},   {1, 0, 1, 2},   {-1, 0, 1, 2},   {0, 1, 1, 2},
    {1, 1, 1, 3},   {-1, 1, 1, 3},   {0, -1, 1, 2},  {1, -1, 1, 3},  {-1, -1, 1, 3},  {0, 0, -1, 1},
    {1, 0, -1, 2},  {-1, 0, -1, 2},  {0, 1, -1, 2},  {1, 1, -1, 3},  {-1, 1, -1, 3},  {0, -1, -1, 2},
    {1, -1, -1, 3}, {-1, -1, -1, 3}};

template <int NL>
__device__ __forceinline__ float nnss_transfer(const NNSSParams& P, float v1, float v2) {
  float in[16];
  in[0] = v1;
  in[1] = v2;
#pragma unroll
  for (int k = 0; k < 14; ++k) in[2 + k] = P.w[k];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    float out[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) {
      const int o = 14 + l * 272 + n * 17;
      float acc = 0.f;
#pragma unroll
      for (int i = 0; i < 16; ++i) acc = fmaf(P.w[o + i], in[i], acc);
      acc = acc + P.w[o + 16];
      out[n] = tanhf(acc);
    }
#pragma unroll
    for (int n = 0; n < 16; ++n) in[n] = out[n];
  }
  const int o = 14 + NL * 272;
  float acc = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) acc = fmaf(P.w[o + i], in[i], acc);
  acc = acc + P.w[o + 16];
  return acc * acc;
}

template <int NL>
__global__ void __launch_bounds__(256) nnss_kernel(const __grid_constant__ NNSSParams P, int nx, int ny, int nz,
                                                   double gridstep, const float* __restrict__ qube,
                                                   float* __restrict__ qout) {
  const int64_t plane = (int64_t)nx * ny, npts = plane * nz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < npts;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(idx % nx), y = (int)((idx / nx) % ny), z = (int)(idx / plane);
    const float v1 = __ldg(qube + npts + idx);
    float fin = 0.f;
    for (int k = 0; k < 26; ++k) {
      int xx = x + c_nnss_nb[k][0], yy = y + c_nnss_nb[k][1], zz = z + c_nnss_nb[k][2];
      xx = xx < 0 ? nx - 1 : (xx == nx ? 0 : xx);
      yy = yy < 0 ? ny - 1 : (yy == ny ? 0 : yy);
      zz = zz < 0 ? nz - 1 : (zz == nz ? 0 : zz);
      const float v2 = __ldg(qube + npts + xx + (int64_t)yy * nx + (int64_t)zz * plane);
      const float t = nnss_transfer<NL>(P, v1, v2);
      const float factor = (float)((double)rsqrtf((float)c_nnss_nb[k][3]) / gridstep);
      fin = fmaf(t, factor, fin);
    }
    qout[idx] = (float)((double)(v1 * fin) * 0.05234482976098482);
  }
}

template <int NL>
static qmt_status launch_nnss(const NNSSParams& P, int nx, int ny, int nz, double gs, const float* q, float* out,
                              cudaStream_t s) {
  const int64_t npts = (int64_t)nx * ny * nz;
  const int blocks = (int)std::min<int64_t>((npts + 255) / 256, (int64_t)sm_count() * 8);
  nnss_kernel<NL><<<blocks, 256, 0, s>>>(P, nx, ny, nz, gs, q, out);
  QMT_CHECK_LAUNCH("nnss_kernel");
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_nn_singleshot(int nx, int ny, int nz, double gridstep, const float* qube_dev,
                                        float* qout_dev, const float* params, int nparams, int nlayers,
                                        void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !qube_dev || !qout_dev || !params || !(gridstep > 0))
    return fail(QMT_BAD_ARG, "bad automaton arguments");
  if (nlayers < 1 || nlayers > NNSS_MAX_LAYERS)
    return fail(QMT_BAD_ARG, "automaton supports 1 to 8 hidden layers");
  const int need = 272 * nlayers + 29;   // reference DNASIZE: 16*16*NL + 16*NL + 17 + 12
  if (nparams != need) return fail(QMT_BAD_ARG, "automaton parameter count must be 272 * nlayers + 29");
  NNSSParams P;
  for (int i = 0; i < NNSS_MAXP; ++i) P.w[i] = i < nparams ? params[i] : 0.f;
  cudaStream_t s = as_stream(stream);
  switch (nlayers) {
    case 1: return launch_nnss<1>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 2: return launch_nnss<2>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 3: return launch_nnss<3>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 4: return launch_nnss<4>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 5: return launch_nnss<5>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 6: return launch_nnss<6>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    case 7: return launch_nnss<7>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
    default: return launch_nnss<8>(P, nx, ny, nz, gridstep, qube_dev, qout_dev, s);
  }
}

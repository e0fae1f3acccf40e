// FFT Poisson solve (in-house FFT) -- entry point.
#include "mol.cuh"

using namespace qmt;

extern "C" qmt_status qmt_fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step, float ox, float oy,
                                      float oz, float sigma, float cutoff, int padded, const float* q_dev,
                                      float* out_dev, void* stream) {
  (void)mol; (void)nx; (void)ny; (void)nz; (void)step; (void)ox; (void)oy; (void)oz; (void)sigma;
  (void)cutoff; (void)padded; (void)q_dev; (void)out_dev; (void)stream;
  return fail(QMT_BAD_ARG, "FFT Poisson solve not built");
}

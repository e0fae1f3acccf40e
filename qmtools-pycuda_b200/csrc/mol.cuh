// Host-side molecule handle and device buffers.
#pragma once

#include <vector>

#include "gto.cuh"
#include "qmt_common.cuh"

namespace qmt {

// Owned device allocation that only grows.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  qmt_status reserve(size_t n);
  void release();
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

int sm_count();

}  // namespace qmt

struct qmt_mol {
  int natoms = 0, norbs = 0, npad = 0, nshells = 0;
  double qtot = 0;
  std::vector<int> types;
  std::vector<float> coords;
  std::vector<qmt::Shell> shells;
  std::vector<int> atom_shell;  // shells of atom a are [atom_shell[a], atom_shell[a+1])
  std::vector<float> alpha, coeff;
  std::vector<double> alpha64, coeff64;
  std::vector<double> P64;      // symmetric (from the lower triangle), npad x npad; host copy built on
                                // demand from the staged matrix (host_P64), the device copies by a kernel
  bool p64_host_valid = false;
  const std::vector<double>& host_P64();
  std::vector<float> dm_host;   // the caller's density matrix as given (latest upload)
  qmt::DevBuf d_dm_raw;         // the matrix as given, norbs x norbs
  bool basis_ops_ready = false; // column scales and producer tables (depend on the basis only)
  qmt::DevBuf d_gscale;         // device {max, 2^g, 2^-g} of the split density matrix
  std::vector<double> fbound;   // per-function bound on |phi|

  qmt::DevBuf d_atom_shell;
  int fused_prec = -1;          // precision of the fused-path operands below
  qmt::DevBuf d_fused_B;        // scaled density matrix pieces for the fused path (hi then lo)
  qmt::DevBuf d_split_scale;    // 2^-s_j per function for the device split of the density matrix
  std::vector<double> split_inv; // the same on the host
  int fact_prec = -1;           // precision of the factored-path operands below (-1: not built)
  int fact_rank = 0;            // rank of the density-matrix factor P = L L^T (0: not factored)
  std::vector<double> fact_Lr_host, fact_d_host;   // host work buffers of the factorisation
  int fact_r16 = 0;             // the rank rounded up to 16 (the MMA N)
  qmt::DevBuf d_fact_B;         // scaled factor pieces, K-step blocks of fact_r16 rows (hi then lo)
  qmt::DevBuf d_fact_L;         // the factor (FP64, row by row) and a flag, for the residual check
  int fact_rows_prec = -1;      // precision of d_fact_Bs (-1: not built for the current factor)
  qmt::DevBuf d_fact_Bs;        // the factor as the staged path's B operand (fact_rows_kernel)
  const int* fact_gate = nullptr; // that flag: 0 when the factor reproduces P, 1 when it does not
  qmt::DevBuf d_fact_scale;     // per factor column k: 2^-2h_k, 2^h_k (FP64), then 2^-h_k (FP32)
  qmt::DevBuf d_fused_tab;      // fused path: packed shell records, then (alpha, scaled coefficient) pairs
  qmt::DevBuf d_coords, d_types, d_shells, d_alpha, d_coeff, d_alpha64, d_coeff64;
  qmt::DevBuf d_P32, d_P64;
  // tensor-core operands
  int tc_prec = -1;             // precision the operands below were built for
  qmt::DevBuf d_tc_P;           // split, scaled density matrix (hi then lo)
  qmt::DevBuf d_Phi_hi, d_Phi_lo;
  // scratch
  qmt::DevBuf d_partials, d_scalars, d_work;
  // analytic potential: primitive-pair table (FP64), and the FP32 kernels' tables (gto.cu)
  bool gto_ready = false;
  int gto_npairs = 0;
  size_t gto_doff_bytes = 0;
  qmt::DevBuf d_pairs;
  qmt::DevBuf d_pairs32;        // storage of gto32 (device pointers into it)
  qmt::Gto32Tables gto32{};
  std::vector<double> gto32_work;   // cumulative estimated work of the FP32 off-site pairs
  std::vector<double> gto64_work;   // and of the FP64 ones
  qmt::DevBuf d_gto_part;       // FP64 partial sums of the off-site pair slices

  ~qmt_mol();
  qmt_status upload_coords(const float* c, cudaStream_t s);
  qmt_status upload_dm(const float* dm, cudaStream_t s);
  qmt::MolView view() const;
};

// Library state, status strings and the molecule handle (device-resident basis,
// coordinates and density matrix).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "mol.cuh"

namespace qmt {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

qmt_status fail(qmt_status code, const std::string& msg) {
  set_error(msg);
  return code;
}

qmt_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return QMT_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return QMT_NO_DEVICE;
  return QMT_CUDA_ERR;
}

qmt_status DevBuf::reserve(size_t n) {
  if (n <= bytes) return QMT_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  bytes = n;
  return QMT_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

static std::atomic<uint64_t> g_launches{0};
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

constexpr uint64_t kDefaultWaitNs = 2000000000ull;   // 2 s
static std::atomic<uint64_t> g_wait_ns{kDefaultWaitNs};
uint64_t wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }

int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Bound on max_r |phi| for a shell: s: sum|c|; p: sum|c| max_r r e^{-a r^2}; d: sum|c| max r^2 e^{-a r^2},
// times the largest angular constant.  Used only to pick power-of-two operand scales.
static double shell_bound(int L, const float* al, const float* co, int n) {
  double b = 0;
  for (int k = 0; k < n; ++k) {
    const double a = al[k], c = std::fabs((double)co[k]);
    if (L == 0) b += c;
    else if (L == 1) b += c / std::sqrt(2.0 * std::exp(1.0) * a);
    else b += c / (std::exp(1.0) * a);
  }
  const double ang = L == 0 ? YS : (L == 1 ? YP : 2 * YD0 + YD1);
  return b * ang;
}

}  // namespace qmt

using namespace qmt;

qmt_mol::~qmt_mol() {
  for (DevBuf* b : {&d_coords, &d_types, &d_shells, &d_alpha, &d_coeff, &d_alpha64, &d_coeff64,
                    &d_P32, &d_P64, &d_Phi_hi, &d_Phi_lo, &d_tc_P, &d_partials,
                    &d_scalars, &d_pairs, &d_work, &d_atom_shell, &d_fused_B, &d_fact_B, &d_fact_scale, &d_fact_L, &d_fact_Bs,
                    &d_fused_tab, &d_split_scale,
                    &d_dm_raw, &d_gscale, &d_pairs32, &d_gto_part})
    b->release();
}

namespace qmt {
// P (npad x npad, FP64 and FP32) symmetric from the lower triangle of the caller's matrix,
// zero in the padding.
__global__ void sym_dm_kernel(const float* __restrict__ raw, int n, int np, double* __restrict__ P64,
                              float* __restrict__ P32) {
  const int64_t tot = (int64_t)np * np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / np), c = (int)(i - (int64_t)r * np);
    float v = 0.f;
    if (r < n && c < n) v = c <= r ? raw[(size_t)r * n + c] : raw[(size_t)c * n + r];
    P64[i] = v;
    P32[i] = v;
  }
}
}  // namespace qmt

const std::vector<double>& qmt_mol::host_P64() {
  if (!p64_host_valid) {
    const int n = norbs, np = npad;
    P64.assign((size_t)np * np, 0.0);
    for (int p = 0; p < n; ++p)
      for (int q = 0; q <= p; ++q) {
        const double v = dm_host[(size_t)p * n + q];
        P64[(size_t)p * np + q] = v;
        P64[(size_t)q * np + p] = v;
      }
    p64_host_valid = true;
  }
  return P64;
}

static qmt_status upload(DevBuf& b, const void* src, size_t n, cudaStream_t s) {
  qmt_status st = b.reserve(n);
  if (st) return st;
  QMT_CUDA(cudaMemcpyAsync(b.ptr, src, n, cudaMemcpyHostToDevice, s));
  return QMT_OK;
}

qmt_status qmt_mol::upload_coords(const float* c, cudaStream_t s) {
  coords.assign(c, c + 3 * natoms);
  for (float v : coords)
    if (!std::isfinite(v)) return fail(QMT_NAN, "non-finite coordinate");
  return upload(d_coords, coords.data(), coords.size() * sizeof(float), s);
}

qmt_status qmt_mol::upload_dm(const float* dm, cudaStream_t s) {
  const int n = norbs, np = npad;
  const size_t bytes = (size_t)n * n * sizeof(float);
  // the lower triangle is the matrix (the reference reads it that way)
  for (int p = 0; p < n; ++p) {
    const float* row = dm + (size_t)p * n;
    for (int q = 0; q <= p; ++q)
      if (!std::isfinite(row[q])) return fail(QMT_NAN, "non-finite density matrix entry");
  }
  // host copy (the analytic-potential path reads it); the pageable upload returns once the data
  // is staged, so the copy may be overwritten by the next call without synchronisation
  dm_host.assign(dm, dm + (size_t)n * n);
  p64_host_valid = false;
  qmt_status st;
  if ((st = d_dm_raw.reserve(bytes)) || (st = d_P64.reserve((size_t)np * np * sizeof(double))) ||
      (st = d_P32.reserve((size_t)np * np * sizeof(float))))
    return st;
  QMT_CUDA(cudaMemcpyAsync(d_dm_raw.ptr, dm_host.data(), bytes, cudaMemcpyHostToDevice, s));
  const int64_t tot = (int64_t)np * np;
  const int blocks = (int)std::min<int64_t>((tot + 255) / 256, (int64_t)sm_count() * 4);
  sym_dm_kernel<<<std::max(blocks, 1), 256, 0, s>>>(d_dm_raw.as<float>(), n, np, d_P64.as<double>(),
                                                    d_P32.as<float>());
  QMT_CHECK_LAUNCH("sym_dm_kernel");
  tc_prec = -1;
  fused_prec = -1;
  fact_prec = -1;
  gto_ready = false;
  return QMT_OK;
}

// (Re)initialises `m` for a molecule; device buffers already held by `m` are reused.
static qmt_status mol_init(qmt_mol* m, int natoms, const int32_t* types, const float* coords, int norbs,
                           const int16_t* almos, int nparams, const float* alphas, const float* coeffs,
                           const float* dm, cudaStream_t s) {
  if (!types || !coords || !almos || !alphas || !coeffs || !dm) return fail(QMT_BAD_ARG, "null argument");
  if (natoms <= 0 || norbs <= 0 || nparams <= 0) return fail(QMT_BAD_ARG, "empty molecule");
  m->shells.clear();
  m->alpha.clear();
  m->coeff.clear();
  m->tc_prec = -1;
  m->fused_prec = -1;
  m->fact_prec = -1;
  m->gto_ready = false;
  m->basis_ops_ready = false;
  m->natoms = natoms;
  m->norbs = norbs;
  m->npad = (norbs + 31) / 32 * 32;
  m->types.assign(types, types + natoms);
  m->qtot = 0;
  for (int a = 0; a < natoms; ++a) m->qtot += types[a];
  // group the per-function ALMO rows into shells (qmtools/qmtools.py:163-171)
  static const int mord[3][5] = {{0}, {0, 1, -1}, {0, 1, -1, 2, -2}};
  int f = 0;
  m->fbound.assign(m->npad, 0.0);
  while (f < norbs) {
    const int a = almos[4 * f + 0], L = almos[4 * f + 1], so = almos[4 * f + 3];
    if (a < 0 || a >= natoms) {
      return fail(QMT_BAD_ARG, "ALMO atom index out of range");
    }
    if (L < 0 || L > MAX_L) {
      return fail(QMT_UNSUPPORTED_L, "basis shell with L > 2");
    }
    if (f + 2 * L + 1 > norbs || so < 0 || so + MAXAOC > nparams) {
      return fail(QMT_BAD_ARG, "truncated shell in ALMO table");
    }
    for (int k = 0; k < 2 * L + 1; ++k) {
      const int16_t* r = almos + 4 * (f + k);
      if (r[0] != a || r[1] != L || r[3] != so || r[2] != mord[L][k]) {
          return fail(QMT_BAD_ARG, "ALMO rows of a shell must follow the m order of the basis");
      }
    }
    Shell sh{};
    sh.atom = a;
    sh.L = L;
    sh.func = f;
    sh.prim = (int)m->alpha.size();
    int np = 0;
    for (int k = 0; k < MAXAOC; ++k) {
      if (coeffs[so + k] == 0.0f) continue;  // padded slots contribute exactly zero
      m->alpha.push_back(alphas[so + k]);
      m->coeff.push_back(coeffs[so + k]);
      ++np;
    }
    sh.nprim = np;
    if (!m->shells.empty()) {
      const Shell& pv = m->shells.back();
      bool same = pv.atom == a && pv.nprim == np && np <= 8;
      for (int k = 0; same && k < np; ++k) same = m->alpha[pv.prim + k] == m->alpha[sh.prim + k];
      sh.same_exp = same ? 1 : 0;
    }
    const double bnd = shell_bound(L, m->alpha.data() + sh.prim, m->coeff.data() + sh.prim, np);
    for (int k = 0; k < 2 * L + 1; ++k) m->fbound[f + k] = bnd;
    m->shells.push_back(sh);
    f += 2 * L + 1;
  }
  m->nshells = (int)m->shells.size();
  m->atom_shell.assign(natoms + 1, 0);
  for (int a = 0, sidx = 0; a <= natoms; ++a) {
    while (sidx < m->nshells && m->shells[sidx].atom < a) ++sidx;
    m->atom_shell[a] = sidx;
  }
  for (int sidx = 1; sidx < m->nshells; ++sidx)
    if (m->shells[sidx].atom < m->shells[sidx - 1].atom) {
      return fail(QMT_BAD_ARG, "basis functions must be grouped by atom in atom order");
    }
  m->alpha64.assign(m->alpha.begin(), m->alpha.end());
  m->coeff64.assign(m->coeff.begin(), m->coeff.end());
  if (m->alpha.empty()) {
    m->alpha.push_back(0.f);
    m->coeff.push_back(0.f);
    m->alpha64.push_back(0.);
    m->coeff64.push_back(0.);
  }
  qmt_status st;
  if ((st = m->upload_coords(coords, s)) ||
      (st = upload(m->d_types, m->types.data(), natoms * sizeof(int), s)) ||
      (st = upload(m->d_shells, m->shells.data(), m->shells.size() * sizeof(Shell), s)) ||
      (st = upload(m->d_atom_shell, m->atom_shell.data(), m->atom_shell.size() * sizeof(int), s)) ||
      (st = upload(m->d_alpha, m->alpha.data(), m->alpha.size() * sizeof(float), s)) ||
      (st = upload(m->d_coeff, m->coeff.data(), m->coeff.size() * sizeof(float), s)) ||
      (st = upload(m->d_alpha64, m->alpha64.data(), m->alpha64.size() * sizeof(double), s)) ||
      (st = upload(m->d_coeff64, m->coeff64.data(), m->coeff64.size() * sizeof(double), s)) ||
      (st = m->upload_dm(dm, s))) {
    return st;
  }
  // device scratch for sums and the sticky kernel error flag, cleared once here
  if ((st = m->d_scalars.reserve(64 * sizeof(double)))) {
    return st;
  }
  QMT_CUDA(cudaMemsetAsync(m->d_scalars.ptr, 0, 64 * sizeof(double), s));
  QMT_CUDA(cudaStreamSynchronize(s));
  return QMT_OK;
}


extern "C" {

const char* qmt_last_error(void) { return g_last_error.c_str(); }

int qmt_abi_version(void) { return 1; }

uint64_t qmt_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

qmt_status qmt_set_wait_limit_ns(uint64_t ns) {
  if (ns > 60000000000ull) return fail(QMT_BAD_ARG, "wait limit above 60 s");
  g_wait_ns.store(ns ? ns : kDefaultWaitNs, std::memory_order_relaxed);
  return QMT_OK;
}

qmt_status qmt_init(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(QMT_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= n) return fail(QMT_BAD_ARG, "device index out of range");
  QMT_CUDA(cudaSetDevice(device));
  int major = 0;
  QMT_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major != 10) return fail(QMT_NO_DEVICE, "libqmtools_b200 needs an sm_100 device");
  return QMT_OK;
}

qmt_status qmt_mol_create(int natoms, const int32_t* types, const float* coords, int norbs,
                          const int16_t* almos, int nparams, const float* alphas,
                          const float* coeffs, const float* dm, void* stream, qmt_mol** out) {
  if (!out) return fail(QMT_BAD_ARG, "null argument");
  *out = nullptr;
  auto* m = new qmt_mol();
  const qmt_status st = mol_init(m, natoms, types, coords, norbs, almos, nparams, alphas, coeffs, dm,
                                 as_stream(stream));
  if (st) {
    delete m;
    return st;
  }
  *out = m;
  return QMT_OK;
}

qmt_status qmt_mol_reset(qmt_mol* mol, int natoms, const int32_t* types, const float* coords, int norbs,
                         const int16_t* almos, int nparams, const float* alphas, const float* coeffs,
                         const float* dm, void* stream) {
  if (!mol) return fail(QMT_BAD_ARG, "null argument");
  return mol_init(mol, natoms, types, coords, norbs, almos, nparams, alphas, coeffs, dm, as_stream(stream));
}

qmt_status qmt_mol_set_coords(qmt_mol* mol, const float* coords, void* stream) {
  if (!mol || !coords) return fail(QMT_BAD_ARG, "null argument");
  cudaStream_t s = as_stream(stream);
  // the pageable upload returns once the data is staged, so no synchronisation is needed
  qmt_status st = mol->upload_coords(coords, s);
  if (st) return st;
  mol->gto_ready = false;
  return QMT_OK;
}

qmt_status qmt_mol_set_dm(qmt_mol* mol, const float* dm, void* stream) {
  if (!mol || !dm) return fail(QMT_BAD_ARG, "null argument");
  return mol->upload_dm(dm, as_stream(stream));
}

qmt_status qmt_mol_destroy(qmt_mol* mol) {
  if (!mol) return QMT_OK;
  cudaDeviceSynchronize();
  delete mol;
  return QMT_OK;
}

}  // extern "C"

MolView qmt_mol::view() const {
  MolView v;
  v.natoms = natoms;
  v.nshells = nshells;
  v.norbs = norbs;
  v.npad = npad;
  v.coords = (const float*)d_coords.ptr;
  v.types = (const int*)d_types.ptr;
  v.shells = (const Shell*)d_shells.ptr;
  v.atom_shell = (const int*)d_atom_shell.ptr;
  v.alpha = (const float*)d_alpha.ptr;
  v.coeff = (const float*)d_coeff.ptr;
  v.alpha64 = (const double*)d_alpha64.ptr;
  v.coeff64 = (const double*)d_coeff64.ptr;
  return v;
}

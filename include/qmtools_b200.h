/*
 * qmtools_b200.h -- C ABI of libqmtools_b200.so, the sm_100a implementation of the
 * QMTools grid hot path (electron density, Hartree potential, nuclear terms).
 *
 * The reference (fullmetalfelix/QMTools-pycuda) has no native ABI: its Python facade
 * `QMTools` (qmtools/qmtools.py:2320-2831) JIT-compiles CUDA C with PyCUDA and launches
 * kernels with `prepared_call`.  Each entry point below replaces one of those facade
 * methods (or the kernel it launches); the citation on each line names it.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Pointers named *_dev are device pointers; every
 *     other pointer is host memory and is copied in before the call returns.
 *   - Grids are float32, x-fastest (idx = x + y*nx + z*nx*ny), the reference layout
 *     (qmtools/cuda/kernel_density.cu:151-154).  Lengths in bohr unless stated.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls are asynchronous on that stream unless they return a host scalar.
 *   - Every function returns a qmt_status; qmt_last_error() gives a message for the
 *     last failure on the calling thread.  Nothing exits or aborts.
 *   - A qmt_mol handle owns its device memory; qmt_mol_destroy frees it.  Handles may be
 *     used from different host threads as long as one handle is not used concurrently.
 */
#ifndef QMTOOLS_B200_H
#define QMTOOLS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int qmt_status;
enum {
  QMT_OK = 0,
  QMT_BAD_ARG = 1,        /* invalid argument or shape                         */
  QMT_OOM = 2,            /* device allocation failed                          */
  QMT_NOT_CONVERGED = 3,  /* iterative solver stopped at its sweep cap         */
  QMT_NAN = 4,            /* non-finite value in an input or a result          */
  QMT_UNSUPPORTED_L = 5,  /* basis shell with angular momentum > 2             */
  QMT_CUDA_ERR = 6,       /* CUDA runtime error                                */
  QMT_NO_DEVICE = 7       /* no usable sm_100 device                           */
};

/* Precision of the density contraction T = Phi * P (row-dot and sums stay FP32/FP64). */
enum {
  QMT_PREC_FP64 = 0,      /* SIMT FP64                                                  */
  QMT_PREC_FP32 = 1,      /* SIMT FP32 (the plain path)                                 */
  QMT_PREC_TF32 = 2,      /* tcgen05 kind::tf32, one product                            */
  QMT_PREC_TF32X3 = 3,    /* tcgen05 kind::tf32, hi/lo split, 3 products                */
  QMT_PREC_BF16 = 4,      /* tcgen05 kind::f16 (bf16), one product                      */
  QMT_PREC_BF16X3 = 5,    /* tcgen05 kind::f16 (bf16), hi/lo split, 3 products          */
  QMT_PREC_FP16X3 = 6     /* tcgen05 kind::f16 (fp16), power-of-two scaled hi/lo split, */
                          /* 3 products                                                 */
};

typedef struct qmt_mol qmt_mol;

/* ---- library ------------------------------------------------------------------------ */
const char* qmt_last_error(void);
int qmt_abi_version(void);
/* Selects the device for this host thread and checks it is sm_100. */
qmt_status qmt_init(int device);
/* Number of kernel launches this library has made in the process so far (new; no reference
 * counterpart): read it before and after a region to count the region's launches. */
uint64_t qmt_launch_count(void);
/* Limit, in nanoseconds, of every bounded wait inside the kernels (grid barriers of the Jacobi
 * solve, pipeline barriers of the tensor-core density kernels); 0 restores the default of 2 s.
 * A wait that runs out makes the kernel return early with an error flag that the host reads
 * (QMT_CUDA_ERR), leaving the context usable.  Process-wide; new, for tests of those paths. */
qmt_status qmt_set_wait_limit_ns(uint64_t ns);

/* ---- molecule (BasisSet + Molecule device upload) ------------------------------------ */
/* Replaces the uploads of BasisSet.__init__ (qmtools/qmtools.py:97-103) and
 * Molecule.__init__ (qmtools/qmtools.py:174-178).  Inputs are the reference's own host
 * arrays: types[natoms] int32, coords[natoms*3] float32 bohr, almos[norbs*4] int16
 * (atom, L, m, shellOffset), alphas/coeffs[nparams] float32 padded to 20 per shell,
 * dm[norbs*norbs] float32 row-major.  Only the lower triangle p >= q of dm is read,
 * as the reference kernels do (kernel_density.cu:87, kernel_hartree.cu:353). */
qmt_status qmt_mol_create(int natoms, const int32_t* types, const float* coords,
                          int norbs, const int16_t* almos,
                          int nparams, const float* alphas, const float* coeffs,
                          const float* dm, void* stream, qmt_mol** out);
/* Re-initialises an existing handle for another molecule (same arguments as qmt_mol_create),
 * reusing its device allocations: a serving loop keeps one handle per slot and never calls
 * cudaMalloc/cudaFree in steady state.  New entry point. */
qmt_status qmt_mol_reset(qmt_mol* mol, int natoms, const int32_t* types, const float* coords,
                         int norbs, const int16_t* almos, int nparams, const float* alphas,
                         const float* coeffs, const float* dm, void* stream);
/* Molecule.Translate upload (qmtools/qmtools.py:182-188): new coords[natoms*3] bohr.
 * Stream-ordered: returns once the host array has been copied; later calls on `stream` see it. */
qmt_status qmt_mol_set_coords(qmt_mol* mol, const float* coords, void* stream);
/* New density matrix (same norbs).  Stream-ordered like qmt_mol_set_coords: the caller's array
 * may be reused on return; the device operands are re-derived on `stream`. */
qmt_status qmt_mol_set_dm(qmt_mol* mol, const float* dm, void* stream);
qmt_status qmt_mol_destroy(qmt_mol* mol);
/* FP64 Tr(P S) with the analytic overlap S, computed on the device (new; no reference
 * counterpart -- the electron count the density grid must integrate to, before x2). */
qmt_status qmt_mol_trace_ps(qmt_mol* mol, double* trace_out, void* stream);

/* ---- density -------------------------------------------------------------------------- */
/* QMTools.Compute_density (qmtools/qmtools.py:2381-2430) with gpu_densityqube_shmem_subgrid
 * (kernel_density.cu:34-155): q_v = 2 h^3 s^-3 sum_sub sum_pq P_pq phi_p phi_q at voxel-centre
 * sub-points, into qube_dev[nx*ny*nz].  If rescale != 0 the grid is then scaled so that its
 * sum equals the total nuclear charge (qmtools/qmtools.py:2419-2424), on the device.
 * sum_out (host, may be NULL) receives the FP64 sum before rescaling; with sum_out the call
 * blocks and reports kernel failures, without it the call is fully asynchronous on `stream`
 * (capturable in a CUDA graph once the molecule's operands exist) and failures are reported
 * by the next call on this molecule that returns a sum. */
qmt_status qmt_density(qmt_mol* mol, int nx, int ny, int nz, float step,
                       float ox, float oy, float oz, int subgrid, int precision,
                       int rescale, float* qube_dev, double* sum_out, void* stream);

/* Selects the tensor-core density implementation (new; process-wide): 0 = automatic (fused
 * when the contraction is fp16/bf16 and N <= 320, staged otherwise; with the factored density
 * matrix when it has one), 1 = staged (basis values through HBM), 2 = fused (basis values
 * stay in shared memory), 3 = the factored density matrix: P = L L^T from a pivoted Cholesky
 * factorisation (FP64, on the host, once per matrix) and rho = sum_k (Phi L)_k^2, which needs
 * rank(P) columns instead of N -- for a positive semi-definite P of rank at most min(128, N/2)
 * (an SCF density matrix has the rank of its occupied orbitals), on the fused path when N <= 320
 * and the rank <= 64, else on the staged path (fp16 / bf16); QMT_BAD_ARG when the factorisation
 * finds P indefinite or of higher rank.  What the factor leaves out is checked on
 * the device (max |P - L L^T| <= 2e-7 max |P|), which runs the unfactored kernel instead when the
 * check fails, without a host round trip. */
qmt_status qmt_set_density_path(int mode);

/* Rank of the factor the last density call on `mol` contracted with (new): 0 when it ran the
 * unfactored kernel.  Synchronises `stream` (the device-side check decides). */
qmt_status qmt_density_factor_rank(qmt_mol* mol, int* rank_out, void* stream);

/* ---- batches of molecules (new; no reference counterpart) ---------------------------- */
/* The reference evaluates one molecule per Compute_density call (qmtools/qmtools.py:2381-2430).
 * A batch evaluates the densities of many molecules together: the molecules whose contraction
 * takes the fused path share one persistent launch over all their tiles (one for those with a
 * factored density matrix, one for the others); the rest (N > 320 or tf32) get the staged path,
 * one molecule after another; then each grid is summed and, with rescale, scaled to its nuclear
 * charge.  Inputs: shapes[3 i + (0,1,2)] = nx, ny, nz and geoms[4 i + (0,1,2,3)] = step, ox, oy,
 * oz (bohr) of molecule i; qube_devs[i] its grid (device, nx ny nz floats, x-fastest); paths[i]
 * 0 = automatic (fused or staged), 1 = staged, 2 = fused, 3 = fused or staged with the factored
 * density matrix when it has one that passes its check (as qmt_set_density_path mode 3), else
 * unfactored (NULL: automatic).  A factored molecule's factor is built at creation: refresh != 0
 * is refused for a batch that holds one.
 * qmt_batch_create builds every operand (it synchronises `stream`); qmt_batch_density then
 * allocates nothing and is fully asynchronous, so a CUDA graph can capture it.  With refresh != 0
 * it first re-derives each molecule's split density matrix on the device from the matrix last
 * uploaded with qmt_mol_set_dm, so a captured graph follows new uploads.  The molecules must not
 * be used by other calls while a batch call on them is in flight, and must outlive the batch. */
typedef struct qmt_batch qmt_batch;
qmt_status qmt_batch_create(int nmol, qmt_mol* const* mols, const int32_t* shapes, const float* geoms,
                            int subgrid, int precision, const int32_t* paths, float* const* qube_devs,
                            void* stream, qmt_batch** out);
qmt_status qmt_batch_density(qmt_batch* batch, int rescale, int refresh, void* stream);
/* FP64 grid sums before rescaling, sums[nmol] (host); synchronous; reports and clears the kernels'
 * barrier-timeout flags (QMT_CUDA_ERR). */
qmt_status qmt_batch_sums(qmt_batch* batch, double* sums, void* stream);
/* Molecules of the batch on the fused launches, and those with a factored density matrix (fused
 * or staged) (-1 for NULL). */
int qmt_batch_fused_count(const qmt_batch* batch);
int qmt_batch_factored_count(const qmt_batch* batch);
qmt_status qmt_batch_destroy(qmt_batch* batch);

/* ---- analytic GTO potential --------------------------------------------------------- */
/* QMTools.Compute_hartree (qmtools/qmtools.py:2436-2489) with gpu_hartree_GTO
 * (kernel_hartree.cu:288-869): V(C) = -2 sum_pq P_pq (phi_p phi_q | 1/|r-C|) + sum_A Z_A/|C-R_A|
 * at voxel corners C = origin + i h, written into v_dev[nx*ny*nz] (a.u.). */
qmt_status qmt_hartree_gto(qmt_mol* mol, int nx, int ny, int nz, float step,
                           float ox, float oy, float oz, float* v_dev, void* stream);
/* Same potential at npts arbitrary points pts_dev[npts*3] (bohr); used for Dirichlet
 * boundaries.  New entry point. */
qmt_status qmt_hartree_gto_points(qmt_mol* mol, int npts, const float* pts_dev,
                                  float* v_dev, void* stream);
/* Same potential on the outer shell of an nx*ny*nz grid at voxel centres
 * origin + (i + 1/2) h, written into those voxels of v_dev (interior untouched); the
 * Dirichlet boundary of qmt_jacobi_dirichlet.  New entry point. */
qmt_status qmt_hartree_gto_boundary(qmt_mol* mol, int nx, int ny, int nz, float step,
                                    float ox, float oy, float oz, float* v_dev, void* stream);
/* Arithmetic of the three analytic-potential entry points above (new; process-wide):
 * QMT_PREC_FP32 (default) is mixed: the largest off-site primitive pairs (95% of the total size)
 * and the on-site pairs, the near field and the nuclei in FP64; the other off-site pairs in FP32
 * (asymptotic Boys functions where p |P - C|^2 >= 30), less those below 1e-11 of the total
 * size, summed in FP64; QMT_PREC_FP64 keeps every pair and every operation in FP64 (the checker
 * of the mixed kernels). */
qmt_status qmt_set_gto_precision(int precision);

/* ---- Jacobi relaxation ---------------------------------------------------------------- */
/* QMTools.Compute_hartree_iter (qmtools/qmtools.py:2497-2573) with gpu_hartree_iteration
 * (kernel_hartree.cu:85-171): sweeps V' = (sum of 6 neighbours - Q/h)/6 with a zero outer
 * shell, Q = rho_dev.  v_dev holds the start value and receives the result; t_dev is a
 * scratch grid of the same size.  Every check_every sweep pairs the FP64 sum |V - T| is
 * compared with tol (the reference checks every 100 pairs); the solve stops there or at
 * max_sweeps (returning QMT_NOT_CONVERGED).  sweeps_out/delta_out are host, may be NULL. */
qmt_status qmt_jacobi(int nx, int ny, int nz, float step, const float* rho_dev,
                      float* v_dev, float* t_dev, int max_sweeps, int check_every,
                      double tol, int* sweeps_out, double* delta_out, void* stream);
/* Physical-unit Jacobi (new): lap V = -4 pi rho (a.u.), Dirichlet values taken from the
 * outer shell of v_dev (e.g. from qmt_hartree_gto_points), interior start value from v_dev.
 * Same stopping rule; FP64 residual norm. */
qmt_status qmt_jacobi_dirichlet(int nx, int ny, int nz, float step, const float* rho_dev,
                                float* v_dev, float* t_dev, int max_sweeps, int check_every,
                                double tol, int* sweeps_out, double* delta_out, void* stream);
/* Selects the Jacobi implementation of the two calls above (new; process-wide): 0 = automatic
 * (the cluster kernel for qmt_jacobi_dirichlet where it applies, else the grid-barrier kernel),
 * 1 = one persistent kernel with a grid barrier between sweeps, 2 = one 16-CTA thread-block
 * cluster holding the field in shared memory (nx % 4 == 0, nx * ny <= 4096, nz <= 64;
 * QMT_BAD_ARG where it does not apply).  Both give identical grids; the residual sums may differ
 * in the last bits. */
qmt_status qmt_set_jacobi_path(int mode);

/* ---- FFT Poisson ---------------------------------------------------------------------- */
/* QMTools.Compute_hartree_fft (qmtools/qmtools.py:2578-2639) with gpu_add_nuclear_charge
 * (kernel_fft.cu:23-79) and gpu_poisson_frequency_solve (kernel_fft.cu:82-107).
 * q_dev: electron grid (x-fastest).  out_dev receives the potential in volts, C-order
 * (i*ny*nz + j*nz + k) like the reference's returned array.
 * padded = 0: the reference's periodic solve; padded = 1: free-space solve on a zero-padded
 * grid of at least 2n per axis with the Hockney Green's function (new). */
qmt_status qmt_fft_poisson(qmt_mol* mol, int nx, int ny, int nz, float step,
                           float ox, float oy, float oz, float sigma, float cutoff,
                           int padded, const float* q_dev, float* out_dev, void* stream);
/* The free-space solve of qmt_fft_poisson(padded = 1) with explicit padded lengths mx >= 2 nx,
 * my >= 2 ny, mz >= 2 nz (lengths whose prime factors are at most 127); new, for callers that
 * pick the transform lengths (the batch autotuner).  The potential does not depend on them
 * beyond FP32 rounding. */
qmt_status qmt_fft_poisson_padded(qmt_mol* mol, int nx, int ny, int nz, float step,
                                  float ox, float oy, float oz, float sigma, float cutoff,
                                  int mx, int my, int mz, const float* q_dev, float* out_dev,
                                  void* stream);

/* ---- grid utilities and nuclear fields ----------------------------------------------- */
/* QMTools.Compute_qtot / gpu_total (qmtools/qmtools.py:2796-2803, kernel_utils.cu:68-98),
 * deterministic FP64 sum of n floats. */
qmt_status qmt_grid_total(const float* q_dev, int64_t n, double* out, void* stream);
/* Grid total that allocates nothing (no counterpart in the reference).  Same result as
 * qmt_grid_total, for callers that must not allocate device memory: a host framework that
 * owns all device memory through its own pool, or a serving loop that cannot accept the
 * device-wide synchronisation cudaMalloc and cudaFree can cause.  The partial sums go to a
 * fixed 32 KiB array compiled into the library, so n is limited to 33,554,432 points
 * (QMT_BAD_ARG beyond that).  The first call on each device looks up that array's device
 * address; make that first call before any stream capture begins.  All calls share the
 * array; every slot a call reads it writes first, so nothing must be cleared, but calls
 * whose work overlaps on the GPU (other streams, other host threads) race on it: order them.
 * The looked-up address is kept for the life of the process; a cudaDeviceReset in between is
 * not supported.  Synchronous like qmt_grid_total. */
qmt_status qmt_grid_total_noalloc(const float* q_dev, int64_t n, double* out, void* stream);
/* QMTools.Compute_qscale / gpu_rescale (qmtools/qmtools.py:2808-2813, kernel_utils.cu:54-65). */
qmt_status qmt_grid_scale(float* q_dev, int64_t n, float factor, void* stream);
/* QMTools.Compute_qdiff / gpu_qdiff(_rel) (qmtools/qmtools.py:2818-2831,
 * kernel_utils.cu:101-167): sum |a-b|, or 100*sum |a-b|/b when rel != 0. */
qmt_status qmt_grid_diff(const float* a_dev, const float* b_dev, int64_t n, int rel,
                         double* out, void* stream);
/* Error report (new): max |a-b|, ||a-b||_2/||b||_2, sum a, sum b, all FP64; out[4]. */
qmt_status qmt_grid_errors(const float* a_dev, const float* b_dev, int64_t n,
                           double* out4, void* stream);
/* QMTools.Compute_qseed / gpu_density_seed (qmtools/qmtools.py:2645-2672,
 * kernel_utils.cu:5-50) into q_dev (not cleared first, like the reference). */
qmt_status qmt_density_seed(qmt_mol* mol, int nx, int ny, int nz, float step,
                            float ox, float oy, float oz, float* q_dev, void* stream);
/* sum_A Z_A/|r - R_A| at voxel centres (gpu_hartree_add_nuclei, kernel_hartree.cu:209-251),
 * added into v_dev when accumulate != 0, else stored. */
qmt_status qmt_vne_point(qmt_mol* mol, int nx, int ny, int nz, float step,
                         float ox, float oy, float oz, int accumulate, float* v_dev,
                         void* stream);
/* QMTools.Compute_VNe_classic / gpu_vne_classic (qmtools/qmtools.py:2750-2790,
 * kernel_vne_classic.cu:13-84). */
qmt_status qmt_vne_classic(qmt_mol* mol, int nx, int ny, int nz, float step,
                           float ox, float oy, float oz, int divisions, float* v_dev,
                           void* stream);
/* QMTools.Compute_VNe / gpu_vne (qmtools/qmtools.py:2677-2745, kernel_vne.cu:13-128):
 * ping-pong pseudo-field; res_dev receives the field, out_dev is scratch; both are cleared
 * first.  Stops when the mean |delta| of a pair falls to tol or after maxiters pairs. */
qmt_status qmt_vne_pseudo(qmt_mol* mol, int nx, int ny, int nz, float step,
                          float ox, float oy, float oz, float ads, float dif, double tol,
                          int maxiters, float* res_dev, float* out_dev, int* iters_out,
                          void* stream);

/* ---- GA single-shot automaton --------------------------------------------------------- */
/* AutomatonSingleShot.Evaluate's kernel (qmtools/automaton_nn_singleshot.py:78-183,
 * gpu_automaton_nn_singleshot, kernel_nn_ss.cu:33-178): qout_dev[v] =
 * field1(v) * sum over the 26 neighbours u (periodic) of MLP(field1(v), field1(u))^2
 * rsqrt(|u - v|_1) / gridstep * 0.05234482976098482.  qube_dev holds two fields of
 * nx*ny*nz floats (field 0 is not read); params is a HOST array of 272*nlayers + 29 floats
 * (the reference's DNASIZE), nlayers 1..8; gridstep is the double the reference writes into
 * its kernel source (the grid step in bohr as printed from float32).  Asynchronous. */
qmt_status qmt_nn_singleshot(int nx, int ny, int nz, double gridstep, const float* qube_dev,
                             float* qout_dev, const float* params, int nparams, int nlayers,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QMTOOLS_B200_H */

// Jacobi relaxation of the Poisson equation on the voxel grid.
//
// Reference mode (gpu_hartree_iteration, kernel_hartree.cu:85-171):
//     V'(interior) = (xm + xp + yp + ym + zp + zm - Q/h) / 6,  V' = 0 on the outer shell,
// summed in that order so FP32 results match the reference update.
// Dirichlet mode (new): V'(interior) = (sum of 6 neighbours + 4 pi h^2 rho) / 6, evaluated as an
// increment of V, and the outer shell keeps its given values.
//
// One cooperative, persistent launch runs every sweep.  A work item is four consecutive x
// points (float4 loads of the row, the four neighbouring rows and Q): the grids of the path
// (three fields up to 192^3 = 85 MB) stay in the 126 MB L2 across sweeps, so the stencil is
// limited by L2 latency and wants many independent loads in flight rather than on-chip reuse.
// Sweeps are separated by a grid barrier of this file (bounded wait: it raises an error flag
// after the library's wait limit, 2 s unless qmt_set_wait_limit_ns changed it).
// V and its copy are rewritten by other CTAs between sweeps, so they are read through L2
// (ld.global.cg), never through the non-coherent L1 paths.  On sweeps that feed a
// convergence check each CTA sums |V' - V| in FP64 over its units; CTA 0 adds the CTA sums in
// CTA order, so the residual is deterministic, and every CTA takes the same stop decision.
//
// Small grids (a plane of at most 4096 points, at most 4 planes per CTA of a 16-CTA cluster:
// the 64^3 grid of the small-molecule configuration) can run as one thread-block cluster instead
// (the automatic choice for the Dirichlet update):
// the field lives in the CTAs' shared memory (two buffers of each CTA's z-slab), each thread
// keeps its column of four-point groups and their charges in registers, neighbours come from
// registers (z inside the slab), warp shuffles (x), shared memory (y, x across warps) and the
// neighbouring CTAs' shared memory (z across slabs, distributed shared memory), and sweeps are
// separated by the hardware cluster barrier -- no global-memory round trip and no software
// grid barrier per sweep.  Both kernels apply jac_point, so their results are identical.
#include "mol.cuh"
#include "reduce.cuh"

namespace qmt {

constexpr int JX = 32, JY = 8;
constexpr int JAC_THREADS = JX * JY;
constexpr int JAC_BLOCKS_PER_SM = 4;

struct JacobiArgs {
  int nx, ny, nz;
  float h, src_scale;
  const float* Q;
  float* V;            // start value in, result out
  float* T;            // second buffer
  int vec4;            // nx % 4 == 0 and 16-byte aligned V, T, Q: groups of four x points
  int max_sweeps, check_every;
  double tol;
  double* part;        // per-CTA partial sums
  unsigned* bar;       // [0] arrivals, [1] generation
  uint64_t wait_ns;    // limit of a grid-barrier wait before the solve gives up
  double* res;         // [0] residual of the last check
  int* out;            // [0] sweeps done, [1] status: 0 running/cap, 1 converged, 2 not finite, 3 barrier timeout
};

__device__ __forceinline__ uint64_t jac_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Sense-counting grid barrier for a cooperative launch (all CTAs co-resident).  Returns false
// on every CTA once any CTA has waited more than `wait_ns` or raised the flag.  Arrivals are
// acquire-release atomics on bar[0] (the CTA's writes are ordered before its arrival by the CTA
// barrier); the last arrival resets the count and releases the generation bar[1], which the
// others read with acquire loads: no full memory fences.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ bool grid_barrier(unsigned* bar, int* flag, unsigned nblocks, uint64_t wait_ns) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile int* vflag = flag;
    const unsigned g = ld_acquire_gpu(bar + 1);
    int ok = 1;
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
    if (old == nblocks - 1) {
      asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(bar) : "memory");
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar + 1) : "memory");
    } else {
      const uint64_t t0 = jac_timer_ns();
      while (ld_acquire_gpu(bar + 1) == g) {
        if (*vflag) {
          ok = 0;
          break;
        }
        if (jac_timer_ns() - t0 > wait_ns) {
          atomicExch(flag, 1);
          ok = 0;
          break;
        }
      }
    }
    ok_s = ok && !*vflag;
  }
  __syncthreads();
  return ok_s != 0;
}

template <bool DIRICHLET>
__device__ __forceinline__ float jac_source(float q, float h, float src_scale) {
  if constexpr (!DIRICHLET) return q / h;
  else return __fmul_rn(src_scale, q);
}

// Update of one point from its six neighbours (in the reference's summation order) and its
// source term.
template <bool DIRICHLET>
__device__ __forceinline__ float jac_point(float xm, float xp, float yp, float ym, float zp, float zm, float src,
                                           float vc, bool edge) {
  if constexpr (!DIRICHLET) {
    float s = xm + xp;
    s = s + yp;
    s = s + ym;
    s = s + zp;
    s = s + zm;
    s = s - src;
    return edge ? 0.f : s / 6.0f;
  } else {
    // increment form V + (sum (nb - V) + 4 pi h^2 rho) / 6: the FP32 rounding of 1/6 and of the
    // neighbour sum then scale only the increment, which vanishes at convergence.  (The direct
    // form (sum nb + 4 pi h^2 rho) * fp32(1/6) biases every sweep the same way; over 2000 sweeps
    // of a 64^3 grid the smooth error modes amplify that to ~1e-5 relative, against ~4e-8 here.)
    const float s = ((xm - vc) + (xp - vc)) + ((yp - vc) + (ym - vc)) + ((zp - vc) + (zm - vc));
    return edge ? vc : fmaf(__fadd_rn(s, src), 1.0f / 6.0f, vc);
  }
}

__device__ __forceinline__ float4 ldcg4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }

// A thread's work items in a sweep: the grid-stride sequence tid, tid + nthreads, ... over
// the groups (or points), as grid coordinates of the first item and of the stride, advanced by
// additions with carries -- no division per item (the stride is below nxq * ny * nz, so each
// carry needs one subtraction).  Set up once per launch.
struct JacWalk {
  int x, y, z;      // first item: x group (vec4) or point
  int sx, sy, sz;   // the stride
};

__device__ JacWalk jac_walk(const JacobiArgs& a) {
  const uint32_t w = a.vec4 ? (uint32_t)(a.nx >> 2) : (uint32_t)a.nx;
  const uint32_t ny = (uint32_t)a.ny;
  const uint32_t nthreads = gridDim.x * JAC_THREADS;   // (the grid is a few CTAs per SM)
  const uint32_t tid = blockIdx.x * JAC_THREADS + threadIdx.y * JX + threadIdx.x;
  const uint32_t r = tid / w, rs = nthreads / w;
  return JacWalk{(int)(tid - r * w), (int)(r % ny), (int)(r / ny), (int)(nthreads - rs * w), (int)(rs % ny),
                 (int)(rs / ny)};
}

// One sweep src -> dst.  Work items are groups of four consecutive x points (float4 loads of
// the row, the four neighbouring rows and Q, scalar loads of the two x halo values), spread over
// all CTAs; every load of a group is independent, so many are in flight per thread.  Returns
// this thread's FP64 sum |dst - src| when `resid` is set.
template <bool DIRICHLET>
__device__ double sweep(const JacobiArgs& a, const float* src, float* dst, bool resid, const JacWalk& wk) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int64_t row = nx, plane = (int64_t)nx * ny;
  const int64_t nthreads = (int64_t)gridDim.x * JAC_THREADS;
  const int64_t tid = (int64_t)blockIdx.x * JAC_THREADS + threadIdx.y * JX + threadIdx.x;
  double dsum = 0.0;
  if (a.vec4) {
    const int nxq = nx >> 2;
    const int64_t ngroups = (int64_t)nxq * ny * nz;
    int xq = wk.x, y = wk.y, z = wk.z;
    const int sx = wk.sx, sy = wk.sy, sz = wk.sz;
    for (int64_t gi = tid; gi < ngroups; gi += nthreads) {
      const int x0 = xq * 4;
      const int64_t b = z * plane + (int64_t)y * row + x0;
      const float4 c = ldcg4(src + b);
      const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 ym = y > 0 ? ldcg4(src + b - row) : zero;
      const float4 yp = y + 1 < ny ? ldcg4(src + b + row) : zero;
      const float4 zm = z > 0 ? ldcg4(src + b - plane) : zero;
      const float4 zp = z + 1 < nz ? ldcg4(src + b + plane) : zero;
      const float4 q4 = __ldg(reinterpret_cast<const float4*>(a.Q + b));
      const float4 q = make_float4(jac_source<DIRICHLET>(q4.x, a.h, a.src_scale),
                                   jac_source<DIRICHLET>(q4.y, a.h, a.src_scale),
                                   jac_source<DIRICHLET>(q4.z, a.h, a.src_scale),
                                   jac_source<DIRICHLET>(q4.w, a.h, a.src_scale));
      const float xl = x0 > 0 ? __ldcg(src + b - 1) : 0.f;
      const float xr = x0 + 4 < nx ? __ldcg(src + b + 4) : 0.f;
      const bool eyz = y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
      float4 o;
      o.x = jac_point<DIRICHLET>(xl, c.y, yp.x, ym.x, zp.x, zm.x, q.x, c.x, eyz || x0 == 0);
      o.y = jac_point<DIRICHLET>(c.x, c.z, yp.y, ym.y, zp.y, zm.y, q.y, c.y, eyz || x0 + 1 == nx - 1);
      o.z = jac_point<DIRICHLET>(c.y, c.w, yp.z, ym.z, zp.z, zm.z, q.z, c.z, eyz || x0 + 2 == nx - 1);
      o.w = jac_point<DIRICHLET>(c.z, xr, yp.w, ym.w, zp.w, zm.w, q.w, c.w, eyz || x0 + 3 == nx - 1);
      __stcg(reinterpret_cast<float4*>(dst + b), o);
      if (resid)
        dsum += (fabs((double)o.x - (double)c.x) + fabs((double)o.y - (double)c.y)) +
                (fabs((double)o.z - (double)c.z) + fabs((double)o.w - (double)c.w));
      xq += sx;
      if (xq >= nxq) {
        xq -= nxq;
        ++y;
      }
      y += sy;
      if (y >= ny) {
        y -= ny;
        ++z;
      }
      z += sz;
    }
  } else {
    const int64_t n = plane * nz;
    int x = wk.x, y = wk.y, z = wk.z;
    const int sx = wk.sx, sy = wk.sy, sz = wk.sz;
    for (int64_t g = tid; g < n; g += nthreads) {
      const float vc = __ldcg(src + g);
      const float xm = x > 0 ? __ldcg(src + g - 1) : 0.f;
      const float xp = x + 1 < nx ? __ldcg(src + g + 1) : 0.f;
      const float ym = y > 0 ? __ldcg(src + g - row) : 0.f;
      const float yp = y + 1 < ny ? __ldcg(src + g + row) : 0.f;
      const float zm = z > 0 ? __ldcg(src + g - plane) : 0.f;
      const float zp = z + 1 < nz ? __ldcg(src + g + plane) : 0.f;
      const bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
      const float o =
          jac_point<DIRICHLET>(xm, xp, yp, ym, zp, zm, jac_source<DIRICHLET>(__ldg(a.Q + g), a.h, a.src_scale), vc, edge);
      __stcg(dst + g, o);
      if (resid) dsum += fabs((double)o - (double)vc);
      x += sx;
      if (x >= nx) {
        x -= nx;
        ++y;
      }
      y += sy;
      if (y >= ny) {
        y -= ny;
        ++z;
      }
      z += sz;
    }
  }
  return dsum;
}

template <bool DIRICHLET>
__global__ void __launch_bounds__(JAC_THREADS, JAC_BLOCKS_PER_SM) jacobi_persistent_kernel(JacobiArgs a) {
  __shared__ double sh[JAC_THREADS / 32];
  const unsigned nb = gridDim.x;
  int* flag = a.out + 2;
  double delta = INFINITY;
  int sweeps = 0, pairs = 0, status = 0;
  const int lin = threadIdx.y * JX + threadIdx.x;
  const JacWalk wk = jac_walk(a);
  while (sweeps + 2 <= a.max_sweeps) {
    ++pairs;
    const bool check = pairs % a.check_every == 0 || sweeps + 4 > a.max_sweeps;
    sweep<DIRICHLET>(a, a.V, a.T, false, wk);
    if (!grid_barrier(a.bar, flag, nb, a.wait_ns)) {
      status = 3;
      break;
    }
    const double ds = sweep<DIRICHLET>(a, a.T, a.V, check, wk);
    sweeps += 2;
    if (!check) {
      if (!grid_barrier(a.bar, flag, nb, a.wait_ns)) {
        status = 3;
        break;
      }
      continue;
    }
    // FP64 residual: warp tree, warps in order, CTAs in order
    double v = ds;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((lin & 31) == 0) sh[lin >> 5] = v;
    __syncthreads();
    if (lin == 0) {
      double r = 0.0;
      for (int w = 0; w < JAC_THREADS / 32; ++w) r += sh[w];
      __stcg(a.part + blockIdx.x, r);
    }
    if (!grid_barrier(a.bar, flag, nb, a.wait_ns)) {
      status = 3;
      break;
    }
    if (blockIdx.x == 0 && lin == 0) {
      double r = 0.0;
      for (unsigned b = 0; b < nb; ++b) r += __ldcg(a.part + b);
      __stcg(a.res, r);
    }
    if (!grid_barrier(a.bar, flag, nb, a.wait_ns)) {
      status = 3;
      break;
    }
    delta = __ldcg(a.res);
    if (!isfinite(delta)) {
      status = 2;
      break;
    }
    if (delta <= a.tol) {
      status = 1;
      break;
    }
  }
  if (blockIdx.x == 0 && lin == 0) {
    a.out[0] = sweeps;
    a.out[1] = status;
    __stcg(a.res + 1, delta);
  }
}

// ---- single-cluster kernel ---------------------------------------------------------------------
constexpr int JAC_CLUSTER = 16;          // CTAs of the cluster (a non-portable size)
constexpr int JAC_CLUSTER_THREADS = 1024;

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t dsmem_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ float4 dsmem_ld4(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(addr)
               : "memory");
  return v;
}

__device__ __forceinline__ double dsmem_ld_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
  return v;
}

// One cluster; CTA c owns planes [c P, c P + np) of the grid.  Thread t owns the four-point group
// (xq, y) = (t % nxq, t / nxq) of every plane of the slab.  Shared memory: buf[2][P][ny][nxq]
// float4 (the field before / after a sweep).  Launched only when nx % 4 == 0, nxq * ny <= 1024,
// ceil(nz / 16) <= P <= 4 and V, Q 16-byte aligned (checked on the host).
template <bool DIRICHLET, int P>
__global__ void __launch_bounds__(JAC_CLUSTER_THREADS, 1) jacobi_cluster_kernel(JacobiArgs a) {
  extern __shared__ float4 jbuf[];
  __shared__ double red[JAC_CLUSTER_THREADS / 32];
  __shared__ double part;
  __shared__ int stop_s;
  const int nx = a.nx, ny = a.ny, nz = a.nz, nxq = nx >> 2;
  const int t = threadIdx.x, lane = t & 31;
  const bool act = t < nxq * ny;
  const int xq = act ? t % nxq : 0, y = act ? t / nxq : 0;
  const uint32_t c = cluster_rank(), ncta = gridDim.x;
  const int z0 = (int)c * P;
  const int np = max(0, min(P, nz - z0));
  const int pstride = nxq * ny;                 // float4 per plane
  float4* buf0 = jbuf;
  float4* buf1 = jbuf + (size_t)P * pstride;
  const int own = y * nxq + xq;
  float4 v[P], q[P];
#pragma unroll
  for (int k = 0; k < P; ++k) {
    v[k] = q[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (act && k < np) {
      const int64_t g = ((int64_t)(z0 + k) * ny + y) * nx + xq * 4;
      v[k] = __ldcg(reinterpret_cast<const float4*>(a.V + g));
      const float4 q4 = __ldg(reinterpret_cast<const float4*>(a.Q + g));   // source terms, once
      q[k] = make_float4(jac_source<DIRICHLET>(q4.x, a.h, a.src_scale), jac_source<DIRICHLET>(q4.y, a.h, a.src_scale),
                         jac_source<DIRICHLET>(q4.z, a.h, a.src_scale), jac_source<DIRICHLET>(q4.w, a.h, a.src_scale));
      buf0[k * pstride + own] = v[k];
    }
  }
  const bool ey = y == 0 || y == ny - 1;
  const bool xlo = xq == 0, xhi = xq == nxq - 1;
  // shuffles give the x neighbours within a warp; at a warp's first / last lane the group beside
  // it (same row) belongs to another warp and is read from shared memory
  const bool left_smem = !xlo && lane == 0, right_smem = !xhi && lane == 31;
  cluster_sync_all();
  int sweeps = 0, pairs = 0, status = 0;
  double delta = INFINITY;
  while (sweeps + 2 <= a.max_sweeps) {
    ++pairs;
    const bool check = pairs % a.check_every == 0 || sweeps + 4 > a.max_sweeps;
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
      float4* src = half == 0 ? buf0 : buf1;
      float4* dst = half == 0 ? buf1 : buf0;
      const bool resid = check && half == 1;
      double ds = 0.0;
      const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 below = zero, above = zero;
      if (act && np > 0) {
        if (z0 > 0) below = dsmem_ld4(dsmem_addr(src + (P - 1) * pstride + own, c - 1));
        if (z0 + np < nz) above = dsmem_ld4(dsmem_addr(src + own, c + 1));
      }
      float4 prev = below;
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const float4 cen = v[k];
        const float wl = __shfl_up_sync(0xffffffffu, cen.w, 1);
        const float xr0 = __shfl_down_sync(0xffffffffu, cen.x, 1);
        if (k < np && act) {
          const float4* pl = src + k * pstride;
          const float4 ym = y > 0 ? pl[own - nxq] : zero;
          const float4 yp = y + 1 < ny ? pl[own + nxq] : zero;
          const float4 zp = k + 1 < np ? v[k + 1] : above;
          const float4 zm = prev;
          const float xl = xlo ? 0.f : (left_smem ? pl[own - 1].w : wl);
          const float xr = xhi ? 0.f : (right_smem ? pl[own + 1].x : xr0);
          const int z = z0 + k;
          const bool eyz = ey || z == 0 || z == nz - 1;
          float4 o;
          o.x = jac_point<DIRICHLET>(xl, cen.y, yp.x, ym.x, zp.x, zm.x, q[k].x, cen.x, eyz || xlo);
          o.y = jac_point<DIRICHLET>(cen.x, cen.z, yp.y, ym.y, zp.y, zm.y, q[k].y, cen.y, eyz || xq * 4 + 1 == nx - 1);
          o.z = jac_point<DIRICHLET>(cen.y, cen.w, yp.z, ym.z, zp.z, zm.z, q[k].z, cen.z, eyz || xq * 4 + 2 == nx - 1);
          o.w = jac_point<DIRICHLET>(cen.z, xr, yp.w, ym.w, zp.w, zm.w, q[k].w, cen.w, eyz || xhi);
          if (resid)
            ds += (fabs((double)o.x - (double)cen.x) + fabs((double)o.y - (double)cen.y)) +
                  (fabs((double)o.z - (double)cen.z) + fabs((double)o.w - (double)cen.w));
          prev = cen;
          v[k] = o;
          dst[k * pstride + own] = o;
        }
      }
      cluster_sync_all();   // every read of src done, every write of dst visible cluster-wide
      if (resid) {
        // FP64 residual: warp tree, warps in order, CTAs in rank order -- every CTA adds the same
        // partials in the same order, so all take the same decision
        for (int o = 16; o > 0; o >>= 1) ds += __shfl_xor_sync(0xffffffffu, ds, o);
        if (lane == 0) red[t >> 5] = ds;
        __syncthreads();
        if (t == 0) {
          double r = 0.0;
          for (int w = 0; w < JAC_CLUSTER_THREADS / 32; ++w) r += red[w];
          part = r;
        }
        cluster_sync_all();
        if (t == 0) {
          double r = 0.0;
          for (uint32_t b = 0; b < ncta; ++b) r += dsmem_ld_f64(dsmem_addr(&part, b));
          delta = r;
          stop_s = !isfinite(r) ? 2 : (r <= a.tol ? 1 : 0);
        }
        __syncthreads();
      }
    }
    sweeps += 2;
    if (check) {
      status = stop_s;
      if (status != 0) break;
    }
  }
  // no CTA may leave while another can still read its shared memory
  cluster_sync_all();
#pragma unroll
  for (int k = 0; k < P; ++k)
    if (act && k < np)
      __stcg(reinterpret_cast<float4*>(a.V + ((int64_t)(z0 + k) * ny + y) * nx + xq * 4), v[k]);
  if (c == 0 && t == 0) {
    a.out[0] = sweeps;
    a.out[1] = status;
    a.res[1] = delta;
  }
}

static int g_jacobi_path = 0;   // 0 automatic, 1 grid barrier per sweep, 2 single cluster

// Planes per CTA of the cluster kernel for this grid (1, 2 or 4), or 0 if it does not apply.
static int cluster_planes(int nx, int ny, int nz, const float* rho, const float* v) {
  if (nx % 4 || (nx / 4) * ny > JAC_CLUSTER_THREADS || nz < 2) return 0;
  if ((reinterpret_cast<uintptr_t>(rho) | reinterpret_cast<uintptr_t>(v)) % 16) return 0;
  const int need = (nz + JAC_CLUSTER - 1) / JAC_CLUSTER;
  int P = 1;
  while (P < need) P *= 2;
  if (P > 4) return 0;   // eight planes of values and sources do not fit in a thread's registers
  const size_t smem = 2ull * P * (size_t)nx * ny * sizeof(float);
  if (smem > 200u * 1024u) return 0;
  return P;
}

template <bool DIRICHLET, int P>
static qmt_status launch_cluster(JacobiArgs& a, cudaStream_t s, bool* launched) {
  *launched = false;
  auto kern = jacobi_cluster_kernel<DIRICHLET, P>;
  const size_t smem = 2ull * P * (size_t)a.nx * a.ny * sizeof(float);
  const int ncta = std::min(JAC_CLUSTER, (a.nz + P - 1) / P);
  QMT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  QMT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(ncta);
  cfg.blockDim = dim3(JAC_CLUSTER_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ncta;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
    cudaGetLastError();   // the persistent kernel takes the solve
    return QMT_OK;
  }
  QMT_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
  note_launches(1);
  *launched = true;
  return QMT_OK;
}

template <bool DIRICHLET>
static qmt_status try_cluster(JacobiArgs& a, int P, cudaStream_t s, bool* launched) {
  switch (P) {
    case 1: return launch_cluster<DIRICHLET, 1>(a, s, launched);
    case 2: return launch_cluster<DIRICHLET, 2>(a, s, launched);
    case 4: return launch_cluster<DIRICHLET, 4>(a, s, launched);
    default: *launched = false; return QMT_OK;
  }
}

template <bool DIRICHLET>
static qmt_status run_jacobi(int nx, int ny, int nz, float step, const float* rho, float* v, float* t,
                             int max_sweeps, int check_every, double tol, int* sweeps_out,
                             double* delta_out, cudaStream_t s) {
  if (nx < 1 || ny < 1 || nz < 1 || !(step > 0.f) || !rho || !v || !t || max_sweeps < 0 || check_every < 1)
    return fail(QMT_BAD_ARG, "bad Jacobi arguments");
  const int nsm = sm_count();
  int per_sm = 0;
  auto kern = jacobi_persistent_kernel<DIRICHLET>;
  QMT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, JAC_THREADS, 0));
  if (per_sm < 1) return fail(QMT_CUDA_ERR, "Jacobi kernel does not fit on an SM");
  per_sm = std::min(per_sm, JAC_BLOCKS_PER_SM);
  const int64_t capacity = (int64_t)nsm * per_sm;

  JacobiArgs a{};
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.h = DIRICHLET ? 0.f : step;
  a.src_scale = DIRICHLET ? (float)(4.0 * 3.14159265358979323846 * (double)step * step) : 0.f;
  a.Q = rho;
  a.V = v;
  a.T = t;
  a.vec4 = (nx % 4 == 0) && ((reinterpret_cast<uintptr_t>(rho) | reinterpret_cast<uintptr_t>(v) |
                                reinterpret_cast<uintptr_t>(t)) % 16 == 0);
  a.max_sweeps = max_sweeps;
  a.check_every = check_every;
  a.tol = tol;
  a.wait_ns = wait_limit_ns();
  const int64_t items = a.vec4 ? (int64_t)(nx / 4) * ny * nz : (int64_t)nx * ny * nz;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((items + JAC_THREADS - 1) / JAC_THREADS, capacity));

  // scratch: CTA partial sums, barrier words, residuals, status words (grows, never freed)
  static thread_local DevBuf scratch;
  const size_t part_bytes = ((size_t)grid * sizeof(double) + 255) / 256 * 256;
  qmt_status st = scratch.reserve(part_bytes + 256);
  if (st) return st;
  uint8_t* base = scratch.as<uint8_t>();
  a.part = reinterpret_cast<double*>(base);
  a.res = reinterpret_cast<double*>(base + part_bytes);          // [0] check sum, [1] last residual
  a.bar = reinterpret_cast<unsigned*>(base + part_bytes + 64);    // [0] arrivals, [1] generation
  a.out = reinterpret_cast<int*>(base + part_bytes + 128);        // [0] sweeps, [1] status, [2] flag
  QMT_CUDA(cudaMemsetAsync(base + part_bytes, 0, 256, s));
  if (max_sweeps >= 2) {
    bool done = false;
    // the cluster kernel where it applies: for the Dirichlet update (measured 3.8 against 4.2 us per
    // 64^3 sweep); the reference update's IEEE division makes it issue-bound on its 16 SMs (4.5
    // against 4.3 us), so automatic selection leaves that one on the grid-barrier kernel
    const bool want_cluster = g_jacobi_path == 2 || (g_jacobi_path == 0 && DIRICHLET);
    const int P = want_cluster ? cluster_planes(nx, ny, nz, rho, v) : 0;
    if (!done && P > 0 && (st = try_cluster<DIRICHLET>(a, P, s, &done))) return st;
    if (g_jacobi_path == 2 && !done)
      return fail(QMT_BAD_ARG, "the single-cluster Jacobi kernel does not apply to this grid or device");
    if (!done) {
      void* params[] = {&a};
      QMT_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(JX, JY), params, 0, s));
      note_launches(1);
    }
  }
  int out[3] = {0, 0, 0};
  double res[2] = {0.0, INFINITY};
  QMT_CUDA(cudaMemcpyAsync(out, a.out, sizeof(out), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaMemcpyAsync(res, a.res, sizeof(res), cudaMemcpyDeviceToHost, s));
  QMT_CUDA(cudaStreamSynchronize(s));
  const double delta = max_sweeps >= 2 ? res[1] : INFINITY;
  if (sweeps_out) *sweeps_out = out[0];
  if (delta_out) *delta_out = delta;
  if (out[1] == 3 || out[2]) return fail(QMT_CUDA_ERR, "Jacobi grid barrier timed out");
  if (out[1] == 2) return fail(QMT_NAN, "Jacobi residual is not finite");
  if (out[1] != 1 && tol > 0) return fail(QMT_NOT_CONVERGED, "Jacobi stopped at its sweep cap");
  return QMT_OK;
}

}  // namespace qmt

using namespace qmt;

extern "C" qmt_status qmt_jacobi(int nx, int ny, int nz, float step, const float* rho_dev, float* v_dev,
                                 float* t_dev, int max_sweeps, int check_every, double tol, int* sweeps_out,
                                 double* delta_out, void* stream) {
  return run_jacobi<false>(nx, ny, nz, step, rho_dev, v_dev, t_dev, max_sweeps, check_every, tol, sweeps_out,
                           delta_out, as_stream(stream));
}

extern "C" qmt_status qmt_jacobi_dirichlet(int nx, int ny, int nz, float step, const float* rho_dev, float* v_dev,
                                           float* t_dev, int max_sweeps, int check_every, double tol,
                                           int* sweeps_out, double* delta_out, void* stream) {
  return run_jacobi<true>(nx, ny, nz, step, rho_dev, v_dev, t_dev, max_sweeps, check_every, tol, sweeps_out,
                          delta_out, as_stream(stream));
}

extern "C" qmt_status qmt_set_jacobi_path(int mode) {
  if (mode < 0 || mode > 2)
    return fail(QMT_BAD_ARG, "Jacobi path must be 0 (automatic), 1 (grid barrier per sweep) or 2 (single cluster)");
  g_jacobi_path = mode;
  return QMT_OK;
}

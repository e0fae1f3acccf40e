"""Oracle: basis functions on points and the electron density grid (test infrastructure).

Restates, in FP64, what `QMTools.Compute_density` (qmtools/qmtools.py:2381-2430)
and the kernel `gpu_densityqube_shmem_subgrid` (qmtools/cuda/kernel_density.cu:34-155)
compute:

    q_v = 2 * h^3 * (1/s^3) * sum_sub sum_{p,q} P_pq phi_p(r) phi_q(r)

at voxel-centre sub-points r = origin + (i + (ix + 1/2)/s) h  (kernel_density.cu:96-100),
stored x-fastest (kernel_density.cu:151-154), then rescaled so that sum_v q_v equals
the total nuclear charge (qmtools/qmtools.py:2419-2424).
"""
import numpy as np

# real solid harmonics times r^l, constants of kernel_density.cu:17-28
C_S = 0.28209479177387814
C_P = 0.4886025119029199
C_D1 = 1.0925484305920792
C_D0 = 0.31539156525252005
C_D2 = 0.5462742152960396


def solid_harmonic(L, m, x, y, z):
    """Y_lm(r) r^l as used for the basis functions (kernel_density.cu:14-31)."""
    if L == 0:
        return np.full_like(x, C_S)
    if L == 1:
        return C_P * {-1: y, 0: z, 1: x}[m]
    if L == 2:
        if m == -2:
            return C_D1 * x * y
        if m == -1:
            return C_D1 * z * y
        if m == 0:
            return C_D0 * (2 * z * z - x * x - y * y)
        if m == 1:
            return C_D1 * x * z
        if m == 2:
            return C_D2 * (x * x - y * y)
    raise IndexError(f"unsupported L={L}, m={m}")


def eval_phi(points, coords, almos, alphas, coeffs):
    """Phi[P, N]: every basis function at every point, FP64.

    points, coords in bohr (same frame); almos = [atom, L, m, shellOffset] per
    function (qmtools/qmtools.py:163-171); alphas/coeffs = the padded
    MAXAOC=20 tables (qmtools/qmtools.py:78-85).
    """
    points = np.asarray(points, dtype=np.float64)
    coords = np.asarray(coords, dtype=np.float64)
    al = np.asarray(alphas, dtype=np.float64)
    co = np.asarray(coeffs, dtype=np.float64)
    N = almos.shape[0]
    phi = np.empty((points.shape[0], N), dtype=np.float64)
    cache = {}
    for f in range(N):
        a, L, m, so = (int(v) for v in almos[f])
        key = (a, so)
        if key not in cache:
            d = points - coords[a]
            r2 = np.einsum("pi,pi->p", d, d)
            a_s = al[so:so + 20]
            c_s = co[so:so + 20]
            nz = c_s != 0
            rad = np.exp(-np.outer(r2, a_s[nz])) @ c_s[nz]
            cache[key] = (d, rad)
        d, rad = cache[key]
        phi[:, f] = solid_harmonic(L, m, d[:, 0], d[:, 1], d[:, 2]) * rad
    return phi


def voxel_centres(shape, step, origin, subgrid=1, ix=0, iy=0, iz=0, zslab=None):
    """Sub-point positions (flat, x-fastest) for sub-offset (ix,iy,iz).

    Mirrors kernel_density.cu:95-100: pos = origin + (i + (ix+1/2)/s) * h.
    zslab=(z0, z1) restricts to z planes z0..z1-1.
    """
    nx, ny, nz = shape
    z0, z1 = (0, nz) if zslab is None else zslab
    h = float(step)
    xs = (np.arange(nx) + (ix + 0.5) / subgrid) * h + float(origin[0])
    ys = (np.arange(ny) + (iy + 0.5) / subgrid) * h + float(origin[1])
    zs = (np.arange(z0, z1) + (iz + 0.5) / subgrid) * h + float(origin[2])
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def density_at(points, coords, almos, alphas, coeffs, dm, chunk=65536):
    """rho(r) = sum_pq P_pq phi_p phi_q  (no spin factor), FP64."""
    dm = np.asarray(dm, dtype=np.float64)
    out = np.empty(points.shape[0], dtype=np.float64)
    for s in range(0, points.shape[0], chunk):
        phi = eval_phi(points[s:s + chunk], coords, almos, alphas, coeffs)
        out[s:s + chunk] = np.einsum("pi,pi->p", phi @ dm, phi)
    return out


def density_qube_unscaled(shape, step, origin, coords, almos, alphas, coeffs, dm,
                          subgrid=1, zslab=None):
    """Electrons per voxel before the qtot rescale (kernel_density.cu:74-154), flat x-fastest."""
    acc = None
    for ix in range(subgrid):
        for iy in range(subgrid):
            for iz in range(subgrid):
                pts = voxel_centres(shape, step, origin, subgrid, ix, iy, iz, zslab)
                r = density_at(pts, coords, almos, alphas, coeffs, dm)
                acc = r if acc is None else acc + r
    h = float(step)
    return 2.0 * acc / subgrid ** 3 * h ** 3


def compute_density(shape, step, origin, coords, types, almos, alphas, coeffs, dm,
                    subgrid=1):
    """`QMTools.Compute_density` result (qmtools/qmtools.py:2381-2430), flat x-fastest.

    Returns (q_scaled, q_unscaled, sum_unscaled).
    """
    q = density_qube_unscaled(shape, step, origin, coords, almos, alphas, coeffs, dm, subgrid)
    tot = q.sum()
    qtot = float(np.sum(types))
    return q * (qtot / tot), q, tot

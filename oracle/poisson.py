"""Oracle: Jacobi relaxation and FFT Poisson solves on voxel grids (test infrastructure).

All grids are flat arrays in the reference's x-fastest order
(idx = x + y*NX + z*NX*NY, kernel_hartree.cu:94), viewed here as [z, y, x].
"""
import numpy as np

R_BOHR = 0.529177211       # kernel_fft.cu:17
EPS0 = 0.0055263494        # kernel_fft.cu:18, e/(V*Ang)
ANG2BOR = 1.8897259886
CUBE_INV_R = 2.3800772417  # (1/h^3) * integral over a voxel cube of 1/|r|, times h


def density_seed(shape, step, origin, coords, types):
    """`gpu_density_seed` (kernel_utils.cu:5-50): Z spread over the 8 nodes around each nucleus.

    Node i0 = floor(x/h) + t (t in {0,1}) gets Z * prod |x - i0 h| / h; the last
    atom to write a node wins (plain stores, one block per atom).  Index and
    weights follow the kernel's FP32 arithmetic, including nvcc's default contraction
    of `x - i0*h` into one fused multiply-add (exact product and sum, one rounding).
    """
    nx, ny, nz = shape
    h = np.float32(step)
    q = np.zeros(nx * ny * nz, dtype=np.float32)
    o = np.asarray(origin, dtype=np.float32)
    for A, Z in zip(np.asarray(coords, dtype=np.float32), types):
        rel = (A - o).astype(np.float32)
        base = np.floor(rel / h).astype(np.int64)
        for tz in range(2):
            for ty in range(2):
                for tx in range(2):
                    i0 = base + np.array([tx, ty, tz])
                    p = np.float32(Z)
                    for d in range(3):
                        diff = np.float32(np.float64(rel[d]) - np.float64(np.float32(i0[d])) * np.float64(h))
                        p = np.float32(p * np.float32(np.abs(diff) / h))
                    q[i0[0] + i0[1] * nx + i0[2] * nx * ny] = p
    return q


def jacobi_sweeps(rho, shape, step, nsweeps, V0=None, dtype=np.float64):
    """`gpu_hartree_iteration` applied nsweeps times (kernel_hartree.cu:85-171).

    V'(interior) = (sum of the 6 neighbours - Q/h) / 6 ; V' = 0 on the outer shell.
    """
    nx, ny, nz = shape
    Q = np.asarray(rho, dtype=dtype).reshape(nz, ny, nx)
    V = np.zeros((nz, ny, nx), dtype=dtype) if V0 is None else np.asarray(V0, dtype=dtype).reshape(nz, ny, nx).copy()
    h = dtype(step)
    six = dtype(6.0)
    for _ in range(nsweeps):
        W = np.zeros_like(V)
        s = (V[1:-1, 1:-1, :-2] + V[1:-1, 1:-1, 2:]) + V[1:-1, 2:, 1:-1]
        s = s + V[1:-1, :-2, 1:-1]
        s = s + V[2:, 1:-1, 1:-1]
        s = s + V[:-2, 1:-1, 1:-1]
        W[1:-1, 1:-1, 1:-1] = (s - Q[1:-1, 1:-1, 1:-1] / h) / six
        V = W
    return V.ravel()


def jacobi_dirichlet(rhs_phys, shape, step, boundary, nsweeps, dtype=np.float64):
    """Physical-unit Jacobi: lap V = -4 pi rho (a.u.), fixed boundary values on the outer shell.

    rhs_phys: charge density rho (e/bohr^3, positive for nuclei); boundary: full grid
    whose outer shell holds the Dirichlet values (interior ignored).  V starts at 0
    inside.  Update: V' = (sum nb + 4 pi h^2 rho) / 6.
    """
    nx, ny, nz = shape
    R = np.asarray(rhs_phys, dtype=dtype).reshape(nz, ny, nx)
    V = np.asarray(boundary, dtype=dtype).reshape(nz, ny, nx).copy()
    V[1:-1, 1:-1, 1:-1] = 0
    f = dtype(4 * np.pi) * dtype(step) ** 2
    for _ in range(nsweeps):
        s = (V[1:-1, 1:-1, :-2] + V[1:-1, 1:-1, 2:] + V[1:-1, 2:, 1:-1] + V[1:-1, :-2, 1:-1]
             + V[2:, 1:-1, 1:-1] + V[:-2, 1:-1, 1:-1])
        W = V.copy()
        W[1:-1, 1:-1, 1:-1] = (s + f * R[1:-1, 1:-1, 1:-1]) / 6
        V = W
    return V.ravel()


def fft_rhs(q, shape, step_bohr, origin_bohr, coords_bohr, types, sigma, cutoff):
    """RHS grid of `gpu_add_nuclear_charge` (kernel_fft.cu:23-79), returned as [x, y, z] (C-order).

    rho_tot = -q/h^3 (h in Ang) + sum_A Z_A g_sigma(r - R_A) within cutoff*sigma;
    returns -rho_tot / EPS0.
    """
    nx, ny, nz = shape
    h = step_bohr / ANG2BOR
    o = np.asarray(origin_bohr, dtype=np.float64) / ANG2BOR
    qx = np.asarray(q, dtype=np.float64).reshape(nz, ny, nx).transpose(2, 1, 0)
    rho = qx / (-h ** 3)
    xs = o[0] + (np.arange(nx) + 0.5) * h
    ys = o[1] + (np.arange(ny) + 0.5) * h
    zs = o[2] + (np.arange(nz) + 0.5) * h
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    norm = 1.0 / (sigma ** 3 * 2 * np.pi * np.sqrt(2 * np.pi))
    cut2 = (cutoff * sigma) ** 2
    for A, Zn in zip(np.asarray(coords_bohr, dtype=np.float64) * R_BOHR, types):
        r2 = (X - A[0]) ** 2 + (Y - A[1]) ** 2 + (Z - A[2]) ** 2
        rho = rho + np.where(r2 <= cut2, Zn * norm * np.exp(-r2 / (2 * sigma ** 2)), 0.0)
    return -rho / EPS0


def fft_poisson_periodic(q, shape, step_bohr, origin_bohr, coords_bohr, types, sigma=0.2, cutoff=6):
    """`Compute_hartree_fft` semantics (qmtools/qmtools.py:2578-2639, kernel_fft.cu:82-107).

    Periodic solve, k in cycles/Ang, V_hat = -RHS_hat / (4 pi^2 |k|^2), V_hat(0) = 0.
    Returns the real potential in volts as an (NX, NY, NZ) C-order array.
    """
    nx, ny, nz = shape
    h = step_bohr / ANG2BOR
    rhs = fft_rhs(q, shape, step_bohr, origin_bohr, coords_bohr, types, sigma, cutoff)
    F = np.fft.fftn(rhs)
    kx = np.fft.fftfreq(nx, d=h)
    ky = np.fft.fftfreq(ny, d=h)
    kz = np.fft.fftfreq(nz, d=h)
    K2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    K2[0, 0, 0] = 1.0
    F = -F / (4 * np.pi ** 2 * K2)
    F[0, 0, 0] = 0.0
    return np.fft.ifftn(F).real


def hockney_green(shape, step_ang, padded_shape):
    """Free-space Green's function 1/(4 pi EPS0 |r|) sampled on the padded grid (minimum image).

    G(0) uses the voxel-cube average of 1/|r|.  Returns the real array on the padded grid.
    """
    M = padded_shape
    h = step_ang
    ax = []
    for m in M:
        i = np.arange(m)
        ax.append(np.minimum(i, m - i) * h)
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    with np.errstate(divide="ignore"):
        G = np.where(r > 0, 1.0 / r, CUBE_INV_R / h)
    return G / (4 * np.pi * EPS0)


def hockney_poisson(q, shape, step_bohr, origin_bohr, coords_bohr, types, sigma=0.2, cutoff=6,
                    padded_shape=None):
    """Free-space (zero-padded, Hockney) solve of the same RHS; returns (NX, NY, NZ) volts.

    V_i = h^3 sum_j G(r_i - r_j) rho_tot_j  with rho_tot = -RHS * EPS0.
    """
    nx, ny, nz = shape
    if padded_shape is None:
        padded_shape = (2 * nx, 2 * ny, 2 * nz)
    h = step_bohr / ANG2BOR
    rho = -fft_rhs(q, shape, step_bohr, origin_bohr, coords_bohr, types, sigma, cutoff) * EPS0
    G = hockney_green(shape, h, padded_shape)
    pad = np.zeros(padded_shape)
    pad[:nx, :ny, :nz] = rho
    V = np.fft.irfftn(np.fft.rfftn(pad) * np.fft.rfftn(G), s=padded_shape, axes=(0, 1, 2))
    return V[:nx, :ny, :nz] * h ** 3

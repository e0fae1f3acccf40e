"""Oracle: grid reductions and nuclear (Vne) fields (test infrastructure).

Flat grids are x-fastest (idx = x + y*NX + z*NX*NY).
"""
import numpy as np


def qtot(q):
    """`Compute_qtot` / `gpu_total` (qmtools/qmtools.py:2796-2803, kernel_utils.cu:68-98): sum of field 0."""
    return float(np.sum(np.asarray(q, dtype=np.float64)))


def qdiff(a, b, rel=False):
    """`Compute_qdiff` (qmtools/qmtools.py:2818-2831, kernel_utils.cu:101-167).

    sum |a-b|, or 100 * sum |a-b|/b when rel.
    """
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    if rel:
        with np.errstate(divide="ignore", invalid="ignore"):
            return float(np.sum(d / b) * 100.0)
    return float(np.sum(d))


def centre_points(shape, step, origin):
    nx, ny, nz = shape
    h = float(step)
    i = np.arange(nx * ny * nz)
    x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
    o = np.asarray(origin, dtype=np.float64)
    return np.stack([(x + 0.5) * h + o[0], (y + 0.5) * h + o[1], (z + 0.5) * h + o[2]], axis=1)


def vne_centres(shape, step, origin, coords, types):
    """sum_A Z_A/|r - R_A| at voxel centres (`gpu_hartree_add_nuclei`, kernel_hartree.cu:209-251)."""
    pts = centre_points(shape, step, origin)
    out = np.zeros(pts.shape[0])
    for A, Z in zip(np.asarray(coords, dtype=np.float64), types):
        out += float(Z) / np.sqrt(np.sum((pts - A) ** 2, axis=1))
    return out


def vne_classic(shape, step, origin, coords, types, divisions=4):
    """`Compute_VNe_classic` (qmtools/qmtools.py:2750-2790, kernel_vne_classic.cu:13-84).

    Per voxel: sub-points x0 + (ii+1/2) dx with x0 = i*DX (corner frame, dx = DX/NDIV);
    average Z/d over every (sub-point, atom) with d != 0, then divide by DX^3.
    """
    nx, ny, nz = shape
    DX = float(step)
    dx = DX / divisions
    o = np.asarray(origin, dtype=np.float64)
    rel = np.asarray(coords, dtype=np.float64) - o
    i = np.arange(nx * ny * nz)
    base = np.stack([i % nx, (i // nx) % ny, i // (nx * ny)], axis=1) * DX
    acc = np.zeros(i.size)
    cnt = np.zeros(i.size)
    for ii in range(divisions):
        for jj in range(divisions):
            for kk in range(divisions):
                pt = base + (np.array([ii, jj, kk]) + 0.5) * dx
                for A, Z in zip(rel, types):
                    d2 = np.sum((pt - A) ** 2, axis=1)
                    ok = d2 != 0
                    with np.errstate(divide="ignore"):
                        acc += np.where(ok, float(Z) / np.sqrt(d2), 0.0)
                    cnt += ok
    return acc / cnt / DX ** 3


def vne_pseudo_step(q, shape, step, origin, coords, types, ads, dif):
    """One `gpu_vne` update (kernel_vne.cu:13-128) in FP64; returns (qout, sum |q - qout|).

    26-neighbour diffusion with periodic wrap, weight DIF/sqrt(|dx|+|dy|+|dz|), self weight
    1 - DIF*16.794682450997072, adsorption -ADS*q, source Z*exp(-d) for d < sqrt(3)*h,
    zero outer shell.
    """
    nx, ny, nz = shape
    V = np.asarray(q, dtype=np.float64).reshape(nz, ny, nx)
    out = np.zeros_like(V)
    for x in (-1, 0, 1):
        for y in (-1, 0, 1):
            for z in (-1, 0, 1):
                d = abs(x) + abs(y) + abs(z)
                if d < 1:
                    continue
                out += dif * np.roll(V, shift=(-z, -y, -x), axis=(0, 1, 2)) / np.sqrt(d)
    out += (1.0 - dif * 16.794682450997072) * V
    out -= V * ads
    h = float(step)
    pts = centre_points(shape, step, (0.0, 0.0, 0.0))
    o = np.asarray(origin, dtype=np.float64)
    src = np.zeros(pts.shape[0])
    for A, Z in zip(np.asarray(coords, dtype=np.float64) - o, types):
        dd = np.sqrt(np.sum((pts - A) ** 2, axis=1))
        src += np.where(dd < np.sqrt(3.0) * h, float(Z) * np.exp(-dd), 0.0)
    out += src.reshape(nz, ny, nx)
    out[0, :, :] = 0
    out[-1, :, :] = 0
    out[:, 0, :] = 0
    out[:, -1, :] = 0
    out[:, :, 0] = 0
    out[:, :, -1] = 0
    return out.ravel(), float(np.sum(np.abs(V - out)))


def vne_pseudo(shape, step, origin, coords, types, ads=0.1, dif=0.01, tolerance=1e-9, maxiters=None):
    """`Compute_VNe` host loop (qmtools/qmtools.py:2677-2745): ping-pong until mean |delta| <= tol.

    The convergence delta is that of the second update of each pair, divided by npts;
    the loop stops after maxiters pairs (default 10 * npts^(1/3)).
    Returns (field, pairs_done).
    """
    nx, ny, nz = shape
    npts = nx * ny * nz
    if maxiters is None:
        maxiters = 10 * np.power(npts, 1.0 / 3)
    res = np.zeros(npts)
    delta = 1.0
    niter = 0
    while delta > tolerance:
        out, _ = vne_pseudo_step(res, shape, step, origin, coords, types, ads, dif)
        res, d = vne_pseudo_step(out, shape, step, origin, coords, types, ads, dif)
        delta = d / npts
        niter += 1
        if niter > maxiters:
            break
    return res, niter

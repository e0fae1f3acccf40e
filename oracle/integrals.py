"""Oracle: Gaussian integrals over the real-solid-harmonic basis (test infrastructure).

McMurchie-Davidson Hermite expansion (Helgaker, Jorgensen, Olsen, "Molecular
Electronic-Structure Theory", ch. 9) in FP64, used to restate:

* the analytic electrostatic potential of the GTO density plus the nuclei,
  computed by `QMTools.Compute_hartree` / `gpu_hartree_GTO`
  (qmtools/qmtools.py:2436-2489, qmtools/cuda/kernel_hartree.cu:288-869):

      V(C) = -2 sum_{pq} P_pq (phi_p phi_q | 1/|r-C|) + sum_A Z_A / |C - R_A|

  at voxel corners C = origin + i h (kernel_hartree.cu:343-345); the nuclear term
  skips |C - R_A| <= 1e-8 (kernel_hartree.cu:852-865).  The reference sums the
  lower triangle p >= q with factor (2 - delta_pq) (kernel_hartree.cu:836-838);
  here P is symmetrised from its lower triangle, which is the same sum.

* the overlap matrix S (for Tr(PS)).

The reference evaluates closed forms for each (L, m) pair (kernel_hartree.cu:432-823);
the general Hermite route gives the same integrals for L <= 2.
"""
import math

import numpy as np

from .density import C_S, C_P, C_D0, C_D1, C_D2

# Cartesian expansion of Y_lm r^l: list of (coef, (i, j, k))  (kernel_density.cu:17-28)
CART = {
    (0, 0): [(C_S, (0, 0, 0))],
    (1, -1): [(C_P, (0, 1, 0))],
    (1, 0): [(C_P, (0, 0, 1))],
    (1, 1): [(C_P, (1, 0, 0))],
    (2, -2): [(C_D1, (1, 1, 0))],
    (2, -1): [(C_D1, (0, 1, 1))],
    (2, 0): [(2 * C_D0, (0, 0, 2)), (-C_D0, (2, 0, 0)), (-C_D0, (0, 2, 0))],
    (2, 1): [(C_D1, (1, 0, 1))],
    (2, 2): [(C_D2, (2, 0, 0)), (-C_D2, (0, 2, 0))],
}


def hermite_e(la, lb, a, b, xa, xb):
    """E[i][j][t] Hermite expansion coefficients in one direction (without exp(-mu X^2))."""
    p = a + b
    xp = (a * xa + b * xb) / p
    xpa, xpb = xp - xa, xp - xb
    E = np.zeros((la + 1, lb + 1, la + lb + 2))
    E[0, 0, 0] = 1.0
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            for t in range(i + j + 1):
                if i > 0:
                    v = xpa * E[i - 1, j, t]
                    if t > 0:
                        v += E[i - 1, j, t - 1] / (2 * p)
                    v += (t + 1) * E[i - 1, j, t + 1]
                else:
                    v = xpb * E[i, j - 1, t]
                    if t > 0:
                        v += E[i, j - 1, t - 1] / (2 * p)
                    v += (t + 1) * E[i, j - 1, t + 1]
                E[i, j, t] = v
    return E


def boys(nmax, T):
    """F_n(T) for n = 0..nmax, FP64, vectorised: series + downward recursion, asymptote for T > 40."""
    T = np.asarray(T, dtype=np.float64)
    out = np.empty((nmax + 1,) + T.shape)
    small = T <= 40.0
    Ts = T[small]
    if Ts.size:
        # F_nmax(T) = exp(-T) sum_k (2T)^k / ((2n+1)(2n+3)...(2n+2k+1))
        term = np.full_like(Ts, 1.0 / (2 * nmax + 1))
        acc = term.copy()
        for k in range(1, 200):
            term = term * (2 * Ts) / (2 * nmax + 2 * k + 1)
            acc += term
        et = np.exp(-Ts)
        f = et * acc
        out[nmax][small] = f
        for n in range(nmax - 1, -1, -1):
            f = (2 * Ts * f + et) / (2 * n + 1)
            out[n][small] = f
    big = ~small
    Tb = T[big]
    if Tb.size:
        for n in range(nmax + 1):
            dfact = 1.0
            for k in range(1, 2 * n, 2):
                dfact *= k
            out[n][big] = dfact / 2 ** (n + 1) * np.sqrt(np.pi / Tb ** (2 * n + 1))
    return out


def hermite_r(lmax, p, PC):
    """R_{tuv}(p, PC) for t+u+v <= lmax, dict {(t,u,v): array over points}."""
    X, Y, Z = PC[:, 0], PC[:, 1], PC[:, 2]
    T = p * (X * X + Y * Y + Z * Z)
    F = boys(lmax, T)
    # R^n_000
    Rn = {}
    for n in range(lmax + 1):
        Rn[(n, 0, 0, 0)] = (-2 * p) ** n * F[n]

    def R(n, t, u, v):
        key = (n, t, u, v)
        if key in Rn:
            return Rn[key]
        if t > 0:
            val = X * R(n + 1, t - 1, u, v)
            if t > 1:
                val = val + (t - 1) * R(n + 1, t - 2, u, v)
        elif u > 0:
            val = Y * R(n + 1, t, u - 1, v)
            if u > 1:
                val = val + (u - 1) * R(n + 1, t, u - 2, v)
        else:
            val = Z * R(n + 1, t, u, v - 1)
            if v > 1:
                val = val + (v - 1) * R(n + 1, t, u, v - 2)
        Rn[key] = val
        return val

    out = {}
    for t in range(lmax + 1):
        for u in range(lmax + 1 - t):
            for v in range(lmax + 1 - t - u):
                out[(t, u, v)] = R(0, t, u, v)
    return out


def shells_from_almos(almos, alphas, coeffs):
    """Group the per-function ALMO rows into shells: [(atom, L, alphas, coeffs, [functions], [m])]."""
    shells = []
    key = None
    for f in range(almos.shape[0]):
        a, L, m, so = (int(v) for v in almos[f])
        if key != (a, so):
            al = np.asarray(alphas[so:so + 20], dtype=np.float64)
            co = np.asarray(coeffs[so:so + 20], dtype=np.float64)
            nz = co != 0
            shells.append([a, L, al[nz], co[nz], [], []])
            key = (a, so)
        shells[-1][4].append(f)
        shells[-1][5].append(m)
    return shells


def sym_lower(dm):
    """Symmetric matrix built from the lower triangle p >= q (the part the reference reads)."""
    dm = np.asarray(dm, dtype=np.float64)
    lo = np.tril(dm)
    return lo + np.tril(dm, -1).T


def electron_potential(points, coords, almos, alphas, coeffs, dm):
    """sum_{pq} P_pq (phi_p phi_q | 1/|r - C|) at every point C, FP64 (no sign, no spin factor)."""
    coords = np.asarray(coords, dtype=np.float64)
    points = np.asarray(points, dtype=np.float64)
    P = sym_lower(dm)
    shells = shells_from_almos(almos, alphas, coeffs)
    V = np.zeros(points.shape[0])
    for iA, (aA, LA, alA, coA, fA, mA) in enumerate(shells):
        A = coords[aA]
        for iB, (aB, LB, alB, coB, fB, mB) in enumerate(shells):
            if iB < iA:
                continue
            fac = 1.0 if iA == iB else 2.0
            B = coords[aB]
            blk = P[np.ix_(fA, fB)]
            AB2 = float(np.sum((A - B) ** 2))
            for a, ca in zip(alA, coA):
                for b, cb in zip(alB, coB):
                    p = a + b
                    K = math.exp(-a * b / p * AB2)
                    if K * abs(ca * cb) < 1e-300:
                        continue
                    Pc = (a * A + b * B) / p
                    Ex = hermite_e(LA, LB, a, b, A[0], B[0])
                    Ey = hermite_e(LA, LB, a, b, A[1], B[1])
                    Ez = hermite_e(LA, LB, a, b, A[2], B[2])
                    D = {}
                    for ia, m1 in enumerate(mA):
                        for ib, m2 in enumerate(mB):
                            w = blk[ia, ib]
                            if w == 0.0:
                                continue
                            for c1, (i, k, mm) in CART[(LA, m1)]:
                                for c2, (j, l, n) in CART[(LB, m2)]:
                                    cc = w * c1 * c2
                                    for t in range(i + j + 1):
                                        for u in range(k + l + 1):
                                            for v in range(mm + n + 1):
                                                key = (t, u, v)
                                                D[key] = D.get(key, 0.0) + cc * Ex[i, j, t] * Ey[k, l, u] * Ez[mm, n, v]
                    if not D:
                        continue
                    R = hermite_r(LA + LB, p, Pc[None, :] - points)
                    pref = fac * ca * cb * K * 2 * math.pi / p
                    acc = np.zeros(points.shape[0])
                    for key, d in D.items():
                        acc += d * R[key]
                    V += pref * acc
    return V


def nuclear_potential(points, coords, types, rmin=1e-8):
    """sum_A Z_A / |C - R_A|, skipping |C - R_A| <= rmin (kernel_hartree.cu:852-865)."""
    points = np.asarray(points, dtype=np.float64)
    out = np.zeros(points.shape[0])
    for A, Z in zip(np.asarray(coords, dtype=np.float64), types):
        r = np.sqrt(np.sum((points - A) ** 2, axis=1))
        with np.errstate(divide="ignore"):
            out += np.where(r > rmin, float(Z) / r, 0.0)
    return out


def total_potential(points, coords, types, almos, alphas, coeffs, dm):
    """V(C) of `gpu_hartree_GTO`: -2 sum P (phi phi | 1/r_C) + sum Z/r (kernel_hartree.cu:836-865)."""
    return (-2.0 * electron_potential(points, coords, almos, alphas, coeffs, dm)
            + nuclear_potential(points, coords, types))


def voxel_corners(shape, step, origin, idx=None):
    """Corner points origin + i h, flat x-fastest (kernel_hartree.cu:343-345); idx selects flat indices."""
    nx, ny, nz = shape
    if idx is None:
        idx = np.arange(nx * ny * nz)
    idx = np.asarray(idx)
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    h = float(step)
    return np.stack([x * h + float(origin[0]), y * h + float(origin[1]), z * h + float(origin[2])], axis=1)


def overlap_matrix(coords, almos, alphas, coeffs):
    """S_pq = <phi_p | phi_q>, FP64."""
    coords = np.asarray(coords, dtype=np.float64)
    shells = shells_from_almos(almos, alphas, coeffs)
    N = almos.shape[0]
    S = np.zeros((N, N))
    for (aA, LA, alA, coA, fA, mA) in shells:
        A = coords[aA]
        for (aB, LB, alB, coB, fB, mB) in shells:
            B = coords[aB]
            AB2 = float(np.sum((A - B) ** 2))
            for a, ca in zip(alA, coA):
                for b, cb in zip(alB, coB):
                    p = a + b
                    K = math.exp(-a * b / p * AB2) * (math.pi / p) ** 1.5 * ca * cb
                    Ex = hermite_e(LA, LB, a, b, A[0], B[0])
                    Ey = hermite_e(LA, LB, a, b, A[1], B[1])
                    Ez = hermite_e(LA, LB, a, b, A[2], B[2])
                    for ia, m1 in enumerate(mA):
                        for ib, m2 in enumerate(mB):
                            s = 0.0
                            for c1, (i, k, mm) in CART[(LA, m1)]:
                                for c2, (j, l, n) in CART[(LB, m2)]:
                                    s += c1 * c2 * Ex[i, j, 0] * Ey[k, l, 0] * Ez[mm, n, 0]
                            S[fA[ia], fB[ib]] += K * s
    return S

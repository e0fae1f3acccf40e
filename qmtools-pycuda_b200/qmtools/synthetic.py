"""Seeded synthetic molecules, density matrices and grids for the benchmark workloads.

No public benchmark or dataset exists for this path; every input is generated here:

* geometry: uniform coordinates in a cube, rejection-sampled to a minimum pair
  separation of 1.8 bohr;
* elements: C0 is 2 C + 6 H; the others draw C:H:N:O = 10:14:3:3 (exact counts when the
  atom count is a multiple of 30, otherwise per-atom draws with those weights);
* density matrix: S = analytic FP64 overlap of the cc-pVDZ functions, Q = seeded random
  orthogonal matrix (QR of a Gaussian matrix, signs fixed), C = (S^-1/2 Q)[:, :n_occ],
  total density matrix P = 2 C C^T, so Tr(PS) = 2 n_occ.  n_occ = floor(sum Z / 2)
  (an odd electron count gives the +1 cation).  The reference convention stores the
  spin-up matrix P/2 = C C^T, which is what `Molecule` receives;
* grids: the cube's centre at the grid's centre (C0-C2), or bounding box + 3 bohr per side
  rounded up to a multiple of 8 points (batched and serving workloads).
"""
import math

import numpy as np

ANG2BOR = 1.8897259886
ELEMENTS = (6, 1, 7, 8)
WEIGHTS = (10, 14, 3, 3)

CONFIGS = {
    # name: (natoms or None, cube side bohr, grid points per axis, step bohr, seed)
    "c0": dict(natoms=8, side=6.0, n=64, step=0.2, seed=0, n_occ=7),
    "c1": dict(natoms=30, side=12.0, n=128, step=0.15, seed=1),
    "c2": dict(natoms=60, side=18.0, n=192, step=0.12, seed=2),
}


def element_list(natoms, rng, c0=False):
    if c0:
        return [6, 6] + [1] * (natoms - 2)
    if natoms % 30 == 0:
        k = natoms // 30
        lst = [6] * 10 * k + [1] * 14 * k + [7] * 3 * k + [8] * 3 * k
        rng.shuffle(lst)
        return lst
    p = np.array(WEIGHTS, dtype=float) / sum(WEIGHTS)
    return list(rng.choice(ELEMENTS, size=natoms, p=p))


def random_geometry(natoms, side, rng, min_sep=1.8, max_tries=200000):
    pts = []
    tries = 0
    while len(pts) < natoms:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the requested separation")
        x = rng.uniform(0.0, side, size=3)
        if all(np.sum((x - q) ** 2) >= min_sep * min_sep for q in pts):
            pts.append(x)
    return np.array(pts)


def cube_side(natoms):
    """Cube side (bohr) used for the batched and serving workloads: 12 (n/30)^(1/3)."""
    return 12.0 * (natoms / 30.0) ** (1.0 / 3.0)


# ---- FP64 overlap -----------------------------------------------------------------------
_YS = 0.28209479177387814
_YP = 0.4886025119029199
_YD1 = 1.0925484305920792
_YD0 = 0.31539156525252005
_YD2 = 0.5462742152960396
_CART = {
    0: [[(_YS, (0, 0, 0))]],
    1: [[(_YP, (0, 0, 1))], [(_YP, (1, 0, 0))], [(_YP, (0, 1, 0))]],
    2: [[(2 * _YD0, (0, 0, 2)), (-_YD0, (2, 0, 0)), (-_YD0, (0, 2, 0))],
        [(_YD1, (1, 0, 1))], [(_YD1, (0, 1, 1))],
        [(_YD2, (2, 0, 0)), (-_YD2, (0, 2, 0))], [(_YD1, (1, 1, 0))]],
}


def _e0_table(la, lb, a, b, xa, xb):
    """E^{ij}_0 for i <= la, j <= lb, vectorised over primitive pairs (no exp prefactor)."""
    p = a + b
    xp = (a * xa + b * xb) / p
    pa, pb, i2p = xp - xa, xp - xb, 0.5 / p
    E = {}
    one = np.ones_like(a)
    E[(0, 0, 0)] = one
    zero = np.zeros_like(a)
    for i in range(la + 1):
        for j in range(lb + 1):
            if i == 0 and j == 0:
                continue
            for t in range(i + j + 1):
                if i > 0:
                    v = pa * E.get((i - 1, j, t), zero) + (t + 1) * E.get((i - 1, j, t + 1), zero)
                    if t > 0:
                        v = v + i2p * E.get((i - 1, j, t - 1), zero)
                else:
                    v = pb * E.get((i, j - 1, t), zero) + (t + 1) * E.get((i, j - 1, t + 1), zero)
                    if t > 0:
                        v = v + i2p * E.get((i, j - 1, t - 1), zero)
                E[(i, j, t)] = v
    return {(i, j): E[(i, j, 0)] for i in range(la + 1) for j in range(lb + 1)}


def overlap(coords_bohr, almos, alphas, coeffs):
    """S (FP64) for the basis described by the reference ALMO table and padded tables."""
    coords = np.asarray(coords_bohr, dtype=np.float64)
    prims = {0: [], 1: [], 2: []}   # L -> rows (atom, alpha, coeff, func0)
    f = 0
    while f < almos.shape[0]:
        a, L, _, so = (int(v) for v in almos[f])
        for k in range(20):
            c = float(coeffs[so + k])
            if c != 0.0:
                prims[L].append((a, float(alphas[so + k]), c, f))
        f += 2 * L + 1
    Nf = almos.shape[0]
    S = np.zeros(Nf * Nf)
    for LA in (0, 1, 2):
        for LB in (0, 1, 2):
            if not prims[LA] or not prims[LB]:
                continue
            PA = np.array(prims[LA])
            PB = np.array(prims[LB])
            ia = np.repeat(np.arange(len(PA)), len(PB))
            ib = np.tile(np.arange(len(PB)), len(PA))
            atA = PA[ia, 0].astype(int)
            atB = PB[ib, 0].astype(int)
            a = PA[ia, 1]
            b = PB[ib, 1]
            ca = PA[ia, 2]
            cb = PB[ib, 2]
            fA = PA[ia, 3].astype(int)
            fB = PB[ib, 3].astype(int)
            A = coords[atA]
            B = coords[atB]
            p = a + b
            K = np.exp(-a * b / p * np.sum((A - B) ** 2, axis=1)) * (np.pi / p) ** 1.5 * ca * cb
            E = [_e0_table(LA, LB, a, b, A[:, d], B[:, d]) for d in range(3)]
            for k1, terms1 in enumerate(_CART[LA]):
                for k2, terms2 in enumerate(_CART[LB]):
                    s = np.zeros_like(a)
                    for c1, (i, k, m) in terms1:
                        for c2, (j, l, n) in terms2:
                            s = s + c1 * c2 * E[0][(i, j)] * E[1][(k, l)] * E[2][(m, n)]
                    idx = (fA + k1) * Nf + (fB + k2)
                    S += np.bincount(idx, weights=K * s, minlength=Nf * Nf)
    return S.reshape(Nf, Nf)


def random_orthogonal(n, rng):
    Q, R = np.linalg.qr(rng.standard_normal((n, n)))
    return Q * np.sign(np.diag(R))


def density_matrix(S, n_occ, rng):
    """Spin-up density matrix C C^T with C = (S^-1/2 Q)[:, :n_occ] (total P = 2 C C^T)."""
    w, U = np.linalg.eigh(S)
    if w.min() <= 1e-10:
        raise ValueError("overlap matrix is not positive definite")
    Sm12 = (U / np.sqrt(w)) @ U.T
    Q = random_orthogonal(S.shape[0], rng)
    C = Sm12 @ Q[:, :n_occ]
    return C @ C.T


class SyntheticMolecule:
    """Everything a workload needs for one molecule; `molecule(basis)` builds the API object."""

    def __init__(self, types, coords_bohr, n_occ, grid_shape, step_bohr, origin_bohr, seed):
        self.types = np.asarray(types, dtype=np.int32)
        self.coords_bohr = np.asarray(coords_bohr, dtype=np.float64)
        self.n_occ = int(n_occ)
        self.grid_shape = tuple(int(v) for v in grid_shape)
        self.step_bohr = float(step_bohr)
        self.origin_bohr = tuple(float(v) for v in origin_bohr)
        self.seed = seed
        self.dm = None

    def xyz_list(self):
        ang = self.coords_bohr / ANG2BOR
        return [[int(z), float(x), float(y), float(w)] for z, (x, y, w) in zip(self.types, ang)]

    def molecule(self, basis, Molecule):
        """Build `Molecule` (reference API) with the seeded density matrix."""
        if self.dm is None:
            almos, coords32 = self._almos_coords(basis)
            S = overlap(coords32, almos, basis.alphas, basis.coeffs)
            self.dm = density_matrix(S, self.n_occ, np.random.default_rng(1000 + self.seed))
        return Molecule(self.xyz_list(), self.dm, basis)

    def _almos_coords(self, basis):
        m = np.array(self.xyz_list(), dtype=np.float64)
        m[:, 1:] *= ANG2BOR
        coords32 = np.array(m[:, 1:], dtype=np.float32)
        rows = []
        for a, Z in enumerate(self.types):
            aos = basis.atomOffset[Z]
            for s in range(basis.nshells[Z]):
                L = basis.Ls[aos + s]
                for mi in range(2 * L + 1):
                    rows.append((a, L, basis.global_m_values[L, mi], basis.shellOffset[aos + s]))
        return np.array(rows, dtype=np.int16).reshape(-1, 4), coords32

    def grid(self, Grid):
        g = Grid((1,) + self.grid_shape, self.step_bohr / ANG2BOR, list(self.origin_bohr))
        return g


def config_molecule(name):
    """C0 / C1 / C2 of the benchmark definitions."""
    c = CONFIGS[name]
    rng = np.random.default_rng(c["seed"])
    types = element_list(c["natoms"], rng, c0=(name == "c0"))
    xyz = random_geometry(c["natoms"], c["side"], rng)
    n_occ = c.get("n_occ", int(sum(types)) // 2)
    ext = c["n"] * c["step"]
    centre = c["side"] / 2.0
    origin = (centre - ext / 2.0,) * 3
    return SyntheticMolecule(types, xyz, n_occ, (c["n"],) * 3, c["step"], origin, c["seed"])


def extent_molecule(natoms, seed, step=0.15, pad=3.0):
    """Molecule in a cube of side 12 (n/30)^(1/3) with a grid of its bounding box + pad per side."""
    rng = np.random.default_rng(seed)
    types = element_list(natoms, rng)
    xyz = random_geometry(natoms, cube_side(natoms), rng)
    lo = xyz.min(axis=0) - pad
    hi = xyz.max(axis=0) + pad
    n = np.ceil((hi - lo) / step / 8.0).astype(int) * 8
    n_occ = int(sum(types)) // 2
    return SyntheticMolecule(types, xyz, n_occ, tuple(n), step, tuple(lo), seed)


def batch_molecules(count=64, seed=3, lo=5, hi=60):
    """Batched workload: atom counts uniform in lo..hi."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(lo, hi + 1, size=count)
    return [extent_molecule(int(n), seed * 100000 + i) for i, n in enumerate(sizes)]


def serving_stream(rate, count, seed=4, lo=3, hi=120):
    """Serving workload: Poisson arrivals at `rate` req/s, atom counts log-uniform in lo..hi."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrivals = np.cumsum(gaps)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).round().astype(int)
    return [(float(t), extent_molecule(int(n), seed * 100000 + i)) for i, (t, n) in enumerate(zip(arrivals, sizes))]

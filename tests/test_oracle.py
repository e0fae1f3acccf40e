"""Oracle self-checks on known answers (CPU only).

The reference ships no tests or golden vectors; these known-answer checks pin the
oracle's mathematics, and tests/test_golden.py pins it against the reference kernels'
own outputs.
"""
import math

import numpy as np
import pytest
from scipy import special

import qmtools
from qmtools import synthetic as syn
from oracle import basis as ob
from oracle import density as od
from oracle import gridops as og
from oracle import integrals as oi
from oracle import poisson as op


def test_basis_layout_and_almos(basis):
    tabs = ob.reference_tables(qmtools.BASIS_CCPVDZ)
    for k in ("atomOffset", "nshells", "shellOffset", "Ls", "alphas", "coeffs"):
        assert np.array_equal(tabs[k], getattr(basis, k)), k
    b64 = ob.read_basis_fp64(qmtools.BASIS_CCPVDZ)
    assert [(L, len(a)) for L, a, _ in b64[6]] == [(0, 8), (0, 8), (0, 1), (1, 3), (1, 1), (2, 1)]
    assert [(L, len(a)) for L, a, _ in b64[1]] == [(0, 3), (0, 1), (1, 1)]
    assert 19 not in b64


def test_radial_normalisation():
    """Coefficients are normalised so that int r^(2L+2) R(r)^2 dr = 1 for every shell."""
    b64 = ob.read_basis_fp64(qmtools.BASIS_CCPVDZ)
    for Z in (1, 6, 7, 8, 17, 35):
        for L, a, c in b64[Z]:
            s = 0.0
            for ai, ci in zip(a, c):
                for aj, cj in zip(a, c):
                    s += ci * cj * math.gamma(L + 1.5) / (2 * (ai + aj) ** (L + 1.5))
            assert abs(s - 1.0) < 2e-6, (Z, L, s)


def test_boys_function_known_values():
    T = np.array([0.0, 1e-6, 0.5, 3.0, 12.0, 39.9, 40.1, 200.0])
    F = oi.boys(4, T)
    ref0 = np.where(T > 0, 0.5 * np.sqrt(np.pi / np.maximum(T, 1e-300)) * special.erf(np.sqrt(T)), 1.0)
    assert np.allclose(F[0], ref0, rtol=1e-13, atol=0)
    # F_n(0) = 1/(2n+1)
    assert np.allclose(F[:, 0], [1, 1 / 3, 1 / 5, 1 / 7, 1 / 9], rtol=1e-14)
    # derivative identity F_n' = -F_{n+1} (finite difference)
    d = 1e-5
    Fp = oi.boys(4, T[2:6] + d)
    Fm = oi.boys(4, T[2:6] - d)
    assert np.allclose((Fp[:4] - Fm[:4]) / (2 * d), -F[1:5, 2:6], rtol=1e-6)


def test_s_gaussian_potential_closed_form():
    """Potential of a normalised s Gaussian charge: erf(sqrt(2a) r) / r."""
    a = 0.7
    c = (2 * a / np.pi) ** 0.75 / oi.C_S  # so that phi = C_S * c e^{-a r^2} is normalised
    almos = np.array([[0, 0, 0, 0]], dtype=np.int16)
    alphas = np.zeros(20, dtype=np.float64)
    coeffs = np.zeros(20, dtype=np.float64)
    alphas[0] = a
    coeffs[0] = c
    pts = np.array([[0.3, 0.2, -0.1], [2.0, 0.0, 0.0], [0.0, 5.0, 1.0]])
    V = oi.electron_potential(pts, np.zeros((1, 3)), almos, alphas, coeffs, np.ones((1, 1)))
    r = np.linalg.norm(pts, axis=1)
    assert np.allclose(V, special.erf(np.sqrt(2 * a) * r) / r, rtol=1e-12)


def test_density_integrates_to_trace_ps(basis):
    """sum_v q_v approaches 2 Tr(PS) (reference convention) as the grid is refined."""
    sm = syn.config_molecule("c0")
    mol = sm.molecule(basis, qmtools.Molecule)
    S = oi.overlap_matrix(mol.coords, mol.ALMOs, basis.alphas, basis.coeffs)
    tr = float(np.sum(oi.sym_lower(mol.dm) * S))
    assert abs(tr - sm.n_occ) < 1e-5
    shape = (40, 40, 40)
    h = 0.33
    o = np.asarray(mol.coords, dtype=np.float64).mean(axis=0) - 20 * h
    q = od.density_qube_unscaled(shape, h, o, mol.coords, mol.ALMOs, basis.alphas, basis.coeffs, mol.dm)
    assert abs(q.sum() - 2 * tr) < 0.25   # quadrature error of the 0.33-bohr grid near the C nuclei


def test_gto_potential_far_field_is_net_charge(basis):
    """Far from the molecule V -> (sum Z - N_e) / r."""
    sm = syn.config_molecule("c0")
    mol = sm.molecule(basis, qmtools.Molecule)
    c = mol.coords.mean(axis=0).astype(np.float64)
    pts = c + np.array([[600.0, 0, 0], [0, -700.0, 0]])
    V = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, basis.alphas, basis.coeffs, mol.dm)
    r = np.linalg.norm(pts - c, axis=1)
    net = mol.qtot - 2 * sm.n_occ
    assert np.allclose(V * r, net, atol=0.02)   # dipole term ~ |d|/r


def test_jacobi_quadratic_known_answer():
    """Reference update on V = x^2+y^2+z^2-like fixed point: lap V = 6 -> Q/h^3 = 6 with zero BC."""
    n = 12
    h = 0.5
    Q = np.full(n ** 3, 6.0 * h ** 3)
    V = op.jacobi_sweeps(Q, (n, n, n), h, 3000)
    # discrete Poisson with zero Dirichlet data: compare with a direct sparse solve
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    m = n - 2
    I = sp.identity(m)
    D = sp.diags([1, -2, 1], [-1, 0, 1], shape=(m, m))
    Lap = (sp.kron(sp.kron(I, I), D) + sp.kron(sp.kron(I, D), I) + sp.kron(sp.kron(D, I), I)) / h ** 2
    rhs = np.full(m ** 3, 6.0)
    sol = spl.spsolve(Lap.tocsc(), rhs)
    got = V.reshape(n, n, n)[1:-1, 1:-1, 1:-1].ravel()
    assert np.allclose(got, sol, rtol=1e-6, atol=1e-9)


def test_periodic_fft_matches_direct_frequency_solve():
    rng = np.random.default_rng(0)
    shape = (8, 16, 8)
    q = rng.uniform(0, 0.01, size=np.prod(shape))
    V = op.fft_poisson_periodic(q, shape, 0.3, (0, 0, 0), np.array([[1.0, 1.2, 0.8]]), [6], sigma=0.3, cutoff=3)
    assert V.shape == shape
    # V solves lap V = RHS (spectral sense): check via FFT of V
    h = 0.3 / op.ANG2BOR
    rhs = op.fft_rhs(q, shape, 0.3, (0, 0, 0), np.array([[1.0, 1.2, 0.8]]), [6], 0.3, 3)
    k = [np.fft.fftfreq(n, d=h) for n in shape]
    K2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    lapV = np.fft.ifftn(-4 * np.pi ** 2 * K2 * np.fft.fftn(V)).real
    assert np.allclose(lapV, rhs - rhs.mean(), atol=1e-9 * np.abs(rhs).max())


def test_hockney_point_charge_is_coulomb():
    """A unit charge in one voxel: free-space solve gives 1/(4 pi eps0 r) away from it."""
    n = 16
    step_b = 0.4
    h = step_b / op.ANG2BOR
    q = np.zeros(n ** 3)
    q[8 + 8 * n + 8 * n * n] = -1.0   # electron grid convention: rho = -q/h^3 -> +1 e
    V = op.hockney_poisson(q, (n, n, n), step_b, (0, 0, 0), np.zeros((0, 3)), [], sigma=0.2, cutoff=6)
    i, j, k = 8 + 5, 8, 8
    r = 5 * h
    assert abs(V[i, j, k] - 1.0 / (4 * np.pi * op.EPS0 * r)) < 1e-10


def test_vne_classic_and_seed_conserve():
    types = [6, 1]
    coords = np.array([[1.03, 1.27, 1.11], [2.2, 1.3, 1.4]], dtype=np.float32)
    q = op.density_seed((8, 8, 8), 0.5, (0, 0, 0), coords, types)
    assert abs(q.sum() - 7.0) < 1e-5
    v = og.vne_classic((8, 8, 8), 0.5, (0, 0, 0), coords, types, divisions=2)
    assert np.all(v > 0)

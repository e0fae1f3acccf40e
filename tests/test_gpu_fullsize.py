"""Full-size and large-basis parity: the configurations the benchmark quotes, against the FP64
oracle and the reference kernels' checksums.

* C1 (30 atoms, N = 294) on the full 128^3 grid at 0.15 bohr, the default fp16x3 contraction;
* C2 (60 atoms, N = 588) on a small grid: the tensor-core contraction needs three output
  panels, the staged path (N > 320), which no smaller molecule reaches;
* C0's physical Hartree route: the analytic GTO potential on the grid's outer shell, then 2000
  Jacobi sweeps of lap V = -4 pi rho with that Dirichlet boundary and an FP64 residual.
"""
import ctypes as C

import numpy as np
import pytest

import qmtools
from qmtools import _native as N
from qmtools import synthetic as syn
from oracle import density as od
from oracle import integrals as oi
from oracle import poisson as op
from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

# rel-L2 tolerances against the FP64 oracle (the same bars as tests/test_gpu_density.py)
TOL = {"fp64": 1e-7, "fp32": 1e-6, "fp16x3": 1e-6, "tf32x3": 2e-6, "bf16x3": 1e-4}


@pytest.fixture(scope="module")
def c1(basis):
    sm = syn.config_molecule("c1")
    return sm, sm.molecule(basis, qmtools.Molecule)


def test_c1_full_grid_against_reference_checksum_and_oracle_planes(c1):
    """The bench's density (C1, 128^3 at 0.15 bohr, fp16x3) on the full grid: its FP64 sum against
    the reference kernel's on the same inputs (tests/golden/c1_bench.npz, made by
    tests/golden/make_golden.py from the reference's gpu_densityqube_shmem_subgrid), and six
    z-planes spread over the grid against the FP64 oracle."""
    sm, mol = c1
    g = sm.grid(qmtools.Grid)
    gold = dict(np.load(GOLDEN / "c1_bench.npz"))
    assert tuple(gold["shape"]) == g.space_shape()
    out = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False)
    # the reference accumulates per DM pair in FP32: 1e-6 of the total
    assert abs(out.qsum - float(gold["density_raw_s1"])) <= 1e-6 * float(gold["density_raw_s1"])
    scaled = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3")
    assert abs(float(np.sum(scaled.qube, dtype=np.float64)) - float(gold["density_s1"])) <= 1e-5 * float(gold["density_s1"])
    nx, ny, nz, h, ox, oy, oz = g._geom()
    q = out.qube.reshape(nz, ny, nx)          # numpy qube is (nf, nx, ny, nz) over x-fastest data
    got, ref = [], []
    for z in (0, 25, 51, 77, 102, 127):
        ref.append(od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs,
                                            mol.basisset.alphas, mol.basisset.coeffs, mol.dm, zslab=(z, z + 1)))
        got.append(q[z].ravel())
    got = np.concatenate(got)
    ref = np.concatenate(ref)
    err = rel_l2(got, ref)
    assert err <= TOL["fp16x3"], f"full-size C1 planes: rel-L2 {err:.3e}"


@pytest.fixture(scope="module")
def c2(basis):
    sm = syn.config_molecule("c2")
    return sm, sm.molecule(basis, qmtools.Molecule)


@pytest.mark.parametrize("prec", ["fp16x3", "tf32x3", "bf16x3", "fp32", "fp64"])
def test_c2_three_panels(c2, prec):
    """N = 588: kpad 640 gives three 224-column output panels in the staged tensor-core path
    (the automatic choice above N = 320), against the FP64 oracle on a 24^3 grid over the
    whole 18-bohr molecule."""
    sm, mol = c2
    assert mol.norbs == 588
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    n, step = 24, 0.85
    g = qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(c - n * step / 2 + 0.021))
    nx, ny, nz, h, ox, oy, oz = g._geom()
    ref = od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs,
                                   mol.basisset.alphas, mol.basisset.coeffs, mol.dm)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    err = rel_l2(out.qube.ravel(), ref)
    assert err <= TOL[prec], f"C2 {prec}: rel-L2 {err:.3e}"
    assert abs(out.qsum - ref.sum()) <= 10 * TOL[prec] * abs(ref.sum())


@pytest.fixture(scope="module")
def c0_route(basis):
    """C0 (8 atoms, N = 58) on 64^3 at 0.2 bohr: density (FP64, as the configuration asks), the
    analytic boundary and 2000 Dirichlet Jacobi sweeps through the facade."""
    sm = syn.config_molecule("c0")
    mol = sm.molecule(basis, qmtools.Molecule)
    g = sm.grid(qmtools.Grid)
    q = qmtools.QMTools.Compute_density(g, mol, precision="fp64")
    v = qmtools.QMTools.Compute_hartree_dirichlet(q, mol, max_sweeps=2000)
    return sm, mol, g, q, v


def _shell_index(nx, ny, nz):
    i = np.arange(nx * ny * nz)
    x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
    return i[(x == 0) | (x == nx - 1) | (y == 0) | (y == ny - 1) | (z == 0) | (z == nz - 1)]


def test_c0_boundary_is_the_analytic_potential(c0_route):
    """qmt_hartree_gto_boundary on the 64^3 shell (voxel centres) against the FP64
    McMurchie-Davidson oracle (oracle/integrals.py, restating gpu_hartree_GTO's potential,
    kernel_hartree.cu:288-869), on every 5th shell voxel."""
    sm, mol, g, q, v = c0_route
    nx, ny, nz, h, ox, oy, oz = g._geom()
    idx = _shell_index(nx, ny, nz)[::5]
    x, y, zz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    hd = float(h)
    pts = np.stack([ox + (x + 0.5) * hd, oy + (y + 0.5) * hd, oz + (zz + 0.5) * hd], axis=1)
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    got = v.qube.ravel()[idx]
    assert rel_l2(got, ref) <= 1e-6


def test_c0_dirichlet_jacobi_matches_fp64_oracle(c0_route):
    """2000 sweeps in FP32 on the device against the same sweeps in FP64 (oracle/poisson.py
    `jacobi_dirichlet`) from the same boundary values and charge grid: rel-L2 <= 1e-5.  The
    FP64 residual sum |V_2000 - V_1999| is reported and agrees with the oracle's."""
    sm, mol, g, q, v = c0_route
    nx, ny, nz, h, *_ = g._geom()
    assert v.sweeps == 2000
    rho = v.rho.field(0).cpu().numpy().astype(np.float64)
    bnd = v.qube.ravel().astype(np.float64)       # the outer shell is kept by the solve
    v1999 = op.jacobi_dirichlet(rho, (nx, ny, nz), float(h), bnd, 1999)
    w = v1999.reshape(nz, ny, nx).copy()
    s = (w[1:-1, 1:-1, :-2] + w[1:-1, 1:-1, 2:] + w[1:-1, 2:, 1:-1] + w[1:-1, :-2, 1:-1]
         + w[2:, 1:-1, 1:-1] + w[:-2, 1:-1, 1:-1])
    v2000 = w.copy()
    v2000[1:-1, 1:-1, 1:-1] = (s + 4 * np.pi * float(h) ** 2 * rho.reshape(nz, ny, nx)[1:-1, 1:-1, 1:-1]) / 6
    err = rel_l2(v.qube.ravel(), v2000.ravel())
    assert err <= 1e-5, f"Dirichlet Jacobi: rel-L2 {err:.3e}"
    ref_delta = float(np.abs(v2000 - w).sum())
    assert np.isfinite(v.delta) and v.delta > 0
    assert 0.5 * ref_delta <= v.delta <= 2.0 * ref_delta, (v.delta, ref_delta)


def test_c0_dirichlet_to_tolerance_stops_early(c0_route):
    """With a tolerance the solve stops at the first check whose FP64 residual is below it."""
    sm, mol, g, q, v = c0_route
    tol = 2.0 * v.delta
    w = qmtools.QMTools.Compute_hartree_dirichlet(q, mol, max_sweeps=20000, tolerance=tol, check_every=50)
    assert w.delta <= tol
    assert w.sweeps % 100 == 0 and w.sweeps <= 2000

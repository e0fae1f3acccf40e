"""Density parity: the CUDA path (every precision) against the FP64 oracle.

The oracle restates `gpu_densityqube_shmem_subgrid` (kernel_density.cu:34-155) and the
qtot rescale of `Compute_density` (qmtools/qmtools.py:2419-2424).
"""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import density as od
from conftest import rel_l2

pytestmark = pytest.mark.gpu

# rel-L2 tolerance of the unscaled grid against the FP64 oracle, per precision (the grid is
# stored in float32, so even the FP64 path carries ~3e-8 of output rounding)
TOL = {"fp64": 1e-7, "fp32": 1e-6, "fp16x3": 1e-6, "tf32x3": 2e-6, "bf16x3": 1e-4,
       "tf32": 5e-3, "bf16": 5e-2}


def _small_grid(sm, n, step):
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    o = c - n * step / 2
    return qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(o))


def _oracle(grid, mol, subgrid=1):
    nx, ny, nz, h, ox, oy, oz = grid._geom()
    return od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs,
                                    mol.basisset.alphas, mol.basisset.coeffs, mol.dm, subgrid)


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


@pytest.fixture(scope="module")
def c1(basis):
    sm = syn.config_molecule("c1")
    return sm, sm.molecule(basis, qmtools.Molecule)


@pytest.mark.parametrize("prec", list(TOL))
def test_density_c0_all_precisions(c0, prec):
    sm, mol = c0
    g = _small_grid(sm, 32, 0.4)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    got = out.qube.ravel()
    err = rel_l2(got, ref)
    assert err <= TOL[prec], f"{prec}: rel-L2 {err:.3e}"
    assert abs(out.qsum - ref.sum()) <= max(10 * TOL[prec], 1e-9) * abs(ref.sum())


@pytest.mark.parametrize("density_path", [1, 2, 3])
@pytest.mark.parametrize("shape", [(13, 7, 5), (33, 17, 9), (8, 4, 4)])
def test_density_partial_tile_blocks(c0, density_path, shape):
    """Grids that are not a multiple of the 8 x 4 x 4 voxel tiles, through the C ABI (the Grid
    class only makes multiples of 8): staged and fused paths, and the SIMT path for fp32.  Every
    voxel is written once and the edge tiles' unused rows nowhere."""
    import ctypes as C
    import torch
    from qmtools import _native as N
    sm, mol = c0
    nx, ny, nz = shape
    h = 0.45
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    o = (c - np.array(shape) * h / 2).astype(np.float32)   # the kernel's float32 origin
    ref = od.density_qube_unscaled((nx, ny, nz), np.float32(h), tuple(float(v) for v in o), mol.coords, mol.ALMOs,
                                   mol.basisset.alphas, mol.basisset.coeffs, mol.dm, 1)
    q = torch.full((nx * ny * nz + 64,), -7.0, dtype=torch.float32, device="cuda")   # sentinel tail
    N.call("qmt_set_density_path", density_path)
    try:
        for prec in ("fp16x3", "fp32"):
            s = C.c_double()
            N.call("qmt_density", mol.handle, nx, ny, nz, C.c_float(h), C.c_float(o[0]), C.c_float(o[1]),
                   C.c_float(o[2]), 1, N.PREC[prec], 0, C.c_void_p(q.data_ptr()), C.byref(s), N.stream_handle())
            got = q.cpu().numpy()
            assert np.all(got[nx * ny * nz:] == -7.0), "write beyond the grid"
            err = rel_l2(got[:nx * ny * nz], ref)
            assert err <= TOL[prec], f"{prec} {shape}: rel-L2 {err:.3e}"
            assert abs(s.value - ref.sum()) <= 10 * TOL[prec] * abs(ref.sum())
    finally:
        N.call("qmt_set_density_path", 0)


@pytest.mark.parametrize("prec", ["fp32", "fp16x3", "tf32x3", "bf16x3"])
def test_density_two_panels(c1, prec):
    """N = 294 needs two output panels in the tensor-core kernel."""
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp32", "fp16x3"])
def test_density_subgrid2(c0, prec):
    sm, mol = c0
    g = _small_grid(sm, 16, 0.6)
    ref = _oracle(g, mol, subgrid=2)
    out = qmtools.QMTools.Compute_density(g, mol, subgrid=2, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16x3"])
def test_density_sample_molecule(sample_molecule, prec):
    """Real molecule with Br/Cl (d shells with 5 primitives) and a CCSD density matrix."""
    mol = sample_molecule
    g = qmtools.Grid.DensityGrid(mol, 0.35, 1.0)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


def test_density_rescale_matches_reference_convention(c0):
    """After Compute_density the grid sums to the nuclear charge (qmtools/qmtools.py:2419-2424)."""
    sm, mol = c0
    g = _small_grid(sm, 32, 0.4)
    q, _, _ = od.compute_density(g.space_shape(), np.float32(g.step), g._geom()[4:], mol.coords, mol.types,
                                 mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs, mol.dm)
    out = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    assert abs(float(np.sum(out.qube, dtype=np.float64)) - float(mol.qtot)) < 1e-3
    assert rel_l2(out.qube.ravel(), q) <= 2e-6


def test_trace_ps(c0):
    from oracle import integrals as oi
    sm, mol = c0
    S = oi.overlap_matrix(mol.coords, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs)
    P = oi.sym_lower(mol.dm)
    assert abs(mol.trace_ps() - float(np.sum(P * S))) < 1e-10


def test_density_deterministic(c1):
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    a = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3")
    b = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3")
    assert np.array_equal(a.qube, b.qube)
    assert a.qsum == b.qsum


@pytest.fixture(params=[1, 2, 3], ids=["staged", "fused", "factored"])
def density_path(request):
    """Run a test once through each tensor-core implementation (the factored one takes the synthetic
    molecules' rank-n_occ density matrices), then restore automatic choice."""
    from qmtools import _native as N
    N.call("qmt_set_density_path", request.param)
    yield request.param
    N.call("qmt_set_density_path", 0)


@pytest.mark.parametrize("prec", ["fp16x3", "bf16x3", "bf16"])
def test_density_paths_agree_with_oracle(c1, density_path, prec):
    """Staged (HBM), fused (shared-memory) and factored tensor-core paths, N = 294."""
    sm, mol = c1
    g = _small_grid(sm, 24, 0.8)
    ref = _oracle(g, mol)
    out = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL[prec]


@pytest.mark.parametrize("sub", [1, 2, 3])
def test_fused_path_subgrids_and_small_basis(c0, density_path, sub):
    """N = 58 (one 64-wide K block), partial last tile, sub-point averaging."""
    sm, mol = c0
    g = _small_grid(sm, 16 if sub > 1 else 24, 0.6)
    ref = _oracle(g, mol, subgrid=sub)
    out = qmtools.QMTools.Compute_density(g, mol, subgrid=sub, precision="fp16x3", rescale=False)
    assert rel_l2(out.qube.ravel(), ref) <= TOL["fp16x3"]


def test_set_dm_and_translate_update_the_handle(basis):
    """A handle whose density matrix is replaced (and restored) and whose molecule is moved gives
    the density of a molecule built with those inputs: the device copies, the split operands and
    the host copy read by the analytic potential all follow the upload."""
    sm = syn.config_molecule("c0")
    mol = sm.molecule(basis, qmtools.Molecule)
    g = _small_grid(sm, 24, 0.45)
    qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False)   # operands built
    v0 = qmtools.Grid((1, 8, 8, 8), 0.9 / qmtools.ANG2BOR, list(np.asarray(sm.coords_bohr).mean(axis=0) - 3.6))
    qmtools.QMTools.Compute_hartree(v0, mol)                                     # host copy built
    rng = np.random.default_rng(5)
    dm1 = np.array(mol.dm, dtype=np.float64)
    dm2 = dm1 * (1.0 + 0.1 * rng.standard_normal(dm1.shape))
    dm2 = 0.5 * (dm2 + dm2.T)
    for dm in (dm2, dm1, dm2):
        mol.set_dm(dm)
        ref = _oracle(g, mol)
        for prec in ("fp16x3", "fp64"):
            got = qmtools.QMTools.Compute_density(g, mol, precision=prec, rescale=False).qube.ravel()
            assert rel_l2(got, ref) <= TOL[prec], prec
        fresh = qmtools.Molecule(sm.xyz_list(), np.array(dm, dtype=np.float32), basis)
        va = qmtools.Grid.emptyAs(v0)
        vb = qmtools.Grid.emptyAs(v0)
        qmtools.QMTools.Compute_hartree(va, mol)
        qmtools.QMTools.Compute_hartree(vb, fresh)
        assert rel_l2(va.qube.ravel(), vb.qube.ravel()) <= 1e-12
        fresh.release()
    mol.Translate(0.2, -0.1, 0.05)
    ref = _oracle(g, mol)
    got = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False).qube.ravel()
    assert rel_l2(got, ref) <= TOL["fp16x3"]
    mol.release()


def test_factored_path_needs_a_low_rank_psd_matrix(basis):
    """A density matrix that is not positive semi-definite is not factored (the host factorisation
    finds it indefinite): the automatic choice falls back to the unfactored fused path (same grid
    as asking for it), and asking for the factored path is an error.  The synthetic matrix (rank
    n_occ) is factored, and its grid matches the unfactored one."""
    import ctypes as C
    from qmtools import _native as N
    sm = syn.config_molecule("c0")
    mol = sm.molecule(basis, qmtools.Molecule)
    g = _small_grid(sm, 24, 0.45)
    try:
        grids = {}
        for path in (2, 3, 0):
            N.call("qmt_set_density_path", path)
            grids[path] = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False).qube.ravel()
        assert rel_l2(grids[3], grids[2]) <= 1e-6
        assert np.array_equal(grids[0], grids[3])
        rng = np.random.default_rng(11)
        dm = np.array(mol.dm, dtype=np.float64)
        dm = dm + 0.05 * rng.standard_normal(dm.shape)
        mol.set_dm(0.5 * (dm + dm.T))
        ref = _oracle(g, mol)
        N.call("qmt_set_density_path", 0)
        auto = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False).qube.ravel()
        assert rel_l2(auto, ref) <= TOL["fp16x3"]
        N.call("qmt_set_density_path", 2)
        fused = qmtools.QMTools.Compute_density(g, mol, precision="fp16x3", rescale=False).qube.ravel()
        assert np.array_equal(auto, fused)
        N.call("qmt_set_density_path", 3)
        nx, ny, nz, h, ox, oy, oz = g._geom()
        import torch
        q = torch.zeros(nx * ny * nz, device="cuda")
        st = N.load().qmt_density(mol.handle, nx, ny, nz, C.c_float(h), C.c_float(ox), C.c_float(oy), C.c_float(oz),
                                  1, N.PREC["fp16x3"], 0, C.c_void_p(q.data_ptr()), None, N.stream_handle())
        assert st == N.BAD_ARG
        assert b"factored" in N.load().qmt_last_error()
    finally:
        N.call("qmt_set_density_path", 0)
        mol.release()

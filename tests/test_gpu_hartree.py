"""Hartree routes against the oracle: analytic GTO potential, Jacobi, FP64 trace."""
import numpy as np
import pytest

import qmtools
from qmtools import synthetic as syn
from oracle import integrals as oi
from oracle import poisson as op
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c0(basis):
    sm = syn.config_molecule("c0")
    return sm, sm.molecule(basis, qmtools.Molecule)


def _grid(sm, n, step):
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    return qmtools.Grid((1, n, n, n), step / qmtools.ANG2BOR, list(c - n * step / 2 + 0.013))


def test_gto_potential_corners(c0):
    """Compute_hartree at voxel corners vs the McMurchie-Davidson oracle (FP64 vs FP64)."""
    sm, mol = c0
    g = _grid(sm, 16, 0.7)
    qmtools.QMTools.Compute_hartree(g, mol)
    pts = oi.voxel_corners(g.space_shape(), g.step, g._geom()[4:])
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    assert rel_l2(g.qube.ravel(), ref) < 1e-6


def test_gto_potential_sample_molecule_points(sample_molecule):
    """d shells, many primitives, real CCSD density matrix; arbitrary points."""
    import ctypes as C
    import torch
    mol = sample_molecule
    rng = np.random.default_rng(7)
    pts = (mol.coords.mean(axis=0) + rng.uniform(-6, 6, size=(300, 3))).astype(np.float32)
    pt = torch.from_numpy(pts.ravel()).cuda()
    out = torch.empty(300, dtype=torch.float32, device="cuda")
    from qmtools import _native as N
    N.call("qmt_hartree_gto_points", mol.handle, 300, C.c_void_p(pt.data_ptr()), C.c_void_p(out.data_ptr()),
           N.stream_handle())
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6


def test_jacobi_reference_update(c0):
    """gpu_hartree_iteration semantics (kernel_hartree.cu:85-171), FP32 against an FP32 restatement."""
    import ctypes as C
    import torch
    from qmtools import _native as N
    sm, mol = c0
    g = _grid(sm, 24, 0.5)
    q = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    seed = qmtools.QMTools.Compute_qseed(g, mol)
    rho = (seed.qube.ravel() - q.qube.ravel()).astype(np.float32)
    nx, ny, nz, h, *_ = g._geom()
    r = torch.from_numpy(rho).cuda()
    v = torch.zeros_like(r)
    t = torch.zeros_like(r)
    sw = C.c_int()
    dl = C.c_double()
    N.call("qmt_jacobi", nx, ny, nz, h, C.c_void_p(r.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(t.data_ptr()),
           40, 100, 0.0, C.byref(sw), C.byref(dl), N.stream_handle())
    ref32 = op.jacobi_sweeps(rho, (nx, ny, nz), np.float32(h), 40, dtype=np.float32)
    got = v.cpu().numpy()
    assert sw.value == 40
    assert np.max(np.abs(got - ref32)) <= 1e-6 * np.max(np.abs(ref32))
    ref64 = op.jacobi_sweeps(rho, (nx, ny, nz), h, 40, dtype=np.float64)
    assert rel_l2(got, ref64) < 1e-5


def test_compute_hartree_iter_stops_at_cap(c0):
    sm, mol = c0
    g = _grid(sm, 16, 0.5)
    q = qmtools.QMTools.Compute_density(g, mol, precision="fp32")
    with pytest.warns(UserWarning):
        v = qmtools.QMTools.Compute_hartree_iter(q, mol, tolerance=1e-30, max_sweeps=400)
    assert v.sweeps == 400


@pytest.fixture(scope="module")
def c1(basis):
    sm = syn.config_molecule("c1")
    return sm, sm.molecule(basis, qmtools.Molecule)


def _boundary(mol, g, precision):
    import ctypes as C
    import torch
    from qmtools import _native as N
    nx, ny, nz, h, ox, oy, oz = g._geom()
    v = torch.zeros(nx * ny * nz, device="cuda")
    N.call("qmt_set_gto_precision", N.PREC[precision])
    try:
        N.call("qmt_hartree_gto_boundary", mol.handle, nx, ny, nz, h, ox, oy, oz, C.c_void_p(v.data_ptr()),
               N.stream_handle())
    finally:
        N.call("qmt_set_gto_precision", N.PREC["fp32"])
    return v.cpu().numpy()


def _shell(nx, ny, nz):
    i = np.arange(nx * ny * nz)
    x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
    return i[(x == 0) | (x == nx - 1) | (y == 0) | (y == ny - 1) | (z == 0) | (z == nz - 1)]


def test_gto_boundary_fp32_against_fp64_kernel_c1(c1):
    """The default FP32 kernel (asymptotic Boys functions in the far field, FP64 accumulation) on
    all 96,776 boundary voxels of the medium molecule's 128^3 grid against the FP64 kernel, and
    the interior left untouched by both."""
    sm, mol = c1
    g = sm.grid(qmtools.Grid)
    nx, ny, nz = g.space_shape()
    v32 = _boundary(mol, g, "fp32")
    v64 = _boundary(mol, g, "fp64")
    sh = _shell(nx, ny, nz)
    assert sh.size == 96776
    assert rel_l2(v32[sh], v64[sh]) <= 1e-6
    inner = np.setdiff1d(np.arange(nx * ny * nz), sh)
    assert not np.any(v32[inner]) and not np.any(v64[inner])


def test_gto_boundary_fp32_against_oracle_c1(c1):
    """FP32 kernel against the FP64 McMurchie-Davidson oracle on 300 boundary voxels of C1."""
    sm, mol = c1
    g = sm.grid(qmtools.Grid)
    nx, ny, nz, h, ox, oy, oz = g._geom()
    v32 = _boundary(mol, g, "fp32")
    idx = _shell(nx, ny, nz)[::323]
    x, y, z = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    hd = float(h)
    pts = np.stack([ox + (x + 0.5) * hd, oy + (y + 0.5) * hd, oz + (z + 0.5) * hd], axis=1)
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             mol.dm)
    assert rel_l2(v32[idx], ref) <= 1e-6


def test_gto_fp32_near_field_corners(c0):
    """Corners of a 16^3 grid through the molecule (most terms near-field) in both precisions."""
    sm, mol = c0
    g = _grid(sm, 16, 0.7)
    from qmtools import _native as N
    out = {}
    for prec in ("fp32", "fp64"):
        N.call("qmt_set_gto_precision", N.PREC[prec])
        try:
            v = qmtools.Grid.emptyAs(g)
            qmtools.QMTools.Compute_hartree(v, mol)
            out[prec] = v.qube.ravel()
        finally:
            N.call("qmt_set_gto_precision", N.PREC["fp32"])
    assert rel_l2(out["fp32"], out["fp64"]) <= 1e-6


def _jacobi_call(name, shape, h, rho, v, t, sweeps, check_every=100, tol=0.0):
    import ctypes as C
    from qmtools import _native as N
    nx, ny, nz = shape
    so, dl = C.c_int(), C.c_double()
    st = getattr(N.load(), name)(nx, ny, nz, C.c_float(h), C.c_void_p(rho.data_ptr()), C.c_void_p(v.data_ptr()),
                                 C.c_void_p(t.data_ptr()), sweeps, check_every, tol, C.byref(so), C.byref(dl),
                                 N.stream_handle())
    return st, so.value, dl.value


@pytest.mark.parametrize("mode", ["qmt_jacobi", "qmt_jacobi_dirichlet"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 48, 40), (16, 16, 17), (8, 8, 2)])
def test_jacobi_kernels_give_identical_grids(mode, shape):
    """The persistent grid-barrier kernel and the single-cluster kernel (field in the CTAs' shared
    memory, cluster barrier per sweep) give identical grids: slabs of 4, 3, 2 and 1 planes per CTA
    (a ragged last slab), x neighbours across warp boundaries (nx = 32, 16, 8), 302 sweeps with a
    check every 25 pairs."""
    import torch
    from qmtools import _native as N
    N.ensure_device()
    n = int(np.prod(shape))
    g = torch.Generator(device="cuda").manual_seed(11)
    rho = torch.rand(n, device="cuda", generator=g) - 0.5
    v0 = torch.rand(n, device="cuda", generator=g)
    out = {}
    for path in (1, 2):
        N.call("qmt_set_jacobi_path", path)
        try:
            v = v0.clone()
            t = torch.zeros_like(v)
            st, sw, dl = _jacobi_call(mode, shape, 0.2, rho, v, t, 302, check_every=25, tol=-1.0)
        finally:
            N.call("qmt_set_jacobi_path", 0)
        assert st == N.OK, (path, N.load().qmt_last_error())
        assert sw == 302
        out[path] = (v.cpu().numpy(), dl)
    assert np.array_equal(out[1][0], out[2][0])
    assert abs(out[1][1] - out[2][1]) <= 1e-12 * abs(out[1][1])


def test_jacobi_kernels_stop_at_tolerance():
    """The cluster kernel's FP64 residual stops the solve at the first check below tol, like the
    grid-barrier kernel."""
    import torch
    from qmtools import _native as N
    N.ensure_device()
    shape = (64, 64, 64)
    rho = torch.zeros(64 ** 3, device="cuda")
    v0 = torch.rand(64 ** 3, device="cuda")
    res = {}
    for path in (1, 2):
        N.call("qmt_set_jacobi_path", path)
        try:
            v = v0.clone()
            t = torch.zeros_like(v)
            st, sw, dl = _jacobi_call("qmt_jacobi_dirichlet", shape, 0.2, rho, v, t, 100000, check_every=10,
                                      tol=50.0)
        finally:
            N.call("qmt_set_jacobi_path", 0)
        assert st == N.OK and dl <= 50.0 and sw % 20 == 0
        res[path] = (sw, v.cpu().numpy())
    assert res[1][0] == res[2][0]
    assert np.array_equal(res[1][1], res[2][1])

"""Bounded device waits that run out: the kernel returns early with an error flag, the call
reports QMT_CUDA_ERR, the flag is cleared, and the next call on the same context is correct.

The wait limit is shortened to 1 ns with qmt_set_wait_limit_ns, so a wait that cannot be
satisfied at once (a grid barrier that other CTAs have not reached yet, a pipeline barrier
whose producer has not finished) gives up.  No wait is left unbounded and nothing faults: the
kernels drain their own copies and tensor-core work before they leave, with a separate limit.
"""
import ctypes as C

import numpy as np
import pytest

import qmtools
from qmtools import _native as N
from qmtools import synthetic as syn

pytestmark = pytest.mark.gpu


def _jacobi(n, sweeps, rho, v, t):
    so, dl = C.c_int(), C.c_double()
    st = N.load().qmt_jacobi(n, n, n, C.c_float(0.2), C.c_void_p(rho.data_ptr()), C.c_void_p(v.data_ptr()),
                             C.c_void_p(t.data_ptr()), sweeps, 100, 0.0, C.byref(so), C.byref(dl),
                             N.stream_handle())
    return st, so.value


@pytest.fixture
def grid_barrier_path():
    """The persistent Jacobi kernel (the one with a software grid barrier between sweeps)."""
    N.call("qmt_set_jacobi_path", 1)
    try:
        yield
    finally:
        N.call("qmt_set_jacobi_path", 0)


def test_jacobi_grid_barrier_gives_up_and_recovers(grid_barrier_path):
    import torch
    N.ensure_device()
    n = 64
    g = torch.Generator(device="cuda").manual_seed(3)
    rho = torch.rand(n ** 3, device="cuda", generator=g)
    ref_v = torch.zeros_like(rho)
    t = torch.zeros_like(rho)
    assert _jacobi(n, 200, rho, ref_v, t) == (N.OK, 200)
    v = torch.zeros_like(rho)
    N.call("qmt_set_wait_limit_ns", 1)
    try:
        st, sweeps = _jacobi(n, 200, rho, v, t)
    finally:
        N.call("qmt_set_wait_limit_ns", 0)
    assert st == N.CUDA_ERR, N.STATUS_NAMES.get(st, st)
    assert b"timed out" in N.load().qmt_last_error()
    assert sweeps < 200
    v.zero_()
    assert _jacobi(n, 200, rho, v, t) == (N.OK, 200)
    assert torch.equal(v, ref_v)


@pytest.mark.parametrize("path", [2, 1, 3], ids=["fused", "staged", "factored"])
def test_density_pipeline_waits_give_up_and_recover(basis, path):
    """Both tensor-core kernels (fused: shared-memory Phi'; staged: TMA-fed) give up on their
    pipeline barriers; the sticky flag is reported by the call that returns the sum, cleared,
    and the next call gives the same grid as before."""
    import torch
    sm = syn.config_molecule("c1")
    mol = sm.molecule(basis, qmtools.Molecule)
    c = np.asarray(sm.coords_bohr).mean(axis=0)
    g = qmtools.Grid((1, 32, 32, 32), 0.6 / qmtools.ANG2BOR, list(c - 16 * 0.6))
    nx, ny, nz, h, ox, oy, oz = g._geom()
    q = torch.zeros(nx * ny * nz, device="cuda")

    def density():
        s = C.c_double()
        st = N.load().qmt_density(mol.handle, nx, ny, nz, h, ox, oy, oz, 1, N.PREC["fp16x3"], 0,
                                  C.c_void_p(q.data_ptr()), C.byref(s), N.stream_handle())
        return st, s.value

    N.call("qmt_set_density_path", path)
    try:
        st, ref_sum = density()
        assert st == N.OK
        ref = q.clone()
        N.call("qmt_set_wait_limit_ns", 1)
        try:
            st, _ = density()
        finally:
            N.call("qmt_set_wait_limit_ns", 0)
        assert st == N.CUDA_ERR, N.STATUS_NAMES.get(st, st)
        assert b"gave up waiting" in N.load().qmt_last_error()
        q.zero_()
        st, s = density()
        assert st == N.OK
        assert s == ref_sum
        assert torch.equal(q, ref)
    finally:
        N.call("qmt_set_density_path", 0)
        mol.release()

"""The sm_100a kernels against the reference kernels' own outputs (golden fixtures)."""
from pathlib import Path

import numpy as np
import pytest

import qmtools
from oracle import ref_cases as rc
from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = [c for c in rc.CASES if c != "c1_bench" and (GOLDEN / f"{c}.npz").exists()]


@pytest.fixture(scope="module")
def inputs(basis):
    cache = {}

    def get(case):
        if case not in cache:
            cache[case] = rc.case_inputs(case, basis)
        return cache[case]
    return get


@pytest.mark.parametrize("prec", ["fp32", "fp16x3"])
@pytest.mark.parametrize("case", CASES)
def test_density_vs_reference(case, prec, inputs):
    g = dict(np.load(GOLDEN / f"{case}.npz"))
    mol, grid = inputs(case)
    for key in [k for k in g if k.startswith("density_raw_s")]:
        s = int(key.rsplit("s", 1)[1])
        raw = qmtools.QMTools.Compute_density(grid, mol, subgrid=s, precision=prec, rescale=False)
        assert rel_l2(raw.qube.ravel(), g[key]) < 1e-4
        out = qmtools.QMTools.Compute_density(grid, mol, subgrid=s, precision=prec)
        assert rel_l2(out.qube.ravel(), g[f"density_s{s}"]) < 1e-4
        assert abs(out.qsum - float(g[f"density_total_s{s}"])) < 1e-4 * out.qsum


@pytest.mark.parametrize("case", CASES)
def test_gto_ss_block_vs_reference(case, inputs, basis):
    """The S-S part, where the reference's closed form is exact, against the reference kernel."""
    g = dict(np.load(GOLDEN / f"{case}.npz"))
    if "hartree_gto_ss" not in g:
        pytest.skip("no analytic potential in this case")
    mol, grid = inputs(case)
    s_only = mol.ALMOs[:, 1] == 0
    dm_ss = np.where(np.outer(s_only, s_only), mol.dm, 0).astype(np.float32)
    m2 = qmtools.Molecule([[int(z), *(c / qmtools.ANG2BOR)] for z, c in zip(mol.types, mol.coords.astype(np.float64))],
                          dm_ss, basis)
    m2.coords = mol.coords.copy()
    v = qmtools.Grid.emptyAs(grid)
    qmtools.QMTools.Compute_hartree(v, m2)
    assert rel_l2(v.qube.ravel(), g["hartree_gto_ss"]) < 1e-5   # the reference kernel is FP32


def test_seed_jacobi_fft_vne_vs_reference(inputs):
    import ctypes as C
    import torch
    from qmtools import _native as N
    if "c0_32" not in CASES:
        pytest.skip("c0_32 fixture missing")
    g = dict(np.load(GOLDEN / "c0_32.npz"))
    mol, grid = inputs("c0_32")
    T = qmtools.QMTools
    seed = T.Compute_qseed(grid, mol)
    assert np.array_equal(seed.qube.ravel(), g["seed"])
    nx, ny, nz, h, *_ = grid._geom()
    rho = torch.from_numpy(g["jacobi_rho"]).cuda()
    v = torch.zeros_like(rho)
    t = torch.zeros_like(rho)
    N.call("qmt_jacobi", nx, ny, nz, h, C.c_void_p(rho.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(t.data_ptr()),
           40, 100, 0.0, None, None, N.stream_handle())
    ref = g["jacobi_40"]
    assert np.max(np.abs(v.cpu().numpy() - ref)) <= 2e-6 * np.max(np.abs(ref))
    q = qmtools.Grid.emptyAs(grid)
    q.LoadFromNPY(g["density_s1"].reshape(q.shape))
    V = T.Compute_hartree_fft(q, mol, sigma=rc.FFT_PARAMS["sigma"], cutoff=rc.FFT_PARAMS["cutoff"])
    assert rel_l2(V.ravel(), g["fft_periodic"]) < 1e-4
    vc = T.Compute_VNe_classic(grid, mol, divisions=3)
    assert rel_l2(vc.qube.ravel(), g["vne_classic"]) < 1e-5
    vp = T.Compute_VNe(grid, mol, adsorb=rc.VNE_PARAMS["adsorb"], diff=rc.VNE_PARAMS["diff"], tolerance=-1.0,
                       maxiters=5)
    assert vp.iterations == 6
    assert rel_l2(vp.qube.ravel(), g["vne_pseudo_6"]) < 1e-5
    a = qmtools.Grid.emptyAs(grid)
    b = qmtools.Grid.emptyAs(grid)
    a.LoadFromNPY(g["density_s1"].reshape(a.shape))
    b.LoadFromNPY((g["density_raw_s1"] + np.float32(1e-3)).reshape(b.shape))
    assert abs(T.Compute_qdiff(a, b) - g["qdiff_rel0"]) < 1e-4 * g["qdiff_rel0"]
    assert abs(T.Compute_qdiff(a, b, rel=True) - 100 * g["qdiff_rel1"]) < 1e-3 * 100 * g["qdiff_rel1"]

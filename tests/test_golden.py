"""Pin the oracle against the reference's own kernel outputs (CPU).

tests/golden/<case>.npz hold outputs of the reference CUDA kernels, compiled from the
reference sources with the reference host's substitutions (oracle/build_ref.py) and run on
a B200 by tests/golden/make_golden.py.  The reference computes in FP32; tolerances below
are the FP32-vs-FP64 agreement measured for each quantity.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import density as od
from oracle import gridops as og
from oracle import integrals as oi
from oracle import poisson as op
from oracle import ref_cases as rc
from conftest import rel_l2

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = [c for c in rc.CASES if c != "c1_bench" and (GOLDEN / f"{c}.npz").exists()]


def _load(case):
    return dict(np.load(GOLDEN / f"{case}.npz"))


@pytest.fixture(scope="module")
def inputs(basis):
    cache = {}

    def get(case):
        if case not in cache:
            cache[case] = rc.case_inputs(case, basis)
        return cache[case]
    return get


def test_golden_fixtures_present():
    assert CASES, "no golden fixtures under tests/golden"


@pytest.mark.parametrize("case", CASES)
def test_density_matches_reference_kernel(case, inputs):
    g = _load(case)
    mol, grid = inputs(case)
    shape = tuple(int(v) for v in g["shape"])
    for key in [k for k in g if k.startswith("density_raw_s")]:
        s = int(key.rsplit("s", 1)[1])
        ref = od.density_qube_unscaled(shape, g["step"], g["origin"], mol.coords, mol.ALMOs, mol.basisset.alphas,
                                       mol.basisset.coeffs, mol.dm, s)
        assert rel_l2(g[key], ref) < 1e-4, key          # reference: FP32 per-pair accumulation
        assert abs(float(g[f"density_total_s{s}"]) - ref.sum()) < 1e-4 * ref.sum()
        scaled = ref * (float(mol.qtot) / ref.sum())
        assert rel_l2(g[f"density_s{s}"], scaled) < 1e-4


def _gto_cases():
    return [c for c in CASES if "hartree_gto_ss" in _load(c)]


@pytest.mark.parametrize("case", _gto_cases())
def test_gto_ss_block_matches_reference_kernel(case, inputs):
    """S-S products: the reference's closed form (kernel_hartree.cu:432-434) is exact."""
    g = _load(case)
    mol, grid = inputs(case)
    shape = tuple(int(v) for v in g["shape"])
    idx = np.arange(0, int(np.prod(shape)), 5)
    pts = oi.voxel_corners(shape, g["step"], g["origin"], idx=idx)
    s_only = mol.ALMOs[:, 1] == 0
    dm_ss = np.where(np.outer(s_only, s_only), mol.dm, 0).astype(np.float32)
    ref = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                             dm_ss)
    assert rel_l2(g["hartree_gto_ss"][idx], ref) < 1e-5    # the reference kernel computes in FP32


def test_sp_product_potential_matches_quadrature():
    """Exact s-p product potential (brute-force quadrature) = McMurchie-Davidson oracle.

    The reference's S-P closed form (kernel_hartree.cu:436-449) gives -1.43 x this value for
    the same pair, which is why its full analytic potential (with p and d functions) differs
    from the exact one; tests/test_golden.py::test_reference_gto_with_p_d_is_not_exact shows it.
    """
    a, b = 0.9, 0.6
    A = np.array([0.3, -0.2, 0.1])
    B = np.array([-0.4, 0.5, 0.2])
    C = np.array([2.5, 1.7, -1.9])
    h = 0.04                       # C is not a quadrature node
    ax = np.arange(-4, 4, h)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    ga = np.exp(-a * ((X - A[0]) ** 2 + (Y - A[1]) ** 2 + (Z - A[2]) ** 2))
    gb = np.exp(-b * ((X - B[0]) ** 2 + (Y - B[1]) ** 2 + (Z - B[2]) ** 2))
    r = np.sqrt((X - C[0]) ** 2 + (Y - C[1]) ** 2 + (Z - C[2]) ** 2)
    brute = np.sum(ga * (X - B[0]) * gb / r) * h ** 3
    # the oracle's (s | p_x) potential for unit coefficients, stripped of the Y_lm constants
    almos = np.array([[0, 0, 0, 0], [1, 1, 1, 20]], dtype=np.int16)
    al = np.zeros(40)
    co = np.zeros(40)
    al[0], co[0], al[20], co[20] = a, 1.0, b, 1.0
    dm = np.array([[0.0, 0.0], [1.0, 0.0]])      # lower triangle: P_10 = 1 -> 2 * (phi_1 phi_0 | 1/r)
    v = oi.electron_potential(C[None, :], np.stack([A, B]), almos, al, co, dm)[0]
    v /= 2 * oi.C_S * oi.C_P
    assert abs(v - brute) < 1e-8 * abs(brute)


@pytest.mark.parametrize("case", _gto_cases())
def test_reference_gto_with_p_d_is_not_exact(case, inputs):
    """With p and d functions the reference's analytic potential departs from the exact one."""
    g = _load(case)
    mol, grid = inputs(case)
    shape = tuple(int(v) for v in g["shape"])
    idx = np.arange(0, int(np.prod(shape)), 11)
    pts = oi.voxel_corners(shape, g["step"], g["origin"], idx=idx)
    exact = oi.total_potential(pts, mol.coords, mol.types, mol.ALMOs, mol.basisset.alphas, mol.basisset.coeffs,
                               mol.dm)
    assert rel_l2(g["hartree_gto"][idx], exact) > 0.05


def test_seed_jacobi_fft_vne_match_reference_kernels(inputs):
    if "c0_32" not in CASES:
        pytest.skip("c0_32 fixture missing")
    g = _load("c0_32")
    mol, grid = inputs("c0_32")
    shape = tuple(int(v) for v in g["shape"])
    seed = op.density_seed(shape, g["step"], g["origin"], mol.coords, mol.types)
    assert np.array_equal(seed, g["seed"])
    j32 = op.jacobi_sweeps(g["jacobi_rho"], shape, g["step"], 40, dtype=np.float32)
    assert np.max(np.abs(j32 - g["jacobi_40"])) <= 2e-6 * np.max(np.abs(g["jacobi_40"]))
    rhs = op.fft_rhs(g["density_s1"], shape, float(g["step"]), g["origin"], mol.coords, mol.types, 0.2, 6)
    assert rel_l2(g["fft_rhs"], rhs.ravel()) < 1e-5
    V = op.fft_poisson_periodic(g["density_s1"], shape, float(g["step"]), g["origin"], mol.coords, mol.types, 0.2, 6)
    assert rel_l2(g["fft_periodic"], V.ravel()) < 1e-4
    vc = og.vne_classic(shape, g["step"], g["origin"], mol.coords, mol.types, divisions=3)
    assert rel_l2(g["vne_classic"], vc) < 1e-5
    v6, _ = og.vne_pseudo(shape, g["step"], g["origin"], mol.coords, mol.types, ads=rc.VNE_PARAMS["adsorb"],
                          dif=rc.VNE_PARAMS["diff"], tolerance=-1.0, maxiters=5)
    assert rel_l2(g["vne_pseudo_6"], v6) < 1e-5
    a = g["density_s1"]
    b = g["density_raw_s1"] + np.float32(1e-3)
    assert abs(g["qdiff_rel0"] - og.qdiff(a, b)) < 1e-4 * og.qdiff(a, b)
    # the kernel returns sum |a-b|/b; Compute_qdiff multiplies by 100 (qmtools/qmtools.py:2829)
    assert abs(100 * g["qdiff_rel1"] - og.qdiff(a, b, rel=True)) < 1e-3 * og.qdiff(a, b, rel=True)


@pytest.mark.parametrize("nl", [1, 4])
def test_automaton_oracle_matches_reference_kernel(nl):
    """The single-shot automaton oracle against gpu_automaton_nn_singleshot's own output
    (kernel_nn_ss.cu, tests/golden/c0_32.nn_ss.npz; FP32 kernel vs FP64-emulated oracle)."""
    from oracle import automaton as oa
    g = np.load(GOLDEN / "c0_32.nn_ss.npz")
    shape = tuple(int(v) for v in g["shape"])
    gs = float(str(np.float32(g["step"])))
    got = oa.nn_singleshot_grid(g[f"nn_ss_l{nl}_field1"], shape, g[f"nn_ss_l{nl}_params"], nl, gs)
    assert rel_l2(got, g[f"nn_ss_l{nl}_out"]) < 1e-6


def test_automaton_neighbour_order_covers_the_26_neighbours():
    from oracle import automaton as oa
    nb = oa.neighbour_order()
    assert len(nb) == 26 and len({t[:3] for t in nb}) == 26 and (0, 0, 0) not in {t[:3] for t in nb}

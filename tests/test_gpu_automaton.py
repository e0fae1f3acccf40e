"""The GA single-shot automaton kernel and element on the GPU.

Against the reference kernel's own output (tests/golden/c0_32.nn_ss.npz, bit for bit), the
FP64-emulated oracle, and a whole AutomatonSingleShot.Evaluate / GA generation on a molecule.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import qmtools
from qmtools import _native as N
from qmtools.GAEngine import GA
from qmtools.automaton_nn_singleshot import AutomatonSingleShot
from qmtools.cidhelper import CIDHelper
from oracle import automaton as oa
from conftest import rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def run(field1, shape, params, nl, gs):
    import torch
    N.ensure_device(None)
    n = int(np.prod(shape))
    qube = torch.zeros(2 * n, device="cuda")
    qube[n:] = torch.from_numpy(np.ascontiguousarray(field1, dtype=np.float32)).cuda()
    out = torch.zeros(n, device="cuda")
    p = np.ascontiguousarray(params, dtype=np.float32)
    N.call("qmt_nn_singleshot", *shape, gs, C.c_void_p(qube.data_ptr()), C.c_void_p(out.data_ptr()),
           C.c_void_p(p.ctypes.data), int(p.size), nl, N.stream_handle())
    return out.cpu().numpy()


@pytest.mark.parametrize("nl", [1, 4])
def test_kernel_is_bitwise_the_reference_kernel(nl):
    g = np.load(GOLDEN / "c0_32.nn_ss.npz")
    shape = tuple(int(v) for v in g["shape"])
    got = run(g[f"nn_ss_l{nl}_field1"], shape, g[f"nn_ss_l{nl}_params"], nl, float(str(np.float32(g["step"]))))
    assert np.array_equal(got, g[f"nn_ss_l{nl}_out"])


@pytest.mark.parametrize("nl,shape", [(2, (16, 8, 24)), (3, (8, 16, 8))])
def test_kernel_matches_oracle(nl, shape):
    rng = np.random.default_rng(nl)
    f1 = rng.uniform(0.0, 2.0, size=int(np.prod(shape))).astype(np.float32)
    p = (2 * rng.random(oa.dna_size(nl)) - 1).astype(np.float32)
    gs = float(str(np.float32(0.37)))
    assert rel_l2(run(f1, shape, p, nl, gs), oa.nn_singleshot_grid(f1, shape, p, nl, gs)) < 1e-6


def test_bad_arguments():
    import torch
    N.ensure_device(None)
    x = torch.zeros(2 * 512, device="cuda")
    p = np.zeros(10, dtype=np.float32)
    lib = N.load()
    st = lib.qmt_nn_singleshot(8, 8, 8, 0.2, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                               C.c_void_p(p.ctypes.data), 10, 4, None)
    assert st == N.BAD_ARG


@pytest.fixture(scope="module")
def molecules():
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    out = []
    for cid in (7, 12):
        d = CIDHelper.GetMolecule(cid)
        mol = qmtools.Molecule(d["xyz"], d["D-CCSD"], basis)
        grid = qmtools.Grid.DensityGrid(mol, 0.25, 1.5)
        qgrid = qmtools.QMTools.Compute_density(grid, mol, subgrid=1, copyBack=True)
        gvne = qmtools.QMTools.Compute_VNe(grid, mol, adsorb=0.05, diff=0.02, tolerance=1e-9, maxiters=40,
                                           copyBack=True)
        out.append({"CID": cid, "mol": mol, "qgrid": qgrid, "gvne": gvne})
    return out


def test_evaluate_matches_oracle_fitness(molecules):
    np.random.seed(1)
    atm = AutomatonSingleShot.Random(nlayers=4, pscale=0.3)
    np.random.seed(2)
    fit = atm.Evaluate(molecules=molecules, nEvalMols=2)
    np.random.seed(2)
    chosen = np.random.choice(molecules, size=2, replace=False)
    expect = 0.0
    for m in chosen:
        shape = tuple(int(v) for v in m["qgrid"].shape[1:])
        f1 = m["gvne"].qube.reshape(-1)[:int(np.prod(shape))]
        q = oa.nn_singleshot_grid(f1, shape, atm.params, 4, float(str(np.float32(m["qgrid"].step))))
        q = (q * np.float32(float(m["mol"].qtot) / q.astype(np.float64).sum())).astype(np.float32)
        qref = m["qgrid"].qube.reshape(-1)[:q.size]
        expect -= np.abs(q.astype(np.float64) - qref).sum()
    expect /= 2
    assert np.isfinite(fit) and abs(fit - expect) < 1e-4 * abs(expect)


def test_two_ga_generations(molecules, tmp_path):
    np.random.seed(5)
    ga = GA(populationSize=4, mutationRate=0.5, logfile=str(tmp_path / "ga.log"),
            rstfile=str(tmp_path / "ga.restart.bin"))
    ga.elementTemplate = AutomatonSingleShot
    ga.elementInitDict = {"nlayers": 2}
    ga.Initialize()
    for _ in range(2):
        ga.Evolve(molecules=molecules, nEvalMols=1)
        assert np.all(np.isfinite(ga.fits))
    ga.flog.close()
    dna = 16 * 16 * 2 + 16 * 2 + 17 + 12
    assert (tmp_path / "ga.restart.bin").stat().st_size == 4 * 4 * (dna + 1)
    assert len((tmp_path / "ga.log").read_text().splitlines()) == 2

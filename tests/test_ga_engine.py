"""The GA engine and the single-shot element against the reference engine's own traces.

tests/golden/ga_engine.npz was recorded from the reference's qmtools/GAEngine.py by
tests/golden/make_ga_golden.py; the same seeded steps run here on qmtools.GAEngine must give
the same numbers bit for bit (same NumPy draws in the same order, same restart bytes).
"""
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))

import make_ga_golden  # noqa: E402
from qmtools import GAEngine  # noqa: E402
from qmtools import automaton_nn_singleshot as ass  # noqa: E402

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "ga_engine.npz")


@pytest.fixture(scope="module")
def ours():
    with tempfile.TemporaryDirectory() as td:
        return make_ga_golden.traces(GAEngine, td)


@pytest.mark.parametrize("key", ["rand_a", "rand_b", "mix", "mutate_05", "mutate_10", "serialized", "opts",
                                 "run_fits", "run_offspring", "run_restart", "restart_offspring"])
def test_matches_reference_engine(ours, key):
    assert np.array_equal(ours[key], GOLD[key]), key


def test_mutation_quirk_kept():
    """Amount < 1: the reference's mask is zeroed right after being set, so nothing changes."""
    np.random.seed(3)
    e = GAEngine.GAElement.Random()
    before = e.params.copy()
    e.Mutate(0.5, 1.0)
    assert np.array_equal(e.params, before)


def test_singleshot_element_layout_and_restart_bytes():
    np.random.seed(4)
    a = ass.AutomatonSingleShot.Random(nlayers=4, pscale=0.5)
    b = ass.AutomatonSingleShot.Random(nlayers=4, pscale=0.5)
    assert a._dnasize == 16 * 16 * 4 + 16 * 4 + 17 + 12 == a.params.size
    assert a.params.dtype == np.float32 and np.abs(a.params).max() <= 0.5
    c = ass.AutomatonSingleShot.Mix(a, b)
    assert c.nlayers == 4 and c.params.dtype == np.float32
    assert np.all((c.params == a.params) | (c.params == b.params))
    c.fitness = -3.5
    blob = c.Serialize()
    assert len(blob) == 4 * (c.params.size + 1)
    d = ass.AutomatonSingleShot.Random(nlayers=4)
    assert d.Deserialize(blob) == len(blob)
    assert np.array_equal(d.params, c.params) and d.fitness == -3.5


def test_read_parameters_types():
    o = GAEngine.GA.ReadParameters(["x", "--populationSize", "16", "--pscale", "0.5", "--restart", "r.bin"])
    assert o == {"populationSize": 16, "pscale": 0.5, "restart": "r.bin"}


def test_offline_cidhelper_gives_molecules():
    from qmtools.cidhelper import CIDHelper
    import qmtools
    assert len(CIDHelper.CIDs) >= 256
    d = CIDHelper.GetMolecule(7)
    assert d["CID"] == 7 and d["source"] == "synthetic"
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    mol = qmtools.Molecule(d["xyz"], d["D-CCSD"], basis)
    assert mol.dm.shape == (int(mol.norbs), int(mol.norbs))
    assert CIDHelper.GetMolecule(10 ** 9) is None

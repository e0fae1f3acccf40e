"""Parity cases on which the reference's own CUDA kernels are run (test infrastructure).

Each case fixes a molecule and a grid; `oracle/build_ref.py` specialises the reference
kernels for it with the reference host's text substitutions, and
`tests/golden/make_golden.py` runs them.  Grid construction matches the GPU tests:
origin = centroid - n*step/2 (bohr), step given to `Grid` in Angstrom.
"""
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def _qm():
    import sys
    p = str(ROOT / "qmtools-pycuda_b200")
    if p not in sys.path:
        sys.path.insert(0, p)
    import qmtools
    qmtools.set_verbose(False)
    return qmtools


def centred_grid(qmtools, coords_bohr, n, step_bohr):
    c = np.asarray(coords_bohr, dtype=np.float64).mean(axis=0)
    return qmtools.Grid((1, n, n, n), step_bohr / qmtools.ANG2BOR, list(c - n * step_bohr / 2))


def case_inputs(name, basis=None):
    """(molecule, density/potential grid) of a case, built through the drop-in API."""
    qmtools = _qm()
    from qmtools import synthetic as syn
    basis = basis or qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    if name == "c0_32":
        sm = syn.config_molecule("c0")
        mol = sm.molecule(basis, qmtools.Molecule)
        return mol, centred_grid(qmtools, sm.coords_bohr, 32, 0.4)
    if name == "c0_16":
        sm = syn.config_molecule("c0")
        mol = sm.molecule(basis, qmtools.Molecule)
        return mol, centred_grid(qmtools, sm.coords_bohr, 16, 0.6)
    if name == "c1_24":
        sm = syn.config_molecule("c1")
        mol = sm.molecule(basis, qmtools.Molecule)
        return mol, centred_grid(qmtools, sm.coords_bohr, 24, 0.8)
    if name == "sample":
        d = GOLDEN / "molecule_29766_0"
        mol = qmtools.Molecule(str(d / "GEOM-B3LYP.xyz"), str(d / "D-CCSD.npy"), basis)
        return mol, qmtools.Grid.DensityGrid(mol, 0.35, 1.0)
    if name == "c0_64":
        sm = syn.config_molecule("c0")
        return sm.molecule(basis, qmtools.Molecule), sm.grid(qmtools.Grid)
    if name == "c1_bench":
        sm = syn.config_molecule("c1")
        return sm.molecule(basis, qmtools.Molecule), sm.grid(qmtools.Grid)
    raise KeyError(name)


# case -> kernel families to build: density subgrids, and which other families
CASES = {
    "c0_32": {"density": [1, 2], "hartree_gto": True, "hartree_iter": True, "fft": True, "vne": True,
              "vne_classic": 3, "nn_ss": [4, 1]},
    "c0_16": {"density": [1, 3], "hartree_gto": True},
    "c1_24": {"density": [1], "hartree_gto": True},
    "sample": {"density": [1], "hartree_gto": False},
    "c1_bench": {"density": [1], "fft": True},
    "c0_64": {"hartree_gto": True, "hartree_iter": True},   # timing only (bench), no fixture
}
VNE_PARAMS = {"adsorb": 0.05, "diff": 0.02}
NN_SEED = 4242          # seeded pseudo-field and parameters of the automaton cases
FFT_PARAMS = {"sigma": 0.2, "cutoff": 6}

"""Molecule source of the training scripts (drop-in for qmtools.cidhelper), offline.

The reference's CIDHelper (qmtools/cidhelper.py:11-81) downloads geometries and CCSD density
matrices from a remote server and queries it at import.  This one makes no network call: it
serves molecules saved as `molecule.<CID>.pickle` (the dicts that MakeBatch of
scripts/train-singleshot.py writes, with 'xyz' and 'D-CCSD') from CIDHelper.DATADIR, and any
other CID as a seeded synthetic closed-shell molecule (elements C:H:N:O = 10:14:3:3, 3-20
atoms, density matrix 2 C C^T from the cc-pVDZ overlap), with the same dict layout.
"""
import glob
import os
import pickle
import re

import numpy


class CIDHelper:

    SERVER = None                                   # offline: no server is contacted
    DATADIR = os.environ.get("QMTOOLS_MOLECULE_DIR", "data")
    SYNTHETIC = 256                                 # synthetic CIDs 1..SYNTHETIC
    CIDs = []
    _basis = None

    def _saved():
        out = {}
        for f in glob.glob(os.path.join(CIDHelper.DATADIR, "molecule.*.pickle")):
            m = re.search(r"molecule\.(\d+)\.pickle$", f)
            if m:
                out[int(m.group(1))] = f
        return out

    def GetCIDs():
        CIDHelper.CIDs = sorted(set(CIDHelper._saved()) | set(range(1, CIDHelper.SYNTHETIC + 1)))
        return CIDHelper.CIDs

    def Init():
        CIDHelper.GetCIDs()

    def _synthetic(CID):
        from . import synthetic as syn
        from .qmtools import BASIS_CCPVDZ, BasisSet, Molecule
        if CIDHelper._basis is None:
            CIDHelper._basis = BasisSet(BASIS_CCPVDZ)
        rng = numpy.random.default_rng(9_000_000 + int(CID))
        sm = syn.extent_molecule(int(rng.integers(3, 21)), 9_000_000 + int(CID), step=0.1 * syn.ANG2BOR)
        sm.molecule(CIDHelper._basis, Molecule)          # builds the seeded density matrix
        return {"CID": CID, "xyz": sm.xyz_list(), "D-CCSD": numpy.asarray(sm.dm, dtype=numpy.float64),
                "source": "synthetic"}

    def GetMolecule(CID):
        """dict with 'CID', 'xyz' ([[Z, x, y, z]] in Angstrom) and 'D-CCSD' (N x N), or None."""
        if CID not in CIDHelper.CIDs:
            print('molecule {} not available'.format(CID))
            return None
        saved = CIDHelper._saved()
        if CID in saved:
            with open(saved[CID], "rb") as f:
                d = pickle.load(f)
            d = {k: d[k] for k in ("xyz", "D-CCSD") if k in d}
            d["CID"] = CID
            d["source"] = saved[CID]
            return d
        return CIDHelper._synthetic(CID)

    def GetRandomMolecule():
        return CIDHelper.GetMolecule(numpy.random.choice(CIDHelper.CIDs))


CIDHelper.Init()

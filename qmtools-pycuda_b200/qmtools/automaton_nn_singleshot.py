"""Single-shot neural-network automaton (drop-in for qmtools.automaton_nn_singleshot).

AutomatonSingleShot (qmtools/automaton_nn_singleshot.py:12-292) is the GA element of
`scripts/train-singleshot.py`: a small perceptron maps the pseudo-field Vne of a voxel and of
each of its 26 neighbours to a charge transfer; the element's fitness is minus the grid
difference between its predicted density and the reference density.  The reference
JIT-compiles its kernel per call with PyCUDA and keeps the parameters in __constant__ memory;
here one precompiled sm_100a kernel (`qmt_nn_singleshot`) takes the parameters with each
launch, so the element needs no compilation and two elements never share state.
"""
import ctypes as C

import numpy

from . import _native as N
from .GAEngine import GAElement
from .qmtools import Grid, QMTools


def _gridstep(grid):
    # the reference writes str(grid.step) (a float32) into its kernel source, where it becomes a
    # double literal (qmtools/automaton_nn_singleshot.py:113, kernel_nn_ss.cu:8,169)
    return float(str(numpy.float32(grid.step)))


def _run_kernel(params, nlayers, cgrid, ogrid):
    nx, ny, nz = (int(v) for v in cgrid.shape[1:])
    p = numpy.ascontiguousarray(params, dtype=numpy.float32)
    N.ensure_device()
    N.call("qmt_nn_singleshot", nx, ny, nz, _gridstep(cgrid), C.c_void_p(cgrid.tensor().data_ptr()),
           C.c_void_p(ogrid.field(0).data_ptr()), C.c_void_p(p.ctypes.data), int(p.size), int(nlayers),
           N.stream_handle())


class AutomatonSingleShot(GAElement):
    """NN automaton with 2+2 inputs per voxel pair (the charge and the pseudo-field; the
    kernel reads the pseudo-field) whose output is the charge transfer between the voxels."""

    def __init__(self):
        super().__init__()
        self.nlayers = 0
        # float32 parameters (restart files store 4-byte values)
        self._precision = 4
        self._format = 'f'

    def Random(**kwargs):
        """Random element: `nlayers` hidden layers of 16 neurons [4], parameters uniform in
        [-pscale, pscale] [1.0]."""
        atm = AutomatonSingleShot()
        atm.nlayers = kwargs.get('nlayers', 4)
        pscale = kwargs.get('pscale', 1.0)
        atm._dnasize = 16 * 16 * atm.nlayers + 16 * atm.nlayers + (16 * 1 + 1) + 12
        atm.params = ((2 * numpy.random.random(atm._dnasize) - 1) * pscale).astype(numpy.float32)
        return atm

    def Mix(a, b):
        r = super(AutomatonSingleShot, AutomatonSingleShot).Mix(a, b)
        r.params = r.params.astype(numpy.float32)
        r.nlayers = a.nlayers
        return r

    def Evaluate(self, **kwargs):
        """Mean over `nEvalMols` [4] molecules drawn from kwargs['molecules'] (dicts with 'CID',
        'mol', 'gvne' and 'qgrid') of minus sum |q - qref| after rescaling q to the nuclear
        charge.  `debugElement` prints progress; `copyBack` leaves the result on the host."""
        molecules = kwargs['molecules']
        debug = kwargs.get('debugElement', False)
        copyBack = kwargs.get('copyBack', False)
        nmols = kwargs.get('nEvalMols', 4)
        mols = numpy.random.choice(molecules, size=nmols, replace=False)
        fitness = 0
        for minfo in mols:
            mol, vne, qref = minfo['mol'], minfo['gvne'], minfo['qgrid']
            if debug:
                print("evaluating on CID {}".format(minfo['CID']))
            # compute grid: field 0 zero, field 1 the pseudo-field
            cgrid = Grid.emptyAs(qref, nfields=2)
            cgrid.tensor().zero_()
            cgrid.field(1).copy_(vne.field(0))
            ogrid = Grid.emptyAs(cgrid, nfields=1)
            _run_kernel(self.params, self.nlayers, cgrid, ogrid)
            qtot = QMTools.Compute_qtot(ogrid)
            QMTools.Compute_qscale(ogrid, mol.qtot / qtot)
            qdiff = QMTools.Compute_qdiff(ogrid, qref, rel=False)
            if debug:
                print("automaton NN[SS] qdiff {}".format(qdiff))
            if copyBack:
                ogrid.qube = ogrid.tensor().cpu().numpy().reshape(ogrid.shape)
            if numpy.isnan(qdiff):
                print("diff is nan!")
                qdiff = 9999
            fitness -= qdiff
        self.fitness = fitness / len(mols)
        return self.fitness

    def SingleShot(self, mol, cgrid, qref, debug=False, copyBack=False):
        """One evaluation on a prepared two-field grid (q and the pseudo-field), without the
        rescale: returns minus sum |q - qref| (-999 if not finite)."""
        ogrid = Grid.emptyAs(cgrid)
        _run_kernel(numpy.asarray(self.params, dtype=numpy.float32), self.nlayers, cgrid, ogrid)
        qdiff = QMTools.Compute_qdiff(ogrid, qref, rel=False)
        if debug:
            print("automaton NN[SS] qdiff {}".format(qdiff))
        if copyBack:
            cgrid.qube = ogrid.tensor().cpu().numpy().reshape(ogrid.shape)
        if numpy.isnan(qdiff):
            print("diff is nan")
            return -999
        return -qdiff

    def CompareQ(self, cgrid, qref, rel=False):
        qdiff = QMTools.Compute_qdiff(cgrid, qref, rel)
        self.fitness = -9999 + numpy.random.random() if numpy.isnan(qdiff) else -qdiff
        return self.fitness

"""Drop-in replacement of `qmtools.qmtools` (fullmetalfelix/QMTools-pycuda) on sm_100a.

Same classes, signatures and conventions as the reference (qmtools/qmtools.py):

* `BasisSet(filename)`  -- cc-pvdz.bin layout (qmtools/qmtools.py:30-108)
* `Molecule(xyz, dm, basisset)` and `.Translate` (qmtools/qmtools.py:111-191)
* `Grid(shape, step, origin)`, `Grid.DensityGrid`, `Grid.emptyAs`, load/save
  (qmtools/qmtools.py:194-432)
* `QMTools.Compute_*` (qmtools/qmtools.py:2320-2831)

Device memory is held in torch CUDA tensors and every computation runs in
libqmtools_b200.so through its C ABI.  Importing this module needs no GPU; device
buffers are created on first use.  There is no CPU fallback.
"""
import math
import pickle
import struct
import warnings
from pathlib import Path

import numpy

from . import _native as N

ANG2BOR = 1.8897259886     # qmtools/qmtools.py:17
MAXAOS = 15
MAXAOC = 20
MOLFAT = 2.0

sizeofInt = 4
sizeofFloat = 4
sizeofDouble = 8

VERBOSE = True

# The cc-pVDZ basis in the reference's binary layout (qmtools/qmtools.py:33-91).
BASIS_CCPVDZ = str(Path(__file__).resolve().parent / "data" / "cc-pvdz.bin")

float3 = numpy.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4")])
uint3 = numpy.dtype([("x", "<u4"), ("y", "<u4"), ("z", "<u4")])


def make_float3(x, y, z):
    """A float3 scalar with ['x'], ['y'], ['z'] fields, like pycuda's gpuarray.vec.make_float3."""
    return numpy.array((x, y, z), dtype=float3)[()]


def make_uint3(x, y, z):
    return numpy.array((x, y, z), dtype=uint3)[()]


def set_verbose(flag):
    global VERBOSE
    VERBOSE = bool(flag)


def _log(*a):
    if VERBOSE:
        print(*a)


def _torch():
    import torch
    return torch


class DeviceBuffer:
    """Device allocation handle: int(buf) is the device address (pycuda DeviceAllocation style)."""

    def __init__(self, tensor):
        self.tensor = tensor

    def __int__(self):
        return self.tensor.data_ptr()

    __index__ = __int__

    @property
    def nbytes(self):
        return self.tensor.numel() * self.tensor.element_size()


## Stores the basis set information (qmtools/qmtools.py:30-108).
class BasisSet:

    def __init__(self, filename):
        _log("reading basis set from: ", filename)
        with open(filename, "rb") as f:
            data = f.read()
        off = 0

        def take(fmt):
            nonlocal off
            v = struct.unpack_from("<" + fmt, data, off)
            off += struct.calcsize("<" + fmt)
            return v

        (natm,) = take("i")
        self.atomOffset = numpy.zeros(100).astype(numpy.int32) - 1
        self.nshells = numpy.zeros(MAXAOS * 100).astype(numpy.int32)
        self.shellOffset = numpy.zeros(MAXAOS * 100).astype(numpy.int32)
        self.Ls = numpy.zeros(MAXAOS * 100).astype(numpy.int32)
        self.alphas = numpy.zeros(MAXAOS * MAXAOC * 100).astype(numpy.float32)
        self.coeffs = numpy.zeros(MAXAOS * MAXAOC * 100).astype(numpy.float32)
        self.global_m_values = numpy.asarray([[0, 0, 0, 0, 0], [0, 1, -1, 0, 0], [0, 1, -1, 2, -2]]).astype(numpy.int32)
        self.shells64 = {}   # Z -> [(L, alphas fp64, coeffs fp64)]
        offset = 0
        orbcount = 0
        ncmax = 0
        maxorbs = 0
        for _ in range(natm):
            z, nsh = take("ii")
            self.atomOffset[z] = orbcount
            self.nshells[z] = nsh
            maxorbs = max(maxorbs, nsh)
            lst = []
            for _ in range(nsh):
                L, nc = take("ii")
                a = numpy.array(take("d" * nc))
                c = numpy.array(take("d" * nc))
                self.Ls[orbcount] = L
                self.shellOffset[orbcount] = offset
                self.alphas[offset:offset + nc] = a.astype(numpy.float32)
                self.coeffs[offset:offset + nc] = c.astype(numpy.float32)
                lst.append((L, a, c))
                ncmax = max(ncmax, nc)
                orbcount += 1
                offset += MAXAOC
            self.shells64[z] = lst
        self.nparams = offset
        _log("basis set read - maxorbs={}  ncmax={} - nparams={}\n".format(maxorbs, ncmax, offset))


## Stores a molecule in BOHR (qmtools/qmtools.py:111-191).
class Molecule:

    def __init__(self, filexyz, filedm, basisset):
        self.basisset = basisset
        if isinstance(filexyz, list):
            m = numpy.asarray(filexyz, dtype=numpy.float64)
        elif isinstance(filexyz, numpy.ndarray):
            m = numpy.array(filexyz, dtype=numpy.float64)
        else:
            _log("opening molecule (ang):", filexyz)
            m = numpy.loadtxt(filexyz)
            if len(m.shape) == 1:
                m = numpy.asarray([m])
        m = numpy.array(m, dtype=numpy.float64)
        m[:, 1:] *= ANG2BOR
        self.types = numpy.array(m[:, 0], dtype=numpy.int32)
        self.coords = numpy.array(m[:, 1:], dtype=numpy.float32)
        self.natoms = numpy.int32(self.types.shape[0])
        self.qtot = numpy.int32(numpy.sum(self.types))

        if isinstance(filedm, numpy.ndarray):
            dm = filedm
        else:
            _log("opening density matrix:", filedm)
            dm = numpy.load(filedm)
        self.dm = numpy.array(dm, dtype=numpy.float32)
        self.norbs = numpy.int32(dm.shape[0])
        _log("# of orbitals:", self.norbs)

        rows = []
        for a in range(self.natoms):
            Z = self.types[a]
            aos = basisset.atomOffset[Z]
            if aos < 0:
                raise KeyError(f"element Z={Z} is not in the basis set")
            for s in range(basisset.nshells[Z]):
                L = basisset.Ls[aos + s]
                for mi in range(2 * L + 1):
                    rows.append((a, L, basisset.global_m_values[L, mi], basisset.shellOffset[aos + s]))
        self.ALMOs = numpy.array(rows, dtype=numpy.int16).reshape(-1, 4)
        if self.ALMOs.shape[0] != self.norbs:
            raise ValueError(f"density matrix is {self.norbs}x{self.norbs} but the basis has "
                             f"{self.ALMOs.shape[0]} functions")
        self._handle = None
        self._dev = None

    # -- device handle --------------------------------------------------------------------
    @property
    def handle(self):
        if self._handle is None:
            import ctypes as C
            dev = N.ensure_device()
            bs = self.basisset
            h = C.c_void_p()
            types = numpy.ascontiguousarray(self.types, dtype=numpy.int32)
            coords = numpy.ascontiguousarray(self.coords, dtype=numpy.float32)
            almos = numpy.ascontiguousarray(self.ALMOs, dtype=numpy.int16)
            al = numpy.ascontiguousarray(bs.alphas, dtype=numpy.float32)
            co = numpy.ascontiguousarray(bs.coeffs, dtype=numpy.float32)
            dm = numpy.ascontiguousarray(self.dm, dtype=numpy.float32)
            N.call("qmt_mol_create", int(self.natoms), types.ctypes.data, coords.ctypes.data,
                   int(self.norbs), almos.ctypes.data, int(al.size), al.ctypes.data, co.ctypes.data,
                   dm.ctypes.data, N.stream_handle(), C.byref(h))
            self._handle = h
            self._dev = dev
        return self._handle

    def release(self):
        if self._handle is not None:
            try:
                N.load().qmt_mol_destroy(self._handle)
            finally:
                self._handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __getstate__(self):
        d = dict(self.__dict__)
        d["_handle"] = None
        d["_dev"] = None
        return d

    def set_dm(self, dm):
        """Replace the density matrix (same size) and upload it."""
        self.dm = numpy.array(dm, dtype=numpy.float32)
        if self._handle is not None:
            d = numpy.ascontiguousarray(self.dm)
            N.call("qmt_mol_set_dm", self._handle, d.ctypes.data, N.stream_handle())

    def Translate(self, dx=0, dy=0, dz=0):
        self.coords[:, 0] += dx
        self.coords[:, 1] += dy
        self.coords[:, 2] += dz
        if self._handle is not None:
            c = numpy.ascontiguousarray(self.coords, dtype=numpy.float32)
            N.call("qmt_mol_set_coords", self._handle, c.ctypes.data, N.stream_handle())

    def trace_ps(self):
        """FP64 Tr(P S) on the device (the DM as given, lower triangle)."""
        import ctypes as C
        out = C.c_double()
        N.call("qmt_mol_trace_ps", self.handle, C.byref(out), N.stream_handle())
        return out.value


# Multifield grid (qmtools/qmtools.py:194-432).
class Grid:

    def __init__(self, shape, step, origin=[0, 0, 0]):
        if len(shape) == 3:
            _log("WARNING: augmenting the grid shape!")
            shape = (1, shape[0], shape[1], shape[2])
        if len(shape) != 4:
            raise ValueError("shape has to be 4-dimensional: nfields, nx, ny, nz")
        self.shape = tuple(int(s) for s in shape)
        grd = numpy.asarray(self.shape).astype(numpy.int32)[1:]
        blk = numpy.floor(grd / 8).astype(numpy.int32)
        if not numpy.array_equal(grd, blk * 8):
            raise ValueError("shape for xyz have to be multiple of 8")
        self.GPUblocks = tuple([x.item() for x in blk])
        self.qube = numpy.zeros(self.shape).astype(numpy.float32)
        self.npts = numpy.uint32(self.shape[1] * self.shape[2] * self.shape[3])
        self.nfields = numpy.uint32(self.shape[0])
        self.step = numpy.float32(step * ANG2BOR)
        self.origin = make_float3(origin[0], origin[1], origin[2])
        self.lattice = numpy.asarray([[1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=numpy.float32)
        self._t = None

    def __str__(self):
        return "origin: {}\nshape: {} -- points: {} gpublocks: {}".format(
            self.origin, self.shape, self.npts, self.GPUblocks)

    # -- device storage ---------------------------------------------------------------------
    def tensor(self):
        """Flat float32 CUDA tensor holding all fields (x-fastest per field)."""
        if self._t is None:
            torch = _torch()
            N.ensure_device()
            self._t = torch.from_numpy(numpy.ascontiguousarray(self.qube, dtype=numpy.float32).ravel()).cuda()
        return self._t

    def field(self, f=0):
        n = int(self.npts)
        return self.tensor()[f * n:(f + 1) * n]

    @property
    def d_qube(self):
        return DeviceBuffer(self.tensor())

    def _upload(self):
        if self._t is None:
            self.tensor()
        else:
            torch = _torch()
            self._t.copy_(torch.from_numpy(numpy.ascontiguousarray(self.qube, dtype=numpy.float32).ravel()))

    def _download(self):
        if self._t is not None:
            self.qube = self._t.cpu().numpy().reshape(self.shape).copy()

    def CopyBack(self):
        self._download()
        return self.qube

    def space_shape(self):
        return (self.shape[1], self.shape[2], self.shape[3])

    def space_shape_uint3(self):
        return make_uint3(self.shape[1], self.shape[2], self.shape[3])

    def _geom(self):
        o = self.origin
        return (int(self.shape[1]), int(self.shape[2]), int(self.shape[3]), float(self.step),
                float(o["x"]), float(o["y"]), float(o["z"]))

    ### Creates a cartesian grid around a molecule (qmtools/qmtools.py:243-261).
    def DensityGrid(molecule, step, fat):
        xyz = numpy.array(molecule.coords, copy=True)
        crdmax = numpy.amax(xyz, axis=0) + fat * ANG2BOR
        crdmin = numpy.amin(xyz, axis=0) - fat * ANG2BOR
        grd = crdmax - crdmin
        grd = grd / (step * ANG2BOR)
        grd = grd / 8.0
        grd = numpy.ceil(grd).astype(numpy.uint32) * 8
        shape = (1, grd[0], grd[1], grd[2])
        grid = Grid(shape, step)
        grid.origin = make_float3(crdmin[0], crdmin[1], crdmin[2])
        return grid

    ### Same shape and step, zero everywhere (qmtools/qmtools.py:268-278).
    def emptyAs(g, nfields=None):
        shape = g.shape
        if nfields is not None:
            shape = (nfields, shape[1], shape[2], shape[3])
        grid = Grid(shape, 1.0)
        grid.origin = g.origin
        grid.lattice = g.lattice
        grid.step = g.step
        return grid

    def LoadData(self, filename):
        self.qube = numpy.load(filename)
        self._upload()

    def Save(self, filename):
        d = {"shape": self.shape, "origin": self.origin, "step": self.step,
             "lattice": self.lattice, "qube": self.qube}
        with open(filename, "wb") as f:
            pickle.dump(d, f)

    def Load(molecule, filename):
        with open(filename, "rb") as f:
            d = pickle.load(f)
        grid = Grid(d["shape"], 0.1)
        o = d["origin"]
        grid.origin = make_float3(o["x"], o["y"], o["z"])
        grid.step = numpy.float32(d["step"])
        grid.lattice = d["lattice"]
        grid.qube = numpy.asarray(d["qube"], dtype=numpy.float32)
        return grid

    def LoadFromNPY(self, npyarray):
        if len(npyarray.shape) != len(self.qube.shape):
            raise ValueError("dimensionality mismatch")
        for i in range(len(self.qube.shape)):
            if npyarray.shape[i] != self.qube.shape[i]:
                raise ValueError("array shape mismatch {} (expected {})".format(npyarray.shape, self.qube.shape))
        self.qube = npyarray.astype(numpy.float32)
        self._upload()

    def _bin_header(self, mol):
        out = bytearray()
        if mol is None:
            out += struct.pack("i", 0)
        else:
            out += struct.pack("i", int(mol.natoms))
            for i in range(int(mol.natoms)):
                out += struct.pack("i", int(mol.types[i]))
                out += struct.pack("fff", *(float(v) for v in mol.coords[i]))
        out += struct.pack("iii", self.shape[1], self.shape[2], self.shape[3])
        o = self.origin
        out += struct.pack("ffff", float(self.step), float(o["x"]), float(o["y"]), float(o["z"]))
        return bytes(out)

    ### Binary format, first field only (qmtools/qmtools.py:331-374).
    def SaveBIN(self, filename, mol=None):
        with open(filename, "wb") as f:
            f.write(self._bin_header(mol))
            f.write(numpy.ascontiguousarray(self.qube[0], dtype=numpy.float32).tobytes())

    ### One file per field, named <filename>-<f>.bin (qmtools/qmtools.py:377-410).
    def SaveBINmulti(self, filename, mol=None):
        for f in range(self.shape[0]):
            with open("{}-{}.bin".format(filename, f), "wb") as fo:
                fo.write(self._bin_header(mol))
                fo.write(numpy.ascontiguousarray(self.qube[f], dtype=numpy.float32).tobytes())

    ### Load a .bin grid (qmtools/qmtools.py:414-432); vectorised read of the same bytes.
    def LoadBIN(filename):
        with open(filename, "rb") as f:
            data = f.read()
        (natm,) = struct.unpack_from("i", data, 0)
        off = 4 + 16 * natm
        shape = struct.unpack_from("iii", data, off)
        off += 12
        (step,) = struct.unpack_from("f", data, off)
        origin = struct.unpack_from("fff", data, off + 4)
        off += 16
        n = shape[0] * shape[1] * shape[2]
        linear = numpy.frombuffer(data, dtype="<f4", count=n, offset=off).astype(numpy.float32)
        grid = Grid(shape, step)
        grid.step = numpy.float32(step)
        grid.origin = make_float3(origin[0], origin[1], origin[2])
        grid.qube = linear.reshape(grid.shape).copy()
        return grid


def _new_like(g, nfields=None):
    out = Grid.emptyAs(g, nfields)
    out.tensor()
    return out


class QMTools:
    """Static facade of the hot path (qmtools/qmtools.py:2320-2831)."""

    default_precision = "fp16x3"
    jacobi_max_sweeps = 200000

    ### Electron density grid (qmtools/qmtools.py:2381-2430).
    def Compute_density(grid, molecule, subgrid=1, copyBack=True, debug=False, precision=None,
                        rescale=True):
        import ctypes as C
        prec = QMTools.default_precision if precision is None else precision
        cgrid = _new_like(grid)
        nx, ny, nz, h, ox, oy, oz = grid._geom()
        s = C.c_double()
        N.call("qmt_density", molecule.handle, nx, ny, nz, h, ox, oy, oz, int(subgrid), N.PREC[prec],
               1 if rescale else 0, C.c_void_p(cgrid.field(0).data_ptr()), C.byref(s), N.stream_handle())
        cgrid.qsum = s.value
        if copyBack:
            cgrid._download()
        return cgrid

    ### Analytic potential at voxel corners, written into vgrid (qmtools/qmtools.py:2436-2489).
    def Compute_hartree(vgrid, molecule, copyBack=True):
        import ctypes as C
        nx, ny, nz, h, ox, oy, oz = vgrid._geom()
        N.call("qmt_hartree_gto", molecule.handle, nx, ny, nz, h, ox, oy, oz,
               C.c_void_p(vgrid.field(0).data_ptr()), N.stream_handle())
        if copyBack:
            vgrid._download()
        return

    ### Jacobi relaxation (qmtools/qmtools.py:2497-2573); capped at max_sweeps.
    def Compute_hartree_iter(qgrid, molecule, tolerance=1.0e-24, copyBack=True, max_sweeps=None,
                             check_every=100):
        import ctypes as C
        torch = _torch()
        max_sweeps = QMTools.jacobi_max_sweeps if max_sweeps is None else int(max_sweeps)
        gqsd = QMTools.Compute_qseed(qgrid, molecule, copyBack=False)
        rho = _new_like(qgrid, 1)
        torch.sub(gqsd.field(0), qgrid.field(0), out=rho.field(0))
        vgrid = _new_like(qgrid)
        tgrid = _new_like(qgrid)
        nx, ny, nz, h, _, _, _ = qgrid._geom()
        sw = C.c_int()
        dl = C.c_double()
        st = N.load().qmt_jacobi(nx, ny, nz, h, C.c_void_p(rho.field(0).data_ptr()),
                                 C.c_void_p(vgrid.field(0).data_ptr()), C.c_void_p(tgrid.field(0).data_ptr()),
                                 max_sweeps, int(check_every), float(tolerance), C.byref(sw), C.byref(dl),
                                 N.stream_handle())
        if st == N.NOT_CONVERGED:
            warnings.warn(f"Jacobi not converged after {sw.value} sweeps (delta {dl.value:.3e})")
        else:
            N.check(st, "qmt_jacobi")
        vgrid.sweeps = sw.value
        vgrid.delta = dl.value
        if copyBack:
            vgrid._download()
        return vgrid

    ### Jacobi relaxation in physical units with the analytic boundary (new facade method).
    def Compute_hartree_dirichlet(qgrid, molecule, max_sweeps=2000, tolerance=0.0, check_every=100,
                                  copyBack=True):
        """Total electrostatic potential (a.u.) at voxel centres by Jacobi relaxation of
        lap V = -4 pi rho, rho = (nuclear seed charges - electrons per voxel) / h^3, with the
        outer shell held at the analytic GTO potential of the molecule (electrons and nuclei).

        The reference's Compute_hartree_iter (qmtools/qmtools.py:2497-2573) relaxes the same
        charge grid in its own units (no 4 pi) with a zero outer shell; this variant fixes the
        boundary from gpu_hartree_GTO's potential (kernel_hartree.cu:288-869), so the interior
        converges to the free-space potential.  The FP64 residual sum |V - T| of the last check
        is returned as `.delta`, the sweeps done as `.sweeps`.  tolerance 0 runs max_sweeps."""
        import ctypes as C
        torch = _torch()
        nx, ny, nz, h, ox, oy, oz = qgrid._geom()
        seed = QMTools.Compute_qseed(qgrid, molecule, copyBack=False)
        rho = _new_like(qgrid, 1)
        torch.sub(seed.field(0), qgrid.field(0), out=rho.field(0))
        rho.field(0).mul_(1.0 / float(h) ** 3)
        vgrid = _new_like(qgrid, 1)
        tgrid = _new_like(qgrid, 1)
        N.call("qmt_hartree_gto_boundary", molecule.handle, nx, ny, nz, h, ox, oy, oz,
               C.c_void_p(vgrid.field(0).data_ptr()), N.stream_handle())
        sw = C.c_int()
        dl = C.c_double()
        st = N.load().qmt_jacobi_dirichlet(nx, ny, nz, h, C.c_void_p(rho.field(0).data_ptr()),
                                           C.c_void_p(vgrid.field(0).data_ptr()),
                                           C.c_void_p(tgrid.field(0).data_ptr()), int(max_sweeps),
                                           int(check_every), float(tolerance), C.byref(sw), C.byref(dl),
                                           N.stream_handle())
        if st == N.NOT_CONVERGED:
            warnings.warn(f"Jacobi not converged after {sw.value} sweeps (delta {dl.value:.3e})")
        else:
            N.check(st, "qmt_jacobi_dirichlet")
        vgrid.sweeps = sw.value
        vgrid.delta = dl.value
        vgrid.rho = rho
        if copyBack:
            vgrid._download()
        return vgrid

    ### FFT Poisson solve (qmtools/qmtools.py:2578-2639); returns (NX,NY,NZ) volts, C-order.
    def Compute_hartree_fft(qgrid, molecule, sigma=0.2, cutoff=6, padded=False):
        import ctypes as C
        torch = _torch()
        nx, ny, nz, h, ox, oy, oz = qgrid._geom()
        out = torch.empty(nx * ny * nz, dtype=torch.float32, device="cuda")
        N.call("qmt_fft_poisson", molecule.handle, nx, ny, nz, h, ox, oy, oz, float(sigma), float(cutoff),
               1 if padded else 0, C.c_void_p(qgrid.field(0).data_ptr()), C.c_void_p(out.data_ptr()),
               N.stream_handle())
        return out.cpu().numpy().reshape(nx, ny, nz)

    ### Nuclear seed charges (qmtools/qmtools.py:2645-2672).
    def Compute_qseed(grid, molecule, copyBack=True):
        import ctypes as C
        qgrid = _new_like(grid, 1)
        nx, ny, nz, h, ox, oy, oz = grid._geom()
        N.call("qmt_density_seed", molecule.handle, nx, ny, nz, h, ox, oy, oz,
               C.c_void_p(qgrid.field(0).data_ptr()), N.stream_handle())
        if copyBack:
            qgrid._download()
        return qgrid

    ### Nuclear pseudo-field (qmtools/qmtools.py:2677-2745).
    def Compute_VNe(grid, molecule, adsorb=0.1, diff=0.01, tolerance=1.0e-9, maxiters=None, copyBack=True):
        import ctypes as C
        if maxiters is None:
            maxiters = 10 * numpy.power(grid.npts, 1.0 / 3)
        gridres = _new_like(grid, 1)
        gridout = _new_like(grid, 1)
        nx, ny, nz, h, ox, oy, oz = grid._geom()
        it = C.c_int()
        N.call("qmt_vne_pseudo", molecule.handle, nx, ny, nz, h, ox, oy, oz, float(adsorb), float(diff),
               float(tolerance), int(math.floor(maxiters)), C.c_void_p(gridres.field(0).data_ptr()),
               C.c_void_p(gridout.field(0).data_ptr()), C.byref(it), N.stream_handle())
        if it.value > maxiters:
            _log("VNe not converged!", maxiters)
        gridres.iterations = it.value
        if copyBack:
            gridres._download()
        return gridres

    ### Subsampled sum Z/r (qmtools/qmtools.py:2750-2790).
    def Compute_VNe_classic(grid, molecule, divisions=4, copyBack=True):
        import ctypes as C
        gridout = _new_like(grid, 1)
        nx, ny, nz, h, ox, oy, oz = grid._geom()
        N.call("qmt_vne_classic", molecule.handle, nx, ny, nz, h, ox, oy, oz, int(divisions),
               C.c_void_p(gridout.field(0).data_ptr()), N.stream_handle())
        if copyBack:
            gridout._download()
        return gridout

    ### sum Z/r at voxel centres (kernel_hartree.cu:209-251; new facade method).
    def Compute_VNe_point(grid, molecule, copyBack=True):
        import ctypes as C
        gridout = _new_like(grid, 1)
        nx, ny, nz, h, ox, oy, oz = grid._geom()
        N.call("qmt_vne_point", molecule.handle, nx, ny, nz, h, ox, oy, oz, 0,
               C.c_void_p(gridout.field(0).data_ptr()), N.stream_handle())
        if copyBack:
            gridout._download()
        return gridout

    ### Total charge of field 0 (qmtools/qmtools.py:2796-2803), FP64 sum.
    def Compute_qtot(grid):
        import ctypes as C
        out = C.c_double()
        N.call("qmt_grid_total", C.c_void_p(grid.field(0).data_ptr()), int(grid.npts), C.byref(out),
               N.stream_handle())
        return float(out.value)

    ### Scale field 0 (qmtools/qmtools.py:2808-2813).
    def Compute_qscale(grid, factor, copyBack=False):
        import ctypes as C
        N.call("qmt_grid_scale", C.c_void_p(grid.field(0).data_ptr()), int(grid.npts), float(factor),
               N.stream_handle())
        if copyBack:
            grid._download()
        return

    ### sum |a-b| (or 100 * sum |a-b|/b) over field 0 (qmtools/qmtools.py:2818-2831).
    def Compute_qdiff(grid1, grid2, rel=False):
        import ctypes as C
        out = C.c_double()
        N.call("qmt_grid_diff", C.c_void_p(grid1.field(0).data_ptr()), C.c_void_p(grid2.field(0).data_ptr()),
               int(grid1.npts), 1 if rel else 0, C.byref(out), N.stream_handle())
        return float(out.value)

    ### Error report of field 0 against a reference grid (new).
    def Compute_errors(grid, ref):
        import ctypes as C
        out = (C.c_double * 4)()
        N.call("qmt_grid_errors", C.c_void_p(grid.field(0).data_ptr()), C.c_void_p(ref.field(0).data_ptr()),
               int(grid.npts), out, N.stream_handle())
        return {"max_abs": out[0], "rel_l2": out[1], "sum": out[2], "sum_ref": out[3]}


__all__ = ["ANG2BOR", "BASIS_CCPVDZ", "MAXAOS", "MAXAOC", "BasisSet", "Molecule", "Grid", "QMTools", "DeviceBuffer",
           "make_float3", "make_uint3", "set_verbose"]

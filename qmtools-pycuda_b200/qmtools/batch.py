"""Batched density + Hartree evaluation of many molecules in one captured CUDA graph (new; the
reference evaluates one molecule per facade call, qmtools/qmtools.py:2381-2639).

`BatchEvaluator(molecules, grids)`:

* keeps every molecule's operands, its density grid and its potential grid on the device (one
  flat buffer each, 256-byte aligned slices);
* evaluates all densities through `qmt_batch_density`: the molecules whose contraction takes the
  fused path share persistent launches over all their tiles (one for those whose density matrix
  has a low-rank factor, one for the others), the rest take the staged path; every grid is then
  scaled to its nuclear charge;
* solves the free-space (Hockney) FFT Poisson problem of every molecule with the padded lengths
  the autotuner picked (`qmtools.autotune`);
* captures all of it into one CUDA graph after a first eager run (which builds every operand,
  Green's function and twiddle table), so `run()` is a single graph launch.

With `refresh=True` the graph also re-derives each molecule's split density matrix from the
matrix last uploaded (`Molecule.set_dm`), so new density matrices need no re-capture.
"""
import ctypes as C

import numpy as np

from . import _native as N
from .autotune import Tuner


def _align(n, a=64):
    return (n + a - 1) // a * a


class BatchEvaluator:
    def __init__(self, molecules, grids, precision="fp16x3", hartree=True, sigma=0.2, cutoff=6.0, tuner=None,
                 refresh=False, capture=True):
        import torch
        if len(molecules) != len(grids) or not molecules:
            raise ValueError("one grid per molecule")
        N.ensure_device()
        self.molecules = list(molecules)
        self.grids = list(grids)
        self.precision = precision
        self.hartree = hartree
        self.sigma, self.cutoff = float(sigma), float(cutoff)
        self.refresh = bool(refresh)
        self.tuner = tuner if tuner is not None else Tuner()
        self.stream = torch.cuda.Stream()
        geo = [g._geom() for g in self.grids]
        self.npts = [int(nx * ny * nz) for nx, ny, nz, *_ in geo]
        self.offsets = np.concatenate([[0], np.cumsum([_align(n) for n in self.npts])]).astype(np.int64)
        total = int(self.offsets[-1])
        self.q = torch.zeros(total, dtype=torch.float32, device="cuda")
        self.v = torch.zeros(total, dtype=torch.float32, device="cuda") if hartree else None
        # tuned choices; every molecule takes its factored density matrix when it has one, on the
        # fused path when it fits (a batch that re-derives its operands in the graph keeps the
        # unfactored matrices)
        from .autotune import PATH_FACTORED
        self.paths = [self.tuner.density_path(m, n, precision) for m, n in zip(self.molecules, self.npts)]
        if not self.refresh and not precision.startswith("tf32"):
            self.paths = [PATH_FACTORED for _ in self.paths]
        self.fft_lengths = []
        if hartree:
            for m, (nx, ny, nz, *_) in zip(self.molecules, geo):
                self.fft_lengths.append(tuple(self.tuner.fft_length(k, m) for k in (nx, ny, nz)))
        # the batch
        nm = len(self.molecules)
        handles = (C.c_void_p * nm)(*[m.handle.value for m in self.molecules])
        shapes = np.array([[nx, ny, nz] for nx, ny, nz, *_ in geo], dtype=np.int32)
        geoms = np.array([[h, ox, oy, oz] for _, _, _, h, ox, oy, oz in geo], dtype=np.float32)
        paths = np.array(self.paths, dtype=np.int32)
        qptrs = (C.c_void_p * nm)(*[self.q.data_ptr() + 4 * int(o) for o in self.offsets[:-1]])
        b = C.c_void_p()
        with torch.cuda.stream(self.stream):
            N.call("qmt_batch_create", nm, handles, shapes.ctypes.data, geoms.ctypes.data, 1, N.PREC[precision],
                   paths.ctypes.data, qptrs, C.c_void_p(self.stream.cuda_stream), C.byref(b))
        self.batch = b
        self.fused_count = N.load().qmt_batch_fused_count(b)
        self.factored_count = N.load().qmt_batch_factored_count(b)
        self.graph = None
        # eager runs: the first builds the Green's functions and twiddle tables, the second finds
        # them built, so that the captured calls make no allocation and no event call
        for _ in range(2 if capture else 1):
            self._enqueue()
            self.stream.synchronize()
        lib = N.load()
        l0 = lib.qmt_launch_count()
        if capture:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, stream=self.stream, capture_error_mode="relaxed"):
                self._enqueue()
            self.stream.synchronize()
        # kernels of this library in one evaluation (the captured ones when capturing)
        self.launches_per_run = lib.qmt_launch_count() - l0 if capture else None

    def _enqueue(self):
        s = C.c_void_p(self.stream.cuda_stream)
        N.call("qmt_batch_density", self.batch, 1, 1 if self.refresh else 0, s)
        if not self.hartree:
            return
        for i, (m, g) in enumerate(zip(self.molecules, self.grids)):
            nx, ny, nz, h, ox, oy, oz = g._geom()
            mx, my, mz = self.fft_lengths[i]
            o = int(self.offsets[i])
            N.call("qmt_fft_poisson_padded", m.handle, nx, ny, nz, h, ox, oy, oz, self.sigma, self.cutoff, mx, my, mz,
                   C.c_void_p(self.q.data_ptr() + 4 * o), C.c_void_p(self.v.data_ptr() + 4 * o), s)

    def run(self):
        """Enqueue one evaluation of every molecule on the batch's stream (asynchronous)."""
        import torch
        if self.graph is not None:
            with torch.cuda.stream(self.stream):
                self.graph.replay()
        else:
            with torch.cuda.stream(self.stream):
                self._enqueue()

    def synchronize(self):
        self.stream.synchronize()

    def sums(self):
        """FP64 density sums before scaling (reports kernel give-up flags)."""
        out = (C.c_double * len(self.molecules))()
        N.call("qmt_batch_sums", self.batch, out, C.c_void_p(self.stream.cuda_stream))
        return np.array(out[:])

    def density(self, i):
        """Electrons per voxel of molecule i (x-fastest flat array)."""
        o = int(self.offsets[i])
        return self.q[o:o + self.npts[i]].cpu().numpy()

    def potential(self, i):
        """Potential of molecule i in volts, C-order (nx, ny, nz)."""
        nx, ny, nz = self.grids[i].space_shape()
        o = int(self.offsets[i])
        return self.v[o:o + self.npts[i]].cpu().numpy().reshape(nx, ny, nz)

    def close(self):
        if self.graph is not None:
            self.graph = None
        if self.batch is not None:
            N.load().qmt_batch_destroy(self.batch)
            self.batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""Batched evaluation and continuous-batching serving of density + Hartree requests.

New (no counterpart in the reference, whose facade evaluates one molecule per call and
JIT-compiles kernels on every call, qmtools/qmtools.py:2381-2639).

`Engine` keeps `slots` requests in flight.  Each slot owns a CUDA stream, one molecule handle
(re-initialised per request with `qmt_mol_reset`, so no device allocation happens in steady
state), device grids and pinned host buffers that only grow.  A single scheduler loop:

* admits waiting requests whose arrival time has passed while a slot is free and the request's
  estimated HBM footprint fits the budget;
* enqueues, asynchronously on the slot's stream, the density (tensor-core path, rescaled to the
  nuclear charge on the device), the free-space FFT Hartree potential and the device-to-host
  copies, then records an event;
* retires slots whose event has completed, stamping per-request latency.

Work of different requests overlaps on the device.  Every kernel reduces in a fixed order, so a
request's result does not depend on what else is in flight (tests/test_gpu_serving.py).
"""
import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


@dataclass
class Request:
    molecule: object            # qmtools.Molecule (host data only is used)
    grid: object                # qmtools.Grid: geometry only (shape, step, origin)
    arrival: float = 0.0        # seconds after the engine starts
    rid: int = 0
    hartree: bool = True
    sigma: float = 0.2
    cutoff: float = 6.0
    density: np.ndarray = None  # electrons per voxel, x-fastest flat (result)
    potential: np.ndarray = None  # volts, C-order (nx, ny, nz) (result)
    t_admit: float = None
    t_done: float = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival

    @property
    def npts(self):
        s = self.grid.shape
        return int(s[1] * s[2] * s[3])


def _nice(n):
    m = n
    while True:
        k = m
        for r in (2, 3, 5, 7):
            while k % r == 0:
                k //= r
        if k == 1:
            return m
        m += 1


def footprint(req, precision="fp16x3"):
    """Estimated device bytes of one request (grids, FFT work grid, molecule operands)."""
    nx, ny, nz = (int(v) for v in req.grid.shape[1:])
    npts = nx * ny * nz
    n = int(req.molecule.norbs)
    kpad = (n + 63) // 64 * 64
    b = 8 * npts                                   # density + potential grids
    if req.hartree:
        b += 8 * _nice(2 * nx) * _nice(2 * ny) * nz  # complex work planes z < nz
    b += 24 * kpad * kpad                          # P (FP32 + FP64) and split operands
    if kpad > 320 or precision.startswith("tf32"):
        tiles = (npts + 127) // 128
        b += min(2 << 30, tiles * 128 * kpad * 4)  # staged basis values
    return b + (16 << 20)


class _Slot:
    def __init__(self, device):
        import torch
        self.stream = torch.cuda.Stream(device=device)
        self.handle = None
        self.q = None
        self.v = None
        self.q_host = None
        self.v_host = None
        self.event = None
        self.req = None
        self.bytes = 0

    def ensure(self, npts):
        import torch
        if self.q is None or self.q.numel() < npts:
            with torch.cuda.stream(self.stream):
                self.q = torch.empty(npts, dtype=torch.float32, device="cuda")
                self.v = torch.empty(npts, dtype=torch.float32, device="cuda")
            self.q_host = torch.empty(npts, dtype=torch.float32).pin_memory()
            self.v_host = torch.empty(npts, dtype=torch.float32).pin_memory()


class Engine:
    def __init__(self, slots=4, precision="fp16x3", hbm_budget=None, device=None):
        import torch
        self.device = N.ensure_device(device)
        self.precision = precision
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info()
            hbm_budget = int(0.6 * free)
        self.budget = hbm_budget
        self.slots = [_Slot(self.device) for _ in range(slots)]
        self.in_use = 0

    # ---- one request ----------------------------------------------------------------------
    def _launch(self, slot, req):
        mol = req.molecule
        bs = mol.basisset
        s = C.c_void_p(slot.stream.cuda_stream)
        types = np.ascontiguousarray(mol.types, dtype=np.int32)
        coords = np.ascontiguousarray(mol.coords, dtype=np.float32)
        almos = np.ascontiguousarray(mol.ALMOs, dtype=np.int16)
        al = np.ascontiguousarray(bs.alphas, dtype=np.float32)
        co = np.ascontiguousarray(bs.coeffs, dtype=np.float32)
        dm = np.ascontiguousarray(mol.dm, dtype=np.float32)
        if slot.handle is None:
            h = C.c_void_p()
            N.call("qmt_mol_create", int(mol.natoms), types.ctypes.data, coords.ctypes.data, int(mol.norbs),
                   almos.ctypes.data, int(al.size), al.ctypes.data, co.ctypes.data, dm.ctypes.data, s, C.byref(h))
            slot.handle = h
        else:
            N.call("qmt_mol_reset", slot.handle, int(mol.natoms), types.ctypes.data, coords.ctypes.data,
                   int(mol.norbs), almos.ctypes.data, int(al.size), al.ctypes.data, co.ctypes.data, dm.ctypes.data, s)
        nx, ny, nz, h_, ox, oy, oz = req.grid._geom()
        npts = nx * ny * nz
        slot.ensure(npts)
        q, v = slot.q, slot.v
        N.call("qmt_density", slot.handle, nx, ny, nz, h_, ox, oy, oz, 1, N.PREC[self.precision], 1,
               C.c_void_p(q.data_ptr()), None, s)
        if req.hartree:
            N.call("qmt_fft_poisson", slot.handle, nx, ny, nz, h_, ox, oy, oz, float(req.sigma), float(req.cutoff), 1,
                   C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), s)
        import torch
        with torch.cuda.stream(slot.stream):
            slot.q_host[:npts].copy_(q[:npts], non_blocking=True)
            if req.hartree:
                slot.v_host[:npts].copy_(v[:npts], non_blocking=True)
            slot.event = torch.cuda.Event()
            slot.event.record(slot.stream)
        slot.req = req

    def _retire(self, slot, now):
        req = slot.req
        n = req.npts
        req.density = slot.q_host[:n].numpy().copy()
        if req.hartree:
            nx, ny, nz = (int(v) for v in req.grid.shape[1:])
            req.potential = slot.v_host[:n].numpy().copy().reshape(nx, ny, nz)
        req.t_done = now
        slot.req = None
        slot.event = None
        self.in_use -= slot.bytes
        slot.bytes = 0

    # ---- scheduler ------------------------------------------------------------------------
    def run(self, requests, realtime=True):
        """Process `requests` (arrival times in seconds); returns them with results and timings.

        realtime=False admits everything at t=0 (batched evaluation).
        """
        pending = sorted(requests, key=lambda r: r.arrival)
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        for r in pending:
            if footprint(r, self.precision) > self.budget:
                raise N.QMToolsError(N.OOM, "serving", f"request {r.rid} needs more than the HBM budget")
        t0 = time.perf_counter()
        busy = []
        free = list(self.slots)
        i = 0
        while i < len(pending) or busy:
            now = time.perf_counter() - t0
            progressed = False
            for slot in list(busy):
                if slot.event.query():
                    self._retire(slot, time.perf_counter() - t0)
                    busy.remove(slot)
                    free.append(slot)
                    progressed = True
            while i < len(pending) and free and pending[i].arrival <= now:
                need = footprint(pending[i], self.precision)
                if self.in_use + need > self.budget and busy:
                    break
                slot = free.pop()
                slot.bytes = need
                self.in_use += need
                pending[i].t_admit = time.perf_counter() - t0
                self._launch(slot, pending[i])
                busy.append(slot)
                i += 1
                progressed = True
            if not progressed:
                time.sleep(5e-5)
        return requests

    def warm(self, requests):
        """Serve every one of `requests` once on every slot (results discarded), so that serving
        them later allocates nothing: each slot's device grids and pinned host buffers, and its
        molecule handle's operands, Phi staging and FFT work grids, reach the largest size any
        request needs (each of those buffers peaks on a different request), and the Green's
        functions and FFT twiddles of every padded shape are built.  Growing a device buffer calls
        cudaFree/cudaMalloc, and cudaFree synchronises the whole device: an unwarmed slot that a
        larger request outgrows stalls every other slot (requests of 50-240 ms at 200 req/s instead
        of 17-40 ms).  Costs about one evaluation of every request per slot."""
        import dataclasses
        order = sorted(requests, key=lambda r: -footprint(r, self.precision))
        for slot in self.slots:
            for r in order:
                r2 = dataclasses.replace(r, density=None, potential=None, t_admit=None, t_done=None)
                self._launch(slot, r2)
                slot.event.synchronize()
                self._retire(slot, 0.0)
        self.in_use = 0

    def close(self):
        for s in self.slots:
            if s.handle is not None:
                N.load().qmt_mol_destroy(s.handle)
                s.handle = None


def latency_stats(requests):
    lat = np.array([r.latency for r in requests if r.latency is not None])
    if lat.size == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "n": int(lat.size)}

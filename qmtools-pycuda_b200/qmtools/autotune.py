"""Autotuner for batched density + Hartree evaluation (new; the reference has no tuning).

Two choices are measured on the device the first time a bucket is met and cached on disk:

* the density path of a molecule with N <= 320 basis functions (`fused`: basis values stay in
  shared memory, one persistent launch shared by the batch; `staged`: basis values through HBM,
  then the TMA-fed contraction), per (N rounded up to 32, grid points rounded to a power of two,
  precision) -- timed on the molecule itself on a 32^3 grid through its centre;
* the padded transform length of the free-space FFT solve per grid edge n: candidates are the
  lengths >= 2n whose prime factors are 2, 3, 5 and 7, up to 1.3 x 2n, and 256 / 128 (the lengths
  with register kernels) when they qualify -- timed as a cubic n^3 solve.

The cache is a JSON file, `$QMTOOLS_TUNE_CACHE` or ~/.cache/qmtools_b200/tune.json, keyed by the
device name; set QMTOOLS_TUNE=0 to skip measuring (defaults are used and nothing is written).
"""
import ctypes as C
import json
import os
import threading
from pathlib import Path

import numpy as np

from . import _native as N

PATH_STAGED, PATH_FUSED, PATH_FACTORED = 1, 2, 3


def _nice(n):
    for r in (2, 3, 5, 7):
        while n % r == 0:
            n //= r
    return n == 1


def fft_candidates(n):
    lo = 2 * n
    hi = int(1.3 * lo)
    cands = [m for m in range(lo, hi + 1) if _nice(m)]
    return cands[:6] if cands else [lo]


class Tuner:
    def __init__(self, path=None, measure=None):
        if path is None:
            path = os.environ.get("QMTOOLS_TUNE_CACHE",
                                  str(Path.home() / ".cache" / "qmtools_b200" / "tune.json"))
        self.path = Path(path)
        self.measure = (os.environ.get("QMTOOLS_TUNE", "1") != "0") if measure is None else measure
        self._lock = threading.Lock()
        self._data = None
        self.measured = 0     # decisions measured by this instance (not read from the cache)

    # ---- cache ----------------------------------------------------------------------------
    def _device_key(self):
        import torch
        return torch.cuda.get_device_name()

    def _load(self):
        if self._data is None:
            try:
                self._data = json.loads(self.path.read_text())
            except Exception:
                self._data = {}
        return self._data.setdefault(self._device_key(), {})

    def _store(self):
        if not self.measure:
            return
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self._data, indent=1, sort_keys=True))
        tmp.replace(self.path)

    # ---- density path ---------------------------------------------------------------------
    @staticmethod
    def density_key(norbs, npts, precision):
        nb = (int(norbs) + 31) // 32 * 32
        gb = 1 << max(0, int(np.ceil(np.log2(max(int(npts), 1)))))
        return f"density:{precision}:N{nb}:P{gb}"

    def density_path(self, molecule, npts, precision):
        """PATH_FUSED or PATH_STAGED for this molecule (N <= 320 only; larger ones are staged)."""
        if int(molecule.norbs) > 320 or precision.startswith("tf32"):
            return PATH_STAGED
        key = self.density_key(molecule.norbs, npts, precision)
        with self._lock:
            d = self._load()
            if key in d:
                return d[key]["choice"]
            if not self.measure:
                return PATH_FUSED
            times = {p: self._time_density(molecule, precision, p) for p in (PATH_FUSED, PATH_STAGED)}
            choice = min(times, key=times.get)
            d[key] = {"choice": choice, "ms": {str(k): v for k, v in times.items()}}
            self.measured += 1
            self._store()
            return choice

    @staticmethod
    def _time_density(molecule, precision, path, n=32, reps=3):
        import torch
        c = np.asarray(molecule.coords, dtype=np.float64).mean(axis=0)
        h = 0.3
        o = c - n * h / 2
        q = torch.empty(n ** 3, device="cuda")
        st = N.stream_handle()
        N.call("qmt_set_density_path", path)
        try:
            def run():
                N.call("qmt_density", molecule.handle, n, n, n, C.c_float(h), C.c_float(o[0]), C.c_float(o[1]),
                       C.c_float(o[2]), 1, N.PREC[precision], 0, C.c_void_p(q.data_ptr()), None, st)
            run()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            e1.synchronize()
            return e0.elapsed_time(e1) / reps
        finally:
            N.call("qmt_set_density_path", 0)

    # ---- FFT padding ----------------------------------------------------------------------
    def fft_length(self, n, molecule):
        """Padded transform length (>= 2n) for a grid edge of n points."""
        key = f"fft:n{int(n)}"
        with self._lock:
            d = self._load()
            if key in d:
                return d[key]["choice"]
            cands = fft_candidates(int(n))
            if not self.measure or len(cands) == 1:
                return cands[0]
            times = {m: self._time_fft(int(n), m, molecule) for m in cands}
            choice = min(times, key=times.get)
            d[key] = {"choice": choice, "ms": {str(k): v for k, v in times.items()}}
            self.measured += 1
            self._store()
            return choice

    @staticmethod
    def _time_fft(n, m, molecule, reps=3):
        import torch
        c = np.asarray(molecule.coords, dtype=np.float64).mean(axis=0)
        h = 0.28
        o = c - n * h / 2
        q = torch.rand(n ** 3, device="cuda")
        v = torch.empty(n ** 3, device="cuda")
        st = N.stream_handle()

        def run():
            N.call("qmt_fft_poisson_padded", molecule.handle, n, n, n, C.c_float(h), C.c_float(o[0]),
                   C.c_float(o[1]), C.c_float(o[2]), C.c_float(0.2), C.c_float(6.0), m, m, m,
                   C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), st)
        run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

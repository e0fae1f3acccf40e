"""Benchmark: density + Hartree grid points per second on the medium-molecule workload.

Workload (one step): a 30-atom molecule (C10 H14 N3 O3 drawn from a seed in a 12-bohr cube,
cc-pVDZ, N = 294 basis functions, closed-shell seeded density matrix) on a 128^3 grid at
0.15 bohr:
  1. electron density (tensor-core split contraction, default fp16x3), reference convention
     (electrons per voxel, rescaled to the nuclear charge);
  2. Hartree potential by the zero-padded (Hockney, free-space) FFT Poisson solve on a 256^3
     grid, nuclei as Gaussian charges (sigma 0.2 A), in FP32.
value = grid points (128^3 per step, summed over ranks) / second.  One process per GPU;
each rank evaluates its own copy of the workload (replicas, no collective on the path).

Timing: W warm-up steps, then K steps each bracketed by CUDA events on the launching
stream; before each timed step a 512 MiB buffer is written to flush L2.  Barrier and
synchronise on both sides; the reported time is the max over ranks.

`e2e` runs the same step through the public API starting from pinned host buffers
(coordinates and density matrix uploaded into the molecule handle, which re-derives its
device operands) and reads the potential grid back to the host every step.

Beside the headline step, rank 0 also reports (not part of `value`):
  * `plain_fp32`: the same step with the plain FP32 SIMT density path (the reference's
    precision), and the speed-up of the mixed-precision path over it;
  * `accuracy`: density rel-L2 / max-abs of the mixed path against this library's FP64
    density, and the FP64 electron-count error;
  * `batched`: 64 molecules of 5-60 atoms (grids = bounding box + 3 bohr per side at
    0.15 bohr) through the continuous-batching engine, against serial plain FP32;
  * `serving`: a Poisson request stream (atoms log-uniform 3-120) through the engine with
    p50/p99 latency, against serial plain FP32;
  * `cpu_baseline`: the FP64 NumPy/SciPy evaluation on a bounded sample, which also checks
    the mixed result against it (density on the sampled planes, Hartree on the full grid).

`--impl reference` times the reference's own implementation of this path.  The reference is
GPU-only CUDA C driven from Python; its kernels, compiled from its sources into oracle/_ref,
run here with the reference facade's launch shapes and host steps (density kernel, grid
total and rescale, periodic cuFFT Poisson route).  Without those builds the FP64 CPU port
of its algorithm is timed instead.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "qmtools-pycuda_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "grid pts/s density+Hartree & req p50/p99, mixed vs plain FP32 at 1e-6 rel err"
UNIT = "grid_pts/s"
WORKLOAD = "medium molecule: 30 atoms C10H14N3O3, cc-pVDZ N=294, 128^3 grid @ 0.15 bohr, density + Hockney FFT Poisson on 256^3"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("bf16_tflops", 1590.0), d.get("hbm_gbs", 6650.0), "measured"
    return 1590.0, 6650.0, "fallback"


class NvmlClockSampler:
    """SM clock and clock-event reasons polled through NVML every 10 ms in a thread."""

    def __init__(self, local):
        import pynvml
        import torch
        self.nv = pynvml
        pynvml.nvmlInit()
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
        self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode() if isinstance(uuid, str) else uuid)
        self.max = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.samples = []
        self._stop = threading.Event()

    def _run(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                              getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))
        while not self._stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                                     int(get_reasons(self.h)) if get_reasons else 0))
            except Exception:
                pass
            self._stop.wait(0.01)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.th.join(timeout=2)

    def summary(self):
        nv = self.nv
        bits = {"hw_slowdown": "HwSlowdown", "hw_thermal_slowdown": "HwThermalSlowdown",
                "sw_thermal_slowdown": "SwThermalSlowdown", "sw_power_cap": "SwPowerCap"}
        reasons = set()
        for _, r in self.samples:
            for name, suffix in bits.items():
                b = getattr(nv, "nvmlClocksEventReason" + suffix, getattr(nv, "nvmlClocksThrottleReason" + suffix, 0))
                if r & b:
                    reasons.add(name)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median([c for c, _ in self.samples])), "sm_max_mhz": self.max,
                "reasons": sorted(reasons), "samples": len(self.samples), "source": "nvml 10 ms"}


def clock_sampler(local):
    try:
        return NvmlClockSampler(local)
    except Exception:
        return ClockSampler(local)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region (NVML fallback)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend="nccl"):
    """One process per GPU (replicas): torchrun environment, short process-group timeout."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=60))
        pg = dist
    return world, rank, local, pg


def _dev(pg):
    import torch
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def barrier(pg):
    if pg is not None:
        import torch
        pg.barrier()
        if _dev(pg) == "cuda":
            torch.cuda.synchronize()


def max_over_ranks(pg, v):
    """Timed regions are reported as the max over ranks."""
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline_c1(sm, basis, qmtools, check=None):
    """FP64 NumPy/SciPy evaluation of the same step on a bounded sample, per grid point.

    Density: 4 z-planes (4*128^2 points) of the 128^3 grid through the oracle (chunked Phi,
    BLAS Phi@P, row-dot), extrapolated per point.  Hartree: one scipy.fft rfftn/irfftn
    Hockney convolution on the full 256^3 padded grid with all host cores.  With `check`
    (host copies of the mixed-precision results) the FP64 results also score them: density
    on the sampled planes, and the FP64 Hockney potential of the same density on the full
    grid.
    """
    import scipy.fft
    from oracle import density as od
    from oracle import poisson as op
    mol = sm.molecule(basis, qmtools.Molecule)
    g = sm.grid(qmtools.Grid)
    nx, ny, nz, h, ox, oy, oz = g._geom()
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    nzs = 4
    z0 = nz // 2
    q = od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs, basis.alphas,
                                 basis.coeffs, mol.dm, zslab=(z0, z0 + nzs))
    t_dens = (time.perf_counter() - t0) / q.size
    M = 2 * nx
    rho = np.zeros((M, M, M))
    rho[:nx, :ny, :nz] = np.random.default_rng(0).random((nx, ny, nz))
    G = op.hockney_green((nx, ny, nz), h / op.ANG2BOR, (M, M, M))
    t1 = time.perf_counter()
    Gh = scipy.fft.rfftn(G, workers=cores)
    V = scipy.fft.irfftn(scipy.fft.rfftn(rho, workers=cores) * Gh, s=(M, M, M), workers=cores)
    t_fft = time.perf_counter() - t1
    npts = nx * ny * nz
    per_pt = t_dens + t_fft / npts
    out = {"value": 1.0 / per_pt, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"density on {nzs} z-planes ({nzs * nx * ny} pts, FP64 NumPy, extrapolated per point) + "
                     f"one full {M}^3 scipy.fft Hockney convolution (workers={cores})",
           "density_s_per_pt": t_dens, "fft_s": t_fft}
    if check is not None:
        ref = np.asarray(q, dtype=np.float64).ravel()
        got = check["q_raw"].reshape(nz, ny, nx)[z0:z0 + nzs].ravel().astype(np.float64)
        vref = op.hockney_poisson(check["q"], (nx, ny, nz), h, (ox, oy, oz), mol.coords, mol.types, 0.2, 6)
        vref = np.asarray(vref, dtype=np.float64).ravel()
        vgot = check["v"].astype(np.float64).ravel()
        out["check_vs_fp64"] = {
            "density_rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "density_max_abs": float(np.abs(got - ref).max()),
            "density_points": int(ref.size),
            "hartree_rel_l2": float(np.linalg.norm(vgot - vref) / np.linalg.norm(vref)),
            "hartree_max_abs_volt": float(np.abs(vgot - vref).max())}
    return out


def _requests(mols, basis, qmtools, serving, arrivals=None):
    out = []
    for i, m in enumerate(mols):
        out.append(serving.Request(m.molecule(basis, qmtools.Molecule), m.grid(qmtools.Grid),
                                   arrival=0.0 if arrivals is None else arrivals[i], rid=i))
    return out


def _engine_run(serving, reqs, slots, precision, realtime):
    import torch
    eng = serving.Engine(slots=slots, precision=precision)
    eng.warm(reqs)                              # steady state: slots grown to the largest requests
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng.run(reqs, realtime=realtime)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    eng.close()
    return wall


def batched_and_serving(basis, qmtools, precision):
    """C3-like batch and C4-like request stream through the continuous-batching engine."""
    from qmtools import serving
    from qmtools import synthetic as syn
    res = {}
    bm = syn.batch_molecules(64)
    pts = sum(int(np.prod(m.grid_shape)) for m in bm)
    t_mix = _engine_run(serving, _requests(bm, basis, qmtools, serving), 8, precision, False)
    t_fp32 = _engine_run(serving, _requests(bm, basis, qmtools, serving), 1, "fp32", False)
    res["batched"] = {"molecules": len(bm), "atoms": "uniform 5-60", "grid_pts": pts,
                      "value": pts / t_mix, "unit": UNIT, "wall_s": t_mix, "slots": 8,
                      "serial_plain_fp32": {"value": pts / t_fp32, "wall_s": t_fp32},
                      "speedup_vs_serial_plain_fp32": t_fp32 / t_mix,
                      "timing": "host wall clock around the whole batch (set-up, H2D, density, Hockney FFT, D2H); "
                                "slots grown to the largest requests beforehand"}
    rate, count = 200.0, 32
    stream = syn.serving_stream(rate, count)
    arr = [t for t, _ in stream]
    mols = [m for _, m in stream]
    pts = sum(int(np.prod(m.grid_shape)) for m in mols)
    reqs = _requests(mols, basis, qmtools, serving, arr)
    t_mix = _engine_run(serving, reqs, 8, precision, True)
    lat = serving.latency_stats(reqs)
    t_fp32 = _engine_run(serving, _requests(mols, basis, qmtools, serving), 1, "fp32", False)
    res["serving"] = {"requests": count, "rate_req_s": rate, "atoms": "log-uniform 3-120", "grid_pts": pts,
                      "p50_ms": lat["p50_ms"], "p99_ms": lat["p99_ms"], "mean_ms": lat["mean_ms"],
                      "value": pts / t_mix, "unit": UNIT, "makespan_s": t_mix, "slots": 8,
                      "serial_plain_fp32": {"value": pts / t_fp32, "wall_s": t_fp32},
                      "speedup_vs_serial_plain_fp32": t_fp32 / t_mix}
    return res


def run_ours(args, world, rank, local, pg):
    import ctypes as C
    import torch
    import qmtools
    from qmtools import _native as N
    from qmtools import synthetic as syn
    qmtools.set_verbose(False)
    torch.cuda.set_device(local)
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    sm = syn.config_molecule("c1")
    mol = sm.molecule(basis, qmtools.Molecule)
    g = sm.grid(qmtools.Grid)
    if args.grid:
        # the same molecule on a smaller cube of the same spacing, centred on it (profiling cases)
        c = np.asarray(sm.coords_bohr).mean(axis=0)
        hb = sm.step_bohr
        g = qmtools.Grid((1, args.grid, args.grid, args.grid), hb / qmtools.ANG2BOR, list(c - args.grid * hb / 2))
    nx, ny, nz, h, ox, oy, oz = g._geom()
    npts = nx * ny * nz
    qgrid = qmtools.Grid.emptyAs(g)
    q = qgrid.tensor()
    vout = torch.empty(npts, dtype=torch.float32, device="cuda")
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    prec = N.PREC[args.precision]
    stream = torch.cuda.current_stream()
    sh = C.c_void_p(stream.cuda_stream)
    qsum = C.c_double()
    handle = mol.handle

    def step():
        N.call("qmt_density", handle, nx, ny, nz, h, ox, oy, oz, 1, prec, 1, C.c_void_p(q.data_ptr()),
               C.byref(qsum), sh)
        N.call("qmt_fft_poisson", handle, nx, ny, nz, h, ox, oy, oz, 0.2, 6.0, 1, C.c_void_p(q.data_ptr()),
               C.c_void_p(vout.data_ptr()), sh)

    def timed(fn, k, with_density_events=False):
        tot = 0.0
        dens = 0.0
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        for _ in range(k):
            flush.fill_(1.0)
            ev[0].record(stream)
            if with_density_events:
                N.call("qmt_density", handle, nx, ny, nz, h, ox, oy, oz, 1, prec, 1, C.c_void_p(q.data_ptr()),
                       C.byref(qsum), sh)
                ev[1].record(stream)
                N.call("qmt_fft_poisson", handle, nx, ny, nz, h, ox, oy, oz, 0.2, 6.0, 1,
                       C.c_void_p(q.data_ptr()), C.c_void_p(vout.data_ptr()), sh)
            else:
                fn()
                ev[1].record(stream)
            ev[2].record(stream)
            ev[2].synchronize()
            tot += ev[0].elapsed_time(ev[2])
            dens += ev[0].elapsed_time(ev[1])
        return tot / k, dens / k

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(pg)
    with clock_sampler(local) as clk:
        ms, dens_ms = timed(step, args.steps, with_density_events=True)
    torch.cuda.synchronize()
    barrier(pg)
    ms = max_over_ranks(pg, ms)

    # end to end through the public API from pinned host buffers
    coords_h = torch.from_numpy(np.ascontiguousarray(mol.coords, dtype=np.float32)).pin_memory()
    dm_h = torch.from_numpy(np.ascontiguousarray(mol.dm, dtype=np.float32)).pin_memory()
    v_h = torch.empty(npts, dtype=torch.float32).pin_memory()

    def e2e_step():
        N.call("qmt_mol_set_coords", handle, C.c_void_p(coords_h.data_ptr()), sh)
        N.call("qmt_mol_set_dm", handle, C.c_void_p(dm_h.data_ptr()), sh)
        step()
        v_h.copy_(vout, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    barrier(pg)
    e2e_ms, _ = timed(e2e_step, args.steps)
    e2e_ms = max_over_ranks(pg, e2e_ms)

    launches = kernel_launches_per_step(args.precision)
    out = {
        "metric": METRIC, "value": world * npts / (ms / 1000.0), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
        "data": "synthetic (seeded geometry and density matrix; no public dataset exists for this path)",
        "config": {"workload": WORKLOAD if not args.grid else WORKLOAD.replace("128^3", f"{args.grid}^3"),
                   "grid_pts_per_step": npts, "basis_functions": int(mol.norbs),
                   "density_precision": args.precision, "poisson": "Hockney free-space FFT, 256^3 padded, FP32",
                   "l2": "512 MiB flush written before every timed step", "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * npts / (e2e_ms / 1000.0), "unit": UNIT,
                "h2d_bytes_per_step": int(coords_h.numel() * 4 + dm_h.numel() * 4),
                "d2h_bytes_per_step": int(v_h.numel() * 4)},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    # roofline of the dominant kernel: the density contraction, algorithmic flops npts(2N^2+2N)
    nb = int(mol.norbs)
    flops = npts * (2.0 * nb * nb + 2.0 * nb)
    peak_tf, hbm, kind = peaks()
    achieved = flops / (dens_ms / 1000.0) / 1e12
    out["roofline"] = {"bound": "tensor", "kernel": "qmt_density (basis + tcgen05 contraction + row-dot)",
                       "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s", "frac": achieved / peak_tf,
                       "peak_source": f"bf16_tflops burst, {kind}", "density_ms": dens_ms,
                       "traffic": profiled_traffic() if (args.precision == "fp16x3" and not args.grid) else None,
                       "traffic_unit": "DRAM bytes per launch (ncu, dram__bytes_read.sum + dram__bytes_write.sum)"}
    # the basis evaluation's exponentials, counted separately (npts x primitives of all shells,
    # before screening): what bounds the SIMT half of the kernel
    almos = np.asarray(mol.ALMOs).reshape(-1, 4)
    shells = {(int(r[0]), int(r[3])) for r in almos}
    co = np.asarray(mol.basisset.coeffs)
    nprim = sum(int(np.count_nonzero(co[so:so + 20])) for _, so in shells)
    out["roofline"]["exponentials_per_launch"] = int(npts * nprim)
    out["roofline"]["exponentials_per_s"] = npts * nprim / (dens_ms / 1000.0)
    check = None
    if world == 1 and not args.quick:
        # plain FP32 SIMT density (the reference's precision) on the same step
        p32 = N.PREC["fp32"]

        def step32():
            N.call("qmt_density", handle, nx, ny, nz, h, ox, oy, oz, 1, p32, 1, C.c_void_p(q.data_ptr()),
                   C.byref(qsum), sh)
            N.call("qmt_fft_poisson", handle, nx, ny, nz, h, ox, oy, oz, 0.2, 6.0, 1, C.c_void_p(q.data_ptr()),
                   C.c_void_p(vout.data_ptr()), sh)

        step32()
        ms32, _ = timed(step32, 5)
        out["plain_fp32"] = {"value": npts / (ms32 / 1000.0), "unit": UNIT, "ms_per_step": ms32,
                             "speedup_of_mixed": ms32 / ms}
        # accuracy of the mixed path against this library's FP64 density (raw electrons/voxel)
        q64 = torch.empty_like(q)
        s64, smx = C.c_double(), C.c_double()
        N.call("qmt_density", handle, nx, ny, nz, h, ox, oy, oz, 1, N.PREC["fp64"], 0, C.c_void_p(q64.data_ptr()),
               C.byref(s64), sh)
        N.call("qmt_density", handle, nx, ny, nz, h, ox, oy, oz, 1, prec, 0, C.c_void_p(q.data_ptr()),
               C.byref(smx), sh)
        tr = C.c_double()
        N.call("qmt_mol_trace_ps", handle, C.byref(tr), sh)
        d = (q.double() - q64.double())
        out["accuracy"] = {"density_rel_l2_vs_fp64": float(d.norm() / q64.double().norm()),
                           "density_max_abs_vs_fp64": float(d.abs().max()),
                           "grid_electrons_fp64": s64.value, "grid_electrons_mixed": smx.value,
                           "electron_count_trace_ps_fp64": 2.0 * tr.value,
                           "reference": "this library's FP64 density path (checked against the FP64 oracle by the tests)"}
        q_raw = q.cpu().numpy()
        step()
        torch.cuda.synchronize()
        check = {"q_raw": q_raw, "q": q.cpu().numpy(), "v": vout.cpu().numpy()}
        out.update(batched_and_serving(basis, qmtools, args.precision))
        out["kernels"] = other_kernels(basis, qmtools, N, hbm, ms - dens_ms, {"n3": npts, "M": 2 * nx})
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_c1(sm, basis, qmtools, check)
    return out


def other_kernels(basis, qmtools, N, hbm_peak, fft_ms, nfft):
    """Rooflines of the other kernels of the path (rank 0, not part of `value`)."""
    import ctypes as C
    import torch
    from qmtools import synthetic as syn
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {}
    jac = {}
    for name, n, sweeps in (("c0_64^3_2000_sweeps", 64, 2000), ("c1_128^3_400_sweeps", 128, 400)):
        npts = n ** 3
        rho = torch.rand(npts, device="cuda")
        v = torch.zeros(npts, device="cuda")
        t = torch.zeros(npts, device="cuda")
        so, d = C.c_int(), C.c_double()
        args = lambda k: (n, n, n, 0.2, C.c_void_p(rho.data_ptr()), C.c_void_p(v.data_ptr()),
                          C.c_void_p(t.data_ptr()), k, 100, 0.0, C.byref(so), C.byref(d), s)
        N.call("qmt_jacobi", *args(20))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        N.call("qmt_jacobi", *args(sweeps))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        gbs = 12.0 * npts * sweeps / (ms / 1e3) / 1e9
        jac[name] = {"ms": ms, "us_per_sweep": 1e3 * ms / sweeps, "achieved_GBps": gbs,
                     "frac_of_hbm_peak": gbs / hbm_peak}
    out["jacobi"] = dict(jac, bytes_per_point_sweep=12, kernel="jacobi_persistent_kernel (one cooperative launch)")
    # GA single-shot automaton: 26 neighbour MLPs (4 hidden layers of 16) per voxel, 96^3 grid
    n, nl = 96, 4
    npts = n ** 3
    qube = torch.rand(2 * npts, device="cuda")
    qo = torch.empty(npts, device="cuda")
    p = ((2 * np.random.default_rng(0).random(272 * nl + 29) - 1) * 0.5).astype(np.float32)
    call = lambda: N.call("qmt_nn_singleshot", n, n, n, 0.2, C.c_void_p(qube.data_ptr()),
                          C.c_void_p(qo.data_ptr()), C.c_void_p(p.ctypes.data), int(p.size), nl, s)
    call()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        call()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    fma = 26.0 * (272 * nl + 17)
    out["automaton_nnss_96^3_nl4"] = {"ms": ms, "voxels_per_s": npts / (ms / 1e3),
                                      "fp32_tflops": 2 * fma * npts / (ms / 1e3) / 1e12,
                                      "flop_definition": "2 x 26 x (272 NL + 17) FMA per voxel (tanh not counted)"}
    if nfft is not None:
        H = nfft["M"] ** 2 * (nfft["M"] // 2 + 1)
        fbytes = 8.0 * nfft["n3"] + 100.0 * H
        out["fft_hockney"] = {"ms": fft_ms, "algorithmic_bytes": fbytes,
                              "achieved_GBps": fbytes / (fft_ms / 1e3) / 1e9,
                              "frac_of_hbm_peak": fbytes / (fft_ms / 1e3) / 1e9 / hbm_peak,
                              "definition": "8 n^3 + 100 H bytes, H = M^2 (M/2+1), M = 2n"}
        sm = syn.config_molecule("c1")
        mol = sm.molecule(basis, qmtools.Molecule)
        g = sm.grid(qmtools.Grid)
        nx, ny, nz, h, ox, oy, oz = g._geom()
        v = torch.zeros(nx * ny * nz, device="cuda")
        call = lambda: N.call("qmt_hartree_gto_boundary", mol.handle, nx, ny, nz, h, ox, oy, oz,
                              C.c_void_p(v.data_ptr()), s)
        call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        call()
        e1.record()
        torch.cuda.synchronize()
        nb = nx * ny * nz - (nx - 2) * (ny - 2) * (nz - 2)
        ms = e0.elapsed_time(e1)
        out["gto_boundary_c1"] = {"ms": ms, "boundary_points": nb, "points_per_s": nb / (ms / 1e3),
                                  "precision": "FP64 McMurchie-Davidson"}
    return out


def profiled_traffic():
    """DRAM bytes (read + write) per launch of the fused density kernel at the bench size, from
    the one-pass ncu capture summarised in profiles/density_fused_kernel_c1.md."""
    import re
    f = ROOT / "profiles" / "density_fused_kernel_c1.md"
    if not f.exists():
        return None
    txt = f.read_text().split("## DRAM traffic at the bench size", 1)[-1]
    rd = re.search(r"dram__bytes_read\.sum \| ([\d,]+) B", txt)
    wr = re.search(r"dram__bytes_write\.sum \| ([\d,]+) B", txt)
    if not (rd and wr):
        return None
    return int(rd.group(1).replace(",", "")) + int(wr.group(1).replace(",", ""))


def kernel_launches_per_step(prec):
    """Launches of this library's kernels per timed step (density + Hockney FFT)."""
    dens = 3        # density kernel (fused tensor-core or SIMT), partial-sum reduction, rescale
    fft = 5         # x forward with the RHS, y forward, z forward x G x z inverse, y inverse, x inverse
    return dens + fft


def _ref_libs():
    ref = ROOT / "oracle" / "_ref"
    paths = [ref / "utils.so", ref / "c1_bench" / "density_s1.so", ref / "c1_bench" / "fft.so"]
    return paths if all(p.exists() for p in paths) else None


def run_reference_gpu(args, world, rank, local, paths):
    """The reference path on the same B200: its density kernel (kernel_density.cu), grid total
    and rescale (kernel_utils.cu) and the periodic FFT route (kernel_fft.cu around cuFFT), with
    the launch shapes and host steps of its facade (Compute_density, Compute_hartree_fft)."""
    import ctypes as C
    import torch
    import qmtools
    from qmtools import synthetic as syn
    qmtools.set_verbose(False)
    torch.cuda.set_device(local)
    ut, dl, fl_ = (C.CDLL(str(p)) for p in paths)
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    sm = syn.config_molecule("c1")
    mol = sm.molecule(basis, qmtools.Molecule)
    g = sm.grid(qmtools.Grid)
    nx, ny, nz = g.space_shape()
    gx, gy, gz = g.GPUblocks
    n = nx * ny * nz
    h = float(g.step)
    ox, oy, oz = (float(g.origin[k]) for k in "xyz")
    dev = "cuda"
    pin = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt).ravel()).pin_memory()
    coords_h, dm_h = pin(mol.coords, np.float32), pin(mol.dm, np.float32)
    coords, dm = coords_h.to(dev), dm_h.to(dev)
    types = torch.from_numpy(np.ascontiguousarray(mol.types, dtype=np.int32)).to(dev)
    almos = torch.from_numpy(np.ascontiguousarray(mol.ALMOs, dtype=np.int16)).to(dev)
    alphas = torch.from_numpy(np.ascontiguousarray(basis.alphas, dtype=np.float32)).to(dev)
    coeffs = torch.from_numpy(np.ascontiguousarray(basis.coeffs, dtype=np.float32)).to(dev)
    q = torch.zeros(n, device=dev)
    tot = torch.zeros(1, device=dev)
    wr, c1, c2, v = (torch.zeros(k * n, device=dev) for k in (1, 2, 2, 1))
    v_h = torch.empty(n, dtype=torch.float32).pin_memory()
    vp = lambda t: C.c_void_p(t.data_ptr())
    f = C.c_float

    def step(e2e=False):
        if e2e:
            coords.copy_(coords_h, non_blocking=True)
            dm.copy_(dm_h, non_blocking=True)
        assert dl.ref_density(gx, gy, gz, f(h), f(ox), f(oy), f(oz), vp(coords), vp(alphas), vp(coeffs), vp(almos),
                              vp(dm), vp(q)) == 0
        assert ut.ref_total(gx, gy, gz, vp(q), vp(tot)) == 0
        factor = np.float32(mol.qtot / float(tot.item()))
        assert ut.ref_rescale(gx, gy, gz, vp(q), f(factor)) == 0
        assert fl_.ref_fft_route(gx, gy, gz, nx, ny, nz, vp(q), vp(types), vp(coords), vp(wr), vp(c1), vp(c2),
                                 vp(v)) == 0
        if e2e:
            v_h.copy_(v)
        torch.cuda.synchronize()

    def timed(k, e2e, budget_s):
        # up to k steps, stopping once budget_s of wall time is spent (a reference step takes
        # seconds): the run stays within a few minutes at any --steps
        ts = []
        t_start = time.perf_counter()
        for _ in range(k):
            t0 = time.perf_counter()
            step(e2e)
            ts.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start > budget_s:
                break
        return float(np.mean(ts)), len(ts)

    for _ in range(min(args.warmup, 3)):
        step()
    ms, nsteps = timed(args.steps, False, 60.0)
    e2e_ms, _ = timed(max(1, args.steps // 2), True, 30.0)
    ms *= 1000.0
    e2e_ms *= 1000.0
    v_ = n / (ms / 1000.0)
    return {"metric": METRIC, "value": v_, "unit": UNIT, "n_gpus": world, "steps": nsteps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD.replace("density + Hockney FFT Poisson on 256^3",
                                                   "density + periodic FFT Poisson on 128^3 (the reference's solve)"),
                       "grid_pts_per_step": n, "timing": "host wall clock around each synchronised step; up to --steps steps within 60 s (end to end: 30 s)"},
            "cpu_baseline": {"value": v_, "unit": UNIT, "cores": 0, "kind": "reference",
                             "sample": "the full step on the GPU: the reference's kernels compiled from its sources "
                                       "for sm_100a (oracle/_ref/c1_bench), no host cores used"},
            "e2e": {"value": n / (e2e_ms / 1000.0), "unit": UNIT,
                    "h2d_bytes_per_step": int(4 * (coords_h.numel() + dm_h.numel())), "d2h_bytes_per_step": 4 * n}}


def run_reference(args, world, rank, local, pg):
    """The reference's implementation of this path, timed on the same workload (rank 0 only)."""
    if rank != 0:
        return None
    paths = _ref_libs()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if paths is not None and has_gpu:
        return run_reference_gpu(args, world, rank, local, paths)
    import qmtools
    from qmtools import synthetic as syn
    qmtools.set_verbose(False)
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    sm = syn.config_molecule("c1")
    # CPU oracle port of the reference algorithm (FP64 density + FFT solve)
    samples = []
    for _ in range(args.warmup):
        cpu_baseline_c1(sm, basis, qmtools)
    for _ in range(args.steps):
        samples.append(cpu_baseline_c1(sm, basis, qmtools))
    v = float(np.median([s["value"] for s in samples]))
    cb = dict(samples[0])
    cb["value"] = v
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * (128 ** 3) / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "FP64 CPU port of the reference algorithm on the host cores (reference kernel builds absent)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp16x3")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="headline step only (no plain-FP32, batch, serving)")
    ap.add_argument("--grid", type=int, default=0, help="cube edge of a smaller grid for the same molecule")
    ap.add_argument("--only", default="", choices=["", "jacobi"], help="run one kernel family alone (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local, pg = dist_setup()
    if args.only == "jacobi":
        # the Jacobi solve alone (64^3 for 2000 sweeps, 128^3 for 400): its profiling case
        import torch
        import qmtools
        from qmtools import _native as N
        qmtools.set_verbose(False)
        torch.cuda.set_device(local)
        N.ensure_device(None)
        print(json.dumps(other_kernels(None, qmtools, N, peaks()[1], 0.0, None)["jacobi"]))
        return
    try:
        if args.impl == "reference":
            out = run_reference(args, world, rank, local, pg)
        else:
            out = run_ours(args, world, rank, local, pg)
        if rank == 0 and out is not None:
            print(json.dumps(out))
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()

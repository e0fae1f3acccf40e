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

`--impl reference` times the reference implementation of this path instead (see
DESIGN.md: the reference is GPU-only CUDA C; its kernels are compiled from source into
oracle/_ref when available, otherwise the CPU oracle port of its algorithm is timed).
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


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

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


def cpu_baseline_c1(sm, basis, qmtools):
    """FP64 NumPy/SciPy evaluation of the same step on a bounded sample, per grid point.

    Density: 4 z-planes (4*128^2 points) of the 128^3 grid through the oracle (chunked Phi,
    BLAS Phi@P, row-dot), extrapolated per point.  Hartree: one scipy.fft rfftn/irfftn
    Hockney convolution on the full 256^3 padded grid with all host cores.
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
    q = od.density_qube_unscaled((nx, ny, nz), np.float32(h), (ox, oy, oz), mol.coords, mol.ALMOs, basis.alphas,
                                 basis.coeffs, mol.dm, zslab=(nz // 2, nz // 2 + nzs))
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
    return {"value": 1.0 / per_pt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"density on {nzs} z-planes ({nzs * nx * ny} pts, FP64 NumPy, extrapolated per point) + "
                      f"one full {M}^3 scipy.fft Hockney convolution (workers={cores})",
            "density_s_per_pt": t_dens, "fft_s": t_fft}


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
    with ClockSampler(local) as clk:
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
        "config": {"workload": WORKLOAD, "grid_pts_per_step": npts, "basis_functions": int(mol.norbs),
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
                       "traffic": None}
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_c1(sm, basis, qmtools)
    return out


def kernel_launches_per_step(prec):
    """Launches of this library's kernels per step (density + Hockney FFT)."""
    # density: tensor-core path = staging + contraction per chunk, partial reduction, rescale
    dens = 4 + 2 if prec not in ("fp32", "fp64") else 3
    fft = 1 + 3 + 1 + 3 + 1    # RHS, 3 forward axis passes, G multiply, 3 inverse passes, C-order write
    return dens + fft


def run_reference(args, world, rank, local, pg):
    """The reference's implementation of this path, timed on the same workload."""
    if rank != 0:
        return None
    import qmtools
    from qmtools import synthetic as syn
    qmtools.set_verbose(False)
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    sm = syn.config_molecule("c1")
    ref_lib = ROOT / "oracle" / "_ref"
    # CPU oracle port of the reference algorithm (density per voxel centre + periodic FFT solve)
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
            "note": "oracle port (FP64 NumPy/SciPy) of the reference algorithm on the host cores"
            + ("" if ref_lib.exists() else "; reference CUDA harness not built")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp16x3")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local, pg = dist_setup()
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

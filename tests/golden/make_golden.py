"""Generate golden fixtures from the reference's own CUDA kernels (run on a B200).

Loads the reference kernels compiled from their sources by oracle/build_ref.py
(oracle/_ref/*.so), runs them on each parity case of oracle/ref_cases.py with the launch
shapes and host-side steps of the reference facade (qmtools/qmtools.py), and writes the
outputs to <outdir>/<case>.npz (default golden_out).  The committed tests/golden/*.npz were
produced by

    python tests/golden/make_golden.py <outdir>

on a B200; tests/test_golden.py checks the oracle against them (CPU) and
tests/test_gpu_golden.py checks the sm_100a kernels against them (GPU).
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "qmtools-pycuda_b200"))

from oracle import ref_cases as rc  # noqa: E402

REF = ROOT / "oracle" / "_ref"


def lib(path):
    L = C.CDLL(str(path))
    return L


def vp(t):
    return C.c_void_p(t.data_ptr())


def run_case(case, outdir):
    import torch
    import qmtools
    qmtools.set_verbose(False)
    mol, grid = rc.case_inputs(case)
    spec = rc.CASES[case]
    dev = "cuda"
    f32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)
    coords = f32(mol.coords.ravel())
    types = torch.from_numpy(np.ascontiguousarray(mol.types, dtype=np.int32)).to(dev)
    almos = torch.from_numpy(np.ascontiguousarray(mol.ALMOs, dtype=np.int16)).to(dev)
    alphas = f32(mol.basisset.alphas)
    coeffs = f32(mol.basisset.coeffs)
    dm = f32(mol.dm.ravel())
    nx, ny, nz = grid.space_shape()
    gx, gy, gz = grid.GPUblocks
    n = nx * ny * nz
    h = float(grid.step)
    ox, oy, oz = (float(grid.origin[k]) for k in "xyz")
    ut = lib(REF / "utils.so")
    out = {"shape": np.array([nx, ny, nz]), "step": np.float32(grid.step),
           "origin": np.array([ox, oy, oz], dtype=np.float32)}
    fl = C.c_float
    for s in spec.get("density", []):
        L = lib(REF / case / f"density_s{s}.so")
        q = torch.zeros(n, device=dev)
        rc_ = L.ref_density(gx, gy, gz, fl(h), fl(ox), fl(oy), fl(oz), vp(coords), vp(alphas), vp(coeffs), vp(almos),
                            vp(dm), vp(q))
        assert rc_ == 0, rc_
        out[f"density_raw_s{s}"] = q.cpu().numpy()
        # Compute_density: qtot via gpu_total, then gpu_rescale by qtot/sum (qmtools/qmtools.py:2420-2424)
        tot = torch.zeros(1, device=dev)
        assert ut.ref_total(gx, gy, gz, vp(q), vp(tot)) == 0
        total = float(tot.item())
        factor = np.float32(mol.qtot / total)
        assert ut.ref_rescale(gx, gy, gz, vp(q), fl(factor)) == 0
        out[f"density_total_s{s}"] = np.float64(total)
        out[f"density_s{s}"] = q.cpu().numpy()
    if spec.get("hartree_gto"):
        L = lib(REF / case / "hartree_gto.so")
        v = torch.zeros(n, device=dev)
        assert L.ref_hartree_gto(gx, gy, gz, vp(types), vp(coords), vp(alphas), vp(coeffs), vp(almos), vp(dm),
                                 vp(v)) == 0
        out["hartree_gto"] = v.cpu().numpy()
        # same kernel with the density matrix restricted to its s-s block: isolates the
        # reference's S-S closed form (kernel_hartree.cu:432-434)
        s_only = (mol.ALMOs[:, 1] == 0)
        dm_ss = np.where(np.outer(s_only, s_only), mol.dm, 0).astype(np.float32)
        dss = f32(dm_ss.ravel())
        v.zero_()
        assert L.ref_hartree_gto(gx, gy, gz, vp(types), vp(coords), vp(alphas), vp(coeffs), vp(almos), vp(dss),
                                 vp(v)) == 0
        out["hartree_gto_ss"] = v.cpu().numpy()
    if spec.get("hartree_iter"):
        # Compute_hartree_iter (qmtools/qmtools.py:2522-2561): seed, rho = seed - q, 20 sweep pairs
        L = lib(REF / case / "hartree_iter.so")
        q = torch.from_numpy(out["density_s1"]).to(dev)
        seed = torch.zeros(n, device=dev)
        assert ut.ref_seed(int(mol.natoms), fl(h), fl(ox), fl(oy), fl(oz), nx, ny, nz, vp(types), vp(coords),
                           vp(seed)) == 0
        out["seed"] = seed.cpu().numpy()
        rho = seed - q
        V = torch.zeros(n, device=dev)
        T = torch.zeros(n, device=dev)
        for _ in range(20):
            assert L.ref_hartree_iteration(gx, gy, gz, vp(rho), vp(V), vp(T)) == 0
            assert L.ref_hartree_iteration(gx, gy, gz, vp(rho), vp(T), vp(V)) == 0
        d = torch.zeros(1, device=dev)
        assert ut.ref_qdiff(gx, gy, gz, vp(V), vp(T), vp(d), 0) == 0
        out["jacobi_rho"] = rho.cpu().numpy()
        out["jacobi_40"] = V.cpu().numpy()
        out["jacobi_delta"] = np.float64(d.item())
    if spec.get("fft"):
        L = lib(REF / case / "fft.so")
        q = torch.from_numpy(out["density_s1"]).to(dev)
        wr = torch.zeros(n, device=dev)
        c1 = torch.zeros(2 * n, device=dev)
        c2 = torch.zeros(2 * n, device=dev)
        vout = torch.zeros(n, device=dev)
        assert L.ref_fft_route(gx, gy, gz, nx, ny, nz, vp(q), vp(types), vp(coords), vp(wr), vp(c1), vp(c2),
                               vp(vout)) == 0
        out["fft_rhs"] = wr.cpu().numpy()
        out["fft_periodic"] = vout.cpu().numpy()
    if spec.get("vne"):
        # Compute_VNe loop (qmtools/qmtools.py:2713-2740) for 6 pairs
        L = lib(REF / case / "vne.so")
        res = torch.zeros(n, device=dev)
        o2 = torch.zeros(n, device=dev)
        d = torch.zeros(1, device=dev)
        deltas = []
        for _ in range(6):
            assert L.ref_vne(gx, gy, gz, vp(types), vp(coords), fl(ox), fl(oy), fl(oz), fl(h), vp(res), vp(o2),
                             vp(d)) == 0
            d.zero_()
            assert L.ref_vne(gx, gy, gz, vp(types), vp(coords), fl(ox), fl(oy), fl(oz), fl(h), vp(o2), vp(res),
                             vp(d)) == 0
            deltas.append(float(d.item()) / n)
            d.zero_()
        out["vne_pseudo_6"] = res.cpu().numpy()
        out["vne_pseudo_deltas"] = np.array(deltas)
    if spec.get("vne_classic"):
        L = lib(REF / case / "vne_classic.so")
        v = torch.zeros(n, device=dev)
        assert L.ref_vne_classic(gx, gy, gz, vp(types), vp(coords), vp(v)) == 0
        out["vne_classic"] = v.cpu().numpy()
    if "density_s1" in out and case != "c1_bench":
        a = torch.from_numpy(out["density_s1"]).to(dev)
        b = torch.from_numpy(out["density_raw_s1"]).to(dev) + 1e-3
        for rel in (0, 1):
            d = torch.zeros(1, device=dev)
            assert ut.ref_qdiff(gx, gy, gz, vp(a), vp(b), vp(d), rel) == 0
            out[f"qdiff_rel{rel}"] = np.float64(d.item())
    torch.cuda.synchronize()
    path = Path(outdir) / f"{case}.npz"
    if case == "c1_bench":
        # full-size outputs are not fixtures: keep checksums only
        out = {k: (np.float64(np.sum(v, dtype=np.float64)) if isinstance(v, np.ndarray) and v.size > 4096 else v)
               for k, v in out.items()}
    np.savez_compressed(path, **out)
    return path


def run_nn_ss(case, outdir):
    """The single-shot automaton kernel on seeded inputs, as AutomatonSingleShot.Evaluate
    launches it (qmtools/automaton_nn_singleshot.py:90-140): a two-field grid (field 0 zero,
    field 1 the pseudo-field), the element's parameters in cParams, 8x8x8 blocks."""
    import torch
    import qmtools
    qmtools.set_verbose(False)
    _, grid = rc.case_inputs(case)
    nx, ny, nz = grid.space_shape()
    gx, gy, gz = grid.GPUblocks
    n = nx * ny * nz
    out = {"shape": np.array([nx, ny, nz]), "step": np.float32(grid.step)}
    for nl in rc.CASES[case].get("nn_ss", []):
        rng = np.random.default_rng(rc.NN_SEED + nl)
        field1 = rng.uniform(0.0, 1.0, size=n).astype(np.float32)
        dna = 16 * 16 * nl + 16 * nl + (16 * 1 + 1) + 12
        params = ((2 * rng.random(dna) - 1) * 1.0).astype(np.float32)
        qube = torch.zeros(2 * n, device="cuda")
        qube[n:] = torch.from_numpy(field1).cuda()
        qout = torch.zeros(n, device="cuda")
        L = lib(REF / case / f"nn_ss_l{nl}.so")
        assert L.ref_nn_ss(gx, gy, gz, vp(qube), vp(qout), params.ctypes.data_as(C.c_void_p), dna) == 0
        out[f"nn_ss_l{nl}_field1"] = field1
        out[f"nn_ss_l{nl}_params"] = params
        out[f"nn_ss_l{nl}_out"] = qout.cpu().numpy()
    path = Path(outdir) / f"{case}.nn_ss.npz"
    np.savez_compressed(path, **out)
    return path


def main():
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    outdir = Path(args[0] if args else "golden_out")
    outdir.mkdir(parents=True, exist_ok=True)
    cases = args[1:] or list(rc.CASES)
    for case in cases:
        if "--nn-ss" in sys.argv:
            if rc.CASES[case].get("nn_ss"):
                print("wrote", run_nn_ss(case, outdir), flush=True)
        else:
            print("wrote", run_case(case, outdir), flush=True)


if __name__ == "__main__":
    main()

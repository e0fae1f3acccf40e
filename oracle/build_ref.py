"""Compile the reference's CUDA kernels from their sources for sm_100a (test infrastructure).

The reference (fullmetalfelix/QMTools-pycuda) is CUDA C that its Python host specialises by
text substitution of PYCUDA_* tokens and JIT-compiles with PyCUDA.  PyCUDA is not available
here, so this recipe performs the same substitutions, in the same order and with the same
value formatting as the reference host (qmtools/qmtools.py:2384-2391, 2439-2455, 2500-2515,
2581-2595, 2682-2689, 2756-2769), on the reference sources where they lie under
/root/reference, appends a small launcher of this repository (oracle/ref_launch/*.inc) and
compiles each specialisation with nvcc into oracle/_ref/<case>/<family>.so.  Nothing here is
copied into the repository: the substituted sources live only in a temporary directory during
the compile, and the libraries under oracle/_ref/ are git-ignored build products.  The GPU tests and tests/golden/make_golden.py load these libraries.

    python oracle/build_ref.py [--force]
"""
import hashlib
import os
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
REF_CUDA = Path("/root/reference/qmtools/cuda")
OUT = HERE / "_ref"
LAUNCH = HERE / "ref_launch"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler", "-fPIC",
         "-I", str(REF_CUDA), "-I", str(LAUNCH), "-diag-suppress", "177,550,128,2464"]


def _ff(v):
    """str() of a value as the reference host writes it into kernel source."""
    return str(v)


def subst(text, pairs):
    for k, v in pairs:
        text = text.replace(k, v)
    return text


def density_src(mol, subgrid):
    # qmtools/qmtools.py:2384-2391
    t = (REF_CUDA / "kernel_density.cu").read_text()
    return subst(t, [("PYCUDA_NATOMS", _ff(mol.natoms)), ("PYCUDA_NORBS", _ff(mol.norbs)),
                     ("PYCUDA_SUBGRIDN", _ff(subgrid)), ("PYCUDA_SUBGRIDDX1", _ff(1.0 / subgrid) + "f"),
                     ("PYCUDA_SUBGRIDDX2", _ff(1.0 / (subgrid * 2)) + "f"),
                     ("PYCUDA_SUBGRIDiV", _ff(1.0 / (subgrid * subgrid * subgrid)) + "f")])


def hartree_src(mol, grid, with_norb):
    # qmtools/qmtools.py:2439-2455 (Compute_hartree) and 2500-2515 (Compute_hartree_iter, NORB left 0)
    t = (REF_CUDA / "kernel_hartree.cu").read_text()
    pairs = [("PYCUDA_NATOMS", _ff(mol.natoms)), ("PYCUDA_GRID_STEP", _ff(grid.step) + "f"),
             ("PYCUDA_GRID_X0", _ff(grid.origin["x"]) + "f"), ("PYCUDA_GRID_Y0", _ff(grid.origin["y"]) + "f"),
             ("PYCUDA_GRID_Z0", _ff(grid.origin["z"]) + "f"), ("PYCUDA_GRID_NX", _ff(grid.shape[1])),
             ("PYCUDA_GRID_NY", _ff(grid.shape[2])), ("PYCUDA_GRID_NZ", _ff(grid.shape[3]))]
    if with_norb:
        pairs.append(("#define NORB 0", "#define NORB {}".format(mol.norbs)))
    else:
        # Compute_hartree_iter leaves `#define NORB 0`; nvcc 12.9 rejects the zero-sized
        # shared arrays this gives gpu_hartree_GTO (kernel_hartree.cu:300-301).
        # gpu_hartree_iteration never reads NORB, so NORB=1 builds the same iteration kernel.
        pairs.append(("#define NORB 0", "#define NORB 1"))
    return subst(t, pairs)


def fft_src(mol, grid, sigma, cutoff, ang2bor):
    # qmtools/qmtools.py:2581-2595; step and origin are converted back to Angstrom there.
    t = (REF_CUDA / "kernel_fft.cu").read_text()
    sh = grid.space_shape()
    return subst(t, [("PYCUDA_NATOMS", _ff(mol.natoms)),
                     ("PYCUDA_GRID_STEP", _ff(float(grid.step) / ang2bor) + "f"),
                     ("PYCUDA_GRID_X0", _ff(float(grid.origin["x"]) / ang2bor) + "f"),
                     ("PYCUDA_GRID_Y0", _ff(float(grid.origin["y"]) / ang2bor) + "f"),
                     ("PYCUDA_GRID_Z0", _ff(float(grid.origin["z"]) / ang2bor) + "f"),
                     ("PYCUDA_GRID_NX", _ff(sh[0])), ("PYCUDA_GRID_NY", _ff(sh[1])), ("PYCUDA_GRID_NZ", _ff(sh[2])),
                     ("PYCUDA_SIGMA", _ff(sigma) + "f"), ("PYCUDA_CUTOFF_SQ", _ff((cutoff * sigma) ** 2) + "f")])


def vne_src(mol, grid, adsorb, diff):
    # qmtools/qmtools.py:2682-2689
    t = (REF_CUDA / "kernel_vne.cu").read_text()
    return subst(t, [("PYCUDA_NATOMS", _ff(mol.natoms)), ("PYCUDA_NX", _ff(grid.shape[1])),
                     ("PYCUDA_NY", _ff(grid.shape[2])), ("PYCUDA_NZ", _ff(grid.shape[3])),
                     ("PYCUDA_ADS", _ff(adsorb)), ("PYCUDA_DIF", _ff(diff))])


def vne_classic_src(mol, grid, divisions):
    # qmtools/qmtools.py:2756-2769
    t = (REF_CUDA / "kernel_vne_classic.cu").read_text()
    return subst(t, [("PYCUDA_NATOMS", _ff(mol.natoms)), ("PYCUDA_NX", _ff(grid.shape[1])),
                     ("PYCUDA_NY", _ff(grid.shape[2])), ("PYCUDA_NZ", _ff(grid.shape[3])),
                     ("PYCUDA_X0", _ff(grid.origin["x"])), ("PYCUDA_Y0", _ff(grid.origin["y"])),
                     ("PYCUDA_Z0", _ff(grid.origin["z"])), ("PYCUDA_DX", _ff(grid.step)),
                     ("PYCUDA_NDIV", _ff(divisions)), ("PYCUDA_dx", _ff(grid.step / divisions))])


def nn_ss_src(grid, nlayers):
    # AutomatonSingleShot.__WriteCode (qmtools/automaton_nn_singleshot.py:195-207), then the
    # common substitutions of Evaluate (qmtools/automaton_nn_singleshot.py:108-113) on the
    # two-field compute grid (Grid.npts is a uint32, Grid.step a float32, qmtools/qmtools.py:218-221)
    import numpy
    t = (REF_CUDA / "kernel_nn_ss.cu").read_text()
    dna = 16 * 16 * nlayers + 16 * nlayers + (16 * 1 + 1) + 12
    t = subst(t, [("PYCUDA_DNASIZE", _ff(dna)), ("PYCUDA_NL1", _ff(nlayers)), ("PYCUDA_NL2", _ff(0)),
                  ("PYCUDA_ABS_A", _ff(0)), ("PYCUDA_ABS_B", _ff(0))])
    npts = numpy.uint32(grid.shape[1] * grid.shape[2] * grid.shape[3])
    return subst(t, [("PYCUDA_NX", _ff(grid.shape[1])), ("PYCUDA_NY", _ff(grid.shape[2])),
                     ("PYCUDA_NZ", _ff(grid.shape[3])), ("PYCUDA_NPTS", _ff(npts)),
                     ("PYCUDA_GRIDSTEP", _ff(grid.step))])


def targets():
    """[(output .so path, generated source text, launcher include, extra libs)]."""
    from oracle import ref_cases as rc
    qmtools = rc._qm()
    basis = qmtools.BasisSet(qmtools.BASIS_CCPVDZ)
    out = [(OUT / "utils.so", (REF_CUDA / "kernel_utils.cu").read_text(), "utils.inc", [])]
    for case, spec in rc.CASES.items():
        mol, grid = rc.case_inputs(case, basis)
        d = OUT / case
        for s in spec.get("density", []):
            out.append((d / f"density_s{s}.so", density_src(mol, s), "density.inc", []))
        if spec.get("hartree_gto"):
            out.append((d / "hartree_gto.so", hartree_src(mol, grid, True), "hartree.inc", []))
        if spec.get("hartree_iter"):
            out.append((d / "hartree_iter.so", hartree_src(mol, grid, False), "hartree.inc", []))
        if spec.get("fft"):
            out.append((d / "fft.so", fft_src(mol, grid, rc.FFT_PARAMS["sigma"], rc.FFT_PARAMS["cutoff"],
                                              qmtools.ANG2BOR), "fft.inc", ["-lcufft"]))
        if spec.get("vne"):
            out.append((d / "vne.so", vne_src(mol, grid, rc.VNE_PARAMS["adsorb"], rc.VNE_PARAMS["diff"]),
                        "vne.inc", []))
        for nl in spec.get("nn_ss", []):
            out.append((d / f"nn_ss_l{nl}.so", nn_ss_src(grid, nl), "nn_ss.inc", []))
        if spec.get("vne_classic"):
            out.append((d / "vne_classic.so", vne_classic_src(mol, grid, spec["vne_classic"]), "vne_classic.inc",
                        []))
    return out


def _compile(item, force):
    so, src, inc, libs = item
    text = src + f'\n#include "{inc}"\n'
    digest = hashlib.sha256((text + (LAUNCH / inc).read_text() + " ".join(FLAGS)).encode()).hexdigest()
    stamp = so.with_suffix(".so.sha256")
    if not force and so.exists() and stamp.exists() and stamp.read_text() == digest:
        return so, "cached"
    so.parent.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        cu = Path(td) / (so.stem + ".cu")
        cu.write_text(text)
        r = subprocess.run([NVCC, *FLAGS, str(cu), "-o", str(so), *libs], capture_output=True, text=True)
    if r.returncode != 0:
        return so, "FAILED:\n" + r.stderr[-3000:]
    stamp.write_text(digest)
    return so, "built"


def build_all(force=False):
    if not REF_CUDA.exists():
        return []
    items = targets()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        res = list(ex.map(lambda it: _compile(it, force), items))
    bad = [(s, m) for s, m in res if m.startswith("FAILED")]
    if bad:
        raise RuntimeError("reference build failed:\n" + "\n".join(f"{s}: {m}" for s, m in bad))
    return res


if __name__ == "__main__":
    for so, status in build_all(force="--force" in sys.argv):
        print(status, so)

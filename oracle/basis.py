"""Oracle: cc-pVDZ basis parsing and the per-function ALMO table (test infrastructure).

Follows the binary layout read by `BasisSet.__init__` (qmtools/qmtools.py:33-108)
and the ALMO construction of `Molecule.__init__` (qmtools/qmtools.py:150-171).
"""
import struct

import numpy as np

ANG2BOR = 1.8897259886          # qmtools/qmtools.py:17, kernel_common.h:1
MAXAOS = 15                     # qmtools/qmtools.py:19
MAXAOC = 20                     # qmtools/qmtools.py:20
# m order per L: s {0}; p {0,+1,-1}; d {0,+1,-1,+2,-2}  (qmtools/qmtools.py:52)
M_VALUES = {0: (0,), 1: (0, 1, -1), 2: (0, 1, -1, 2, -2)}


def read_basis_fp64(path):
    """Parse cc-pvdz.bin keeping FP64 values.

    Layout (little-endian, qmtools/qmtools.py:42-91): int32 natm; per element
    int32 Z, int32 nshells; per shell int32 L, int32 nc, float64 alpha[nc],
    float64 coeff[nc].  Returns {Z: [(L, alphas[nc], coeffs[nc]), ...]}.
    """
    with open(path, "rb") as f:
        data = f.read()
    off = 0

    def take(fmt):
        nonlocal off
        vals = struct.unpack_from("<" + fmt, data, off)
        off += struct.calcsize("<" + fmt)
        return vals

    (natm,) = take("i")
    out = {}
    for _ in range(natm):
        z, nsh = take("ii")
        shells = []
        for _ in range(nsh):
            L, nc = take("ii")
            a = np.array(take("d" * nc), dtype=np.float64)
            c = np.array(take("d" * nc), dtype=np.float64)
            shells.append((L, a, c))
        out[z] = shells
    if off != len(data):
        raise ValueError("trailing bytes in basis file")
    return out


def reference_tables(path):
    """The reference's padded FP32 tables (qmtools/qmtools.py:44-91).

    Returns dict with atomOffset[100], nshells[1500], Ls[1500],
    shellOffset[1500], alphas[30000] f32, coeffs[30000] f32.  Each shell has a
    MAXAOC=20 slot; unused slots are zero.
    """
    basis = read_basis_fp64(path)
    atomOffset = np.full(100, -1, dtype=np.int32)
    nshells = np.zeros(MAXAOS * 100, dtype=np.int32)
    shellOffset = np.zeros(MAXAOS * 100, dtype=np.int32)
    Ls = np.zeros(MAXAOS * 100, dtype=np.int32)
    alphas = np.zeros(MAXAOS * MAXAOC * 100, dtype=np.float32)
    coeffs = np.zeros(MAXAOS * MAXAOC * 100, dtype=np.float32)
    offset = 0
    orbcount = 0
    for z, shells in basis.items():  # file order (dict keeps insertion order)
        atomOffset[z] = orbcount
        nshells[z] = len(shells)
        for (L, a, c) in shells:
            Ls[orbcount] = L
            shellOffset[orbcount] = offset
            alphas[offset:offset + len(a)] = a.astype(np.float32)
            coeffs[offset:offset + len(c)] = c.astype(np.float32)
            orbcount += 1
            offset += MAXAOC
    return dict(atomOffset=atomOffset, nshells=nshells, shellOffset=shellOffset,
                Ls=Ls, alphas=alphas, coeffs=coeffs)


def almo_table(types, tables):
    """Per-basis-function [atom, L, m, shellOffset] int16 (qmtools/qmtools.py:150-171)."""
    rows = []
    for a, Z in enumerate(types):
        aos = tables["atomOffset"][Z]
        if aos < 0:
            raise KeyError(f"element Z={Z} not in basis")
        for s in range(tables["nshells"][Z]):
            L = int(tables["Ls"][aos + s])
            if L not in M_VALUES:
                raise IndexError(f"L={L} not supported")
            for m in M_VALUES[L]:
                rows.append((a, L, m, tables["shellOffset"][aos + s]))
    return np.array(rows, dtype=np.int16).reshape(-1, 4)


def shells_fp64(types, basis):
    """Shell list [(atom, L, alphas, coeffs, first_function)] in ALMO order, FP64."""
    out = []
    f = 0
    for a, Z in enumerate(types):
        for (L, al, co) in basis[int(Z)]:
            out.append((a, L, al, co, f))
            f += 2 * L + 1
    return out, f

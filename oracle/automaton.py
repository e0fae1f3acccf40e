"""Oracle (test infrastructure): the single-shot NN automaton in NumPy.

Restates gpu_automaton_nn_singleshot (kernel_nn_ss.cu:33-178) as driven by
AutomatonSingleShot.Evaluate (qmtools/automaton_nn_singleshot.py:78-183) in FP32 arithmetic
emulated with FP64 products (one rounding per fused multiply-add); tanh and 1/sqrt are the
correctly rounded FP64 functions, so results agree with the GPU to ~1e-6 relative, not bitwise.
"""
import numpy as np


def neighbour_order():
    """(dx, dy, dz, |d|_1) in the order of the kernel's `deltas` loop (kernel_nn_ss.cu:50-88):
    bits 0-1, 2-3, 4-5 of `deltas` give x, y, z steps (low bit: step, high bit: sign); codes of
    a signed zero step are skipped by bumping the loop variable."""
    out = []
    d = 1
    while d < 64:
        if (d & 3) == 2:
            d += 1
        if (d & 12) == 8:
            d += 4
        if (d & 48) == 32:
            d += 16

        def step(bits):
            s = 1 if d & bits[0] else 0
            return -s if d & bits[1] else s
        dx, dy, dz = step((1, 2)), step((4, 8)), step((16, 32))
        out.append((dx, dy, dz, abs(dx) + abs(dy) + abs(dz)))
        d += 1
    return out


def _f32(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32)


def _fma(a, b, c):
    return _f32(a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64))


def dna_size(nlayers):
    """AutomatonSingleShot.Random (qmtools/automaton_nn_singleshot.py:56-57)."""
    return 16 * 16 * nlayers + 16 * nlayers + (16 * 1 + 1) + 12


def nn_singleshot_grid(field1, shape, params, nlayers, gridstep):
    """field1: the pseudo-field (flat, x-fastest, shape = (nx, ny, nz)); params: the element's
    DNA (dna_size(nlayers) floats); gridstep: the grid step as the kernel source carries it.
    Returns the output grid (flat, x-fastest), before Evaluate's rescale to the nuclear charge."""
    nx, ny, nz = shape
    f = np.asarray(field1, dtype=np.float32).reshape(nz, ny, nx)
    w = np.zeros(dna_size(nlayers) + 2, dtype=np.float32)      # the kernel reads 2 past the end
    w[:dna_size(nlayers)] = np.asarray(params, dtype=np.float32)
    v1 = f
    fin = np.zeros_like(f)
    for dx, dy, dz, cnt in neighbour_order():
        v2 = np.roll(f, shift=(-dz, -dy, -dx), axis=(0, 1, 2))   # field at (x+dx, y+dy, z+dz), periodic
        inp = [v1, v2] + [np.full_like(f, w[k]) for k in range(14)]
        os_ = 14
        for _ in range(nlayers):
            out = []
            for _n in range(16):
                acc = np.zeros_like(f)
                for i in range(16):
                    acc = _fma(np.float32(w[os_]), inp[i], acc)
                    os_ += 1
                acc = _f32(acc.astype(np.float64) + np.float64(w[os_]))
                os_ += 1
                out.append(_f32(np.tanh(acc.astype(np.float64))))
            inp = out
        acc = np.zeros_like(f)
        for i in range(16):
            acc = _fma(np.float32(w[os_]), inp[i], acc)
            os_ += 1
        acc = _f32(acc.astype(np.float64) + np.float64(w[os_]))
        t = _f32(acc.astype(np.float64) * acc.astype(np.float64))
        factor = np.float32((1.0 / np.sqrt(np.float32(cnt))) / gridstep)
        fin = _fma(t, np.full_like(f, factor), fin)
    res = _f32((v1.astype(np.float64) * fin.astype(np.float64)).astype(np.float32).astype(np.float64)
               * 0.05234482976098482)
    return res.ravel()

"""CPU oracle for the QMTools grid hot path -- TEST INFRASTRUCTURE ONLY.

This package is a plain FP64 NumPy restatement of the reference's algorithms
(fullmetalfelix/QMTools-pycuda, `qmtools/qmtools.py` and `qmtools/cuda/*.cu`),
written from the reference's conventions, not from its code.  Every function
cites the reference file:line it follows.

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` may import this package, and only as the checker or as the timed
CPU baseline -- never as the thing measured or shipped.  The product path
(`qmtools-pycuda_b200/`) does not import it and fails loudly when its CUDA
library is missing.

Parity pin: the reference has no tests and no golden vectors.  The oracle is
pinned against outputs of the reference's own CUDA kernels, compiled from the
reference sources with the same PYCUDA_* substitutions the reference host
performs (`oracle/build_ref.py`) and run on a B200; those outputs are committed
as fixtures under `tests/golden/` together with the script that made them.
"""

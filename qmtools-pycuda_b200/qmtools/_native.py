"""ctypes binding of libqmtools_b200.so (the C ABI declared in include/qmtools_b200.h).

Loading the library needs no GPU; the first call that touches the device runs
`qmt_init`.  There is no CPU fallback: if the library is missing every entry point
raises `NativeUnavailable`.
"""
import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libqmtools_b200.so"

OK, BAD_ARG, OOM, NOT_CONVERGED, NAN, UNSUPPORTED_L, CUDA_ERR, NO_DEVICE = range(8)
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "NOT_CONVERGED", 4: "NAN",
                5: "UNSUPPORTED_L", 6: "CUDA_ERR", 7: "NO_DEVICE"}

PREC = {"fp64": 0, "fp32": 1, "tf32": 2, "tf32x3": 3, "bf16": 4, "bf16x3": 5, "fp16x3": 6}

_vp = C.c_void_p
_i = C.c_int
_f = C.c_float
_d = C.c_double
_i64 = C.c_int64
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)

# name -> argtypes (every function returns an int status, except those in OTHER)
SIGNATURES = {
    "qmt_init": [_i],
    "qmt_mol_create": [_i, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp, C.POINTER(_vp)],
    "qmt_mol_reset": [_vp, _i, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp],
    "qmt_mol_set_coords": [_vp, _vp, _vp],
    "qmt_mol_set_dm": [_vp, _vp, _vp],
    "qmt_mol_destroy": [_vp],
    "qmt_mol_trace_ps": [_vp, _pd, _vp],
    "qmt_density": [_vp, _i, _i, _i, _f, _f, _f, _f, _i, _i, _i, _vp, _pd, _vp],
    "qmt_set_density_path": [_i],
    "qmt_density_factor_rank": [_vp, _pi, _vp],
    "qmt_batch_create": [_i, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, C.POINTER(_vp)],
    "qmt_batch_density": [_vp, _i, _i, _vp],
    "qmt_batch_sums": [_vp, _pd, _vp],
    "qmt_batch_destroy": [_vp],
    "qmt_set_wait_limit_ns": [C.c_uint64],
    "qmt_hartree_gto": [_vp, _i, _i, _i, _f, _f, _f, _f, _vp, _vp],
    "qmt_hartree_gto_points": [_vp, _i, _vp, _vp, _vp],
    "qmt_hartree_gto_boundary": [_vp, _i, _i, _i, _f, _f, _f, _f, _vp, _vp],
    "qmt_set_gto_precision": [_i],
    "qmt_jacobi": [_i, _i, _i, _f, _vp, _vp, _vp, _i, _i, _d, _pi, _pd, _vp],
    "qmt_jacobi_dirichlet": [_i, _i, _i, _f, _vp, _vp, _vp, _i, _i, _d, _pi, _pd, _vp],
    "qmt_set_jacobi_path": [_i],
    "qmt_fft_poisson": [_vp, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _vp, _vp, _vp],
    "qmt_fft_poisson_padded": [_vp, _i, _i, _i, _f, _f, _f, _f, _f, _f, _i, _i, _i, _vp, _vp, _vp],
    "qmt_grid_total": [_vp, _i64, _pd, _vp],
    "qmt_grid_total_noalloc": [_vp, _i64, _pd, _vp],
    "qmt_grid_scale": [_vp, _i64, _f, _vp],
    "qmt_grid_diff": [_vp, _vp, _i64, _i, _pd, _vp],
    "qmt_grid_errors": [_vp, _vp, _i64, _pd, _vp],
    "qmt_density_seed": [_vp, _i, _i, _i, _f, _f, _f, _f, _vp, _vp],
    "qmt_vne_point": [_vp, _i, _i, _i, _f, _f, _f, _f, _i, _vp, _vp],
    "qmt_vne_classic": [_vp, _i, _i, _i, _f, _f, _f, _f, _i, _vp, _vp],
    "qmt_vne_pseudo": [_vp, _i, _i, _i, _f, _f, _f, _f, _f, _f, _d, _i, _vp, _vp, _pi, _vp],
    "qmt_nn_singleshot": [_i, _i, _i, _d, _vp, _vp, _vp, _i, _i, _vp],
}
OTHER = {"qmt_last_error": ([], C.c_char_p), "qmt_abi_version": ([], C.c_int),
         "qmt_launch_count": ([], C.c_uint64), "qmt_batch_fused_count": ([_vp], C.c_int),
         "qmt_batch_factored_count": ([_vp], C.c_int)}


class NativeUnavailable(RuntimeError):
    """The CUDA library is not built or cannot be loaded."""


class QMToolsError(RuntimeError):
    def __init__(self, status, fn, msg):
        self.status = status
        super().__init__(f"{fn}: {STATUS_NAMES.get(status, status)}: {msg}")


class NotConverged(QMToolsError):
    pass


_lib = None
_lock = threading.Lock()
_inited = set()


def load():
    """Load the shared library (no device needed) and bind every entry point."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = os.environ.get("QMTOOLS_B200_LIB", str(LIB_PATH))
        if not Path(path).exists():
            raise NativeUnavailable(
                f"{path} is missing: build it with `python qmtools-pycuda_b200/build.py`")
        lib = C.CDLL(path)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        for name, (args, res) in OTHER.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def check(status, fn):
    if status == OK:
        return
    msg = load().qmt_last_error().decode(errors="replace")
    if status == NOT_CONVERGED:
        raise NotConverged(status, fn, msg)
    raise QMToolsError(status, fn, msg)


def call(name, *args):
    lib = load()
    check(getattr(lib, name)(*args), name)


def ensure_device(device=None):
    """Initialise the library on the current torch device (once per device and thread)."""
    import torch
    if not torch.cuda.is_available():
        raise QMToolsError(NO_DEVICE, "qmt_init", "no CUDA device visible")
    dev = torch.cuda.current_device() if device is None else device
    key = (threading.get_ident(), dev)
    if key not in _inited:
        call("qmt_init", dev)
        _inited.add(key)
    return dev


def stream_handle():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)

"""ctypes binding of ``libamg_b200.so`` (the C ABI declared in include/amg_b200.h).

The shared library is built in-tree (``amjax_b200/csrc/build.py``).  There is no CPU
fallback: every compute entry point raises when the library or a CUDA device is missing.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libamg_b200.so"

# enums (include/amg_b200.h)
AMG_OK = 0
STATUS_NAMES = {0: "AMG_OK", 1: "AMG_ERR_INVALID_ARG", 2: "AMG_ERR_UNSUPPORTED", 3: "AMG_ERR_CUDA",
                4: "AMG_ERR_TIMEOUT", 5: "AMG_ERR_BAD_MATRIX"}
CYCLES = {"V": 0, "W": 1, "F": 2}
PREC_F64, PREC_F32, PREC_MIXED, PREC_MIXED_F64CG = 0, 1, 2, 3
SMOOTH_NONE, SMOOTH_JACOBI = 0, 1
COARSE_KINDS = {"pinv": 0, "lu": 1, "qr": 2, "jacobi": 3}


class amg_csr(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("nnz", C.c_int64),
                ("rowptr", C.c_void_p), ("col", C.c_void_p), ("val64", C.c_void_p), ("val32", C.c_void_p)]


class amg_smoother(C.Structure):
    _fields_ = [("kind", C.c_int32), ("iterations", C.c_int32), ("omega", C.c_double)]


class amg_level_desc(C.Structure):
    _fields_ = [("A", amg_csr), ("P", amg_csr), ("R", amg_csr), ("dinv64", C.c_void_p),
                ("dinv32", C.c_void_p), ("pre", amg_smoother), ("post", amg_smoother)]


class amg_coarse_desc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n", C.c_int32), ("m0_64", C.c_void_p), ("m0_32", C.c_void_p),
                ("m1_64", C.c_void_p), ("m1_32", C.c_void_p), ("perm", C.c_void_p),
                ("iterations", C.c_int32), ("omega", C.c_double)]


# name -> (restype, argtypes); mirrors include/amg_b200.h exactly (tests check both ways)
SIGNATURES = {
    "amg_hierarchy_create": (C.c_int, [C.POINTER(amg_level_desc), C.c_int32, C.POINTER(amg_coarse_desc),
                                       C.POINTER(C.c_void_p)]),
    "amg_hierarchy_destroy": (C.c_int, [C.c_void_p]),
    "amg_solve": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_int32,
                            C.c_int32, C.c_int32, C.POINTER(amg_csr), C.POINTER(C.c_int32),
                            C.POINTER(C.c_double), C.c_void_p]),
    "amg_precondition": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_void_p]),
    "amg_pcg": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_double,
                          C.c_int32, C.c_int32, C.c_int32, C.POINTER(amg_csr), C.POINTER(C.c_int32),
                          C.POINTER(C.c_double), C.c_void_p]),
    "amg_pcg_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double,
                               C.c_double, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                               C.POINTER(C.c_double), C.c_void_p]),
    "amg_adjoint": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_double,
                              C.c_double, C.c_int32, C.c_int32, C.c_int32, C.POINTER(amg_csr), C.POINTER(amg_csr),
                              C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_void_p]),
    "amg_pcg_batch": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.POINTER(C.c_int32), C.c_double, C.c_double, C.c_int32,
                                C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_void_p]),
    "amg_jacobi": (C.c_int, [C.POINTER(amg_csr), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_int32, C.c_int32, C.c_double, C.c_void_p]),
    "amg_jacobi_noalloc": (C.c_int, [C.POINTER(amg_csr), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p]),
    "amg_spmv": (C.c_int, [C.POINTER(amg_csr), C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "amg_inverse_diagonal": (C.c_int, [C.POINTER(amg_csr), C.c_int32, C.c_void_p, C.c_void_p]),
    "amg_sampled_outer": (C.c_int, [C.POINTER(amg_csr), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                    C.c_void_p]),
    "amg_time_pcg_ops": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.c_char_p, C.c_int32,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "amg_kernel_launch_count": (C.c_int64, []),
    "amg_last_error": (C.c_char_p, []),
    "amg_version": (C.c_char_p, []),
}

_lib = None


class NativeError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib_path() -> Path:
    return _LIB_PATH


def load(require_cuda: bool = True):
    """Load the shared library (once).  Raises if it is missing, or (by default) if no
    CUDA device is present: the solve phase has no CPU path."""
    global _lib
    if require_cuda:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("amjax_b200 needs a CUDA (sm_100a) device; none is available")
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(f"{_LIB_PATH} is missing: build it with `python -m amjax_b200.csrc.build`")
    lib = C.CDLL(os.fspath(_LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != AMG_OK:
        msg = _lib.amg_last_error().decode() if _lib is not None else ""
        raise NativeError(status, msg)


def call(name, *args):
    lib = load()
    check(getattr(lib, name)(*args))


def time_pcg_ops(handle, k, reps=5, stream=None):
    """Per-kernel timing of one mixed-precision PCG step's fine-level kernels
    (``amg_time_pcg_ops``): a list of (name, microseconds per launch, algorithmic bytes)."""
    m, width = 16, 64
    names = C.create_string_buffer(m * width)
    us = (C.c_double * m)()
    by = (C.c_double * m)()
    n = C.c_int32()
    call("amg_time_pcg_ops", handle, int(k), int(reps), stream_ptr(stream), m, names, width, us, by, C.byref(n))
    raw = names.raw
    return [(raw[i * width:(i + 1) * width].split(b"\0", 1)[0].decode(), us[i], by[i]) for i in range(n.value)]


def kernel_launch_count() -> int:
    """Kernels this library launched so far in this process (read from the device)."""
    return int(load().amg_kernel_launch_count())


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def ptr(t):
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else C.c_void_p(t.data_ptr())

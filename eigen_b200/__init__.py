"""eigen_b200 -- B200 (sm_100a) drop-in for Eigen's dense matrix-matrix product.

The product is the C-ABI shared library ``lib/libeigen_b200.so`` (built by
``python -m eigen_b200.build``).  It exports the Fortran BLAS symbols ``sgemm_`` /
``dgemm_`` (and ILP64 ``_64_`` variants) that Eigen binds for its ``operator*``
under ``EIGEN_USE_BLAS`` (Eigen/src/Core/products/GeneralMatrixMatrix_BLAS.h:53-118),
plus ``eb2_*`` extension calls.  This module is a thin ctypes mirror of that ABI
for Python callers, tests and benchmarks: the call ``dgemm(...)`` takes the same
arguments, in the same order and with the same meaning, as Eigen's
``dgemm_`` (blas/level3_impl.h:12-96), and argument errors surface the same way,
through ``xerbla_``.

Nothing here computes a product: if the library is missing, loading fails.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "lib" / "libeigen_b200.so"
HEADER_PATH = _PKG.parent / "include" / "eigen_b200" / "blas.h"

EB2_OK = 0
EB2_ERR_CUDA = -1
EB2_ERR_ALLOC = -2
EB2_ERR_TIMEOUT = -3
EB2_ERR_ARG = -4
EB2_ERR_NO_DEVICE = -5
EB2_ERR_ACCURACY = -6

METHOD_AUTO = 0
METHOD_NATIVE = 1
METHOD_EMULATED = 2
METHOD_CRT = 3

_lib = None


class CallInfo(ctypes.Structure):
    _fields_ = [
        ("dtype", ctypes.c_int),
        ("method", ctypes.c_int),
        ("slices", ctypes.c_int),
        ("tile_n", ctypes.c_int),
        ("escalations", ctypes.c_int),
        ("nonfinite", ctypes.c_int),
        ("staged", ctypes.c_int),
        ("err_estimate", ctypes.c_double),
        ("kernel_ms", ctypes.c_double),
        ("gemm_kernel_ms", ctypes.c_double),
        ("launches", ctypes.c_int),
        ("spread", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["dtype"] = chr(self.dtype) if self.dtype else ""
        return d


class GemmProblem(ctypes.Structure):
    """eb2_gemm_problem: one product of a grouped launch (device pointers)."""

    _fields_ = [
        ("transa", ctypes.c_char),
        ("transb", ctypes.c_char),
        ("m", ctypes.c_int64),
        ("n", ctypes.c_int64),
        ("k", ctypes.c_int64),
        ("alpha", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("a", ctypes.c_void_p),
        ("lda", ctypes.c_int64),
        ("b", ctypes.c_void_p),
        ("ldb", ctypes.c_int64),
        ("c", ctypes.c_void_p),
        ("ldc", ctypes.c_int64),
    ]


def load(path: str | os.PathLike | None = None, mode: int = ctypes.RTLD_GLOBAL) -> ctypes.CDLL:
    """Load libeigen_b200.so (once) and declare its signatures.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python -m eigen_b200.build`")
    lib = ctypes.CDLL(str(p), mode=mode)
    c_int_p = ctypes.POINTER(ctypes.c_int)
    c_i64_p = ctypes.POINTER(ctypes.c_int64)
    vp = ctypes.c_void_p
    for name, ip in (("dgemm_", c_int_p), ("sgemm_", c_int_p), ("dgemm_64_", c_i64_p), ("sgemm_64_", c_i64_p)):
        f = getattr(lib, name)
        f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ip, ip, ip, vp, vp, ip, vp, ip, vp, vp, ip]
        f.restype = None
    lib.eb2_set_dgemm_method.argtypes = [ctypes.c_int]
    lib.eb2_set_sgemm_method.argtypes = [ctypes.c_int]
    lib.eb2_set_dgemm_slices.argtypes = [ctypes.c_int]
    lib.eb2_set_dgemm_moduli.argtypes = [ctypes.c_int]
    lib.eb2_set_dgemm_tolerance.argtypes = [ctypes.c_double]
    lib.eb2_set_tile_n.argtypes = [ctypes.c_int]
    lib.eb2_set_sgemm_pieces.argtypes = [ctypes.c_int]
    lib.eb2_set_timing.argtypes = [ctypes.c_int]
    lib.eb2_set_slice_tuning.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.eb2_set_wait_limit_ns.argtypes = [ctypes.c_longlong]
    lib.eb2_last_error_string.restype = ctypes.c_char_p
    lib.eb2_last_call_info.argtypes = [ctypes.POINTER(CallInfo)]
    lib.eb2_version.restype = ctypes.c_char_p
    lib.eb2_dgemm_device.argtypes = [ctypes.c_char, ctypes.c_char, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                     ctypes.c_double, vp, ctypes.c_int64, vp, ctypes.c_int64, ctypes.c_double, vp,
                                     ctypes.c_int64, vp, ctypes.c_int]
    lib.eb2_sgemm_device.argtypes = [ctypes.c_char, ctypes.c_char, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                     ctypes.c_float, vp, ctypes.c_int64, vp, ctypes.c_int64, ctypes.c_float, vp,
                                     ctypes.c_int64, vp]
    lib.eb2_dgemm_device_noalloc.argtypes = [ctypes.c_char, ctypes.c_char, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int64, ctypes.c_double, vp, ctypes.c_int64, vp, ctypes.c_int64,
                                             ctypes.c_double, vp, ctypes.c_int64, vp]
    pp = ctypes.POINTER(GemmProblem)
    lib.eb2_grouped_plan_create.argtypes = [ctypes.c_char, ctypes.c_int64, pp, ctypes.POINTER(ctypes.c_void_p)]
    lib.eb2_grouped_plan_execute.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.eb2_grouped_plan_destroy.argtypes = [ctypes.c_void_p]
    lib.eb2_gemm_grouped.argtypes = [ctypes.c_char, ctypes.c_int64, pp, ctypes.c_void_p]
    lib.eb2_gemm_each.argtypes = [ctypes.c_char, ctypes.c_int64, pp, ctypes.c_void_p]
    lib.eb2_set_grouped_classes.argtypes = [ctypes.c_int, ctypes.c_int]
    fp = ctypes.POINTER(ctypes.c_float)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.eb2_picker_set_weights.argtypes = [vp, ctypes.c_int]
    lib.eb2_picker_features.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_char, ctypes.c_double,
                                        ctypes.c_int64, ctypes.c_double, vp]
    lib.eb2_picker_forward_host.argtypes = [vp, vp, vp]
    lib.eb2_picker_predict.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_char, ctypes.c_double,
                                       ctypes.c_int64, ctypes.c_double, ip, ip]
    lib.eb2_set_config.argtypes = [ctypes.c_int]
    lib.eb2_mlp_forward.argtypes = [vp, vp, ctypes.c_int, vp, vp]
    lib.eb2_mlp_backward.argtypes = [vp, vp, vp, vp, ctypes.c_int, vp, vp, vp]
    lib.eb2_mlp_adam.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_float, vp]
    _lib = lib
    return lib


def _ptr(x) -> int | None:
    """Address of a numpy array, torch tensor, or a raw integer address."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    if hasattr(x, "ctypes"):
        return int(x.ctypes.data)
    raise TypeError(f"cannot take the address of {type(x)!r}")


def _gemm(name, ctype, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64=False):
    lib = load()
    it = ctypes.c_int64 if ilp64 else ctypes.c_int
    f = getattr(lib, name + ("_64_" if ilp64 else "_"))
    ta = transa.encode() if isinstance(transa, str) else bytes(transa)
    tb = transb.encode() if isinstance(transb, str) else bytes(transb)
    al, be = ctype(alpha), ctype(beta)
    args = [it(v) for v in (m, n, k, lda, ldb, ldc)]
    f(ta, tb, ctypes.byref(args[0]), ctypes.byref(args[1]), ctypes.byref(args[2]), ctypes.cast(ctypes.byref(al), ctypes.c_void_p),
      _ptr(a), ctypes.byref(args[3]), _ptr(b), ctypes.byref(args[4]), ctypes.cast(ctypes.byref(be), ctypes.c_void_p), _ptr(c),
      ctypes.byref(args[5]))


def dgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64=False):
    """C := alpha*op(A)*op(B) + beta*C through the exported ``dgemm_`` (column-major).

    a, b, c: numpy arrays / torch tensors (host or CUDA) or raw addresses."""
    _gemm("dgemm", ctypes.c_double, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64)


def sgemm(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64=False):
    """Single-precision counterpart through ``sgemm_``."""
    _gemm("sgemm", ctypes.c_float, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64)


def complex_gemm(dtype, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, ilp64=False):
    """C := alpha*op(A)*op(B) + beta*C through ``zgemm_`` (dtype "z") or ``cgemm_`` ("c"):
    alpha, beta Python complex numbers; a, b, c complex numpy arrays / torch tensors (host or
    CUDA, column-major) or raw addresses; op 'N', 'T' or 'C' (conjugate transpose)."""
    lib = load()
    real = ctypes.c_double if dtype == "z" else ctypes.c_float
    it = ctypes.c_int64 if ilp64 else ctypes.c_int
    al = (real * 2)(complex(alpha).real, complex(alpha).imag)
    be = (real * 2)(complex(beta).real, complex(beta).imag)
    dims = [it(v) for v in (m, n, k, lda, ldb, ldc)]
    f = getattr(lib, ("zgemm" if dtype == "z" else "cgemm") + ("_64_" if ilp64 else "_"))
    f.restype = None
    enc = lambda x: x.encode() if isinstance(x, str) else bytes(x)
    f(ctypes.c_char_p(enc(transa)), ctypes.c_char_p(enc(transb)), ctypes.byref(dims[0]), ctypes.byref(dims[1]),
      ctypes.byref(dims[2]), ctypes.cast(al, ctypes.c_void_p), ctypes.c_void_p(_ptr(a)), ctypes.byref(dims[3]),
      ctypes.c_void_p(_ptr(b)), ctypes.byref(dims[4]), ctypes.cast(be, ctypes.c_void_p), ctypes.c_void_p(_ptr(c)),
      ctypes.byref(dims[5]))


# Argument kinds of the other exported level-3 routines, in the order of their Fortran
# signatures: c = character, i = dimension, s = scalar, a = array.
LEVEL3_SIGNATURES = {
    "gemmtr": "cccii" "s" "ai" "ai" "s" "ai",  # uplo transa transb n k alpha a lda b ldb beta c ldc
    "syrk": "ccii" "s" "ai" "s" "ai",          # uplo trans n k alpha a lda beta c ldc
    "syr2k": "ccii" "s" "ai" "ai" "s" "ai",    # uplo trans n k alpha a lda b ldb beta c ldc
    "symm": "ccii" "s" "ai" "ai" "s" "ai",     # side uplo m n alpha a lda b ldb beta c ldc
    "trmm": "ccccii" "s" "ai" "ai",            # side uplo transa diag m n alpha a lda b ldb
    "trsm": "ccccii" "s" "ai" "ai",            # side uplo transa diag m n alpha a lda b ldb
    "hemm": "ccii" "s" "ai" "ai" "s" "ai",     # side uplo m n alpha a lda b ldb beta c ldc (complex)
}


def level3(name: str, *args, ilp64: bool = False) -> None:
    """Call an exported level-3 routine by its BLAS name (``dsyrk``, ``strsm``, ``dgemmtr``,
    ``ztrsm``, ``chemm`` ...) with its Fortran argument list in order (see
    ``LEVEL3_SIGNATURES``): characters as str, dimensions and scalars as Python numbers (complex
    for the z / c routines), matrices as numpy arrays / torch tensors (host or CUDA) or raw
    addresses.  ``ilp64`` calls the ``_64_`` symbol."""
    lib = load()
    dtype, routine = name[0], name[1:]
    kinds = LEVEL3_SIGNATURES[routine]
    if dtype not in "dszc" or len(args) != len(kinds):
        raise ValueError(f"{name}: expected {len(kinds)} arguments")
    ctype = ctypes.c_double if dtype in "dz" else ctypes.c_float
    itype = ctypes.c_int64 if ilp64 else ctypes.c_int
    out, keep = [], []
    for kind, v in zip(kinds, args):
        if kind == "c":
            out.append(ctypes.c_char_p(v.encode() if isinstance(v, str) else bytes(v)))
            continue
        if kind == "a":
            out.append(ctypes.c_void_p(_ptr(v)))
            continue
        if kind == "s" and dtype in "zc":
            x = (ctype * 2)(complex(v).real, complex(v).imag)
        else:
            x = itype(v) if kind == "i" else ctype(v)
        keep.append(x)
        out.append(ctypes.cast(ctypes.byref(x), ctypes.c_void_p))
    f = getattr(lib, name + ("_64_" if ilp64 else "_"))
    f.restype = None
    f(*out)


def dgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=0, check_accuracy=True) -> int:
    """Stream-ordered DGEMM on device pointers (``eb2_dgemm_device``); returns an EB2_* status."""
    return load().eb2_dgemm_device(transa.encode(), transb.encode(), m, n, k, alpha, _ptr(a), lda, _ptr(b), ldb, beta,
                                   _ptr(c), ldc, stream or None, 1 if check_accuracy else 0)


def sgemm_device(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=0) -> int:
    return load().eb2_sgemm_device(transa.encode(), transb.encode(), m, n, k, alpha, _ptr(a), lda, _ptr(b), ldb, beta,
                                   _ptr(c), ldc, stream or None)


def dgemm_device_noalloc(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, stream=0) -> int:
    """eb2_dgemm_device_noalloc: the CRT-form DGEMM with its scratch in a fixed device array
    (no device allocation; for callers whose memory is owned by another allocator)."""
    return load().eb2_dgemm_device_noalloc(transa.encode(), transb.encode(), m, n, k, alpha, _ptr(a), lda, _ptr(b),
                                           ldb, beta, _ptr(c), ldc, stream or None)


def set_dgemm_method(method: int) -> int:
    return load().eb2_set_dgemm_method(method)


def set_sgemm_method(method: int) -> int:
    return load().eb2_set_sgemm_method(method)


def set_dgemm_slices(slices: int) -> int:
    return load().eb2_set_dgemm_slices(slices)


def set_dgemm_moduli(moduli: int) -> int:
    return load().eb2_set_dgemm_moduli(moduli)


def set_sgemm_pieces(pieces: int) -> int:
    return load().eb2_set_sgemm_pieces(pieces)


def set_dgemm_tolerance(tol: float) -> int:
    return load().eb2_set_dgemm_tolerance(tol)


def set_tile_n(tile_n: int) -> int:
    return load().eb2_set_tile_n(tile_n)


def set_slice_tuning(group_m: int, prefetch: int) -> int:
    return load().eb2_set_slice_tuning(group_m, prefetch)


def set_wait_limit_ns(ns: int) -> int:
    """Wall-time bound (ns) of the tcgen05 GEMM's pipeline waits; 0 = the default (2 s)."""
    return load().eb2_set_wait_limit_ns(int(ns))


def set_config(config: int) -> int:
    """Force a configuration class of the picker's first head (-1: automatic); see blas.h."""
    return load().eb2_set_config(int(config))


def set_picker(weights) -> int:
    """Install picker weights (a float32 array of eb2_mlp_param_count() entries) or None."""
    lib = load()
    if weights is None:
        return lib.eb2_picker_set_weights(None, 0)
    import numpy as np

    w = np.ascontiguousarray(weights, dtype=np.float32)
    return lib.eb2_picker_set_weights(w.ctypes.data_as(ctypes.c_void_p), int(w.size))


def set_timing(on: bool) -> int:
    return load().eb2_set_timing(1 if on else 0)


def last_error() -> tuple[int, str]:
    lib = load()
    return lib.eb2_last_error(), lib.eb2_last_error_string().decode()


def clear_error() -> None:
    load().eb2_clear_error()


def routine_calls(name: str) -> int:
    """Calls of the named BLAS routine (e.g. "dtrsm") that reached the device in this process."""
    f = load().eb2_routine_calls
    f.argtypes = [ctypes.c_char_p]
    f.restype = ctypes.c_longlong
    return int(f(name.encode()))


def last_call_info() -> dict:
    """eb2_last_call_info plus eb2_last_call_config (keys "config" and "splits")."""
    lib = load()
    ci = CallInfo()
    lib.eb2_last_call_info(ctypes.byref(ci))
    d = ci.as_dict()
    cfg, splits = ctypes.c_int(), ctypes.c_int()
    lib.eb2_last_call_config(ctypes.byref(cfg), ctypes.byref(splits))
    d["config"], d["splits"] = cfg.value, splits.value
    return d


def problems_array(problems) -> "ctypes.Array":
    """Build a GemmProblem array from dicts with keys transa, transb, m, n, k, alpha, beta,
    a, lda, b, ldb, c, ldc (a/b/c: CUDA tensors or device addresses)."""
    arr = (GemmProblem * len(problems))()
    for i, p in enumerate(problems):
        arr[i] = GemmProblem(p.get("transa", "N").encode(), p.get("transb", "N").encode(), p["m"], p["n"], p["k"],
                             p.get("alpha", 1.0), p.get("beta", 0.0), _ptr(p["a"]), p["lda"], _ptr(p["b"]), p["ldb"],
                             _ptr(p["c"]), p["ldc"])
    return arr


class GroupedPlan:
    """A captured grouped launch (eb2_grouped_plan_*); execute() replays it."""

    def __init__(self, dtype: str, problems):
        self._arr = problems if isinstance(problems, ctypes.Array) else problems_array(problems)
        self._h = ctypes.c_void_p()
        rc = load().eb2_grouped_plan_create(dtype.encode(), len(self._arr), self._arr, ctypes.byref(self._h))
        if rc != EB2_OK:
            raise RuntimeError(f"eb2_grouped_plan_create failed: {rc} {last_error()[1]}")

    def execute(self, stream=0) -> int:
        return load().eb2_grouped_plan_execute(self._h, stream or None)

    def close(self):
        if self._h:
            load().eb2_grouped_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_grouped(dtype: str, problems, stream=0) -> int:
    arr = problems if isinstance(problems, ctypes.Array) else problems_array(problems)
    return load().eb2_gemm_grouped(dtype.encode(), len(arr), arr, stream or None)


def set_grouped_classes(small_max: int = 8, mid_max: int = 16) -> int:
    """Size classes of later grouped plans (eb2_set_grouped_classes)."""
    return load().eb2_set_grouped_classes(small_max, mid_max)


def gemm_each(dtype: str, problems, stream=0) -> int:
    """One launch per product of the same arithmetic (the per-call baseline of the grouped path)."""
    arr = problems if isinstance(problems, ctypes.Array) else problems_array(problems)
    return load().eb2_gemm_each(dtype.encode(), len(arr), arr, stream or None)


def version() -> str:
    return load().eb2_version().decode()

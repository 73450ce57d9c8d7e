"""ctypes binding of ``libfennol_b200.so`` (C ABI in ``include/fennol_b200.h``).

The library is loaded from the package's ``lib/`` folder.  There is no
fallback: if the library is missing or fails to load, every call raises
:class:`LibraryError`.
"""

from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path
from typing import Optional

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libfennol_b200.so"
HEADER = PKG.parent / "include" / "fennol_b200.h"

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_UNSUPPORTED = -3
ERR_WORKSPACE = -4
ERR_STATIC_LIMIT = -5

STATUS_WORDS = 9
ST_NBR_OVERFLOW, ST_NBR_MAXCOUNT, ST_FILTER_OVERFLOW, ST_FILTER_MAXCOUNT = 0, 1, 2, 3
ST_ANG_OVERFLOW, ST_ANG_MAXCOUNT, ST_CELL_OVERFLOW, ST_REBUILD_COUNT = 4, 5, 6, 7
ST_NONFINITE = 8

PBC_NONE, PBC_MINIMUM_IMAGE, PBC_GENERAL = 0, 1, 2
MAX_ANGULAR_NEIGHBORS = 256

AEV_F32, AEV_BF16, AEV_BF16X2, AEV_F16X2 = 0, 1, 2, 3
MLP_FP32, MLP_BF16, MLP_BF16X2, MLP_BF16X3, MLP_F16X3X1, MLP_F16X3X2 = 0, 1, 2, 3, 4, 5
PRECISIONS = {"fp32": MLP_FP32, "bf16": MLP_BF16, "bf16x2": MLP_BF16X2, "bf16x3": MLP_BF16X3,
              "f16x3x1": MLP_F16X3X1, "f16x3x2": MLP_F16X3X2}
F16_FORMS = (MLP_F16X3X1, MLP_F16X3X2)

_ERRNAMES = {ERR_INVALID: "invalid argument", ERR_CUDA: "CUDA launch failure",
             ERR_UNSUPPORTED: "unsupported parameters", ERR_WORKSPACE: "workspace too small",
             ERR_STATIC_LIMIT: "input larger than the fixed in-library scratch"}


class LibraryError(RuntimeError):
    pass


class FennolError(RuntimeError):
    def __init__(self, fn: str, code: int):
        super().__init__(f"{fn} failed: {code} ({_ERRNAMES.get(code, 'unknown')})")
        self.code = code


class NonFiniteError(FloatingPointError):
    """A device check found a NaN or an infinity (status word ST_NONFINITE)."""


class KernelTimeout(RuntimeError):
    """A bounded wait inside the tensor-core MLP ran out (its error word was set)."""


class AEVParams(C.Structure):
    _fields_ = [("num_species", C.c_int), ("radial_divisions", C.c_int),
                ("angular_divisions", C.c_int), ("angle_sections", C.c_int),
                ("radial_cutoff", C.c_double), ("angular_cutoff", C.c_double),
                ("radial_eta", C.c_float), ("angular_eta", C.c_float), ("zeta", C.c_float),
                ("radial_start", C.c_float), ("angular_start", C.c_float)]


class MLPWeights(C.Structure):
    _fields_ = [("n_models", C.c_int), ("n_species", C.c_int), ("dims", C.c_int * 5),
                ("celu_alpha", C.c_float),
                ("w32", C.c_void_p * 4), ("b32", C.c_void_p * 4),
                ("wt_hi", C.c_void_p * 4), ("wt_lo", C.c_void_p * 4),
                ("w_hi", C.c_void_p * 4), ("w_lo", C.c_void_p * 4),
                ("f16_scale", C.c_void_p)]


class NetTrain(C.Structure):
    _fields_ = [("n_species", C.c_int), ("dims", C.c_int * 5), ("celu_alpha", C.c_float),
                ("is_double", C.c_int),
                ("w", (C.c_void_p * 8) * 4), ("b", (C.c_void_p * 8) * 4),
                ("gw", (C.c_void_p * 8) * 4), ("gb", (C.c_void_p * 8) * 4)]


P = C.c_void_p
I = C.c_int
D = C.c_double
F = C.c_float
SZ = C.c_size_t
ULL = C.c_ulonglong

_SIGNATURES = {
    "fennol_version": (C.c_char_p, []),
    "fennol_graph_plan": (I, [I, P, P, D, P, P]),
    "fennol_graph_workspace_bytes": (SZ, [I, I]),
    "fennol_graph_build": (I, [P, I, P, I, P, P, P, P, P, P, I, D, I, P, P, P, P, P, SZ, P, P]),
    "fennol_graph_build_noalloc": (I, [P, I, P, I, P, P, P, P, P, P, I, D, I, P, P, P, P, P, P]),
    "fennol_graph_noalloc_limits": (I, [P, P, P]),
    "fennol_graph_filter": (I, [P, I, P, P, P, P, P, I, D, I, P, P, P, P, P]),
    "fennol_aev_length": (I, [C.POINTER(AEVParams)]),
    "fennol_pack_atoms": (I, [P, P, I, P, P]),
    "fennol_aev_forward": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, I, P, P, I, P, P]),
    "fennol_aev_backward": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, P, I, P, P, P]),
    "fennol_aev_backward_virial": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, P, I, P, P, P, P]),
    "fennol_aev_stage_bytes": (SZ, [I, I]),
    "fennol_aev_forward_staged": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, I, P, P, I, P, SZ, P, P]),
    "fennol_aev_backward_staged": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, P, I, P, P, P, P]),
    "fennol_virial_reduce": (I, [P, I, P, I, D, P, P]),
    "fennol_aev_tangent": (I, [P, I, P, P, P, P, P, I, C.POINTER(AEVParams), P, P, P, I, P, P]),
    "fennol_mlp_workspace_bytes": (SZ, [I, I, I, C.POINTER(MLPWeights)]),
    "fennol_mlp_energy_grad": (I, [I, I, I, P, P, C.POINTER(MLPWeights), P, P, P, P, P, SZ, P]),
    "fennol_mlp_energy_grad_active": (I, [I, I, I, P, P, C.POINTER(MLPWeights), P, P, ULL, P, P, P, SZ, P]),
    "fennol_aev_active_chunks": (ULL, [C.POINTER(AEVParams), C.c_uint]),
    "fennol_energy_workspace_bytes": (SZ, [I, I]),
    "fennol_energy_reduce": (I, [P, P, I, P, I, D, P, P, P, SZ, P]),
    "fennol_forces_finalize": (I, [P, I, F, P, P]),
    "fennol_md_step": (I, [I, D, P, P, P, P, D, D, P, ULL, P, P, P, P, P, D, P, P]),
    "fennol_md_step_systems": (I, [I, I, D, P, P, P, P, D, D, P, P, P, P, P, P, P, P, P, D, P, P]),
    "fennol_md_mark_rebuilt": (I, [I, P, P, P, P]),
    "fennol_md_kinetic": (I, [I, P, P, P, P]),
    "fennol_check_finite": (I, [I, P, P, P, P, P]),
    "fennol_net_loss_grad_workspace_bytes": (SZ, [C.POINTER(NetTrain), P]),
    "fennol_net_loss_grad": (I, [C.POINTER(NetTrain), P, P, P, P, I, P, P, SZ, P]),
    "fennol_mlp_wait_limit": (I, [D]),
    "fennol_mlp_inject_stall": (I, [I]),
    "fennol_capture_if_begin": (I, [P, P, P]),
    "fennol_capture_if_end": (I, [P]),
}

_lib: Optional[C.CDLL] = None


def declared_symbols():
    """Function names declared in the public header."""
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:[a-z_0-9]+\s+)*[a-z_0-9]+\**\s+\**(fennol_[a-z_0-9]+)\s*\(",
                                 txt, flags=re.M)))


def load(path: Optional[os.PathLike] = None) -> C.CDLL:
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise LibraryError(f"{p} not found: build it with `python -m fennol_b200.build`")
    try:
        lib = C.CDLL(str(p))
    except OSError as e:
        raise LibraryError(f"cannot load {p}: {e}") from e
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check_finite(buffers, status, stream: int) -> None:
    """Enqueue ``fennol_check_finite`` on up to four device tensors (float32
    or float64): status[ST_NONFINITE] is set when one holds a NaN or an
    infinity."""
    bufs = [b for b in buffers if b is not None and b.numel() > 0]
    k = len(bufs)
    ptrs = (C.c_void_p * 4)(*[b.data_ptr() for b in bufs])
    counts = (C.c_size_t * 4)(*[b.numel() for b in bufs])
    dbl = (C.c_int * 4)(*[int(b.element_size() == 8) for b in bufs])
    call("fennol_check_finite", k, C.cast(ptrs, C.c_void_p), C.cast(counts, C.c_void_p),
         C.cast(dbl, C.c_void_p), status.data_ptr(), stream)


def call(name: str, *args) -> int:
    """Call ``name`` and raise :class:`FennolError` on a negative status."""
    rc = getattr(load(), name)(*args)
    if isinstance(rc, int) and rc < 0:
        raise FennolError(name, rc)
    return rc

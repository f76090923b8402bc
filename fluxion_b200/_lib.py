"""Loader for ``libfluxion_cuda.so`` and the ctypes view of its C ABI.

The argument and return types of every entry point are read from the C header
(``include/fluxion_cuda.h``), so the Python side cannot drift from the ABI.
There is no fallback: if the shared library is missing or cannot be loaded,
importing the backend raises, and every operation fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# FLUXION_CHECKED=1 loads the checked build (index checks recorded in device status words)
LIB_PATH = os.path.join(HERE, "libfluxion_cuda_checked.so" if os.environ.get("FLUXION_CHECKED") == "1"
                        else "libfluxion_cuda.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "fluxion_cuda.h")

FX_OK = 0
FX_ERR_DIMENSION_MISMATCH = 1
FX_ERR_INVALID_GRID = 2
FX_ERR_INVALID_STENCIL = 3
FX_ERR_BACKEND = 4
FX_ERR_INVALID_ARGUMENT = 5
FX_ERR_UNSUPPORTED = 6
FX_ERR_NO_DEVICE = 7

FX_F32, FX_F64 = 0, 1


class FxBc(C.Structure):
    _fields_ = [("kind", C.c_int), ("a", C.c_double), ("b", C.c_double), ("g", C.c_double)]


class FxBoundaries(C.Structure):
    _fields_ = [("side", FxBc * 4)]


class FxGrid(C.Structure):
    _fields_ = [("rows", C.c_size_t), ("cols", C.c_size_t), ("dx", C.c_double), ("dy", C.c_double)]


class FxStencil(C.Structure):
    _fields_ = [("n", C.c_int), ("dr", C.POINTER(C.c_int)), ("dc", C.POINTER(C.c_int)),
                ("w", C.POINTER(C.c_double))]


class FxStats(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("residual", C.c_double), ("reason", C.c_int)]


class FxMgTuning(C.Structure):
    _fields_ = [("chunk_pct", C.c_int), ("tail_top_points", C.c_size_t)]


class FxMgVertexOpts(C.Structure):
    _fields_ = [("n_pre", C.c_size_t), ("n_post", C.c_size_t), ("omega", C.c_double),
                ("coarse_max", C.c_size_t), ("coarse_sweeps", C.c_size_t), ("dtype", C.c_int),
                ("op_coeff", C.c_double), ("op_stencil", FxStencil)]


_STRUCTS = {
    "fx_bc": FxBc, "fx_boundaries": FxBoundaries, "fx_grid": FxGrid, "fx_stencil": FxStencil,
    "fx_stats": FxStats, "fx_mg_vertex_opts": FxMgVertexOpts, "fx_mg_tuning": FxMgTuning,
}
_OPAQUE = {"fx_ctx", "fx_buf", "fx_precond", "fx_mg", "fx_cg", "fx_pipelined_cg", "fx_bicgstab",
           "fx_gmres", "fx_graph", "fx_ir", "fx_fcg", "fx_fgmres", "fx_op", "fx_cdmg", "fx_lsm", "fx_lsm_data", "fx_batch"}
_SCALARS = {
    "int": C.c_int, "size_t": C.c_size_t, "double": C.c_double, "float": C.c_float,
    "unsigned long long": C.c_ulonglong, "long long": C.c_longlong, "void": None, "char": C.c_char,
}


def _ctype(decl: str):
    """Map one C parameter / return declaration to a ctypes type."""
    d = decl.strip()
    is_array = bool(re.search(r"\[\s*\d*\s*\]\s*$", d))
    d = re.sub(r"\[\s*\d*\s*\]\s*$", "", d)
    nptr = d.count("*") + (1 if is_array else 0)
    d = d.replace("*", " ").replace("const", " ")
    toks = d.split()
    # drop the parameter name if present
    if len(toks) >= 2 and toks[-1] not in _SCALARS and toks[-1] not in _STRUCTS \
            and toks[-1] not in _OPAQUE and not (toks[-2:] == ["long", "long"]):
        toks = toks[:-1]
    base = " ".join(toks)
    if base in _OPAQUE:
        return C.POINTER(C.c_void_p) if nptr >= 2 else C.c_void_p
    if base == "char" and nptr == 1:
        return C.c_char_p
    if base == "void":
        return C.c_void_p if nptr else None
    t = _STRUCTS.get(base) or _SCALARS.get(base)
    if t is None:
        raise TypeError(f"unmapped C type in header: {decl!r}")
    for _ in range(nptr):
        t = C.POINTER(t)
    return t


def parse_header(path: str = HEADER_PATH):
    """Return {name: (restype, [argtypes])} for every function the header declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(fx_\w+)\s*\(([^;{}]*?)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        if "typedef" in ret:
            continue
        ret = ret.strip().split("\n")[-1]
        argl = [] if args.strip() in ("", "void") else [a for a in args.split(",")]
        protos[name] = (_ctype(ret + " x"), [_ctype(a) for a in argl])
    return protos


_lib = None
_lock = threading.Lock()


class LibraryMissing(ImportError):
    pass


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise LibraryMissing(
                    f"{LIB_PATH} is missing: build it with `python -m fluxion_b200.build` "
                    "(the solve path has no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in parse_header().items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    msg = lib().fx_last_error()
    return msg.decode() if msg else ""

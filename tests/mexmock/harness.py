"""Python side of the MEX mock (TEST INFRASTRUCTURE ONLY).

build() compiles tests/mexmock/mexmock.c into libmexmock.so and every gateway
under gbm3d_b200/mex/ into <name>.mexmock.so (linked against libgbm3d.so),
with gcc, into tests/mexmock/_build/.  Gateway(name)(*args, nargout=k) then
calls mexFunction the way MATLAB would: numpy arrays become column-major
numeric mxArrays, lists of arrays with a shape become cell arrays, dicts
become 1x1 structs, str becomes char.  A mexErrMsgIdAndTxt raises MexError.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
MEXDIR = os.path.join(ROOT, "gbm3d_b200", "mex")
OUT = os.path.join(HERE, "_build")
GATEWAYS = ["matchBlocksCPU", "denoiseAndAggregateGPU", "matchBlocksWie", "denoiseAndAggregateWieFast",
            "denoiseAndAggregateWie", "matchBlocksGPU", "matchBlocksV", "denoiseAndAggregateV"]
CLS = {np.dtype(np.float64): 6, np.dtype(np.float32): 7, np.dtype(np.int8): 8, np.dtype(np.uint8): 9,
       np.dtype(np.int32): 12, np.dtype(np.uint32): 13, np.dtype(np.int64): 14, np.dtype(np.bool_): 3}
NP = {v: k for k, v in CLS.items()}


class MexError(RuntimeError):
    def __init__(self, ident, msg):
        super().__init__(f"{ident}: {msg}")
        self.ident, self.msg = ident, msg


class Cell:
    """A MATLAB cell array of the given shape (column-major element order)."""

    def __init__(self, shape, items):
        self.shape, self.items = tuple(shape), list(items)


class GpuArray:
    """Stand-in for a gpuArray argument: opaque until the gateway gathers it."""

    def __init__(self, a):
        self.a = a


_mm = None


def _gcc(args):
    subprocess.run(["gcc", *args], check=True, capture_output=True, text=True)


def build():
    os.makedirs(OUT, exist_ok=True)
    mm = os.path.join(OUT, "libmexmock.so")
    _gcc(["-O1", "-shared", "-fPIC", "-o", mm, os.path.join(HERE, "mexmock.c")])
    lib = os.path.join(ROOT, "gbm3d_b200")
    for g in GATEWAYS:
        _gcc(["-O1", "-shared", "-fPIC", "-I", HERE, "-I", MEXDIR, "-I", os.path.join(ROOT, "include"),
              "-o", os.path.join(OUT, g + ".mexmock.so"), os.path.join(MEXDIR, g + ".c"),
              "-L", OUT, "-lmexmock", "-L", lib, "-lgbm3d", f"-Wl,-rpath,{OUT}:{lib}", "-lm"])
    return OUT


def mm():
    global _mm
    if _mm is None:
        _mm = C.CDLL(os.path.join(OUT, "libmexmock.so"), mode=C.RTLD_GLOBAL)
        P = C.c_void_p
        for name, res, args in [
            ("mm_numeric", P, [C.c_int, C.c_int, C.POINTER(C.c_size_t), P]), ("mm_cell", P, [C.c_size_t, C.c_size_t]),
            ("mm_set_cell", None, [P, C.c_size_t, P]), ("mm_struct", P, []), ("mm_set_field", C.c_int, [P, C.c_char_p, P]),
            ("mm_string", P, [C.c_char_p]), ("mm_gpuarray", P, [P]),
            ("mm_call", C.c_int, [P, C.c_int, C.POINTER(P), C.c_int, C.POINTER(P)]),
            ("mm_err_id", C.c_char_p, []), ("mm_err_msg", C.c_char_p, []), ("mm_run_atexit", None, []),
            ("mm_class", C.c_int, [P]), ("mm_ndim", C.c_int, [P]), ("mm_dim", C.c_size_t, [P, C.c_int]),
            ("mm_numel", C.c_size_t, [P]), ("mm_data", P, [P]), ("mm_get_cell", P, [P, C.c_size_t]),
            ("mm_destroy", None, [P]), ("mm_nfields", C.c_int, [P]), ("mm_field_name", C.c_char_p, [P, C.c_int]),
            ("mm_field_value", P, [P, C.c_int])]:
            f = getattr(_mm, name)
            f.restype, f.argtypes = res, args
    return _mm


def to_mx(v):
    m = mm()
    if isinstance(v, GpuArray):
        return m.mm_gpuarray(to_mx(v.a))
    if isinstance(v, str):
        return m.mm_string(v.encode())
    if isinstance(v, dict):
        s = m.mm_struct()
        for k, x in v.items():
            m.mm_set_field(s, k.encode(), to_mx(x))
        return s
    if isinstance(v, Cell):
        c = m.mm_cell(*v.shape)
        for i, x in enumerate(v.items):
            m.mm_set_cell(c, i, to_mx(x))
        return c
    if isinstance(v, bool):
        v = np.array(v)
    a = np.asarray(v)
    if a.dtype.kind in "iu" and a.dtype not in CLS:
        a = a.astype(np.float64)
    if a.dtype.kind == "f" and a.dtype not in CLS:
        a = a.astype(np.float64)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(1, -1)
    a = np.asfortranarray(a)
    dims = (C.c_size_t * a.ndim)(*a.shape)
    return m.mm_numeric(CLS[a.dtype], a.ndim, dims, a.ctypes.data_as(C.c_void_p))


def from_mx(p):
    m = mm()
    cls = m.mm_class(p)
    shape = tuple(m.mm_dim(p, k) for k in range(m.mm_ndim(p)))
    if cls == 1:  # cell
        n = m.mm_numel(p)
        return Cell(shape, [from_mx(m.mm_get_cell(p, i)) for i in range(n)])
    if cls == 2:  # 1 x 1 struct
        return {m.mm_field_name(p, f).decode(): from_mx(m.mm_field_value(p, f)) for f in range(m.mm_nfields(p))}
    dt = NP[cls]
    n = m.mm_numel(p)
    buf = (C.c_char * (n * dt.itemsize)).from_address(m.mm_data(p))
    return np.frombuffer(bytes(buf), dtype=dt).reshape(shape, order="F").copy()


class Gateway:
    def __init__(self, name):
        self.name = name
        self.lib = C.CDLL(os.path.join(OUT, name + ".mexmock.so"))
        self.fn = C.cast(self.lib.mexFunction, C.c_void_p)

    def __call__(self, *args, nargout=1):
        m = mm()
        prhs = (C.c_void_p * max(len(args), 1))(*[to_mx(a) for a in args])
        plhs = (C.c_void_p * max(nargout, 1))()
        rc = m.mm_call(self.fn, nargout, plhs, len(args), prhs)
        for i in range(len(args)):
            m.mm_destroy(prhs[i])
        if rc:
            raise MexError(m.mm_err_id().decode(), m.mm_err_msg().decode())
        outs = []
        for i in range(nargout):
            outs.append(from_mx(plhs[i]) if plhs[i] else None)
            if plhs[i]:
                m.mm_destroy(plhs[i])
        return outs[0] if nargout == 1 else tuple(outs)

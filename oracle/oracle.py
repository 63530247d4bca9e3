"""ctypes front end of the C++ oracle (liboracle.so) -- TEST INFRASTRUCTURE.

The oracle restates GITM's vertical advance on the CPU (see
gitm_vert_oracle.hpp for the reference files and lines it follows).  This
module builds it on demand with the Makefile beside it and runs it on
numpy arrays in the native layout of include/gitm_vert.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from gitm_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liboracle.so")
    if force or not os.path.exists(path) or _stale(path):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return path


def _stale(path: str) -> bool:
    t = os.path.getmtime(path)
    srcs = [os.path.join(_HERE, f) for f in os.listdir(_HERE) if f.endswith((".cpp", ".hpp"))]
    srcs.append(os.path.join(_HERE, "..", "include", "gitm_vert.h"))
    srcs.append(os.path.join(_HERE, "..", "include", "gitm_hz.h"))
    return any(os.path.getmtime(s) > t for s in srcs if os.path.exists(s))


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path) or _stale(path):
            build()
        L = C.CDLL(path)
        L.oracle_advance_native.restype = C.c_uint32
        L.oracle_advance_native.argtypes = [C.POINTER(abi.GitmVertParams),
                                            C.POINTER(abi.GitmColumnBatch), C.c_int,
                                            C.c_double, C.c_int, C.POINTER(C.c_uint32), C.c_int]
        L.oracle_advance_1d.restype = C.c_uint32
        L.oracle_advance_1d.argtypes = [C.POINTER(abi.GitmVertParams),
                                        C.POINTER(abi.GitmModVerticalBatch), C.c_double,
                                        C.POINTER(C.c_uint32), C.c_int]
        L.oracle_cfl_dt.restype = C.c_double
        L.oracle_cfl_dt.argtypes = [C.POINTER(abi.GitmVertParams),
                                    C.POINTER(abi.GitmColumnBatch), C.c_double]
        L.oracle_count_ops.restype = None
        L.oracle_count_ops.argtypes = [C.POINTER(abi.GitmVertParams),
                                       C.POINTER(abi.GitmModVerticalBatch), C.c_double,
                                       C.POINTER(C.c_double)]
        L.oracle_limiter_mc.restype = C.c_double
        L.oracle_limiter_mc.argtypes = [C.c_double, C.c_double, C.c_double]
        L.oracle_lu_solve.restype = C.c_int
        L.oracle_lu_solve.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_mesh_coefs.restype = None
        L.oracle_mesh_coefs.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_abi_sizes.restype = None
        L.oracle_abi_sizes.argtypes = [C.POINTER(C.c_int64)]
        L.oracle_hz_advance.restype = C.c_uint32
        L.oracle_hz_advance.argtypes = [C.POINTER(abi.GitmHzParams), C.POINTER(abi.GitmHzBlocks), C.c_double,
                                        C.POINTER(C.c_uint32), C.c_int]
        _LIB = L
    return _LIB


def _p(a):
    if a is None:
        return abi.dptr(0)
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return abi.dptr(a.ctypes.data)


def column_batch(m) -> abi.GitmColumnBatch:
    """GitmColumnBatch over a synthetic.Member's numpy arrays (host pointers)."""
    b = abi.GitmColumnBatch()
    b.n_alts = m.n_alts
    b.grid_per_column = 1 if m.altitude.ndim == 2 else 0
    b.n_cols = m.n_cols
    for name, _ in abi.GitmColumnBatch._fields_[3:]:
        setattr(b, name, _p(getattr(m, name, None)))
    return b


def modvertical_batch(d: dict) -> abi.GitmModVerticalBatch:
    b = abi.GitmModVerticalBatch()
    b.n_alts = d["n_alts"]
    b.grid_per_column = 1 if d["altitude"].ndim == 2 else 0
    b.n_cols = d["n_cols"]
    for name, _ in abi.GitmModVerticalBatch._fields_[3:]:
        setattr(b, name, _p(d.get(name)))
    return b


def advance(members, params, dt: float, n_steps: int = 1, nthreads: int | None = None):
    """Advances the members in place; returns the per-column status words."""
    if not isinstance(members, (list, tuple)):
        members = [members]
    arr = (abi.GitmColumnBatch * len(members))(*[column_batch(m) for m in members])
    ncol = sum(m.n_cols for m in members)
    st = np.zeros(ncol, dtype=np.uint32)
    nthreads = nthreads or os.cpu_count() or 1
    lib().oracle_advance_native(C.byref(params), arr, len(members), dt, n_steps,
                                st.ctypes.data_as(C.POINTER(C.c_uint32)), nthreads)
    return st


def advance_1d(d: dict, params, dt: float, nthreads: int | None = None):
    b = modvertical_batch(d)
    st = np.zeros(d["n_cols"], dtype=np.uint32)
    nthreads = nthreads or os.cpu_count() or 1
    lib().oracle_advance_1d(C.byref(params), C.byref(b), dt,
                            st.ctypes.data_as(C.POINTER(C.c_uint32)), nthreads)
    return st


def cfl_dt(m, params, cfl: float) -> float:
    b = column_batch(m)
    return lib().oracle_cfl_dt(C.byref(params), C.byref(b), cfl)


def count_ops(d: dict, params, dt: float) -> dict:
    """Operation counts of one RK4 step of column 0 of a ModVertical batch."""
    out = (C.c_double * 6)()
    lib().oracle_count_ops(C.byref(params), C.byref(modvertical_batch(d)), dt, out)
    keys = ("add", "mul", "div", "sqrt", "trans", "cmp")
    return {k: int(v) for k, v in zip(keys, out)}


def limiter_mc(u: float, d: float, beta: float = 2.0) -> float:
    return lib().oracle_limiter_mc(u, d, beta)


def lu_solve(a: np.ndarray, b: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.float64)
    x = np.ascontiguousarray(b, dtype=np.float64).copy()
    ok = lib().oracle_lu_solve(a.ctypes.data_as(C.POINTER(C.c_double)),
                               x.ctypes.data_as(C.POINTER(C.c_double)))
    return x, bool(ok)


def mesh_coefs(alt: np.ndarray):
    """(GradLogConS stencil [nAlts,5], lower [2,5], upper [2,5]) of a grid."""
    alt = np.ascontiguousarray(alt, dtype=np.float64)
    n = alt.shape[0] - 4
    out = np.zeros(5 * n + 20)
    lib().oracle_mesh_coefs(n, alt.ctypes.data_as(C.POINTER(C.c_double)),
                            out.ctypes.data_as(C.POINTER(C.c_double)))
    return out[: 5 * n].reshape(n, 5), out[5 * n: 5 * n + 10].reshape(2, 5), out[5 * n + 10:].reshape(2, 5)


def hz_advance(blocks, params, dt: float, nthreads: int | None = None):
    """advance_horizontal for every block of host HzBlocks, in place; returns
    the per-block status words."""
    b = blocks.batch()
    st = np.zeros(blocks.n_blocks, dtype=np.uint32)
    nthreads = nthreads or os.cpu_count() or 1
    lib().oracle_hz_advance(C.byref(params), C.byref(b), dt, st.ctypes.data_as(C.POINTER(C.c_uint32)), nthreads)
    return st


def abi_sizes():
    out = (C.c_int64 * 9)()
    lib().oracle_abi_sizes(out)
    return list(out)

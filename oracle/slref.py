"""ctypes front-end of the C restatement oracle (oracle/slref.c).

Test infrastructure only: imported by tests/ and by bench.py's CPU baseline,
never by the product.  Takes the same slgpu_group structures as the engine.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_uint8

import numpy as np

from sparselizard_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslref.so")


class Fragment(ctypes.Structure):
    _fields_ = [("ntr", c_int32), ("ndr", c_int32), ("nr", c_int32), ("nc", c_int64),
                ("rows", POINTER(c_int32)), ("cols", POINTER(c_int32)), ("vals", POINTER(c_double))]


class Csr(ctypes.Structure):
    _fields_ = [("nA", c_int64), ("nD", c_int64), ("nnzA", c_int64), ("nnzD", c_int64),
                ("Arows", POINTER(c_int32)), ("Acols", POINTER(c_int32)), ("Drows", POINTER(c_int32)),
                ("Dcols", POINTER(c_int32)), ("Avals", POINTER(c_double)), ("Dvals", POINTER(c_double))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        l = ctypes.CDLL(LIB_PATH)
        l.slref_element_matrices.argtypes = [POINTER(abi.Group), POINTER(c_double), POINTER(c_int32), POINTER(c_double)]
        l.slref_element_matrices.restype = c_int
        l.slref_matrix.argtypes = [POINTER(abi.Group), c_int, POINTER(c_double), POINTER(POINTER(c_int32)),
                                   POINTER(Fragment), c_int, c_int64, POINTER(c_uint8), POINTER(Csr)]
        l.slref_matrix.restype = c_int
        l.slref_rhs.argtypes = [POINTER(abi.Group), POINTER(c_double), POINTER(c_int32), c_int64, POINTER(c_double)]
        l.slref_rhs.restype = c_int
        l.slref_free.argtypes = [POINTER(Csr)]
        l.slref_set_absmode.argtypes = [c_int]
        _lib = l
    return _lib


def matrix(groups, xyz, conns, ndofs, isconstrained, frags=(), absmode=False):
    """rawmat::process of the groups' element matrices + fragments -> dict of CSR arrays.
    absmode: values are sum |terms| (the rounding-error scale) instead of sum terms."""
    l = lib()
    l.slref_set_absmode(1 if absmode else 0)
    G = (abi.Group * max(1, len(groups)))(*groups)
    C = (POINTER(c_int32) * max(1, len(conns)))(*[abi.i32p(c) for c in conns])
    F = (Fragment * max(1, len(frags)))()
    keep = []
    for i, (ntr, ndr, nr, nc, rows, cols, vals) in enumerate(frags):
        rows = np.ascontiguousarray(rows, np.int32); cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        keep += [rows, cols, vals]
        F[i] = Fragment(ntr, ndr, nr, nc, abi.i32p(rows), abi.i32p(cols), abi.f64p(vals))
    con = np.ascontiguousarray(isconstrained, np.uint8)
    out = Csr()
    xyz = np.ascontiguousarray(xyz, np.float64)
    st = l.slref_matrix(G, len(groups), abi.f64p(xyz), C, F, len(frags), ndofs,
                        con.ctypes.data_as(POINTER(c_uint8)), ctypes.byref(out))
    l.slref_set_absmode(0)
    if st != 0:
        raise RuntimeError("slref_matrix failed")
    nA, nnzA, nnzD = out.nA, out.nnzA, out.nnzD
    res = dict(
        Arows=np.ctypeslib.as_array(out.Arows, (nA + 1,)).copy(),
        Acols=np.ctypeslib.as_array(out.Acols, (max(nnzA, 1),))[:nnzA].copy(),
        Avals=np.ctypeslib.as_array(out.Avals, (max(nnzA, 1),))[:nnzA].copy(),
        Drows=np.ctypeslib.as_array(out.Drows, (nA + 1,)).copy(),
        Dcols=np.ctypeslib.as_array(out.Dcols, (max(nnzD, 1),))[:nnzD].copy(),
        Dvals=np.ctypeslib.as_array(out.Dvals, (max(nnzD, 1),))[:nnzD].copy(),
        nA=nA, nD=out.nD,
    )
    l.slref_free(ctypes.byref(out))
    return res


def rhs(group, xyz, conn, ndofs, absmode=False):
    l = lib()
    l.slref_set_absmode(1 if absmode else 0)
    b = np.zeros(ndofs)
    xyz = np.ascontiguousarray(xyz, np.float64)
    conn = np.ascontiguousarray(conn, np.int32)
    if l.slref_rhs(ctypes.byref(group), abi.f64p(xyz), abi.i32p(conn), ndofs, abi.f64p(b)) != 0:
        raise RuntimeError("slref_rhs failed")
    l.slref_set_absmode(0)
    return np.abs(b) if absmode else b


def element_matrices(group, xyz, conn):
    l = lib()
    K = np.zeros(group.ndests * group.ntf * group.ndof * max(group.nelem, 1))
    xyz = np.ascontiguousarray(xyz, np.float64)
    conn = np.ascontiguousarray(conn, np.int32)
    if l.slref_element_matrices(ctypes.byref(group), abi.f64p(xyz), abi.i32p(conn), abi.f64p(K)) != 0:
        raise RuntimeError("slref_element_matrices failed")
    return K

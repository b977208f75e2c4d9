"""ctypes binding of the slgpu C ABI (include/slgpu.h).

This is the binding a Python caller would add to reach the engine: the
structures mirror the C declarations field by field and every call returns
the C status, raised as ``SlgpuError`` with the engine's message.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint8, c_uint, c_uint64, c_size_t, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libslgpu.so")

OK, E_ARG, E_CUDA, E_UNSUPPORTED, E_BUDGET, E_STATE, E_NODEVICE, E_TIMEOUT = range(8)
CTX_RECORD_ONLY = 1
PREC_FP64, PREC_SPLIT, PREC_FP32 = 0, 1, 2
(OP_CONST, OP_JAC, OP_INVJAC, OP_DETJAC, OP_ELEM, OP_FIELD, OP_COORD, OP_ADD, OP_MUL, OP_INV, OP_NEG,
 OP_POW) = range(12)


class SlgpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"slgpu status {status}: {msg}")
        self.status = status


class Node(ctypes.Structure):
    _fields_ = [("op", c_int32), ("a", c_int32), ("b", c_int32), ("c", c_int32)]


class Table(ctypes.Structure):
    _fields_ = [("rows", c_int32), ("vals", POINTER(c_double))]


class Term(ctypes.Structure):
    _fields_ = [("tf_table", c_int32), ("dof_table", c_int32), ("coef_node", c_int32), ("pad", c_int32),
                ("scale", c_double)]


class Dest(ctypes.Structure):
    _fields_ = [("tfaddr", POINTER(c_int32)), ("dofaddr", POINTER(c_int32)), ("multiplier", c_double)]


class Group(ctypes.Structure):
    _fields_ = [
        ("mesh", c_int32), ("elemtype", c_int32), ("elemdim", c_int32), ("problemdim", c_int32),
        ("nelem", c_int64), ("elems", POINTER(c_int32)), ("orient", POINTER(c_int32)), ("norient", c_int32),
        ("ngp", c_int32), ("weights", POINTER(c_double)), ("ncurvednodes", c_int32), ("lagrange", POINTER(c_double)),
        ("ntf", c_int32), ("ndof", c_int32), ("ntables", c_int32), ("tables", POINTER(Table)),
        ("nnodes", c_int32), ("nodes", POINTER(Node)), ("nconsts", c_int32), ("consts", POINTER(c_double)),
        ("nelemdata", c_int32), ("elemdata", POINTER(POINTER(c_double))),
        ("nfielddata", c_int32), ("fielddata", POINTER(POINTER(c_double))), ("fieldrows", POINTER(c_int32)),
        ("nterms", c_int32), ("terms", POINTER(Term)), ("ndests", c_int32), ("dests", POINTER(Dest)),
    ]


class CsrInfo(ctypes.Structure):
    _fields_ = [("nA", c_int64), ("nD", c_int64), ("nnzA", c_int64), ("nnzD", c_int64), ("ncoo", c_int64),
                ("pattern_reused", c_int32), ("pad", c_int32)]


class Work(ctypes.Structure):
    _fields_ = [("contraction_flops", c_double), ("coef_points", c_int64), ("ncoo", c_int64), ("nvalid", c_int64),
                ("nnz", c_int64), ("nA", c_int64), ("ngroups", c_int32), ("pad", c_int32)]


UPDATE_ELEMDATA, UPDATE_FIELDDATA, UPDATE_SCALES = 0, 1, 2


class GroupDesc(ctypes.Structure):
    _fields_ = [("mesh", c_int32), ("elemtype", c_int32), ("ntf", c_int32), ("ndof", c_int32), ("nterms", c_int32),
                ("ngp", c_int32), ("norient", c_int32), ("ndests", c_int32), ("nelemdata", c_int32),
                ("nfielddata", c_int32), ("fieldrows", c_int32 * 8), ("nelem", c_int64), ("mesh_nelem", c_int64)]


class Update(ctypes.Structure):
    _fields_ = [("group", c_int32), ("kind", c_int32), ("index", c_int32), ("rows", c_int32),
                ("values", POINTER(c_double)), ("count", c_int64)]


class Request(ctypes.Structure):
    _fields_ = [("handle", c_int32), ("precision", c_int32), ("nupdates", c_int32), ("pad", c_int32),
                ("updates", POINTER(Update)), ("Avals", POINTER(c_double)), ("Dvals", POINTER(c_double))]


class RequestStats(ctypes.Structure):
    _fields_ = [("submit_s", c_double), ("start_s", c_double), ("done_s", c_double), ("device_ms", c_double),
                ("slot", c_int32), ("status", c_int32), ("launch_ms", c_double), ("launch_parts_ms", c_double * 3)]


# Every exported symbol with (restype, argtypes); the tests check that the
# library exports each of them.
SIGNATURES = {
    "slgpu_ctx_create": (c_int, [c_int, c_size_t, c_uint, POINTER(c_void_p)]),
    "slgpu_ctx_destroy": (None, [c_void_p]),
    "slgpu_last_error": (c_int, [c_void_p, c_char_p, c_size_t]),
    "slgpu_bytes_in_use": (c_int64, [c_void_p]),
    "slgpu_mesh_set_nodes": (c_int, [c_void_p, c_int, c_int64, POINTER(c_double)]),
    "slgpu_mesh_set_elements": (c_int, [c_void_p, c_int, c_int, c_int, c_int64, POINTER(c_int32)]),
    "slgpu_matrix_create": (c_int, [c_void_p, c_int64, POINTER(c_int)]),
    "slgpu_matrix_destroy": (c_int, [c_void_p, c_int]),
    "slgpu_matrix_clone": (c_int, [c_void_p, c_int, POINTER(c_int)]),
    "slgpu_matrix_add_group": (c_int, [c_void_p, c_int, POINTER(Group), POINTER(c_int)]),
    "slgpu_matrix_add_fragment": (c_int, [c_void_p, c_int, c_int32, c_int32, c_int32, c_int64, POINTER(c_int32),
                                          POINTER(c_int32), POINTER(c_double)]),
    "slgpu_matrix_set_elemdata": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double)]),
    "slgpu_matrix_set_fielddata": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double)]),
    "slgpu_matrix_set_scales": (c_int, [c_void_p, c_int, c_int, POINTER(c_double), POINTER(c_double)]),
    "slgpu_matrix_get_scales": (c_int, [c_void_p, c_int, c_int, POINTER(c_double), POINTER(c_double)]),
    "slgpu_matrix_group_symmetry": (c_int, [c_void_p, c_int, c_int, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
    "slgpu_kernel_launches": (c_int64, [c_void_p]),
    "slgpu_transfer_bytes": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_int64)]),
    "slgpu_tuned_tiles": (c_int, [c_void_p, c_char_p, c_size_t]),
    "slgpu_ctx_set_graphs": (c_int, [c_void_p, c_int]),
    "slgpu_graph_launches": (c_int64, [c_void_p]),
    "slgpu_ctx_set_kernel_timers": (c_int, [c_void_p, c_int]),
    "slgpu_kernel_stats": (c_int, [c_void_p, c_char_p, POINTER(c_double), POINTER(c_int64), POINTER(c_double)]),
    "slgpu_check_coefficient_kernels": (c_int, [c_void_p, c_int, c_char_p, c_size_t]),
    "slgpu_matrix_work": (c_int, [c_void_p, c_int, c_void_p]),
    "slgpu_element_matrices_noalloc": (c_int, [POINTER(Group), c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                               c_void_p, c_char_p, c_size_t]),
    "slgpu_matrix_process": (c_int, [c_void_p, c_int, POINTER(c_uint8), c_int, POINTER(CsrInfo)]),
    "slgpu_matrix_download": (c_int, [c_void_p, c_int, POINTER(c_int32), POINTER(c_int32), POINTER(c_double),
                                      POINTER(c_int32), POINTER(c_int32), POINTER(c_double)]),
    "slgpu_matrix_download_values": (c_int, [c_void_p, c_int, POINTER(c_double), POINTER(c_double)]),
    "slgpu_matrix_pattern_serial": (c_int, [c_void_p, c_int, POINTER(c_uint64)]),
    "slgpu_host_register": (c_int, [c_void_p, c_void_p, c_size_t]),
    "slgpu_matrix_share_addresses": (c_int, [c_void_p, c_int, c_int]),
    "slgpu_host_unregister": (c_int, [c_void_p, c_void_p]),
    "slgpu_matrix_device_csr": (c_int, [c_void_p, c_int] + [POINTER(c_void_p)] * 6),
    "slgpu_matrix_eliminate": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "slgpu_rhs_assemble": (c_int, [c_void_p, POINTER(Group), c_int64, c_int, POINTER(c_double)]),
    "slgpu_rhs_assemble_rows": (c_int, [c_void_p, POINTER(Group), c_int64, c_int, POINTER(c_int32), POINTER(c_double), c_int64,
                                        POINTER(c_int64)]),
    "slgpu_last_timings": (c_int, [c_void_p, POINTER(c_double)]),
    "slgpu_record_count": (c_int, [c_void_p, c_int, POINTER(c_int), POINTER(c_int)]),
    "slgpu_record_group": (c_int, [c_void_p, c_int, c_int, POINTER(Group)]),
    "slgpu_record_fragment": (c_int, [c_void_p, c_int, c_int, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32),
                                      POINTER(c_int64), POINTER(POINTER(c_int32)), POINTER(POINTER(c_int32)),
                                      POINTER(POINTER(c_double))]),
    "slgpu_record_constraints": (c_int, [c_void_p, c_int, POINTER(c_int64), POINTER(POINTER(c_uint8))]),
    "slgpu_record_rhs_count": (c_int, [c_void_p, POINTER(c_int)]),
    "slgpu_record_rhs_group": (c_int, [c_void_p, c_int, POINTER(Group), POINTER(c_int64)]),
    "slgpu_record_mesh": (c_int, [c_void_p, c_int, c_int, POINTER(c_int64), POINTER(POINTER(c_double)), POINTER(c_int),
                                  POINTER(c_int64), POINTER(POINTER(c_int32))]),
    "slgpu_matrix_group_count": (c_int, [c_void_p, c_int, POINTER(c_int)]),
    "slgpu_matrix_group_desc": (c_int, [c_void_p, c_int, c_int, POINTER(GroupDesc)]),
    "slgpu_server_create": (c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    "slgpu_server_prepare": (c_int, [c_void_p, c_int, c_int]),
    "slgpu_server_submit": (c_int, [c_void_p, POINTER(Request), POINTER(c_int64)]),
    "slgpu_server_submit_template": (c_int, [c_void_p, c_int, POINTER(c_uint8), c_int, POINTER(c_int64)]),
    "slgpu_server_wait": (c_int, [c_void_p, c_int64, c_double, POINTER(RequestStats)]),
    "slgpu_server_error": (c_int, [c_void_p, c_int64, c_char_p, c_size_t]),
    "slgpu_server_release": (c_int, [c_void_p, c_int64]),
    "slgpu_server_pending": (c_int64, [c_void_p]),
    "slgpu_server_clock": (c_double, [c_void_p]),
    "slgpu_server_destroy": (None, [c_void_p]),
    "slgpu_host_alloc": (c_int, [c_void_p, c_size_t, POINTER(c_void_p)]),
    "slgpu_host_free": (None, [c_void_p]),
}


def bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib() -> ctypes.CDLL:
    """The engine library; raises if it was not built (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SlgpuError(E_NODEVICE, f"{LIB_PATH} is not built (run __graft_entry__.build())")
        _lib = bind(ctypes.CDLL(LIB_PATH, mode=os.RTLD_LOCAL | os.RTLD_NOW))
    return _lib


def f64p(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def i32p(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int32))


class Context:
    """Owns one slgpu context; methods raise SlgpuError on a non-zero status."""

    def __init__(self, device: int = 0, budget: int = 0, flags: int = 0):
        self.lib = lib()
        h = c_void_p()
        st = self.lib.slgpu_ctx_create(device, budget, flags, ctypes.byref(h))
        if st != OK:
            raise SlgpuError(st, "cannot create a context (no usable CUDA device?)")
        self.h = h

    def error(self) -> str:
        buf = ctypes.create_string_buffer(2048)
        self.lib.slgpu_last_error(self.h, buf, len(buf))
        return buf.value.decode(errors="replace")

    def check(self, st: int):
        if st != OK:
            raise SlgpuError(st, self.error())

    def close(self):
        if getattr(self, "h", None):
            self.lib.slgpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def timings(self) -> np.ndarray:
        out = np.zeros(5)
        self.lib.slgpu_last_timings(self.h, f64p(out))
        return out


class GroupBuilder:
    """Keeps the numpy arrays behind an slgpu_group alive and fills the struct."""

    def __init__(self, *, elemtype, dim, elems, orient, norient, weights, lagrange, ncurvednodes, ntf, ndof,
                 tables, nodes, consts, terms, dests, elemdata=(), fielddata=(), mesh=0):
        self.keep = []
        k = self.keep.append
        self.g = Group()
        g = self.g
        g.mesh, g.elemtype, g.elemdim, g.problemdim = mesh, elemtype, dim, dim
        elems = np.ascontiguousarray(elems, np.int32); k(elems)
        orient = np.ascontiguousarray(orient, np.int32); k(orient)
        g.nelem = elems.size
        g.elems, g.orient, g.norient = i32p(elems), i32p(orient), norient
        weights = np.ascontiguousarray(weights, np.float64); k(weights)
        g.ngp, g.weights = weights.size, f64p(weights)
        lagrange = np.ascontiguousarray(lagrange, np.float64); k(lagrange)
        g.ncurvednodes, g.lagrange = ncurvednodes, f64p(lagrange)
        g.ntf, g.ndof = ntf, ndof
        tabs = (Table * len(tables))()
        for i, t in enumerate(tables):
            t = np.ascontiguousarray(t, np.float64); k(t)
            tabs[i].rows = t.shape[1]
            tabs[i].vals = f64p(t)
        k(tabs)
        g.ntables, g.tables = len(tables), tabs
        nd = (Node * len(nodes))(*[Node(*n) for n in nodes]); k(nd)
        g.nnodes, g.nodes = len(nodes), nd
        consts = np.ascontiguousarray(consts, np.float64); k(consts)
        g.nconsts, g.consts = consts.size, f64p(consts)
        ed = (POINTER(c_double) * max(1, len(elemdata)))()
        for i, a in enumerate(elemdata):
            a = np.ascontiguousarray(a, np.float64); k(a)
            ed[i] = f64p(a)
        k(ed)
        g.nelemdata, g.elemdata = len(elemdata), ed
        fd = (POINTER(c_double) * max(1, len(fielddata)))()
        rows = np.zeros(max(1, len(fielddata)), np.int32)
        for i, a in enumerate(fielddata):
            a = np.ascontiguousarray(a, np.float64); k(a)
            fd[i] = f64p(a)
            rows[i] = a.shape[0]
        k(fd); k(rows)
        g.nfielddata, g.fielddata, g.fieldrows = len(fielddata), fd, i32p(rows)
        tm = (Term * len(terms))(*[Term(t[0], t[1], t[2], 0, t[3]) for t in terms]); k(tm)
        g.nterms, g.terms = len(terms), tm
        ds = (Dest * len(dests))()
        for i, (tfa, dfa, mult) in enumerate(dests):
            tfa = np.ascontiguousarray(tfa, np.int32); k(tfa)
            ds[i].tfaddr = i32p(tfa)
            if dfa is not None:
                dfa = np.ascontiguousarray(dfa, np.int32); k(dfa)
                ds[i].dofaddr = i32p(dfa)
            ds[i].multiplier = mult
        k(ds)
        g.ndests, g.dests = len(dests), ds

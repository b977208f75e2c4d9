"""Python side of the serving loop (include/slgpu.h, slgpu_server_*).

A template is a processed matrix handle; a request recomputes its values with
new per-element data and writes them into host arrays.  `Server.submit`
returns a ticket; `Server.wait` blocks until that request is done and returns
its timing record.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import abi


@dataclass
class UpdateSpec:
    """New per-element data for one array of one group, in mesh element order."""

    group: int
    kind: int          # abi.UPDATE_ELEMDATA, abi.UPDATE_FIELDDATA or abi.UPDATE_SCALES
    index: int
    values: np.ndarray  # [rows][count] float64, count = mesh elements of the group's type;
                        # scales: [nterms + ndests] term scales then destination multipliers


class PinnedArray:
    """Page-locked float64 host array owned by a context (slgpu_host_alloc)."""

    def __init__(self, lib, ctx, n: int):
        self.lib = lib
        p = ctypes.c_void_p()
        st = lib.slgpu_host_alloc(ctx, max(1, n) * 8, ctypes.byref(p))
        if st != abi.OK:
            raise abi.SlgpuError(st, "cannot allocate page-locked host memory")
        self.ptr = p
        self.n = n
        self.array = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), (max(1, n),))[:n]

    def close(self):
        if self.ptr:
            self.lib.slgpu_host_free(self.ptr)
            self.ptr = None


class Server:
    def __init__(self, lib, ctx, nslots: int = 4):
        self.lib = lib
        self.ctx = ctx
        h = ctypes.c_void_p()
        st = lib.slgpu_server_create(ctx, nslots, ctypes.byref(h))
        if st != abi.OK:
            raise abi.SlgpuError(st, "cannot create a server")
        self.h = h
        self._keep = {}

    def submit_template(self, handle: int, constrained, precision: int) -> int:
        """Queues the first process() of an unprocessed matrix (pattern build)."""
        c = np.ascontiguousarray(constrained, dtype=np.uint8) if constrained is not None else None
        self._keep_c = c
        t = ctypes.c_int64()
        ptr = c.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if c is not None else None
        st = self.lib.slgpu_server_submit_template(self.h, handle, ptr, precision, ctypes.byref(t))
        if st != abi.OK:
            buf = ctypes.create_string_buffer(2048)
            self.lib.slgpu_last_error(self.ctx, buf, 2048)
            raise abi.SlgpuError(st, buf.value.decode(errors="replace"))
        return t.value

    def submit(self, handle: int, precision: int, updates, A_out, D_out) -> int:
        """A_out / D_out: float64 arrays (numpy or PinnedArray.array) of nnzA / nnzD values."""
        ups = (abi.Update * max(1, len(updates)))()
        vals = []
        for i, u in enumerate(updates):
            v = np.ascontiguousarray(u.values, dtype=np.float64)
            if v.ndim == 1:
                v = v[:, None] if u.kind == abi.UPDATE_SCALES else v[None, :]
            vals.append(v)
            ups[i].group, ups[i].kind, ups[i].index = u.group, u.kind, u.index
            ups[i].rows, ups[i].count = v.shape[0], v.shape[1]
            ups[i].values = v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r = abi.Request()
        r.handle, r.precision, r.nupdates = handle, precision, len(updates)
        r.updates = ups
        r.Avals = A_out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r.Dvals = D_out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if D_out is not None and D_out.size else None
        t = ctypes.c_int64()
        st = self.lib.slgpu_server_submit(self.h, ctypes.byref(r), ctypes.byref(t))
        if st != abi.OK:
            buf = ctypes.create_string_buffer(2048)
            self.lib.slgpu_last_error(self.ctx, buf, 2048)
            raise abi.SlgpuError(st, buf.value.decode(errors="replace"))
        # Outputs must stay alive until the request is done (inputs are copied).
        self._keep[t.value] = (A_out, D_out)
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0) -> abi.RequestStats:
        s = abi.RequestStats()
        st = self.lib.slgpu_server_wait(self.h, ticket, timeout_s, ctypes.byref(s))
        if st != abi.OK:
            buf = ctypes.create_string_buffer(2048)
            self.lib.slgpu_server_error(self.h, ticket, buf, 2048)
            raise abi.SlgpuError(st, buf.value.decode(errors="replace") or "request not done")
        self.lib.slgpu_server_release(self.h, ticket)
        self._keep.pop(ticket, None)
        return s

    def prepare(self, handle: int, precision: int):
        """Grows every slot's device scratch for requests on a template (no requests pending)."""
        st = self.lib.slgpu_server_prepare(self.h, handle, precision)
        if st != abi.OK:
            buf = ctypes.create_string_buffer(2048)
            self.lib.slgpu_last_error(self.ctx, buf, 2048)
            raise abi.SlgpuError(st, buf.value.decode(errors="replace"))

    def pending(self) -> int:
        return int(self.lib.slgpu_server_pending(self.h))

    def close(self):
        if self.h:
            self.lib.slgpu_server_destroy(self.h)
            self.h = None
            self._keep.clear()

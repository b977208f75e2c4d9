"""ctypes front-end for the sparselizard workload drivers.

A driver library (built from sparselizard_b200/driver/slz_driver.cpp against a
sparselizard build) exposes ``slz_run`` and result getters.  This module runs a
workload through one such library and returns the assembled A/D CSR blocks,
Ainds/Dinds and b as numpy arrays, plus per-phase wall times.

Workload ids and parameters follow ``slz_run``:
  1 Poisson on quads            params = [order]
  2 elasticity on hexes         params = [order, integration delta]
  3 p-adaptive Helmholtz on tets params = []
  4 eddy currents on tets       params = [order, frequency, sigma0..sigma3]
  5 Poisson on quads, non-zero Dirichlet value on the boundary   params = [order]
  6 elasticity on hexes, prescribed displacement of the z = 0 face params = [order]
  7 Poisson on quads, per-element coefficient (slz_set_element_values) params = [order]
  8 Poisson on quads after another formulation was generated         params = [order]
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

POISSON_QUAD, ELASTICITY_HEX, HELMHOLTZ_TET, EDDY_TET, POISSON_DIRICHLET, ELASTICITY_DIRICHLET, POISSON_KFIELD, POISSON_AFTER_OTHER = 1, 2, 3, 4, 5, 6, 7, 8


@dataclass
class Assembled:
    Arows: np.ndarray
    Acols: np.ndarray
    Avals: np.ndarray
    Drows: np.ndarray
    Dcols: np.ndarray
    Dvals: np.ndarray
    Ainds: np.ndarray
    Dinds: np.ndarray
    b: np.ndarray
    ndofs: int
    times: np.ndarray  # [reps, 3]: generate, A, b wall seconds

    @property
    def nnz(self) -> int:
        return int(self.Acols.size + self.Dcols.size)


_LIBS: dict[str, ctypes.CDLL] = {}


def openblas_path() -> str | None:
    """The OpenBLAS shared library bundled with scipy (it exports
    scipy_cblas_dgemm), located through the installed scipy package."""
    import glob
    import importlib.util

    spec = importlib.util.find_spec("scipy")
    if spec is None or not spec.submodule_search_locations:
        return None
    site = os.path.dirname(list(spec.submodule_search_locations)[0])
    hits = sorted(glob.glob(os.path.join(site, "scipy.libs", "libscipy_openblas*.so")))
    return hits[0] if hits else None


def dgemm_name(lib: ctypes.CDLL) -> str:
    """Which dgemm the PETSc/CBLAS stand-in of a driver library uses."""
    f = lib.slshim_dgemm_name
    f.restype = ctypes.c_char_p
    return f().decode(errors="replace")


def load(path: str) -> ctypes.CDLL:
    path = os.path.abspath(path)
    if not os.environ.get("SLSHIM_OPENBLAS"):
        # The stand-in's cblas_dgemm dlopens SLSHIM_OPENBLAS on its first call.
        os.environ["SLSHIM_OPENBLAS"] = openblas_path() or ""
    if path not in _LIBS:
        if not os.path.exists(path):
            raise FileNotFoundError(f"driver library {path} is not built")
        mode = getattr(os, "RTLD_DEEPBIND", 0) | os.RTLD_LOCAL | os.RTLD_NOW
        lib = ctypes.CDLL(path, mode=mode)
        lib.slz_run.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double)]
        lib.slz_run.restype = ctypes.c_int
        lib.slz_last_error.restype = ctypes.c_char_p
        lib.slz_result_size.argtypes = [ctypes.c_int]
        lib.slz_result_size.restype = ctypes.c_longlong
        lib.slz_result_copy.argtypes = [ctypes.c_void_p] * 9
        lib.slz_result_copy.restype = None
        lib.slz_set_threads.argtypes = [ctypes.c_int]
        _LIBS[path] = lib
    return _LIBS[path]


def run(lib_path: str, workload: int, msh: str, params=(), reps: int = 1, threads: int | None = None) -> Assembled:
    lib = load(lib_path)
    if threads is not None:
        lib.slz_set_threads(int(threads))
    p = (ctypes.c_double * max(1, len(params)))(*params)
    times = np.zeros((reps, 3))
    rc = lib.slz_run(workload, msh.encode(), p, reps, times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError(f"slz_run({workload}) failed: {lib.slz_last_error().decode(errors='replace')}")
    size = lambda i: int(lib.slz_result_size(i))
    out = dict(
        Arows=np.empty(size(1), np.int32), Acols=np.empty(size(2), np.int32), Avals=np.empty(size(2), np.float64),
        Drows=np.empty(size(3), np.int32), Dcols=np.empty(size(4), np.int32), Dvals=np.empty(size(4), np.float64),
        Ainds=np.empty(size(5), np.int32), Dinds=np.empty(size(6), np.int32), b=np.empty(size(7), np.float64),
    )
    order = ["Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals", "Ainds", "Dinds", "b"]
    lib.slz_result_copy(*[out[k].ctypes.data for k in order])
    return Assembled(ndofs=size(0), times=times, **out)

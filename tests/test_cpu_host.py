"""CPU-only checks: C-ABI library exports, oracle host logic, mesh files."""
import ctypes
import os
import re

import numpy as np
import pytest

import _pipeline as P
from sparselizard_b200 import abi, meshgen

HEADER = os.path.join(P.ROOT, "include", "slgpu.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t|double)\s+\**(slgpu_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    assert set(names) == set(abi.SIGNATURES), "python binding and header disagree"


def test_no_device_is_a_clean_error():
    """Without a GPU the context refuses to start (there is no CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(abi.SlgpuError) as e:
        abi.Context(0)
    assert e.value.status == abi.E_NODEVICE


def test_record_only_context_records_and_refuses():
    c = abi.Context(0, flags=abi.CTX_RECORD_ONLY)
    L = c.lib
    xyz = np.zeros(12)
    c.check(L.slgpu_mesh_set_nodes(c.h, 0, 4, abi.f64p(xyz)))
    conn = np.array([0, 1, 2, 3], np.int32)
    c.check(L.slgpu_mesh_set_elements(c.h, 0, 3, 4, 1, abi.i32p(conn)))
    h = ctypes.c_int()
    c.check(L.slgpu_matrix_create(c.h, 4, ctypes.byref(h)))
    con = np.zeros(4, np.uint8)
    st = L.slgpu_matrix_process(c.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), 0, None)
    assert st == abi.E_NODEVICE
    c.close()


def test_bad_connectivity_rejected_on_host():
    c = abi.Context(0, flags=abi.CTX_RECORD_ONLY)
    xyz = np.zeros(12)
    c.check(c.lib.slgpu_mesh_set_nodes(c.h, 0, 4, abi.f64p(xyz)))
    conn = np.array([0, 1, 2, 7], np.int32)
    assert c.lib.slgpu_mesh_set_elements(c.h, 0, 3, 4, 1, abi.i32p(conn)) == abi.E_ARG
    c.close()


def test_meshgen_quad(tmp_path):
    p = tmp_path / "q.msh"
    info = meshgen.quad_mesh(str(p), 4, jitter=0.2, seed=1)
    assert info == {"nelem": 16, "nnodes": 25}
    text = p.read_text()
    assert text.startswith("$MeshFormat\n2.2 0 8")
    # same seed -> same file
    p2 = tmp_path / "q2.msh"
    meshgen.quad_mesh(str(p2), 4, jitter=0.2, seed=1)
    assert p2.read_text() == text


def test_meshgen_tets_positive_and_conforming(tmp_path):
    n = 3
    meshgen.tet_mesh(str(tmp_path / "t.msh"), n)
    lines = (tmp_path / "t.msh").read_text().split("$Nodes\n")[1].split("$EndNodes")[0].strip().split("\n")
    nodes = np.array([[float(v) for v in l.split()[1:]] for l in lines[1:]])
    els = (tmp_path / "t.msh").read_text().split("$Elements\n")[1].split("$EndElements")[0].strip().split("\n")[1:]
    tets = np.array([[int(v) for v in l.split()[5:]] for l in els if l.split()[1] == "4"]) - 1
    assert tets.shape == (6 * n ** 3, 4)
    p = nodes[tets]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6
    assert np.all(vol > 0)
    assert abs(vol.sum() - 1.0) < 1e-12
    # conforming: every interior face shared by exactly two tets
    faces = {}
    for t in tets:
        for f in ([0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]):
            k = tuple(sorted(t[f]))
            faces[k] = faces.get(k, 0) + 1
    assert max(faces.values()) == 2
    assert sum(1 for v in faces.values() if v == 1) == 6 * 2 * n * n

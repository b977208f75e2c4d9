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


def test_binding_argument_counts_match_header():
    """Each ctypes signature in abi.SIGNATURES takes as many arguments as
    the header's prototype."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    protos = dict(re.findall(r"^\s*(?:int|void|int64_t|double|const char)\s*\**\s*(slgpu_\w+)\s*\(([^)]*)\)\s*;", text, re.M))
    assert set(protos) == set(abi.SIGNATURES)
    bad = []
    for name, args in protos.items():
        n = 0 if args.strip() in ("", "void") else args.count(",") + 1
        if name in abi.SIGNATURES and len(abi.SIGNATURES[name][1]) != n:
            bad.append((name, n, len(abi.SIGNATURES[name][1])))
    assert not bad, f"argument counts differ (name, header, binding): {bad}"


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


def _add_record_group(c, gb, xyz, conn):
    L = c.lib
    c.check(L.slgpu_mesh_set_nodes(c.h, 0, xyz.size // 3, abi.f64p(xyz)))
    c.check(L.slgpu_mesh_set_elements(c.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))
    h = ctypes.c_int()
    c.check(L.slgpu_matrix_create(c.h, 60, ctypes.byref(h)))
    c.check(L.slgpu_matrix_add_group(c.h, h, ctypes.byref(gb.g), None))
    return h.value


def _symmetry(c, h, nterms, gi=0):
    m = np.zeros(nterms, np.int32)
    s, pt = ctypes.c_int32(), ctypes.c_int32()
    c.check(c.lib.slgpu_matrix_group_symmetry(c.h, h, gi, m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(s),
                                              ctypes.byref(pt)))
    return m, s.value, pt.value


def test_symmetry_detection_synthetic():
    """Mirror terms: copied tables and coefficients that differ only in the
    operand order of a product are found; scales that differ turn the
    symmetric contraction off and back on; one changed constant, or distinct
    tables, leave a group without mirrors."""
    from _synthetic import group

    c = abi.Context(0, flags=abi.CTX_RECORD_ONLY)
    L = c.lib
    gb, xyz, conn = group(np.random.Generator(np.random.PCG64(3)), ntf=6, ndof=6, nterms=5, symmetric=True, ndests=1)
    h = _add_record_group(c, gb, xyz, conn)
    m, s, pt = _symmetry(c, h, 5)
    assert m.tolist() == [1, 0, 3, 2, 4] and s == 1 and pt == -1
    sc = np.zeros(5)
    c.check(L.slgpu_matrix_get_scales(c.h, h, 0, abi.f64p(sc), None))
    sc2 = sc.copy()
    sc2[1] *= 1.0000001
    c.check(L.slgpu_matrix_set_scales(c.h, h, 0, abi.f64p(sc2), None))
    assert _symmetry(c, h, 5)[1] == 0
    c.check(L.slgpu_matrix_set_scales(c.h, h, 0, abi.f64p(sc), None))
    assert _symmetry(c, h, 5)[1] == 1

    # A different constant in one mirror's coefficient: no mirror for it.
    gb, xyz, conn = group(np.random.Generator(np.random.PCG64(3)), ntf=6, ndof=6, nterms=4, symmetric=True, ndests=1)
    nodes = [(gb.g.nodes[k].op, gb.g.nodes[k].a, gb.g.nodes[k].b, gb.g.nodes[k].c) for k in range(gb.g.nnodes)]
    t3 = gb.g.terms[3].coef_node
    gb.g.nodes[t3].b = 2  # x + detJ instead of x + coordinate
    h = _add_record_group(c, gb, xyz, conn)
    m, s, _ = _symmetry(c, h, 4)
    assert (m == -1).all() and s == 0
    assert nodes[t3][0] == abi.OP_ADD

    # Independent random tables: not symmetric.
    gb, xyz, conn = group(np.random.Generator(np.random.PCG64(3)), ntf=6, ndof=6, nterms=4, ndests=1)
    h = _add_record_group(c, gb, xyz, conn)
    m, s, _ = _symmetry(c, h, 4)
    assert (m == -1).all() and s == 0
    c.close()


def test_transposed_partner_detection():
    """Two groups with ntf and ndof swapped and the tables of each term
    swapped are partners; replacing one group's element data or scaling one
    term of one group ends the pairing, and restoring it brings it back.  A
    coefficient that reads another constant is not a partner's."""
    from _synthetic import group

    c = abi.Context(0, flags=abi.CTX_RECORD_ONLY)
    L = c.lib
    rng = np.random.Generator(np.random.PCG64(9))
    gb, xyz, conn = group(rng, ntf=12, ndof=8, nterms=4, ndests=1)
    g1 = gb.g
    g2 = abi.Group.from_buffer_copy(g1)
    g2.ntf, g2.ndof = g1.ndof, g1.ntf
    terms2 = (abi.Term * g1.nterms)(*[abi.Term(g1.terms[t].dof_table, g1.terms[t].tf_table, g1.terms[t].coef_node, 0,
                                               g1.terms[t].scale) for t in range(g1.nterms)])
    g2.terms = terms2
    c.check(L.slgpu_mesh_set_nodes(c.h, 0, xyz.size // 3, abi.f64p(xyz)))
    c.check(L.slgpu_mesh_set_elements(c.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))
    h = ctypes.c_int()
    c.check(L.slgpu_matrix_create(c.h, 60, ctypes.byref(h)))
    c.check(L.slgpu_matrix_add_group(c.h, h, ctypes.byref(g1), None))
    c.check(L.slgpu_matrix_add_group(c.h, h, ctypes.byref(g2), None))
    h = h.value
    partners = lambda: [_symmetry(c, h, 4, gi)[2] for gi in (0, 1)]
    assert partners() == [1, 0]
    e_new = rng.lognormal(0.0, 0.4, g1.nelem)
    e_old = np.ctypeslib.as_array(g1.elemdata[0], (g1.nelem,)).copy()
    c.check(L.slgpu_matrix_set_elemdata(c.h, h, 1, 0, abi.f64p(e_new)))
    assert partners() == [-1, -1]
    c.check(L.slgpu_matrix_set_elemdata(c.h, h, 1, 0, abi.f64p(e_old)))
    assert partners() == [1, 0]
    sc = np.zeros(4)
    c.check(L.slgpu_matrix_get_scales(c.h, h, 0, abi.f64p(sc), None))
    sc2 = sc.copy()
    sc2[2] *= 2.0
    c.check(L.slgpu_matrix_set_scales(c.h, h, 0, abi.f64p(sc2), None))
    assert partners() == [-1, -1]
    c.check(L.slgpu_matrix_set_scales(c.h, h, 1, abi.f64p(sc2), None))
    assert partners() == [1, 0]

    # A partner whose coefficients read another constant: no pair.
    g3 = abi.Group.from_buffer_copy(g2)
    nodes3 = (abi.Node * g1.nnodes)(*[abi.Node(g1.nodes[k].op, g1.nodes[k].a, g1.nodes[k].b, g1.nodes[k].c)
                                      for k in range(g1.nnodes)])
    assert nodes3[1].op == abi.OP_CONST
    nodes3[1].a = 3
    g3.nodes = nodes3
    h3 = ctypes.c_int()
    c.check(L.slgpu_matrix_create(c.h, 60, ctypes.byref(h3)))
    c.check(L.slgpu_matrix_add_group(c.h, h3, ctypes.byref(g1), None))
    c.check(L.slgpu_matrix_add_group(c.h, h3, ctypes.byref(g3), None))
    assert [_symmetry(c, h3.value, 4, gi)[2] for gi in (0, 1)] == [-1, -1]
    c.close()


def test_symmetry_detection_workloads(gpu_lib, tmp_path):
    """On the drop-in's lowering (record-only context): every group of the
    p-adaptive Helmholtz problem (grad-grad and mass terms) has mirror terms,
    pairing d/dx_a with d/dx_b; of the nine component blocks of the
    order-2 elasticity problem, the three diagonal ones do, and the others
    form three transposed pairs; the harmonic hcurl groups are symmetric."""
    n = 2
    rng = np.random.Generator(np.random.PCG64(7))
    tags = meshgen.ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
    msh = str(tmp_path / "t.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=2, element_tags=tags)
    from sparselizard_b200 import workloads as W

    r = P.record_symmetry(W.HELMHOLTZ_TET, msh, [])
    assert len(r["symmetric"]) >= 3 and (r["symmetric"] == 1).all()
    off = 0
    for nt in r["nterms"]:
        m = r["mirror"][off:off + nt]
        assert (m[m] == np.arange(nt)).all() and (m != np.arange(nt)).sum() == 6  # three swapped pairs
        off += nt
    msh = str(tmp_path / "h.msh")
    meshgen.hex_mesh(msh, 2, jitter=0.15, seed=1)
    r = P.record_symmetry(W.ELASTICITY_HEX, msh, [2, -2])
    assert r["symmetric"].tolist() == [2, 0, 0, 0, 2, 0, 0, 0, 2]
    # Off-diagonal blocks (u_a, u_b) and (u_b, u_a) are transposed partners.
    assert r["partner"].tolist() == [-1, 3, 6, 1, -1, 7, 2, 5, -1]
    # Harmonic hcurl eddy currents (curl-curl and sigma dt terms, two harmonics): both groups are
    # symmetric up to the order of factors.
    rng = np.random.Generator(np.random.PCG64(11))
    tags = meshgen.MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
    msh = str(tmp_path / "e.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=4, element_tags=tags)
    r = P.record_symmetry(W.EDDY_TET, msh, [2, 1.0e3, 1e3, 5e5, 2e6, 6e7])
    assert len(r["symmetric"]) >= 1 and (r["symmetric"] > 0).all() and (r["partner"] == -1).all()


def test_bench_roofline_of_dominant_family():
    """bench.roofline_of names the family with the most device time, divides
    its algorithmic work by its event time, and scales the ncu traffic per
    element to the launch (8x the 32^3 capture at 64^3)."""
    import bench

    stats = {"coefficients": {"ms": 8.2, "launches": 10, "work": 3.1e10},
             "contract_split": {"ms": 75.0, "launches": 60, "work": 1.5e17},
             "row_values": {"ms": 84.0, "launches": 10, "work": 2.73e11}}
    r = bench.roofline_of(stats, "c2", 64)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and "k_row_values" in r["kernel"]
    assert abs(r["achieved"] - 2.73e11 / 84e-3 / 1e9) < 1e-6 and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert abs(r["ms_per_launch"] - 8.4) < 1e-12
    assert abs(r["traffic"] - 8 * bench.traffic_per_launch("c2", "row_values", 32, 1)) < 1.0
    stats["contract_split"]["ms"] = 100.0
    r = bench.roofline_of(stats, "c2", 64)
    assert r["bound"] == "tensor" and r["unit"] == "TFLOP/s" and abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert bench.roofline_of(stats, "c3", 32)["traffic"] is None

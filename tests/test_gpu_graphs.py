"""CUDA-graph replay of process() on a resident pattern.

The value path (coefficients, contractions, CSR values) of a matrix is
captured into a graph on the second process() with unchanged launches and
replayed afterwards.  Replays must give the same values bit for bit as the
ungraphed path, also after in-place changes of per-element data, node
coordinates, term scales and destination multipliers (read by the kernels at
run time).  Both CSR value kernels (streaming warps, warp per row) must agree
bit for bit as well.
"""
import ctypes

import numpy as np
import pytest

import _synthetic as S
from sparselizard_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def _setup(ctx, rng, mesh_id, grid, ntf, ndof, nterms, ngp1, ndofs):
    gb, xyz, conn = S.group(rng, nelem_grid=grid, ntf=ntf, ndof=ndof, nterms=nterms, ngp1=ngp1, norient=2, ndests=2,
                            ndofs=ndofs)
    g = gb.g
    g.mesh = mesh_id
    L = ctx.lib
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, mesh_id, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, mesh_id, 3, 4, conn.size // 4, abi.i32p(conn)))
    h = ctypes.c_int()
    ctx.check(L.slgpu_matrix_create(ctx.h, ndofs, ctypes.byref(h)))
    ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g), None))
    con = (rng.random(ndofs) < 0.1).astype(np.uint8)
    return dict(gb=gb, h=h.value, con=con, xyz=xyz, nelem=g.nelem, nterms=g.nterms, ndests=g.ndests, mesh=mesh_id)


def _process(ctx, t, precision):
    L = ctx.lib
    info = abi.CsrInfo()
    ctx.check(L.slgpu_matrix_process(ctx.h, t["h"], t["con"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), precision,
                                     ctypes.byref(info)))
    A, D = np.zeros(max(1, info.nnzA)), np.zeros(max(1, info.nnzD))
    ctx.check(L.slgpu_matrix_download_values(ctx.h, t["h"], abi.f64p(A), abi.f64p(D)))
    return A[: info.nnzA].copy(), D[: info.nnzD].copy()


def _run(ctx, t, precision, graphs, edits):
    """process() after each edit (a callable or None); returns the values."""
    ctx.check(ctx.lib.slgpu_ctx_set_graphs(ctx.h, 1 if graphs else 0))
    out = []
    for e in edits:
        if e is not None:
            e()
        out.append(_process(ctx, t, precision))
    return out


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_SPLIT])
def test_graph_replay_matches_ungraphed(ctx, precision):
    rng = np.random.Generator(np.random.PCG64(21))
    t = _setup(ctx, rng, 11 + precision, 60, 9, 9, 4, 3, 3000)
    L = ctx.lib
    e1 = rng.lognormal(0.0, 0.4, t["nelem"])
    e2 = rng.lognormal(0.0, 0.4, t["nelem"])
    xyz2 = t["xyz"] * 1.01
    scales = rng.uniform(0.5, 2.0, t["nterms"])
    mults = rng.uniform(-2.0, 2.0, t["ndests"])

    def set_e(v):
        return lambda: ctx.check(L.slgpu_matrix_set_elemdata(ctx.h, t["h"], 0, 0, abi.f64p(v)))

    def set_nodes(v):
        return lambda: ctx.check(L.slgpu_mesh_set_nodes(ctx.h, t["mesh"], v.size // 3, abi.f64p(v)))

    def set_scales(ts, dm):
        return lambda: ctx.check(L.slgpu_matrix_set_scales(ctx.h, t["h"], 0, abi.f64p(ts) if ts is not None else None,
                                                           abi.f64p(dm) if dm is not None else None))

    orig_scales = np.zeros(t["nterms"])
    orig_mults = np.zeros(t["ndests"])
    ctx.check(L.slgpu_matrix_get_scales(ctx.h, t["h"], 0, abi.f64p(orig_scales), abi.f64p(orig_mults)))
    edits = [set_e(e1), None, None, set_e(e2), set_nodes(xyz2), set_scales(scales, None), None,
             set_scales(None, mults), None, set_nodes(t["xyz"]), set_scales(orig_scales, orig_mults)]
    g0 = L.slgpu_graph_launches(ctx.h)
    with_graph = _run(ctx, t, precision, True, edits)
    replays = L.slgpu_graph_launches(ctx.h) - g0
    without = _run(ctx, t, precision, False, edits)
    ctx.check(L.slgpu_ctx_set_graphs(ctx.h, 1))
    assert replays >= 8, f"only {replays} graph replays"
    for i, ((a, d), (a0, d0)) in enumerate(zip(with_graph, without)):
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(d)), f"call {i}: non-finite values"
        assert np.array_equal(a, a0) and np.array_equal(d, d0), f"call {i}: graph != ungraphed"
    # The edits changed the values (the replays are not stale copies).
    assert not np.array_equal(with_graph[2][0], with_graph[3][0])
    assert not np.array_equal(with_graph[3][0], with_graph[4][0])
    assert not np.array_equal(with_graph[6][0], with_graph[7][0])


def test_graph_kernel_stats_and_launch_count(ctx):
    rng = np.random.Generator(np.random.PCG64(22))
    t = _setup(ctx, rng, 13, 40, 4, 4, 3, 2, 1200)
    L = ctx.lib
    ctx.check(L.slgpu_ctx_set_graphs(ctx.h, 1))
    for _ in range(3):
        _process(ctx, t, abi.PREC_FP64)
    k0 = L.slgpu_kernel_launches(ctx.h)
    g0 = L.slgpu_graph_launches(ctx.h)
    _process(ctx, t, abi.PREC_FP64)
    assert L.slgpu_graph_launches(ctx.h) == g0 + 1
    # coefficients, contraction, CSR values
    assert L.slgpu_kernel_launches(ctx.h) - k0 == 3
    ms, n, w = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
    for fam in ("coefficients", "contract_fp64", "row_values"):
        ctx.check(L.slgpu_kernel_stats(ctx.h, fam.encode(), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(w)))
        assert n.value == 1 and ms.value > 0 and w.value > 0, fam


def test_value_kernels_agree(tmp_path):
    """The streaming-warp, warp-per-row and thread-per-row CSR value kernels,
    each forced in a child process, give the same values bit for bit
    (incidence widths 4, 9 and 40; the thread kernel on the short rows)."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    res = {}
    for k in ("stream", "warp", "thread"):
        out = str(tmp_path / f"{k}.npz")
        env = dict(os.environ, SLGPU_ROW_KERNEL=k)
        subprocess.run([sys.executable, os.path.join(here, "_rowkernel_child.py"), out], env=env, check=True, timeout=600)
        res[k] = np.load(out)
    for key in res["warp"].files:
        for k in ("stream", "thread"):
            a, b = res[k][key], res["warp"][key]
            assert np.all(np.isfinite(a)), key
            assert np.array_equal(a, b), f"{key}: {k} and warp-per-row value kernels differ"


def test_graph_replay_with_transposed_pair(ctx):
    """A matrix with two transposed-partner groups, edited so that the pairing
    turns off and on again (a scale of one group; element data of one group,
    then of both): replayed graphs give the ungraphed values bit for bit, and
    the pairing follows the edits."""
    rng = np.random.Generator(np.random.PCG64(23))
    ndofs = 2500
    gb, xyz, conn = S.group(rng, nelem_grid=40, ntf=12, ndof=8, nterms=4, ngp1=3, norient=2, ndests=1, ndofs=ndofs)
    g1 = gb.g
    g2 = abi.Group.from_buffer_copy(g1)
    g2.ntf, g2.ndof = g1.ndof, g1.ntf
    terms2 = (abi.Term * g1.nterms)(*[abi.Term(g1.terms[t].dof_table, g1.terms[t].tf_table, g1.terms[t].coef_node, 0,
                                               g1.terms[t].scale) for t in range(g1.nterms)])
    g2.terms = terms2
    dest2 = (abi.Dest * 1)()
    dest2[0].tfaddr, dest2[0].dofaddr, dest2[0].multiplier = g1.dests[0].dofaddr, g1.dests[0].tfaddr, 1.5
    g2.dests = dest2
    mesh_id = 31
    g1.mesh = g2.mesh = mesh_id
    L = ctx.lib
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, mesh_id, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, mesh_id, 3, 4, conn.size // 4, abi.i32p(conn)))
    h = ctypes.c_int()
    ctx.check(L.slgpu_matrix_create(ctx.h, ndofs, ctypes.byref(h)))
    ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g1), None))
    ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g2), None))
    t = dict(h=h.value, con=(rng.random(ndofs) < 0.1).astype(np.uint8))
    sc = np.zeros(g1.nterms)
    ctx.check(L.slgpu_matrix_get_scales(ctx.h, t["h"], 0, abi.f64p(sc), None))
    sc2 = sc.copy()
    sc2[1] *= 3.0
    e_old = np.ctypeslib.as_array(g1.elemdata[0], (g1.nelem,)).copy()
    e_new = rng.lognormal(0.0, 0.4, g1.nelem)

    def set_scales(gi, v):
        return lambda: ctx.check(L.slgpu_matrix_set_scales(ctx.h, t["h"], gi, abi.f64p(v), None))

    def set_e(gi, v):
        return lambda: ctx.check(L.slgpu_matrix_set_elemdata(ctx.h, t["h"], gi, 0, abi.f64p(v)))

    def partner():
        pt = ctypes.c_int32()
        ctx.check(L.slgpu_matrix_group_symmetry(ctx.h, t["h"], 0, None, None, ctypes.byref(pt)))
        return pt.value

    edits = [None, None, set_scales(0, sc2), None, None, set_scales(1, sc2), None, None, set_e(1, e_new), None,
             set_e(0, e_new), None, None, set_e(0, e_old), set_e(1, e_old), set_scales(0, sc), set_scales(1, sc), None]
    paired = [True, True, False, False, False, True, True, True, False, False, True, True, True, False, True, False, True,
              True]

    def run(graphs):
        ctx.check(L.slgpu_ctx_set_graphs(ctx.h, 1 if graphs else 0))
        out = []
        for e, p in zip(edits, paired):
            if e is not None:
                e()
            assert (partner() == 1) == p
            out.append(_process(ctx, t, abi.PREC_SPLIT))
        return out

    g0 = L.slgpu_graph_launches(ctx.h)
    with_graph = run(True)
    replays = L.slgpu_graph_launches(ctx.h) - g0
    without = run(False)
    ctx.check(L.slgpu_ctx_set_graphs(ctx.h, 1))
    ctx.check(L.slgpu_matrix_destroy(ctx.h, t["h"]))
    assert replays >= 5, f"only {replays} graph replays"
    for i, ((a, d), (a0, d0)) in enumerate(zip(with_graph, without)):
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(d)), f"call {i}: non-finite values"
        assert np.array_equal(a, a0) and np.array_equal(d, d0), f"call {i}: graph != ungraphed"
    assert not np.array_equal(with_graph[1][0], with_graph[2][0])


def test_pattern_serial_and_page_locked_downloads(ctx):
    """slgpu_matrix_pattern_serial: unchanged across process() calls on the same
    addresses and constraints, new when the constraints change.  Values
    downloaded into page-locked host memory (slgpu_host_register) equal those
    downloaded into pageable memory, and stay equal after unregistering."""
    rng = np.random.Generator(np.random.PCG64(41))
    t = _setup(ctx, rng, 31, 60, 9, 9, 4, 3, 3000)
    L = ctx.lib
    s = ctypes.c_uint64()
    ctx.check(L.slgpu_matrix_pattern_serial(ctx.h, t["h"], ctypes.byref(s)))
    assert s.value == 0
    A0, D0 = _process(ctx, t, abi.PREC_FP64)
    ctx.check(L.slgpu_matrix_pattern_serial(ctx.h, t["h"], ctypes.byref(s)))
    s0 = s.value
    assert s0 > 0
    _process(ctx, t, abi.PREC_FP64)
    ctx.check(L.slgpu_matrix_pattern_serial(ctx.h, t["h"], ctypes.byref(s)))
    assert s.value == s0

    buf = np.zeros(A0.size + 1024)
    ctx.check(L.slgpu_host_register(ctx.h, buf.ctypes.data, buf.nbytes))
    D = np.zeros(max(1, D0.size))
    ctx.check(L.slgpu_matrix_download_values(ctx.h, t["h"], abi.f64p(buf), abi.f64p(D)))
    assert np.array_equal(buf[: A0.size], A0) and np.array_equal(D[: D0.size], D0)
    ctx.check(L.slgpu_host_unregister(ctx.h, buf.ctypes.data))
    buf[:] = 0
    ctx.check(L.slgpu_matrix_download_values(ctx.h, t["h"], abi.f64p(buf), abi.f64p(D)))
    assert np.array_equal(buf[: A0.size], A0)

    t["con"] = t["con"].copy()
    t["con"][::5] ^= 1
    _process(ctx, t, abi.PREC_FP64)
    ctx.check(L.slgpu_matrix_pattern_serial(ctx.h, t["h"], ctypes.byref(s)))
    assert s.value != s0


def test_shared_address_arrays(ctx):
    """A group added twice with the same host address arrays (the second copy
    with other term scales), with slgpu_matrix_share_addresses on and off:
    the same CSR values bit for bit and the same pattern serial (addresses are
    hashed by content either way)."""
    rng = np.random.Generator(np.random.PCG64(43))
    L = ctx.lib
    gb, xyz, conn = S.group(rng, nelem_grid=40, ntf=9, ndof=9, nterms=4, ngp1=3, norient=2, ndests=2, ndofs=3000)
    g1 = gb.g
    g1.mesh = 33
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, 33, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, 33, 3, 4, conn.size // 4, abi.i32p(conn)))
    g2 = abi.Group.from_buffer_copy(g1)
    terms2 = (abi.Term * g1.nterms)(*[abi.Term(g1.terms[t].tf_table, g1.terms[t].dof_table, g1.terms[t].coef_node, 0,
                                               0.5 + t) for t in range(g1.nterms)])
    g2.terms = terms2
    con = (rng.random(3000) < 0.1).astype(np.uint8)
    out = {}
    for share in (0, 1):
        h = ctypes.c_int()
        ctx.check(L.slgpu_matrix_create(ctx.h, 3000, ctypes.byref(h)))
        ctx.check(L.slgpu_matrix_share_addresses(ctx.h, h, share))
        ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g1), None))
        ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g2), None))
        A, D = _process(ctx, dict(h=h.value, con=con), abi.PREC_FP64)
        s = ctypes.c_uint64()
        ctx.check(L.slgpu_matrix_pattern_serial(ctx.h, h, ctypes.byref(s)))
        out[share] = (A, D, s.value)
        ctx.check(L.slgpu_matrix_destroy(ctx.h, h))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]

"""Serving loop: requests on resident templates, several in flight at once.

Each request carries new per-element coefficients (mesh element order) for a
processed template.  The test submits a mix of requests on several
templates, precisions and sizes to a 4-slot server at once, then runs every
request again alone -- through a 1-slot server and through the plain
set_elemdata + process path -- and requires the same values bit for bit
(the value path has a fixed summation order and no atomics).
"""
import ctypes

import numpy as np
import pytest

import _synthetic as S
from sparselizard_b200 import abi, serving

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def _template(ctx, rng, mesh_id, grid, ntf, ndof, nterms, ngp1, ndofs):
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
    info = abi.CsrInfo()
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), abi.PREC_FP64,
                                     ctypes.byref(info)))
    elems = np.ctypeslib.as_array(g.elems, (g.nelem,)).copy()
    return dict(gb=gb, handle=h.value, con=con, nnzA=info.nnzA, nnzD=info.nnzD, elems=elems, nmesh=conn.size // 4,
                split=ntf * ndof >= 64)


def _plain(ctx, t, values_mesh, precision):
    """The same values through set_elemdata + process (group element order)."""
    L = ctx.lib
    vg = np.ascontiguousarray(values_mesh[t["elems"]])
    ctx.check(L.slgpu_matrix_set_elemdata(ctx.h, t["handle"], 0, 0, abi.f64p(vg)))
    info = abi.CsrInfo()
    ctx.check(L.slgpu_matrix_process(ctx.h, t["handle"], t["con"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
                                     precision, ctypes.byref(info)))
    A, D = np.zeros(max(1, t["nnzA"])), np.zeros(max(1, t["nnzD"]))
    ctx.check(L.slgpu_matrix_download_values(ctx.h, t["handle"], abi.f64p(A), abi.f64p(D)))
    return A[: t["nnzA"]], D[: t["nnzD"]]


def test_served_results_same_alone_and_in_the_mix(ctx):
    rng = np.random.Generator(np.random.PCG64(7))
    temps = [
        _template(ctx, rng, 1, 40, 4, 4, 3, 2, 900),      # small, FP64 only
        _template(ctx, rng, 2, 60, 9, 9, 4, 3, 2000),     # split-eligible
        _template(ctx, rng, 3, 90, 10, 8, 5, 3, 6000),    # split-eligible, more elements
    ]
    reqs = []
    for k in range(18):
        t = temps[k % 3]
        prec = [abi.PREC_FP64, abi.PREC_SPLIT, abi.PREC_FP32][k % 3] if t["split"] else abi.PREC_FP64
        vals = rng.lognormal(0.0, 0.4, t["nmesh"])
        reqs.append((t, prec, vals))

    def run(nslots, which):
        srv = serving.Server(ctx.lib, ctx.h, nslots)
        outs = {}
        tickets = {}
        try:
            for i in which:
                t, prec, vals = reqs[i]
                A = np.full(t["nnzA"], np.nan)
                D = np.full(max(1, t["nnzD"]), np.nan)[: t["nnzD"]]
                up = serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vals)
                tickets[i] = srv.submit(t["handle"], prec, [up], A, D)
                outs[i] = (A, D)
                if nslots == 1:
                    srv.wait(tickets.pop(i))
            for i, tk in tickets.items():
                st = srv.wait(tk)
                assert st.status == abi.OK
        finally:
            srv.close()
        return outs

    mixed = run(4, range(len(reqs)))
    alone = run(1, range(len(reqs)))
    for i, (t, prec, vals) in enumerate(reqs):
        A, D = mixed[i]
        assert np.all(np.isfinite(A)) and np.all(np.isfinite(D))
        assert np.array_equal(A, alone[i][0]) and np.array_equal(D, alone[i][1]), f"request {i}: mixed != alone"
        pA, pD = _plain(ctx, t, vals, prec)
        assert np.array_equal(A, pA) and np.array_equal(D, pD), f"request {i}: served != process()"


def test_server_rejects_bad_requests(ctx):
    rng = np.random.Generator(np.random.PCG64(8))
    t = _template(ctx, rng, 4, 20, 4, 4, 2, 2, 300)
    srv = serving.Server(ctx.lib, ctx.h, 2)
    try:
        A, D = np.zeros(t["nnzA"]), np.zeros(max(1, t["nnzD"]))
        with pytest.raises(abi.SlgpuError):  # wrong element count
            srv.submit(t["handle"], abi.PREC_FP64, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, np.ones(3))], A, D)
        with pytest.raises(abi.SlgpuError):  # unknown template
            srv.submit(9999, abi.PREC_FP64, [], A, D)
        with pytest.raises(abi.SlgpuError):  # array index out of range
            srv.submit(t["handle"], abi.PREC_FP64, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 5, np.ones(t["nmesh"]))], A, D)
        # A valid request still runs after the rejected ones.
        tk = srv.submit(t["handle"], abi.PREC_FP64, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, np.ones(t["nmesh"]))], A, D)
        assert srv.wait(tk).status == abi.OK
    finally:
        srv.close()


def test_pinned_outputs_and_pending_count(ctx):
    rng = np.random.Generator(np.random.PCG64(9))
    t = _template(ctx, rng, 5, 50, 9, 9, 3, 3, 1500)
    srv = serving.Server(ctx.lib, ctx.h, 3)
    pins = []
    try:
        tickets = []
        for k in range(6):
            A = serving.PinnedArray(ctx.lib, ctx.h, t["nnzA"])
            D = serving.PinnedArray(ctx.lib, ctx.h, max(1, t["nnzD"]))
            pins += [A, D]
            vals = rng.lognormal(0.0, 0.3, t["nmesh"])
            tickets.append((srv.submit(t["handle"], abi.PREC_SPLIT, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vals)],
                                       A.array, D.array[: t["nnzD"]]), A, D, vals))
        for tk, A, D, vals in tickets:
            st = srv.wait(tk)
            assert st.status == abi.OK and st.done_s >= st.start_s >= st.submit_s
            pA, pD = _plain(ctx, t, vals, abi.PREC_SPLIT)
            assert np.array_equal(A.array, pA) and np.array_equal(D.array[: t["nnzD"]], pD)
        assert srv.pending() == 0
    finally:
        srv.close()
        for p in pins:
            p.close()


def test_prepare_and_page_locked_inputs(ctx):
    """slgpu_server_prepare sizes every slot ahead of the stream; inputs in
    page-locked memory are read in place.  Results equal process()."""
    rng = np.random.Generator(np.random.PCG64(10))
    t = _template(ctx, rng, 6, 70, 9, 9, 3, 3, 2500)
    srv = serving.Server(ctx.lib, ctx.h, 3)
    pins = []
    try:
        for prec in (abi.PREC_FP64, abi.PREC_SPLIT):
            srv.prepare(t["handle"], prec)
        tickets = []
        for k in range(6):
            prec = abi.PREC_SPLIT if k % 2 else abi.PREC_FP64
            vin = serving.PinnedArray(ctx.lib, ctx.h, t["nmesh"])
            vin.array[:] = rng.lognormal(0.0, 0.3, t["nmesh"])
            A = np.full(t["nnzA"], np.nan)
            D = np.full(max(1, t["nnzD"]), np.nan)[: t["nnzD"]]
            pins.append(vin)
            tk = srv.submit(t["handle"], prec, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vin.array)], A, D)
            tickets.append((tk, prec, vin.array.copy(), A, D))
        for tk, prec, vals, A, D in tickets:
            assert srv.wait(tk).status == abi.OK
            pA, pD = _plain(ctx, t, vals, prec)
            assert np.array_equal(A, pA) and np.array_equal(D, pD)
    finally:
        srv.close()
        for p in pins:
            p.close()


def test_served_frequency_requests(ctx):
    """Requests that carry new term scales and destination multipliers (a
    frequency of a harmonic problem) next to requests with new coefficients,
    in one mix: each result equals the template re-assembled with the same
    scales through slgpu_matrix_set_scales + process(), bit for bit, and the
    template's own scales are left unchanged."""
    rng = np.random.Generator(np.random.PCG64(17))
    t = _template(ctx, rng, 5, 50, 9, 9, 4, 3, 2500)
    g = t["gb"].g
    L = ctx.lib
    ts0, dm0 = np.zeros(g.nterms), np.zeros(g.ndests)
    ctx.check(L.slgpu_matrix_get_scales(ctx.h, t["handle"], 0, abi.f64p(ts0), abi.f64p(dm0)))
    reqs = []
    for k in range(8):
        prec = [abi.PREC_FP64, abi.PREC_SPLIT][k % 2]
        w = 2 * np.pi * 10.0 ** (k - 2)
        scales = np.concatenate([ts0 * (1.0 + 0.5 * w * (np.arange(g.nterms) % 2)), dm0 * (1.0 + 1e-3 * w)])
        reqs.append((prec, scales))
    srv = serving.Server(ctx.lib, ctx.h, 4)
    outs, tickets = [], []
    try:
        for prec, scales in reqs:
            A = np.full(t["nnzA"], np.nan)
            D = np.full(max(1, t["nnzD"]), np.nan)[: t["nnzD"]]
            tickets.append(srv.submit(t["handle"], prec, [serving.UpdateSpec(0, abi.UPDATE_SCALES, 0, scales)], A, D))
            outs.append((A, D))
            vals = rng.lognormal(0.0, 0.4, t["nmesh"])  # a coefficient request in between
            A2, D2 = np.zeros(t["nnzA"]), np.zeros(max(1, t["nnzD"]))[: t["nnzD"]]
            tickets.append(srv.submit(t["handle"], prec, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vals)], A2, D2))
        for tk in tickets:
            assert srv.wait(tk).status == abi.OK
        with pytest.raises(abi.SlgpuError):  # wrong length
            srv.submit(t["handle"], abi.PREC_FP64, [serving.UpdateSpec(0, abi.UPDATE_SCALES, 0, np.ones(3))], A, D)
    finally:
        srv.close()
    ts1, dm1 = np.zeros(g.nterms), np.zeros(g.ndests)
    ctx.check(L.slgpu_matrix_get_scales(ctx.h, t["handle"], 0, abi.f64p(ts1), abi.f64p(dm1)))
    assert np.array_equal(ts0, ts1) and np.array_equal(dm0, dm1), "a request changed the template's scales"
    # The template's element data as the plain path sees it: restore what
    # _template set (the coefficient requests never touch it).
    for (prec, scales), (A, D) in zip(reqs, outs):
        ctx.check(L.slgpu_matrix_set_scales(ctx.h, t["handle"], 0, abi.f64p(np.ascontiguousarray(scales[: g.nterms])),
                                            abi.f64p(np.ascontiguousarray(scales[g.nterms:]))))
        info = abi.CsrInfo()
        ctx.check(L.slgpu_matrix_process(ctx.h, t["handle"], t["con"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), prec,
                                         ctypes.byref(info)))
        pA, pD = np.zeros(max(1, t["nnzA"])), np.zeros(max(1, t["nnzD"]))
        ctx.check(L.slgpu_matrix_download_values(ctx.h, t["handle"], abi.f64p(pA), abi.f64p(pD)))
        assert np.array_equal(A, pA[: t["nnzA"]]) and np.array_equal(D, pD[: t["nnzD"]]), "served != set_scales + process()"
    ctx.check(L.slgpu_matrix_set_scales(ctx.h, t["handle"], 0, abi.f64p(ts0), abi.f64p(dm0)))


def test_server_admits_new_templates(ctx):
    """A new template (groups added, never processed: a new mesh or order)
    goes through the request queue: its first assembly runs when admitted,
    while coefficient requests on another template are in flight, and the
    new template then serves requests.  Its values equal a direct process()
    of an identical matrix."""
    rng = np.random.Generator(np.random.PCG64(23))
    old = _template(ctx, rng, 6, 40, 9, 9, 3, 3, 1500)
    gb, xyz, conn = S.group(rng, nelem_grid=30, ntf=8, ndof=8, nterms=3, ngp1=3, norient=2, ndests=2, ndofs=1200)
    g = gb.g
    g.mesh = 7
    L = ctx.lib
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, 7, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, 7, 3, 4, conn.size // 4, abi.i32p(conn)))
    hs = []
    for _ in range(2):
        h = ctypes.c_int()
        ctx.check(L.slgpu_matrix_create(ctx.h, 1200, ctypes.byref(h)))
        ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g), None))
        hs.append(h.value)
    con = (rng.random(1200) < 0.1).astype(np.uint8)
    srv = serving.Server(ctx.lib, ctx.h, 3)
    try:
        tk = []
        for k in range(4):
            vals = rng.lognormal(0.0, 0.4, old["nmesh"])
            A, D = np.zeros(old["nnzA"]), np.zeros(max(1, old["nnzD"]))[: old["nnzD"]]
            tk.append(srv.submit(old["handle"], abi.PREC_SPLIT, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vals)], A, D))
            if k == 1:
                tt = srv.submit_template(hs[0], con, abi.PREC_FP64)
        assert srv.wait(tt).status == abi.OK
        for t in tk:
            assert srv.wait(t).status == abi.OK
        ref = _direct(ctx, hs[1], con)
        nnzA, nnzD = ref[0].size, ref[1].size
        A, D = np.full(nnzA, np.nan), np.full(max(1, nnzD), np.nan)[:nnzD]
        vals = np.ones(conn.size // 4)
        elems = np.ctypeslib.as_array(g.elems, (g.nelem,))
        vals[elems] = np.ctypeslib.as_array(g.elemdata[0], (g.nelem,))
        t2 = srv.submit(hs[0], abi.PREC_FP64, [serving.UpdateSpec(0, abi.UPDATE_ELEMDATA, 0, vals)], A, D)
        assert srv.wait(t2).status == abi.OK
        assert np.array_equal(A, ref[0]) and np.array_equal(D, ref[1])
    finally:
        srv.close()
    A0, D0 = np.zeros(max(1, nnzA)), np.zeros(max(1, nnzD))
    ctx.check(L.slgpu_matrix_download_values(ctx.h, hs[0], abi.f64p(A0), abi.f64p(D0)))
    assert np.array_equal(A0[:nnzA], ref[0]) and np.array_equal(D0[:nnzD], ref[1])


def _direct(ctx, h, con):
    L = ctx.lib
    info = abi.CsrInfo()
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), abi.PREC_FP64, ctypes.byref(info)))
    A, D = np.zeros(max(1, info.nnzA)), np.zeros(max(1, info.nnzD))
    ctx.check(L.slgpu_matrix_download_values(ctx.h, h, abi.f64p(A), abi.f64p(D)))
    return A[: info.nnzA], D[: info.nnzD]


@pytest.mark.parametrize("order,precision,tol", [(1, abi.PREC_FP64, 1e-12), (3, abi.PREC_SPLIT, 1e-10)])
def test_served_sparselizard_template_matches_reference(ref_lib, gpu_lib, tmp_path, order, precision, tol):
    """A template built through sparselizard (the serving pool's Poisson
    formulation with a per-element coefficient field, assembled once with
    k = 1) serves a request carrying a new field k; the request's matrix must
    equal stock sparselizard's assembly of the same formulation with that k:
    bit-exact pattern, values within the tolerance of the precision."""
    import _pipeline as P
    from sparselizard_b200 import meshgen

    n = 40
    msh = str(tmp_path / "k.msh")
    meshgen.workload_mesh("quad", n, msh)
    ref = P.kfield("ref_kfield", msh, order, n * n, precision)
    got = P.kfield("serve_kfield", msh, order, n * n, precision)
    P.check_pattern(ref, got)
    P.check_values(ref, got, tol)

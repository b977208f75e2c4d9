"""Split-precision (Ozaki INT8 slices on tcgen05 tensor cores) contraction.

Element matrices from the split path are compared with the FP64 path on the
same inputs: relative Frobenius error per element matrix <= 1e-10 for the
split tier and <= 1e-6 for the FP32-level tier.  The drop-in check runs a
small elasticity problem through sparselizard with SLGPU_PRECISION=split.
"""
import ctypes

import numpy as np
import pytest

import _pipeline as P
import _synthetic as S
from sparselizard_b200 import abi, meshgen, workloads as W

pytestmark = pytest.mark.gpu


def _element_matrices(ctx, gb, xyz, conn, precision):
    """Element matrices through slgpu_matrix_* with one row per (element, tf)."""
    g = gb.g
    nelem, ntf, ndof = g.nelem, g.ntf, g.ndof
    tfaddr = (np.arange(nelem)[None, :] * ntf + np.arange(ntf)[:, None]).astype(np.int32)
    dofaddr = np.repeat(np.arange(ndof, dtype=np.int32)[:, None], nelem, axis=1)
    dest = (abi.Dest * 1)()
    dest[0].tfaddr, dest[0].dofaddr, dest[0].multiplier = abi.i32p(tfaddr), abi.i32p(dofaddr), 1.0
    g.ndests, g.dests = 1, dest
    L = ctx.lib
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, 0, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))
    ndofs = nelem * ntf
    h = ctypes.c_int()
    ctx.check(L.slgpu_matrix_create(ctx.h, ndofs, ctypes.byref(h)))
    ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g), None))
    info = abi.CsrInfo()
    con = np.zeros(ndofs, np.uint8)
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), precision,
                                     ctypes.byref(info)))
    rows, cols = np.zeros(ndofs + 1, np.int32), np.zeros(info.nnzA, np.int32)
    vals = np.zeros(info.nnzA)
    ctx.check(L.slgpu_matrix_download(ctx.h, h, abi.i32p(rows), abi.i32p(cols), abi.f64p(vals),
                                      abi.i32p(np.zeros(ndofs + 1, np.int32)), abi.i32p(np.zeros(1, np.int32)),
                                      abi.f64p(np.zeros(1))))
    ctx.check(L.slgpu_matrix_destroy(ctx.h, h))
    return vals.reshape(nelem, ntf * ndof)


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("seed,norient,nterms,ngp1", [(0, 1, 3, 3), (1, 3, 4, 4), (2, 2, 9, 3), (3, 2, 9, 4)])
def test_split_element_matrices(ctx, seed, norient, nterms, ngp1):
    rng = np.random.Generator(np.random.PCG64(seed))
    gb, xyz, conn = S.group(rng, nelem_grid=14, ntf=9, ndof=9, nterms=nterms, ngp1=ngp1, norient=norient, ndests=1)
    ref = _element_matrices(ctx, gb, xyz, conn, abi.PREC_FP64)
    for prec, tol in ((abi.PREC_SPLIT, 1e-10), (abi.PREC_FP32, 1e-6)):
        got = _element_matrices(ctx, gb, xyz, conn, prec)
        err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert err.max() <= tol, f"precision {prec}: per-element Frobenius error {err.max():.3e} > {tol:g}"


@pytest.mark.parametrize("seed,grid,ntf,ndof,norient,nterms,ngp1", [(4, 100, 20, 20, 3, 5, 4), (5, 40, 27, 27, 1, 9, 3)])
def test_split_many_tiles(ctx, seed, grid, ntf, ndof, norient, nterms, ngp1):
    """Several row tiles and more work items than multiprocessors, so that
    every CTA of the persistent kernel reuses its stages and accumulators."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gb, xyz, conn = S.group(rng, nelem_grid=grid, ntf=ntf, ndof=ndof, nterms=nterms, ngp1=ngp1, norient=norient, ndests=1)
    ref = _element_matrices(ctx, gb, xyz, conn, abi.PREC_FP64)
    for prec, tol in ((abi.PREC_SPLIT, 1e-10), (abi.PREC_FP32, 1e-6)):
        got = _element_matrices(ctx, gb, xyz, conn, prec)
        err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert err.max() <= tol, f"precision {prec}: per-element Frobenius error {err.max():.3e} > {tol:g}"


@pytest.mark.parametrize("seed,grid,n,norient,nterms,ngp1", [(6, 14, 9, 2, 5, 3), (7, 60, 20, 3, 4, 4), (8, 30, 27, 1, 9, 3)])
def test_split_symmetric_group(ctx, seed, grid, n, norient, nterms, ngp1):
    """A group with mirror terms: the split contraction computes the upper
    triangle (1 to 3 row tiles, the last one partly filled) and mirrors it.
    The element matrices are symmetric bit for bit and within the split
    tiers' bounds of the FP64 path."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gb, xyz, conn = S.group(rng, nelem_grid=grid, ntf=n, ndof=n, nterms=nterms, ngp1=ngp1, norient=norient, ndests=1,
                            symmetric=True)
    ref = _element_matrices(ctx, gb, xyz, conn, abi.PREC_FP64)
    for prec, tol in ((abi.PREC_SPLIT, 1e-10), (abi.PREC_FP32, 1e-6)):
        got = _element_matrices(ctx, gb, xyz, conn, prec)
        m = got.reshape(-1, n, n)
        assert np.array_equal(m, m.transpose(0, 2, 1)), f"precision {prec}: element matrices not symmetric"
        err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        assert err.max() <= tol, f"precision {prec}: per-element Frobenius error {err.max():.3e} > {tol:g}"


def test_split_symmetry_matches_full_contraction(ref_lib, gpu_lib, tmp_path):
    """The mirrored split contraction against the full one
    (SLGPU_SPLIT_SYMMETRY=0) through the drop-in.  p-adaptive Helmholtz
    tetrahedra, whose mirror coefficients are equal bit for bit: the same
    matrix bit for bit.  Order-2 elasticity, whose diagonal blocks' mirror
    coefficients differ in the order of their factors: within 1e-14 of the
    largest entry.  Both within 1e-10 of the reference."""
    n = 3
    rng = np.random.Generator(np.random.PCG64(7))
    tags = meshgen.ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
    tmsh = str(tmp_path / "t.msh")
    meshgen.tet_mesh(tmsh, n, jitter=0.1, seed=2, element_tags=tags)
    hmsh = str(tmp_path / "h.msh")
    meshgen.hex_mesh(hmsh, 3, jitter=0.15, seed=1)
    for args, exact in (((W.HELMHOLTZ_TET, tmsh, []), True), ((W.ELASTICITY_HEX, hmsh, [2, -2]), False)):
        sym = P.gpu(*args, precision="split")
        full = P.gpu(*args, precision="split", env={"SLGPU_SPLIT_SYMMETRY": "0"})
        P.check_pattern(full, sym)
        for k in ("Avals", "Dvals", "b"):
            if exact:
                assert np.array_equal(sym[k], full[k]), f"workload {args[0]}: {k} differs"
            elif full[k].size:
                d = np.abs(sym[k] - full[k]).max() / max(np.abs(full[k]).max(), 1e-300)
                assert d <= 1e-14, f"workload {args[0]}: {k} differs by {d:.3e}"
        _, _, fro = P.scaled_errors(P.reference(*args), sym)
        assert fro <= 1e-10, f"workload {args[0]}: assembled Frobenius-relative error {fro:.3e}"


def _pair_matrices(ctx, groups, xyz, conn, precision, edit=None):
    """Element matrices of several groups of one matrix, each group's rows in
    a block of its own (row = block base + e ntf + i, column = j).  `edit(h)`
    runs before processing.  Also returns each group's transposed partner."""
    L = ctx.lib
    ctx.check(L.slgpu_mesh_set_nodes(ctx.h, 0, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(L.slgpu_mesh_set_elements(ctx.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))
    keep, base = [], 0
    for g in groups:
        tfaddr = (base + np.arange(g.nelem)[None, :] * g.ntf + np.arange(g.ntf)[:, None]).astype(np.int32)
        dofaddr = np.repeat(np.arange(g.ndof, dtype=np.int32)[:, None], g.nelem, axis=1)
        dest = (abi.Dest * 1)()
        dest[0].tfaddr, dest[0].dofaddr, dest[0].multiplier = abi.i32p(tfaddr), abi.i32p(dofaddr), 1.0
        g.ndests, g.dests = 1, dest
        keep += [tfaddr, dofaddr, dest]
        base += g.nelem * g.ntf
    ndofs = base
    h = ctypes.c_int()
    ctx.check(L.slgpu_matrix_create(ctx.h, ndofs, ctypes.byref(h)))
    for g in groups:
        ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(g), None))
    if edit is not None:
        edit(h.value)
    partners = []
    for gi in range(len(groups)):
        pt = ctypes.c_int32()
        ctx.check(L.slgpu_matrix_group_symmetry(ctx.h, h, gi, None, None, ctypes.byref(pt)))
        partners.append(pt.value)
    info = abi.CsrInfo()
    con = np.zeros(ndofs, np.uint8)
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), precision,
                                     ctypes.byref(info)))
    rows, cols = np.zeros(ndofs + 1, np.int32), np.zeros(info.nnzA, np.int32)
    vals = np.zeros(info.nnzA)
    ctx.check(L.slgpu_matrix_download(ctx.h, h, abi.i32p(rows), abi.i32p(cols), abi.f64p(vals),
                                      abi.i32p(np.zeros(ndofs + 1, np.int32)), abi.i32p(np.zeros(1, np.int32)),
                                      abi.f64p(np.zeros(1))))
    ctx.check(L.slgpu_matrix_destroy(ctx.h, h))
    out, base = [], 0
    for g in groups:
        n = g.nelem * g.ntf * g.ndof
        assert np.array_equal(cols[base:base + n], np.tile(np.arange(g.ndof), g.nelem * g.ntf))
        out.append(vals[base:base + n].reshape(g.nelem, g.ntf, g.ndof))
        base += n
    return out, partners


def test_split_transposed_pair(ctx):
    """Two groups whose element matrices are transposes of each other (ntf 12
    and ndof 8 swapped, tables of each term swapped, the same coefficients and
    data): one split contraction writes both, and the second group's matrices
    are the first's transposed bit for bit, within the split bound of its own
    FP64 result.  Replacing one group's element data ends the pairing; the
    same data in both restores it."""
    rng = np.random.Generator(np.random.PCG64(9))
    gb, xyz, conn = S.group(rng, nelem_grid=30, ntf=12, ndof=8, nterms=4, ngp1=3, norient=2, ndests=1)
    g1 = gb.g
    g2 = abi.Group.from_buffer_copy(g1)
    g2.ntf, g2.ndof = g1.ndof, g1.ntf
    terms2 = (abi.Term * g1.nterms)(*[abi.Term(g1.terms[t].dof_table, g1.terms[t].tf_table, g1.terms[t].coef_node, 0,
                                               g1.terms[t].scale) for t in range(g1.nterms)])
    g2.terms = terms2
    new_e = rng.lognormal(0.0, 0.4, g1.nelem)

    def set_e(groups):
        return lambda h: [ctx.check(ctx.lib.slgpu_matrix_set_elemdata(ctx.h, h, gi, 0, abi.f64p(new_e))) for gi in groups]

    for edit, paired in ((None, True), (set_e([1]), False), (set_e([0, 1]), True)):
        (r1, r2), _ = _pair_matrices(ctx, [g1, g2], xyz, conn, abi.PREC_FP64, edit)
        (m1, m2), partners = _pair_matrices(ctx, [g1, g2], xyz, conn, abi.PREC_SPLIT, edit)
        assert partners == ([1, 0] if paired else [-1, -1])
        if paired:
            assert np.array_equal(m2, m1.transpose(0, 2, 1))
        for got, ref in ((m1, r1), (m2, r2)):
            err = np.linalg.norm((got - ref).reshape(len(got), -1), axis=1) / np.linalg.norm(ref.reshape(len(ref), -1), axis=1)
            assert err.max() <= 1e-10, f"paired={paired}: per-element Frobenius error {err.max():.3e}"


def test_split_dropin_elasticity(ref_lib, gpu_lib, tmp_path):
    msh = str(tmp_path / "h.msh")
    meshgen.hex_mesh(msh, 4, jitter=0.15, seed=1)
    ref = P.reference(W.ELASTICITY_HEX, msh, [2, -2])
    got = P.gpu(W.ELASTICITY_HEX, msh, [2, -2], precision="split")
    P.check_pattern(ref, got)
    _, _, fro = P.scaled_errors(ref, got)
    assert fro <= 1e-10, f"assembled Frobenius-relative error {fro:.3e}"

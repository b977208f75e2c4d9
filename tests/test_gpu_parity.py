"""GPU parity: the CUDA engine against the reference and the C oracle.

Drop-in level: stock sparselizard and sparselizard with the GPU translation
units run the same workload; the A/D CSR pattern must be bit-exact and the
values within 1e-12 (row-relative), b within 1e-12.
C-ABI level: seeded synthetic groups go through slgpu_matrix_* and through
the oracle (oracle/slref.c) with the same structures.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

import _pipeline as P
import _synthetic as S
from sparselizard_b200 import abi, meshgen, workloads as W

sys.path.insert(0, os.path.join(P.ROOT, "oracle"))
import slref  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def tmp(tmp_path_factory):
    return tmp_path_factory.mktemp("gpu_meshes")


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def _full_parity(ref, got, rec):
    """rec: the oracle's record-only run of the same workload, which provides
    the magnitude sums each entry is judged against."""
    P.check_pattern(ref, got)
    P.check_pattern(ref, rec)
    ea, ed = P.check_values(ref, got, TOL, mag=rec)
    eb = P.check_rhs(ref, got["b"], TOL, babs=rec.get("b_abs"))
    assert np.array_equal(ref["Ainds"], got["Ainds"]) and np.array_equal(ref["Dinds"], got["Dinds"])
    return ea, ed, eb


def test_smoke():
    import __graft_entry__

    __graft_entry__.smoke()


@pytest.mark.parametrize("order", [1, 2, 3])
def test_dropin_poisson_quad(ref_lib, gpu_lib, tmp, order):
    msh = str(tmp / f"q{order}.msh")
    meshgen.quad_mesh(msh, 20, jitter=0.2, seed=order)
    args = (W.POISSON_QUAD, msh, [order])
    _full_parity(P.reference(*args), P.gpu(*args), P.record_oracle(*args))


def test_dropin_elasticity_hex(ref_lib, gpu_lib, tmp):
    msh = str(tmp / "h.msh")
    meshgen.hex_mesh(msh, 4, jitter=0.15, seed=1)
    args = (W.ELASTICITY_HEX, msh, [2, -2])
    _full_parity(P.reference(*args), P.gpu(*args), P.record_oracle(*args))


def test_dropin_helmholtz_tet(ref_lib, gpu_lib, tmp):
    n = 4
    rng = np.random.Generator(np.random.PCG64(7))
    tags = meshgen.ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
    msh = str(tmp / "t.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=2, element_tags=tags)
    args = (W.HELMHOLTZ_TET, msh, [])
    _full_parity(P.reference(*args), P.gpu(*args), P.record_oracle(*args))


@pytest.mark.parametrize("freq", [1.0, 1e6])
def test_dropin_eddy_hcurl(ref_lib, gpu_lib, tmp, freq):
    n = 3
    rng = np.random.Generator(np.random.PCG64(11))
    tags = meshgen.MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
    msh = str(tmp / "e.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=4, element_tags=tags)
    p = [2, freq, 1e3, 5e5, 2e6, 6e7]
    args = (W.EDDY_TET, msh, p)
    _full_parity(P.reference(*args), P.gpu(*args), P.record_oracle(*args))


def test_dropin_poisson_full_size(ref_lib, gpu_lib, tmp):
    """The 256 x 256 quadrangle workload at full size."""
    msh = str(tmp / "q256.msh")
    meshgen.quad_mesh(msh, 256, jitter=0.2, seed=1)
    ref = P.reference(W.POISSON_QUAD, msh, [1])
    got = P.gpu(W.POISSON_QUAD, msh, [1], reps=2)
    _full_parity(ref, got, P.record_oracle(W.POISSON_QUAD, msh, [1]))
    assert ref["Acols"].size == 582169 and ref["Dcols"].size == 3056


def test_dropin_repeated_assembly_reuses_host_arrays(ref_lib, gpu_lib, tmp):
    """Three generate()/A()/b() of 12^3 elasticity (8.6M nonzeros): the second
    and third rawmats share the CSR structure downloaded by the first and get
    the value array that the previous rawmat gave back; the last one still
    equals the reference."""
    msh = str(tmp / "h12.msh")
    meshgen.hex_mesh(msh, 12, jitter=0.15, seed=3)
    args = (W.ELASTICITY_HEX, msh, [2, -2])
    ref = P.reference(*args)
    got = P.gpu(*args, reps=3)
    _full_parity(ref, got, P.record_oracle(*args))
    assert ref["Acols"].size > (1 << 21)


@pytest.mark.parametrize("workload,kind,n,params", [(W.POISSON_DIRICHLET, "quad", 24, [1]), (W.POISSON_DIRICHLET, "quad", 24, [2]),
                                                     (W.POISSON_DIRICHLET, "quad", 16, [3]), (W.ELASTICITY_DIRICHLET, "hex", 5, [2])])
def test_dropin_nonzero_dirichlet(ref_lib, gpu_lib, tmp, workload, kind, n, params):
    """Non-zero Dirichlet values: b() projects the constraint expression onto
    the constrained form functions by secondary assemblies (barycenter values
    on the nodes, then projections on the boundary edges / faces: elements of
    lower dimension than the mesh), all through the drop-in on the GPU.  The
    matrix, b and the constrained entries of b must match the reference."""
    msh = str(tmp / f"dir_{kind}_{n}_{params[0]}.msh")
    meshgen.workload_mesh(kind, n, msh)
    ref = P.reference(workload, msh, params)
    got = P.gpu(workload, msh, params)
    P.check_pattern(ref, got)
    assert np.array_equal(ref["Ainds"], got["Ainds"]) and np.array_equal(ref["Dinds"], got["Dinds"])
    P.check_values(ref, got, TOL)
    bd = ref["b"][ref["Dinds"]]
    assert np.abs(bd).max() > 0, "the constraint values must be non-zero"
    P.check_rhs(ref, got["b"], TOL)


def test_dropin_after_another_formulation(ref_lib, gpu_lib, tmp):
    """A formulation assembled after another one on the same mesh (a field of
    another order, its own dofmanager) was generated and left unprocessed: the
    drop-in shares DOF addresses between the contributions of an assembly
    and must keep the two formulations' addresses apart."""
    msh = str(tmp / "after_other.msh")
    meshgen.workload_mesh("quad", 16, msh)
    args = (W.POISSON_AFTER_OTHER, msh, [2])
    ref, got = P.reference(*args), P.gpu(*args)
    P.check_pattern(ref, got)
    P.check_values(ref, got, TOL)
    P.check_rhs(ref, got["b"], TOL)


@pytest.mark.parametrize("order", [1, 3])
def test_gpu_integrate_matches_expression_integrate(ref_lib, gpu_lib, tmp, order):
    """Field interpolation and integration on the GPU: a field set by
    projection, then the integral of an expression of it and of the
    coordinates, against sparselizard's own expression::integrate."""
    msh = str(tmp / f"int_{order}.msh")
    meshgen.workload_mesh("quad", 32, msh)
    ref = P.integrate("ref_integrate", msh, order)
    got = P.integrate("gpu_integrate", msh, order)
    r = float(ref["host"])
    assert abs(float(got["gpu"]) - r) <= TOL * abs(r)
    assert abs(float(got["host"]) - r) <= TOL * abs(r)


@pytest.mark.parametrize("workload,kind,n,params", [(W.POISSON_QUAD, "quad", 64, [2]), (W.ELASTICITY_HEX, "hex", 6, [2, -2])])
def test_device_csr_and_eliminate(ref_lib, gpu_lib, tmp, workload, kind, n, params):
    """Device-resident handoff: slgpu_matrix_device_csr returns the same CSR
    as the download, and slgpu_matrix_eliminate (x_A - D x_D on the device)
    equals the reference's mat::eliminate of the same vector bit for bit."""
    msh = str(tmp / f"elim_{kind}.msh")
    meshgen.workload_mesh(kind, n, msh)
    ref = P.eliminate("ref_elim", workload, msh, params)
    got = P.eliminate("gpu_elim", workload, msh, params)
    assert ref["Dcols"].size > 0
    for k in ("Ainds", "Dinds", "Drows", "Dcols"):
        assert np.array_equal(ref[k], got[k])
    np.testing.assert_array_equal(ref["x"], got["x"])
    # Bit-exact when D's values are; otherwise within the values' tolerance.
    if np.array_equal(ref["Dvals"], got["Dvals"]):
        np.testing.assert_array_equal(got["elim"], ref["elim"])
    bd = ref["x"][ref["Dinds"]]
    rows = np.repeat(np.arange(ref["Ainds"].size), np.diff(ref["Drows"]))
    mag = np.abs(ref["x"][ref["Ainds"]]) + np.bincount(rows, np.abs(ref["Dvals"] * bd[ref["Dcols"]]), ref["Ainds"].size)
    assert np.max(np.abs(got["elim"] - ref["elim"]) / np.maximum(mag, 1e-300)) <= TOL


def _matrix(ctx, groups, ndofs, con, frags=(), precision=abi.PREC_FP64):
    L = ctx.lib
    h = ctypes.c_int()
    ctx.check(L.slgpu_matrix_create(ctx.h, ndofs, ctypes.byref(h)))
    for gb in groups:
        ctx.check(L.slgpu_matrix_add_group(ctx.h, h, ctypes.byref(gb.g), None))
    for (ntr, ndr, nr, nc, rows, cols, vals) in frags:
        ctx.check(L.slgpu_matrix_add_fragment(ctx.h, h, ntr, ndr, nr, nc, abi.i32p(rows), abi.i32p(cols), abi.f64p(vals)))
    info = abi.CsrInfo()
    con = np.ascontiguousarray(con, np.uint8)
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), precision, ctypes.byref(info)))
    out = dict(Arows=np.zeros(info.nA + 1, np.int32), Acols=np.zeros(info.nnzA, np.int32), Avals=np.zeros(info.nnzA),
               Drows=np.zeros(info.nA + 1, np.int32), Dcols=np.zeros(info.nnzD, np.int32), Dvals=np.zeros(info.nnzD))
    ctx.check(L.slgpu_matrix_download(ctx.h, h, abi.i32p(out["Arows"]), abi.i32p(out["Acols"]), abi.f64p(out["Avals"]),
                                      abi.i32p(out["Drows"]), abi.i32p(out["Dcols"]), abi.f64p(out["Dvals"])))
    ctx.check(L.slgpu_matrix_destroy(ctx.h, h))
    out["reused"] = info.pattern_reused
    return out


def _mesh(ctx, xyz, conn):
    ctx.check(ctx.lib.slgpu_mesh_set_nodes(ctx.h, 0, xyz.size // 3, abi.f64p(xyz)))
    ctx.check(ctx.lib.slgpu_mesh_set_elements(ctx.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_abi_synthetic_matrix(ctx, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    ndofs = 80
    gb, xyz, conn = S.group(rng, ndofs=ndofs)
    gb2, _, _ = S.group(np.random.Generator(np.random.PCG64(seed + 100)), ndofs=ndofs, ntf=4, ndof=4, nterms=2, norient=1,
                        ndests=1)
    _mesh(ctx, xyz, conn)
    con = (rng.random(ndofs) < 0.2).astype(np.uint8)
    frag = (3, 2, 6, 5, rng.integers(-1, ndofs, 15).astype(np.int32), rng.integers(-1, ndofs, 10).astype(np.int32),
            rng.standard_normal(30))
    got = _matrix(ctx, [gb, gb2], ndofs, con, [frag])
    ref = slref.matrix([gb.g, gb2.g], xyz, [conn, conn], ndofs, con, [frag])
    mag = slref.matrix([gb.g, gb2.g], xyz, [conn, conn], ndofs, con, [frag], absmode=True)
    P.check_pattern(ref, got)
    P.check_values(ref, got, TOL, mag={"Aabs": mag["Avals"], "Dabs": mag["Dvals"]})


def test_abi_determinism_and_pattern_reuse(ctx):
    rng = np.random.Generator(np.random.PCG64(5))
    gb, xyz, conn = S.group(rng, ndofs=50, nelem_grid=12)
    _mesh(ctx, xyz, conn)
    con = np.zeros(50, np.uint8)
    con[::7] = 1
    a = _matrix(ctx, [gb], 50, con)
    b = _matrix(ctx, [gb], 50, con)
    assert b["reused"] == 1
    for k in ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals"):
        assert np.array_equal(a[k], b[k]), f"{k} not bit-identical across runs"


def test_abi_edge_cases(ctx):
    rng = np.random.Generator(np.random.PCG64(9))
    ndofs = 40
    # every address -1 -> empty CSR
    gb, xyz, conn = S.group(rng, ndofs=ndofs, p_neg=1.1)
    _mesh(ctx, xyz, conn)
    got = _matrix(ctx, [gb], ndofs, np.zeros(ndofs, np.uint8))
    assert got["Acols"].size == 0 and got["Dcols"].size == 0 and np.all(got["Arows"] == 0)
    # every DOF constrained -> no rows
    gb, xyz, conn = S.group(rng, ndofs=ndofs)
    got = _matrix(ctx, [gb], ndofs, np.ones(ndofs, np.uint8))
    assert got["Arows"].size == 1 and got["Acols"].size == 0
    # fragments only (ports / mat(...) constructor path)
    frag = (1, 1, 1, 4, np.array([0, 1, 1, 39], np.int32), np.array([0, 1, 1, 2], np.int32), np.array([1.0, 2.0, 3.0, 4.0]))
    got = _matrix(ctx, [], ndofs, np.zeros(ndofs, np.uint8), [frag])
    ref = slref.matrix([], np.zeros(3), [], ndofs, np.zeros(ndofs, np.uint8), [frag])
    P.check_pattern(ref, got)
    np.testing.assert_array_equal(got["Avals"], ref["Avals"])
    # an address beyond the DOF count is an error, not a fault
    gb, xyz, conn = S.group(rng, ndofs=ndofs + 5)
    with pytest.raises(abi.SlgpuError):
        _matrix(ctx, [gb], ndofs, np.zeros(ndofs, np.uint8))


def test_abi_rhs(ctx):
    rng = np.random.Generator(np.random.PCG64(3))
    ndofs = 70
    gb, xyz, conn = S.group(rng, ndofs=ndofs, rhs=True)
    _mesh(ctx, xyz, conn)
    b = np.zeros(ndofs)
    ctx.check(ctx.lib.slgpu_rhs_assemble(ctx.h, ctypes.byref(gb.g), ndofs, abi.PREC_FP64, abi.f64p(b)))
    ref = slref.rhs(gb.g, xyz, conn, ndofs)
    mag = slref.rhs(gb.g, xyz, conn, ndofs, absmode=True)
    assert np.max(np.abs(b - ref) / np.maximum(mag, 1e-300)) <= TOL
    # The same right-hand side as reached rows and values (ndofs well above
    # the rows reached): the dense result at those rows, zero elsewhere.
    big = 5000
    bd = np.zeros(big)
    ctx.check(ctx.lib.slgpu_rhs_assemble(ctx.h, ctypes.byref(gb.g), big, abi.PREC_FP64, abi.f64p(bd)))
    cap = gb.g.ntf * gb.g.nelem * gb.g.ndests
    rows, vals, n = np.zeros(cap, np.int32), np.zeros(cap), ctypes.c_int64()
    ctx.check(ctx.lib.slgpu_rhs_assemble_rows(ctx.h, ctypes.byref(gb.g), big, abi.PREC_FP64, abi.i32p(rows), abi.f64p(vals), cap,
                                              ctypes.byref(n)))
    rows, vals = rows[: n.value], vals[: n.value]
    assert n.value > 0 and np.all(np.diff(rows) > 0)
    dense = np.zeros(big)
    dense[rows] = vals
    assert np.array_equal(dense, bd)


def test_abi_budget_error(ctx):
    small = abi.Context(0, budget=1 << 18)
    rng = np.random.Generator(np.random.PCG64(1))
    gb, xyz, conn = S.group(rng, ndofs=50, nelem_grid=40)
    with pytest.raises(abi.SlgpuError) as e:
        small.check(small.lib.slgpu_mesh_set_nodes(small.h, 0, xyz.size // 3, abi.f64p(xyz)))
        small.check(small.lib.slgpu_mesh_set_elements(small.h, 0, 3, 4, conn.size // 4, abi.i32p(conn)))
        _matrix(small, [gb], 50, np.zeros(50, np.uint8))
    assert e.value.status == abi.E_BUDGET
    small.close()

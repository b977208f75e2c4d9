"""The allocation-free element-matrix entry point against the regular path.

slgpu_element_matrices_noalloc serves callers that cannot allocate device
memory themselves (their own allocator owns the device heap, or their loop
must not pay for cudaMalloc/cudaFree).  It must give the same element
matrices as the regular entry points.  The regular path is made to expose
element matrices by giving every (element, test function) its own row and
every dof function its own column, so each CSR value is exactly one element
matrix entry.  Two calls in a row check that the shared scratch array is
reused correctly.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import _synthetic as S
from sparselizard_b200 import abi

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _regular_element_matrices(ctx, gb, xyz, conn):
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
    ctx.check(L.slgpu_matrix_process(ctx.h, h, con.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), abi.PREC_FP64,
                                     ctypes.byref(info)))
    assert info.nnzA == nelem * ntf * ndof
    rows, cols = np.zeros(ndofs + 1, np.int32), np.zeros(info.nnzA, np.int32)
    vals = np.zeros(info.nnzA)
    d1, d2 = np.zeros(ndofs + 1, np.int32), np.zeros(1, np.int32)
    ctx.check(L.slgpu_matrix_download(ctx.h, h, abi.i32p(rows), abi.i32p(cols), abi.f64p(vals), abi.i32p(d1),
                                      abi.i32p(d2), abi.f64p(np.zeros(1))))
    ctx.check(L.slgpu_matrix_destroy(ctx.h, h))
    assert np.array_equal(cols.reshape(ndofs, ndof), np.tile(np.arange(ndof), (ndofs, 1)))
    return vals.reshape(nelem, ntf * ndof)


def _noalloc(gb, xyz_dev, conn_dev, mesh_nelem, out_dev, stream, nnodes=None):
    err = ctypes.create_string_buffer(512)
    nnodes = xyz_dev.numel() // 3 if nnodes is None else nnodes
    st = abi.lib().slgpu_element_matrices_noalloc(ctypes.byref(gb.g), ctypes.c_void_p(xyz_dev.data_ptr()), nnodes,
                                                  ctypes.c_void_p(conn_dev.data_ptr()), mesh_nelem,
                                                  ctypes.c_void_p(out_dev.data_ptr()), ctypes.c_void_p(stream), err, 512)
    return st, err.value.decode()


def test_noalloc_matches_regular_path_twice():
    import torch

    ctx = abi.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for seed in (21, 22):  # two calls in a row, different groups, same scratch
        rng = np.random.Generator(np.random.PCG64(seed))
        gb, xyz, conn = S.group(rng, nelem_grid=10 + seed % 3, ntf=6, ndof=4, nterms=3, norient=2, ndests=1)
        xyz_dev = torch.from_numpy(xyz).cuda()
        conn_dev = torch.from_numpy(conn).cuda()
        g = gb.g
        out = torch.full((g.nelem, g.ntf * g.ndof), float("nan"), dtype=torch.float64, device="cuda")
        st, msg = _noalloc(gb, xyz_dev, conn_dev, conn.size // 4, out, stream)
        assert st == abi.OK, msg
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = _regular_element_matrices(ctx, gb, xyz, conn)
        scale = np.abs(want).max()
        err = np.abs(got - want).max() / scale
        assert err <= TOL, f"no-alloc element matrices differ: {err:.3e}"
        results.append(err)
    ctx.close()
    assert len(results) == 2


def test_noalloc_rejects_groups_beyond_its_scratch():
    import torch

    rng = np.random.Generator(np.random.PCG64(5))
    # 400 x 400 elements x 3 terms x 9 Gauss points of coefficients alone exceed 32 MiB
    gb, xyz, conn = S.group(rng, nelem_grid=400, ntf=4, ndof=4, nterms=3, norient=1, ndests=1)
    xyz_dev = torch.from_numpy(xyz).cuda()
    conn_dev = torch.from_numpy(conn).cuda()
    out = torch.empty(16, dtype=torch.float64, device="cuda")
    st, msg = _noalloc(gb, xyz_dev, conn_dev, conn.size // 4, out, torch.cuda.current_stream().cuda_stream)
    assert st == abi.E_BUDGET and "scratch" in msg


def test_noalloc_without_destinations_and_bad_nodes():
    """A group with no destinations is accepted (nothing is assembled), and an
    element whose connectivity names a node beyond `nnodes` gets a NaN matrix
    while the other elements are unaffected."""
    import torch

    rng = np.random.Generator(np.random.PCG64(31))
    gb, xyz, conn = S.group(rng, nelem_grid=6, ntf=4, ndof=4, nterms=2, norient=1, ndests=1)
    g = gb.g
    stream = torch.cuda.current_stream().cuda_stream
    xyz_dev = torch.from_numpy(xyz).cuda()
    conn_dev = torch.from_numpy(conn).cuda()
    good = torch.empty((g.nelem, g.ntf * g.ndof), dtype=torch.float64, device="cuda")
    st, msg = _noalloc(gb, xyz_dev, conn_dev, conn.size // 4, good, stream)
    assert st == abi.OK, msg
    g.ndests, g.dests = 0, None
    bad_conn = conn.copy()
    elems = np.ctypeslib.as_array(g.elems, (g.nelem,)).copy()
    victim = int(elems[0])
    bad_conn[victim * 4 + 1] = xyz.size // 3 + 7
    out = torch.zeros_like(good)
    st, msg = _noalloc(gb, xyz_dev, torch.from_numpy(bad_conn).cuda(), conn.size // 4, out, stream)
    assert st == abi.OK, msg
    torch.cuda.synchronize()
    got, want = out.cpu().numpy(), good.cpu().numpy()
    hit = elems == victim
    assert np.isnan(got[hit]).all()
    assert np.array_equal(got[~hit], want[~hit])

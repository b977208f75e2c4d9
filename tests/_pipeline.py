"""Helpers shared by the parity tests.

Each sparselizard build (stock reference, GPU drop-in, record-only lowering)
runs in its own subprocess so that the two builds' global state never meet
and a record-only context never leaks into a GPU run.  Results come back as
.npz files.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU_LIB = os.path.join(ROOT, "sparselizard_b200", "_build", "libslz_gpu.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libslz_ref.so")

KEYS = ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals", "Ainds", "Dinds", "b")


def _child(mode: str, workload: int, msh: str, params, out: str, env_extra=None, reps: int = 1):
    env = dict(os.environ)
    env.update(env_extra or {})
    code = (
        "import sys; sys.path[:0] = [%r, %r]; import _pipeline; _pipeline._child_main(%r, %d, %r, %r, %r, %d)"
        % (ROOT, os.path.join(ROOT, "tests"), mode, workload, msh, list(params), out, reps)
    )
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"{mode} run failed (rc={r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    d = np.load(out, allow_pickle=False)
    return {k: d[k] for k in d.files}


def _child_main(mode, workload, msh, params, out, reps):
    from sparselizard_b200 import workloads as W

    if mode == "ref":
        r = W.run(REF_LIB, workload, msh, params, reps=reps)
    elif mode == "gpu":
        r = W.run(GPU_LIB, workload, msh, params, reps=reps)
    elif mode == "record":
        np.savez(out, **record_oracle_inproc(workload, msh, params))
        return
    elif mode == "symmetry":
        np.savez(out, **symmetry_inproc(workload, msh, params))
        return
    elif mode.startswith("sweep"):
        np.savez(out, **sweep_inproc(msh, params, mode.split(":")[1]))
        return
    elif mode in ("ref_kfield", "serve_kfield"):
        np.savez(out, **kfield_inproc(mode, msh, params))
        return
    elif mode in ("ref_integrate", "gpu_integrate"):
        lib = W.load(REF_LIB if mode == "ref_integrate" else GPU_LIB)
        out3 = (ctypes.c_double * 2)()
        rc = lib.slz_integrate(msh.encode(), int(params[0]), out3)
        if rc != 0:
            raise RuntimeError(lib.slz_last_error().decode(errors="replace"))
        np.savez(out, host=np.array(out3[0]), gpu=np.array(out3[1]))
        return
    elif mode in ("ref_elim", "gpu_elim"):
        np.savez(out, **eliminate_inproc(mode, workload, msh, params))
        return
    else:
        raise ValueError(mode)
    np.savez(out, ndofs=np.array(r.ndofs), times=r.times, **{k: getattr(r, k) for k in KEYS})


def sweep_inproc(msh, params, precision):
    """Frequency sweep through the drop-in: template assembled at params[1]
    and params[2] (Hz), then re-assembled at each frequency of params[3:] by
    setting fitted scales; returns the A/D values at the last frequency."""
    from sparselizard_b200 import abi, workloads as W

    os.environ["SLGPU_PRECISION"] = precision
    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slz_sweep_prepare.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                      ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_sweep_run.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    lib.slz_sweep_values.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.slz_sweep_values.restype = ctypes.c_longlong
    order, f1, f2, sig = int(params[0]), params[1], params[2], params[3:7]
    freqs = np.array(params[7:], dtype=np.float64)
    sigmas = (ctypes.c_double * 4)(*sig)
    info = (ctypes.c_longlong * 4)()
    if lib.slz_sweep_prepare(msh.encode(), order, sigmas, f1, f2, info) != 0:
        raise RuntimeError(lib.slz_last_error().decode(errors="replace"))
    dev, host = np.zeros(freqs.size), np.zeros(freqs.size)
    prec = {"fp64": abi.PREC_FP64, "split": abi.PREC_SPLIT, "fp32": abi.PREC_FP32}[precision]
    rc = lib.slz_sweep_run(freqs.size, abi.f64p(freqs), prec, abi.f64p(dev), abi.f64p(host))
    if rc != 0:
        raise RuntimeError("sweep failed: " + lib.slz_last_error().decode(errors="replace"))
    nnz = int(info[2])
    nnzA = int(lib.slz_sweep_values(None, None))
    A, D = np.zeros(max(1, nnzA)), np.zeros(max(1, nnz - nnzA))
    lib.slz_sweep_values(abi.f64p(A), abi.f64p(D))
    return dict(Avals=A[:nnzA], Dvals=D[: nnz - nnzA], device_ms=dev, host_ms=host)


def elimination_vector(ndofs, seed=77):
    return np.random.Generator(np.random.PCG64(seed)).standard_normal(ndofs)


def eliminate_inproc(mode, workload, msh, params):
    """Runs the workload, then eliminates the constrained DOFs from a seeded
    random vector x: on the host through mat::eliminate (ref_elim, the stock
    build) or on the device through slgpu_matrix_eliminate (gpu_elim, the
    drop-in, which also checks slgpu_matrix_device_csr against the host CSR)."""
    from sparselizard_b200 import abi, workloads as W

    lib_path = REF_LIB if mode == "ref_elim" else GPU_LIB
    r = W.run(lib_path, workload, msh, params)
    lib = W.load(lib_path)
    x = elimination_vector(r.ndofs)
    out = {k: getattr(r, k) for k in ("Ainds", "Dinds", "Drows", "Dcols", "Dvals")}
    out["x"] = x
    if mode == "ref_elim":
        lib.slz_eliminate.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.slz_eliminate.restype = ctypes.c_longlong
        e = np.zeros(max(1, r.Ainds.size))
        n = lib.slz_eliminate(x.ctypes.data, e.ctypes.data)
        assert n == r.Ainds.size, lib.slz_last_error()
        out["elim"] = e[:n]
        return out
    import torch

    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    h = lib.slz_last_matrix_handle()
    assert h > 0
    ptr = [ctypes.c_void_p() for _ in range(6)]
    assert lib.slgpu_matrix_device_csr(ctx, h, *[ctypes.byref(q) for q in ptr]) == 0
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    host = [r.Arows, r.Acols, r.Avals, r.Drows, r.Dcols, r.Dvals]
    for q, a in zip(ptr, host):
        got = np.empty_like(a)
        if a.size:
            assert cudart.cudaMemcpy(got.ctypes.data, q, a.nbytes, 2) == 0  # device to host
        assert np.array_equal(got, a), "device CSR differs from the downloaded CSR"
    xd = torch.from_numpy(x).cuda()
    ed = torch.empty(max(1, r.Ainds.size), dtype=torch.float64, device="cuda")
    st = lib.slgpu_matrix_eliminate(ctx, h, ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(ed.data_ptr()))
    assert st == 0, st
    out["elim"] = ed.cpu().numpy()[: r.Ainds.size]
    # Host memory is rejected with an error, not read by the device.
    st = lib.slgpu_matrix_eliminate(ctx, h, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(ed.data_ptr()))
    assert st == abi.E_ARG, st
    return out


def kfield_values(nelem, seed=29):
    return np.random.Generator(np.random.PCG64(seed)).lognormal(0.0, 0.3, nelem)


def kfield_inproc(mode, msh, params):
    """Poisson with a per-element coefficient field k on quads.  ref_kfield:
    stock sparselizard assembles it with k = kfield_values (element order).
    serve_kfield: the drop-in assembles the same formulation once with k = 1
    as a serving template (slz_serve_add), then one request through the
    engine's server carries k = kfield_values (mesh element order); returns
    the template's pattern and the request's values."""
    from sparselizard_b200 import abi, serving, workloads as W

    order, nelem, precision = int(params[0]), int(params[1]), int(params[2])
    k = kfield_values(nelem)
    if mode == "ref_kfield":
        lib = W.load(REF_LIB)
        lib.slz_set_element_values.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        lib.slz_set_element_values(k.ctypes.data, k.size)
        r = W.run(REF_LIB, W.POISSON_KFIELD, msh, [order])
        return {key: getattr(r, key) for key in ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals")}
    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    lib.slz_serve_add.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    info = (ctypes.c_longlong * 6)()
    idx = lib.slz_serve_add(1, msh.encode(), 2, order, info)
    if idx < 0:
        raise RuntimeError(lib.slz_last_error().decode(errors="replace"))
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    h, nnzA, nnzD, nmesh, ngroups = int(info[0]), int(info[1]), int(info[2]), int(info[3]), int(info[4])
    assert nmesh == nelem
    # The template's pattern (its last process()).
    ws = abi.Work()
    assert lib.slgpu_matrix_work(ctx, h, ctypes.byref(ws)) == 0
    nA = int(ws.nA)
    pat = dict(Arows=np.zeros(nA + 1, np.int32), Acols=np.zeros(nnzA, np.int32), Avals=np.zeros(max(1, nnzA)),
               Drows=np.zeros(nA + 1, np.int32), Dcols=np.zeros(nnzD, np.int32), Dvals=np.zeros(max(1, nnzD)))
    assert lib.slgpu_matrix_download(ctx, h, *[abi.i32p(pat[x]) if pat[x].dtype == np.int32 else abi.f64p(pat[x])
                                               for x in ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals")]) == 0
    srv = serving.Server(lib, ctx, 2)
    try:
        A, D = np.full(nnzA, np.nan), np.full(max(1, nnzD), np.nan)[:nnzD]
        ups = [serving.UpdateSpec(gi, abi.UPDATE_FIELDDATA, 0, k) for gi in range(ngroups)]
        st = srv.wait(srv.submit(h, precision, ups, A, D))
        assert st.status == abi.OK
    finally:
        srv.close()
    return dict(Arows=pat["Arows"], Acols=pat["Acols"], Avals=A, Drows=pat["Drows"], Dcols=pat["Dcols"], Dvals=D)


def kfield(mode, msh, order, nelem, precision):
    with tempfile.TemporaryDirectory() as d:
        return _child(mode, 0, msh, [order, nelem, precision], os.path.join(d, "o.npz"))


def integrate(mode, msh, order):
    """slz_integrate of the reference build (ref_integrate) or the GPU drop-in
    (gpu_integrate): {"host": expression::integrate, "gpu": the GPU integral}."""
    with tempfile.TemporaryDirectory() as d:
        return _child(mode, 0, msh, [order], os.path.join(d, "o.npz"))


def eliminate(mode, workload, msh, params):
    with tempfile.TemporaryDirectory() as d:
        return _child(mode, workload, msh, params, os.path.join(d, "o.npz"))


def sweep(msh, order, f1, f2, sigmas, freqs, precision="fp64"):
    with tempfile.TemporaryDirectory() as d:
        return _child("sweep:" + precision, 0, msh, [order, f1, f2] + list(sigmas) + list(freqs), os.path.join(d, "o.npz"))


def reference(workload, msh, params, reps=1):
    with tempfile.TemporaryDirectory() as d:
        return _child("ref", workload, msh, params, os.path.join(d, "o.npz"), reps=reps)


def gpu(workload, msh, params, precision="fp64", reps=1, env=None):
    with tempfile.TemporaryDirectory() as d:
        return _child("gpu", workload, msh, params, os.path.join(d, "o.npz"), dict(env or {}, SLGPU_PRECISION=precision),
                      reps=reps)


def record_symmetry(workload, msh, params):
    """Lowers the workload on a record-only context (no GPU) and returns, per
    matrix group, its term count, the mirror term of each term
    (slgpu_matrix_group_symmetry), whether the split contraction would
    compute only the upper triangle, and its transposed partner group."""
    with tempfile.TemporaryDirectory() as d:
        return _child("symmetry", workload, msh, params, os.path.join(d, "o.npz"), {"SLGPU_RECORD_ONLY": "1"})


def symmetry_inproc(workload, msh, params):
    from sparselizard_b200 import abi
    from sparselizard_b200 import workloads as W

    assert os.environ.get("SLGPU_RECORD_ONLY") == "1"
    lib = W.load(GPU_LIB)
    try:
        W.run(GPU_LIB, workload, msh, params)
    except RuntimeError as e:
        assert "record-only" in str(e), str(e)
    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    h = lib.slgpu_adapter_last_handle()
    ng = ctypes.c_int()
    assert lib.slgpu_matrix_group_count(ctx, h, ctypes.byref(ng)) == 0
    nterms, mirror, sym, partner = [], [], [], []
    for gi in range(ng.value):
        desc = abi.GroupDesc()
        assert lib.slgpu_matrix_group_desc(ctx, h, gi, ctypes.byref(desc)) == 0
        m = np.zeros(desc.nterms, np.int32)
        s, pt = ctypes.c_int32(), ctypes.c_int32()
        assert lib.slgpu_matrix_group_symmetry(ctx, h, gi, m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(s),
                                               ctypes.byref(pt)) == 0
        nterms.append(desc.nterms)
        mirror.append(m)
        sym.append(s.value)
        partner.append(pt.value)
    return dict(nterms=np.array(nterms, np.int32), mirror=np.concatenate(mirror) if mirror else np.zeros(0, np.int32),
                symmetric=np.array(sym, np.int32), partner=np.array(partner, np.int32))


def record_oracle(workload, msh, params):
    """Lowers the workload with the drop-in on a record-only context (no GPU)
    and assembles the recorded groups with the C restatement oracle."""
    with tempfile.TemporaryDirectory() as d:
        return _child("record", workload, msh, params, os.path.join(d, "o.npz"), {"SLGPU_RECORD_ONLY": "1"})


def recorded_plan(lib):
    """Groups, constraints, rhs groups and mesh arrays of the last record-only run."""
    from sparselizard_b200 import abi

    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    h = lib.slgpu_adapter_last_handle()
    ng, nf = ctypes.c_int(), ctypes.c_int()
    groups = []
    if h:
        assert lib.slgpu_record_count(ctx, h, ctypes.byref(ng), ctypes.byref(nf)) == 0
        for i in range(ng.value):
            g = abi.Group()
            assert lib.slgpu_record_group(ctx, h, i, ctypes.byref(g)) == 0
            groups.append(g)
    frags = []
    for i in range(nf.value):
        ntr, ndr, nr, nc = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        rp, cp, vp = ctypes.POINTER(ctypes.c_int32)(), ctypes.POINTER(ctypes.c_int32)(), ctypes.POINTER(ctypes.c_double)()
        lib.slgpu_record_fragment(ctx, h, i, *(ctypes.byref(x) for x in (ntr, ndr, nr, nc, rp, cp, vp)))
        frags.append((ntr.value, ndr.value, nr.value, nc.value,
                      np.ctypeslib.as_array(rp, (ntr.value * nc.value,)).copy(),
                      np.ctypeslib.as_array(cp, (ndr.value * nc.value,)).copy(),
                      np.ctypeslib.as_array(vp, (nr.value * nc.value,)).copy()))
    ndofs = ctypes.c_int64()
    cptr = ctypes.POINTER(ctypes.c_uint8)()
    con = None
    if h:
        lib.slgpu_record_constraints(ctx, h, ctypes.byref(ndofs), ctypes.byref(cptr))
        if cptr:
            con = np.ctypeslib.as_array(cptr, (ndofs.value,)).copy()
    nr = ctypes.c_int()
    lib.slgpu_record_rhs_count(ctx, ctypes.byref(nr))
    rhs = []
    for i in range(nr.value):
        g = abi.Group()
        nd = ctypes.c_int64()
        lib.slgpu_record_rhs_group(ctx, i, ctypes.byref(g), ctypes.byref(nd))
        rhs.append((g, nd.value))

    def mesh(elemtype):
        nn, xp, ncn, ne, cp2 = ctypes.c_int64(), ctypes.POINTER(ctypes.c_double)(), ctypes.c_int(), ctypes.c_int64(), ctypes.POINTER(ctypes.c_int32)()
        assert lib.slgpu_record_mesh(ctx, 0, elemtype, *(ctypes.byref(x) for x in (nn, xp, ncn, ne, cp2))) == 0
        return (np.ctypeslib.as_array(xp, (3 * nn.value,)).copy(), np.ctypeslib.as_array(cp2, (ne.value * ncn.value,)).copy())

    return dict(groups=groups, frags=frags, ndofs=ndofs.value, constrained=con, rhs=rhs, mesh=mesh)


def record_oracle_inproc(workload, msh, params):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import slref

    from sparselizard_b200 import workloads as W

    assert os.environ.get("SLGPU_RECORD_ONLY") == "1"
    lib = W.load(GPU_LIB)
    try:
        W.run(GPU_LIB, workload, msh, params)
        raise AssertionError("a record-only run must not assemble")
    except RuntimeError as e:
        assert "record-only" in str(e), str(e)
    plan = recorded_plan(lib)
    out = {}
    # The runtime-generated coefficient kernels of the recorded groups must
    # compile (NVRTC runs on the host, no device needed).
    h = lib.slgpu_adapter_last_handle()
    if h:
        log = ctypes.create_string_buffer(4096)
        ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
        st = lib.slgpu_check_coefficient_kernels(ctx, h, log, 4096)
        assert st == 0, "coefficient kernel does not compile: " + log.value.decode(errors="replace")
    if plan["groups"] or plan["frags"]:
        xyz = None
        conns = []
        for g in plan["groups"]:
            xyz, conn = plan["mesh"](g.elemtype)
            conns.append(conn)
        if xyz is None:
            xyz = np.zeros(3)
        res = slref.matrix(plan["groups"], xyz, conns, plan["ndofs"], plan["constrained"], plan["frags"])
        out.update({k: res[k] for k in ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals")})
        mag = slref.matrix(plan["groups"], xyz, conns, plan["ndofs"], plan["constrained"], plan["frags"], absmode=True)
        out["Aabs"], out["Dabs"] = mag["Avals"], mag["Dvals"]
    b = None
    babs = None
    for g, nd in plan["rhs"]:
        xyz, conn = plan["mesh"](g.elemtype)
        bb = slref.rhs(g, xyz, conn, nd)
        ba = slref.rhs(g, xyz, conn, nd, absmode=True)
        b = bb if b is None else b + bb
        babs = ba if babs is None else babs + ba
    if b is not None:
        out["b_raw"] = b
        out["b_abs"] = babs
    out["ngroups"] = np.array(len(plan["groups"]))
    return out


def check_pattern(ref, other):
    for k in ("Arows", "Acols", "Drows", "Dcols"):
        a, b = np.asarray(ref[k]), np.asarray(other[k])
        assert a.shape == b.shape and np.array_equal(a, b), f"{k} differs from the reference"


def rowwise_rel_err(rows, ref_vals, vals):
    """max over rows of max|vals - ref| / max|ref| within the row (0 for empty rows)."""
    rows = np.asarray(rows, np.int64)
    if ref_vals.size == 0:
        return 0.0
    diff = np.abs(np.asarray(vals) - np.asarray(ref_vals))
    mag = np.abs(np.asarray(ref_vals))
    nz = np.diff(rows) > 0
    starts = rows[:-1][nz]
    dmax = np.maximum.reduceat(diff, starts)
    mmax = np.maximum.reduceat(mag, starts)
    floor = mag.max() * 1e-300 + 1e-300
    return float(np.max(dmax / np.maximum(mmax, floor)))


def scaled_errors(ref, other):
    """Entry-wise errors |a_ij - b_ij| / sqrt(S_i S_j), S = largest magnitude in
    each DOF's row/column of the reference (A and D together).  This is the
    error of the symmetrically scaled matrix D^-1/2 A D^-1/2: an entry that is
    exactly zero in exact arithmetic (e.g. curl-curl of a gradient form
    function) is judged against the scale of the terms that cancel in it, not
    against its own rounding noise.  Also returns the Frobenius-relative error.
    Computed with torch's multi-threaded CPU kernels (full-size workloads hold
    up to a few hundred million entries)."""
    import torch

    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt))
    Arows, Drows = t(ref["Arows"], np.int64), t(ref["Drows"], np.int64)
    Acols, Dcols = t(ref["Acols"], np.int64), t(ref["Dcols"], np.int64)
    Ar, Dr = t(ref["Avals"], np.float64), t(ref["Dvals"], np.float64)
    Ao, Do = t(other["Avals"], np.float64), t(other["Dvals"], np.float64)
    nA = Arows.numel() - 1
    rowA = torch.repeat_interleave(torch.arange(nA), Arows.diff())
    rowD = torch.repeat_interleave(torch.arange(nA), Drows.diff())
    S = torch.zeros(max(nA, 1), dtype=torch.float64)
    if Ar.numel():
        S.scatter_reduce_(0, rowA, Ar.abs(), "amax")
        S.scatter_reduce_(0, Acols, Ar.abs(), "amax")
    if Dr.numel():
        S.scatter_reduce_(0, rowD, Dr.abs(), "amax")
    Cd = torch.zeros(int(Dcols.max()) + 1 if Dcols.numel() else 1, dtype=torch.float64)
    if Dr.numel():
        Cd.scatter_reduce_(0, Dcols, Dr.abs(), "amax")
    floor = 1e-300
    eA = ((Ao - Ar).abs() / (S[rowA] * S[Acols]).sqrt().clamp_min(floor)).max().item() if Ar.numel() else 0.0
    eD = ((Do - Dr).abs() / (S[rowD] * Cd[Dcols]).sqrt().clamp_min(floor)).max().item() if Dr.numel() else 0.0
    num = float(((Ao - Ar) ** 2).sum() + ((Do - Dr) ** 2).sum())
    den = float((Ar ** 2).sum() + (Dr ** 2).sum())
    fro = (num / den) ** 0.5 if den > 0 else (0.0 if num == 0 else float("inf"))
    return float(eA), float(eD), float(fro)


def magnitude_errors(ref, other, mag):
    """max |a_ij - b_ij| / S_ij with S_ij = sum of |terms| summed into entry
    (i,j) (oracle magnitude mode): the relative error of each entry against
    the size of what was added up to form it, i.e. the quantity the standard
    floating-point bound |fl(sum) - sum| <= gamma_n * sum|terms| controls."""
    out = []
    for v, s in (("Avals", "Aabs"), ("Dvals", "Dabs")):
        a, b, S = np.asarray(ref[v]), np.asarray(other[v]), np.asarray(mag[s])
        if a.size == 0:
            out.append(0.0)
            continue
        floor = max(S.max(), 1e-300) * 1e-300
        out.append(float((np.abs(a - b) / np.maximum(S, floor)).max()))
    return out


def check_values(ref, other, tol, mag=None):
    """Values of A and D within tol.  With `mag` (oracle magnitude-mode
    output for the same plan) each entry is judged against the sum of the
    magnitudes of its terms; without it, against the symmetric row/column
    scale (scaled_errors).  The Frobenius-relative error must also be <= tol."""
    ea, ed, fro = scaled_errors(ref, other)
    if mag is not None:
        ea, ed = magnitude_errors(ref, other, mag)
    detail = f"(A {ea:.3e}, D {ed:.3e}, Frobenius {fro:.3e})"
    assert ea <= tol, f"A values: entry-wise error {ea:.3e} > {tol:g} {detail}"
    assert ed <= tol, f"D values: entry-wise error {ed:.3e} > {tol:g} {detail}"
    assert fro <= tol, f"Frobenius-relative error {fro:.3e} > {tol:g} {detail}"
    return ea, ed


def check_rhs(ref, b, tol, unconstrained_only=False, babs=None):
    """b within tol: against the magnitude sums `babs` entry by entry when
    given, else against max |b|."""
    rb = np.asarray(ref["b"])
    b = np.asarray(b)
    mask = np.ones(rb.size, bool)
    if unconstrained_only:
        mask[np.asarray(ref["Dinds"])] = False
    if not mask.any():
        return 0.0
    if babs is not None:
        babs = np.asarray(babs)[mask]
        scale = np.maximum(babs, max(babs.max(), 1e-300) * 1e-300)
    else:
        scale = max(np.abs(rb[mask]).max(), 1e-300)
    err = float((np.abs(rb[mask] - b[mask]) / scale).max())
    assert err <= tol, f"b: relative error {err:.3e} > {tol:g}"
    return err

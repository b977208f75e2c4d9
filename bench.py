#!/usr/bin/env python
"""Assembly benchmark: nnz/s of sparselizard's generate()/A()/b() path on B200.

A step is one assembly pass over the workload on its resident pattern:
geometry + coefficients + element contraction for every element group, then
the A/D CSR values (duplicates summed in a fixed order).  The first
generate()/A()/b() through the drop-in (lowering, upload, pattern build) is
reported separately as `first_assembly`.

value  : device throughput, inputs already in HBM (CUDA events on the engine's
         stream, summed over the K steps; max over ranks).
e2e    : the same metric through sparselizard's own API with the drop-in:
         warm generate() + A() + b() on the resident problem (host lowering,
         DOF addresses, uploads, assembly on the resident pattern and the
         download of the CSR values into the new rawmat that PETSc borrows;
         the rawmat shares the row pointers and column indices that an earlier
         download of the same pattern brought to the host).
--impl reference times stock sparselizard (built from its sources, CPU, all
host threads) on a bounded sample of the same workload (the same config).

The default run (C2) also reports: the plain FP64 GPU path and the FP32-level
tier on the same pattern with their errors, a parity check of the drop-in
against stock sparselizard at the sample size, and a `per_config` block with
the other workloads (C1, C3, C4 sweep, C5 serving) run as child processes.

Multi-GPU: element assembly of independent requests does not shard inside
one matrix without an exchange step, so N ranks run N independent replicas
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sparselizard_b200 import abi, meshgen, workloads as W  # noqa: E402

GPU_LIB = os.path.join(ROOT, "sparselizard_b200", "_build", "libslz_gpu.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libslz_ref.so")
SIGMAS = [1e3, 5.0e5, 2.0e6, 6.0e7]

# Workloads: the elasticity case is the headline (64^3 hexahedra, order-2
# vector field); the others are selectable with --workload.
WORKLOADS = {
    "c1": dict(kind=W.POISSON_QUAD, mesh="quad", n=256, params=[1], ref_n=256,
               name="poisson_q4_256x256_h1_order1"),
    "c2": dict(kind=W.ELASTICITY_HEX, mesh="hex", n=64, params=[2, -2], ref_n=32,
               name="elasticity_hex_64^3_h1xyz_order2"),
    "c3": dict(kind=W.HELMHOLTZ_TET, mesh="tet_orders", n=32, params=[], ref_n=16,
               name="helmholtz_tet_32^3x6_orders1to5"),
    "c4": dict(kind=W.EDDY_TET, mesh="tet_sigma", n=24, params=[2, 1.0e3] + SIGMAS, ref_n=8, sweep=64,
               name="eddy_hcurl_tet_24^3x6_order2_harmonics23_sweep64_1Hz_1MHz"),
    "c5": dict(kind="serve", name="serving_stream_2000req_poisson200rps_16meshes", requests=2000, rate=200.0),
}

# Serving pool: (physics 1 Poisson / 2 elasticity, mesh, n, dim, order); 1e3..1e6
# elements of quads, triangles, hexahedra and tetrahedra, orders 1..4.
SERVE_POOL = [
    (1, "quad", 1000, 2, 1), (1, "quad", 300, 2, 2), (1, "quad", 100, 2, 3), (1, "quad", 32, 2, 4),
    (1, "tri", 700, 2, 1), (1, "tri", 200, 2, 2), (1, "tri", 60, 2, 3), (1, "tri", 25, 2, 4),
    (1, "hex", 80, 3, 1), (2, "hex", 40, 3, 1), (2, "hex", 16, 3, 2), (1, "hex", 12, 3, 3),
    (1, "tet", 50, 3, 1), (2, "tet", 20, 3, 1), (1, "tet", 30, 3, 2), (1, "tet", 8, 3, 4),
]


def serving_per_problem(pool, prob, lat, dev, detail):
    """Per pool problem: requests, latency p50/p99, mean device time, mean
    server-thread launch time (and its input / contraction / value parts),
    mean queueing and submission delay (ms)."""
    out = []
    for i, p in enumerate(pool):
        m = prob == i
        if not m.any():
            continue
        d = detail[m]
        out.append(dict(problem=f'{p["physics"]} {p["mesh"]} n={p["n"]} order {p["order"]}', requests=int(m.sum()),
                        p50_ms=round(float(np.percentile(lat[m], 50) * 1e3), 3),
                        p99_ms=round(float(np.percentile(lat[m], 99) * 1e3), 3),
                        device_ms=round(float(dev[m].mean()), 3), launch_ms=round(float(d[:, 0].mean()), 3),
                        launch_parts_ms=[round(float(x), 3) for x in d[:, 1:4].mean(axis=0)],
                        queue_ms=round(float(d[:, 4].mean()), 3), submit_delay_ms=round(float(d[:, 5].mean()), 3)))
    return out


def write_pool_mesh(kind, n, path):
    {"quad": meshgen.quad_mesh, "tri": meshgen.tri_mesh, "hex": meshgen.hex_mesh, "tet": meshgen.tet_mesh}[kind](path, n)


def write_mesh(spec, n, path):
    meshgen.workload_mesh(spec["mesh"], n, path)


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples taken while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM bytes (read + write) per launch of the dominant kernels, from ncu
# captures of a smaller case of the same workload, per element of the
# launch's group (traffic grows in proportion to the elements).  Summaries
# and the commands that made them are under profiles/.
TRAFFIC_PER_ELEMENT = {
    # profiles/k_contract_split_elasticity_hex32.md, 32768 elements: the one
    # launch of a step (all six contracted groups) reads 417.57 MB and writes
    # 1721.87 MB.
    ("c2", "contract_split"): (417.574912e6 + 1721.872e6) / 32768,
    # profiles/k_row_values_elasticity_hex32.md: 3.140 GB read + 1.187 GB
    # written by the launch over all 9 groups of 32768 elements.
    ("c2", "row_values"): (3.140404e9 + 1.187079e9) / 32768,
}


def traffic_per_launch(workload, family, n, launches):
    per = TRAFFIC_PER_ELEMENT.get((workload, family))
    if per is None:
        return None
    nelem = {"c2": n ** 3, "c1": n * n}.get(workload)
    return None if nelem is None else per * nelem


FAMILIES = ("coefficients", "contract_fp64", "slice_cols", "contract_split", "contract_split_fp32", "row_values")


def kernel_stats(lib, ctx, acc):
    """Adds the per-kernel-family event times of the last process() to acc."""
    for fam in FAMILIES:
        ms, nl, wk = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
        lib.slgpu_kernel_stats(ctx, fam.encode(), ctypes.byref(ms), ctypes.byref(nl), ctypes.byref(wk))
        if nl.value > 0:
            a = acc.setdefault(fam, {"ms": 0.0, "launches": 0, "work": 0.0})
            a["ms"] += ms.value
            a["launches"] += nl.value
            a["work"] += wk.value
    return acc


def dist_setup(n_gpus):
    """One process per GPU (torchrun sets RANK/WORLD_SIZE/LOCAL_RANK).  The
    process group only carries the barrier and the max/sum over replicas:
    NCCL on GPUs, gloo where there is no CUDA device (tests)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def allreduce(vals, op):
    """Element-wise reduction of a list of floats over the replicas."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized():
        return vals
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return t.tolist()


def replica_value(total_units_local, seconds_local):
    """Whole-job throughput of N replicas: units of all ranks / the slowest
    rank's time (max over ranks), as the timing rules ask."""
    import torch.distributed as dist

    if dist.is_initialized():
        secs, = allreduce([seconds_local], dist.ReduceOp.MAX)
        units, = allreduce([float(total_units_local)], dist.ReduceOp.SUM)
    else:
        secs, units = seconds_local, float(total_units_local)
    return units / secs, secs, units


def host_info():
    """Host cores, memory and the dgemm the reference build uses."""
    info = {"nproc": os.cpu_count() or 1}
    try:
        import psutil

        info["host_mem_gb"] = round(psutil.virtual_memory().total / 1e9, 1)
    except Exception:
        pass
    try:
        info["cpu_model"] = next(l.split(":", 1)[1].strip() for l in open("/proc/cpuinfo") if l.startswith("model name"))
    except Exception:
        pass
    return info


def cpu_reference_run(spec, n, reps, warmup, threads, keep=False):
    """Stock sparselizard generate()+A()+b() on the host cores: warm-up
    repetitions, then `reps` timed ones (wall seconds each); with keep=True
    also the last repetition's arrays (for the parity check)."""
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(threads))
    with tempfile.TemporaryDirectory() as d:
        msh = os.path.join(d, "m.msh")
        write_mesh(spec, n, msh)
        r = W.run(REF_LIB, spec["kind"], msh, spec["params"], reps=warmup + reps, threads=threads)
    per = r.times[warmup:].sum(axis=1)
    dg = W.dgemm_name(W.load(REF_LIB))
    return r.nnz, per, dg, (r if keep else None)


def headline_config(spec, n, world):
    """`config` of both arms: the workload as named, its size and the run shape."""
    return {"workload": spec["name"], "n": n, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2" if spec["name"].startswith(("elasticity", "eddy", "helmholtz")) else
            "L2 flushed between steps"}


def run_reference(args, spec):
    """Stock sparselizard on the host cores, all threads, on a bounded sample of
    the workload (n = ref_n): W warm-up and K timed generate()+A()+b()."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n_sample = spec["ref_n"]
    # The W warm-up steps run the same path on the half-size mesh (untimed),
    # so that the K timed steps at the sample size end within a few minutes.
    n_warm = max(4, n_sample // 2)
    if args.warmup > 0:
        cpu_reference_run(spec, n_warm, args.warmup, 0, threads)
    nnz, per, dg, _ = cpu_reference_run(spec, n_sample, args.steps, 0, threads)
    value = nnz / float(np.mean(per))
    sample = (f"{spec['name']} at n={n_sample} ({nnz} nnz) instead of n={spec['n']}: generate()+A()+b() per timed step "
              f"(warm-up steps at n={n_warm}), {threads} threads, dgemm: {dg}")
    line = {
        "impl": "reference", "metric": "assembled_nnz_per_s", "value": value, "unit": "nnz/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(per)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded jittered mesh)",
        "config": headline_config(spec, args.n or spec["n"], args.gpus),
        "sample_n": n_sample,
        "cpu_baseline": {"value": value, "unit": "nnz/s", "cores": threads, "kind": "reference", "sample": sample,
                         "host": host_info(), "dgemm": dg},
        "e2e": {"value": value, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


KERNEL_NAMES = {"coefficients": "slgpu_coef (runtime-compiled)", "contract_fp64": "k_contract_fp64 / k_contract_small",
                "slice_cols": "k_slice_cols", "contract_split": "k_contract_split<7,8>",
                "contract_split_fp32": "k_contract_split<5,6>", "row_values": "k_row_values / k_row_stream (chosen per pattern)"}


def int8_peak_tops(sustained_s=2.0):
    """Dense INT8 tensor throughput of this GPU, measured with torch._int_mm on
    8192^3 int8 operands (2 N^3 ops), CUDA events: the best of 10 single calls
    after warm-up (burst), and the mean over back-to-back calls for
    `sustained_s` seconds (sustained: what the power cap allows a kernel that
    runs inside a long step).  Returns (burst, sustained) in TOPS."""
    import torch

    n = 8192
    a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
    for _ in range(3):
        torch._int_mm(a, b)
    best = float("inf")
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(10, int(sustained_s / (best * 1e-3)))
    e0.record()
    for _ in range(reps):
        torch._int_mm(a, b)
    e1.record()
    e1.synchronize()
    mean = e0.elapsed_time(e1) / reps
    del a, b
    torch.cuda.empty_cache()
    ops = 2.0 * n ** 3
    return ops / (best * 1e-3) / 1e12, ops / (mean * 1e-3) / 1e12


def roofline_of(stats, workload, n, int8_tops=None):
    """Roofline entry of the kernel family with the most device time in `stats`
    (CUDA-event times and algorithmic work summed over launches)."""
    hbm, bf16, peak_kind = peaks()
    dom = max(stats, key=lambda f: stats[f]["ms"])
    k = stats[dom]
    rate = k["work"] / (k["ms"] * 1e-3)
    if dom.startswith("contract_split"):
        if int8_tops:
            burst, sustained = int8_tops
            kind = ("measured INT8 dense, burst (torch._int_mm 8192^3, best of 10, this run); achieved counts INT8 ops; "
                    "peak_sustained: the same GEMM back to back for 2 s under the power cap")
        else:
            burst = sustained = 2.0 * bf16
            kind = f"INT8 dense = 2 x {peak_kind} bf16 burst ({bf16:.0f} TFLOP/s); achieved counts INT8 ops"
        roof = {"kernel": KERNEL_NAMES[dom], "bound": "tensor", "achieved": rate / 1e12, "peak": burst, "unit": "TFLOP/s",
                "peak_kind": kind, "frac": rate / 1e12 / burst, "peak_sustained": sustained,
                "frac_of_sustained": rate / 1e12 / sustained}
    elif dom == "contract_fp64":
        roof = {"kernel": KERNEL_NAMES[dom], "bound": "tensor", "achieved": rate / 1e12, "peak": 40.0, "unit": "TFLOP/s",
                "peak_kind": "nominal B200 FP64 40 TFLOP/s (FP64 vector and tensor rates are equal; not measured here)",
                "frac": rate / 1e12 / 40.0}
    else:
        roof = {"kernel": KERNEL_NAMES[dom], "bound": "hbm", "achieved": rate / 1e9, "peak": hbm, "unit": "GB/s",
                "peak_kind": peak_kind, "frac": rate / 1e9 / hbm}
    roof["ms_per_launch"] = k["ms"] / k["launches"]
    roof["traffic"] = traffic_per_launch(workload, dom, n, k["launches"])
    return roof


def pattern_digest(a):
    import hashlib

    h = hashlib.sha256()
    for k in ("Arows", "Acols", "Drows", "Dcols", "Ainds", "Dinds"):
        h.update(np.ascontiguousarray(getattr(a, k) if not isinstance(a, dict) else a[k], np.int32).tobytes())
    return h.hexdigest()[:16]


def parity_vs_reference(spec, n, ref, precision):
    """The drop-in at the reference's sample size (child process on this GPU)
    against stock sparselizard's arrays `ref` of the same mesh: pattern digest
    of both, entry-wise error against the symmetric row/column scale and the
    Frobenius-relative error of the values, and b."""
    with tempfile.TemporaryDirectory() as d:
        msh, out = os.path.join(d, "m.msh"), os.path.join(d, "g.npz")
        write_mesh(spec, n, msh)
        code = ("import sys, numpy as np; sys.path.insert(0, %r); from sparselizard_b200 import workloads as W; "
                "r = W.run(%r, %d, %r, %r); np.savez(%r, **{k: getattr(r, k) for k in %r})"
                % (ROOT, GPU_LIB, spec["kind"], msh, list(spec["params"]), out,
                   ("Arows", "Acols", "Avals", "Drows", "Dcols", "Dvals", "Ainds", "Dinds", "b")))
        env = dict(os.environ, SLGPU_PRECISION=precision)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            return {"error": (r.stdout + r.stderr)[-400:]}
        g = dict(np.load(out))
    dref, dgot = pattern_digest(ref), pattern_digest(g)
    import torch

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    # Symmetric row/column scale S_i = max |entry| in row/column i of the reference.
    nA = ref.Arows.size - 1
    rowA = torch.repeat_interleave(torch.arange(nA), t(ref.Arows.astype(np.int64)).diff())
    Ar, Ag = t(ref.Avals), t(g["Avals"])
    S = torch.zeros(max(nA, 1), dtype=torch.float64)
    S.scatter_reduce_(0, rowA, Ar.abs(), "amax")
    S.scatter_reduce_(0, t(ref.Acols.astype(np.int64)), Ar.abs(), "amax")
    same = dref == dgot
    ent = float(((Ag - Ar).abs() / (S[rowA] * S[t(ref.Acols.astype(np.int64))]).sqrt().clamp_min(1e-300)).max()) if same else None
    fro = float((((Ag - Ar) ** 2).sum() + ((t(g["Dvals"]) - t(ref.Dvals)) ** 2).sum()).sqrt() /
                ((Ar ** 2).sum() + (t(ref.Dvals) ** 2).sum()).sqrt()) if same else None
    bscale = max(float(np.abs(ref.b).max()), 1e-300)
    return {"sample_n": n, "precision": precision, "nnz": int(ref.nnz), "pattern_digest_reference": dref,
            "pattern_digest_gpu": dgot, "pattern_bit_exact": bool(same), "max_scaled_err": ent, "rel_fro_err": fro,
            "b_max_rel_err": float(np.abs(g["b"] - ref.b).max() / bscale) if g["b"].size == ref.b.size else None}


def cpu_baseline(args, spec, rank, world):
    """Stock sparselizard (oracle/_ref) on the host cores, on the workload's
    bounded sample size, rank 0 of a one-GPU run only.  Returns the baseline
    entry and the last repetition's arrays."""
    if rank != 0 or world != 1 or args.no_cpu_baseline or not os.path.exists(REF_LIB):
        return None, None
    threads = os.cpu_count() or 1
    cnnz, per, dg, r = cpu_reference_run(spec, spec["ref_n"], 2, 1, threads, keep=True)
    return ({"value": cnnz / float(np.mean(per)), "unit": "nnz/s", "cores": threads, "kind": "reference",
             "sample": f"stock sparselizard generate()+A()+b(), {spec['name']} at n={spec['ref_n']} ({cnnz} nnz), "
                       f"mean of 2 after 1 warm-up", "dgemm": dg, "host": host_info()}, r)


def run_ours(args, spec):
    import torch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    os.environ["SLGPU_DEVICE"] = str(local)
    os.environ["SLGPU_PRECISION"] = args.precision
    prec = {"fp64": abi.PREC_FP64, "split": abi.PREC_SPLIT, "fp32": abi.PREC_FP32}[args.precision]
    int8_tops = int8_peak_tops()
    tmpd = tempfile.mkdtemp(prefix=f"slbench{rank}_")
    msh = os.path.join(tmpd, "m.msh")
    n = args.n or spec["n"]
    write_mesh(spec, n, msh)

    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    lib.slz_bench_prepare.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_bench_reassemble.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_bench_constraints.restype = ctypes.POINTER(ctypes.c_uint8)
    params = (ctypes.c_double * max(1, len(spec["params"])))(*spec["params"])
    t3 = (ctypes.c_double * 3)()
    info4 = (ctypes.c_longlong * 4)()
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    h2d0, d2h0 = ctypes.c_int64(), ctypes.c_int64()
    rc = lib.slz_bench_prepare(spec["kind"], msh.encode(), params, t3, info4)
    if rc != 0:
        raise RuntimeError("prepare failed: " + lib.slz_last_error().decode(errors="replace"))
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    handle = int(info4[0])
    ndofs = int(info4[1])
    cons = lib.slz_bench_constraints()
    info = abi.CsrInfo()

    def process(p=None):
        st = lib.slgpu_matrix_process(ctx, handle, cons, prec if p is None else p, ctypes.byref(info))
        if st != 0:
            buf = ctypes.create_string_buffer(2048)
            lib.slgpu_last_error(ctx, buf, 2048)
            raise RuntimeError(f"process failed ({st}): {buf.value.decode()}")
        ms = np.zeros(5)
        lib.slgpu_last_timings(ctx, abi.f64p(ms))
        return ms

    work = abi.Work()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # Timed steps without per-kernel events (a replayed graph then holds only
    # the kernels); the per-kernel breakdown comes from separate steps below.
    lib.slgpu_ctx_set_kernel_timers(ctx, 0)
    for _ in range(args.warmup):
        process()
    lib.slgpu_matrix_work(ctx, handle, ctypes.byref(work))
    nnz = int(work.nnz)
    first = dict(generate_s=t3[0], A_s=t3[1], b_s=t3[2], nnz_per_s=nnz / max(t3[0] + t3[1] + t3[2], 1e-12))
    l2_rule = "inputs larger than L2" if work.nvalid * 8 > 126e6 else "L2 flushed between steps"

    def timed_steps(p, k):
        ph = np.zeros(5)
        for _ in range(k):
            flush.zero_()
            torch.cuda.synchronize()
            ph += process(p)
        return ph

    # ---- device-resident steps
    stats = {}
    launches0 = lib.slgpu_kernel_launches(ctx)
    graphs0 = lib.slgpu_graph_launches(ctx)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        phase = timed_steps(None, args.steps)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
    launches = lib.slgpu_kernel_launches(ctx) - launches0
    graph_replays = lib.slgpu_graph_launches(ctx) - graphs0
    dev_ms = phase[4] / args.steps
    dev_ms_max, = allreduce([dev_ms], torch.distributed.ReduceOp.MAX) if world > 1 else [dev_ms]
    total_nnz, = allreduce([float(nnz)], torch.distributed.ReduceOp.SUM) if world > 1 else [float(nnz)]
    value = total_nnz / (dev_ms_max * 1e-3)

    # ---- values of this precision, then the plain FP64 GPU path and the
    # FP32-level tier on the same resident pattern, each with its error
    # against FP64 on the assembled matrix (A and D values)
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]

    def download():
        """The assembled A and D values, copied on the device (D2D) into one tensor."""
        ptr = [ctypes.c_void_p() for _ in range(6)]
        assert lib.slgpu_matrix_device_csr(ctx, handle, *[ctypes.byref(q) for q in ptr]) == 0
        torch.cuda.synchronize()
        v = torch.empty(info.nnzA + info.nnzD, dtype=torch.float64, device="cuda")
        if info.nnzA:
            assert cudart.cudaMemcpy(v.data_ptr(), ptr[2], 8 * info.nnzA, 3) == 0
        if info.nnzD:
            assert cudart.cudaMemcpy(v.data_ptr() + 8 * info.nnzA, ptr[5], 8 * info.nnzD, 3) == 0
        return v

    def rel_fro(a, b):
        num = den = 0.0
        for i in range(0, a.numel(), 1 << 28):
            d = a[i:i + (1 << 28)] - b[i:i + (1 << 28)]
            num += float(d @ d)
            den += float(b[i:i + (1 << 28)] @ b[i:i + (1 << 28)])
        return (num / den) ** 0.5 if den > 0 else 0.0

    tiers = {}
    mine = download()
    if prec != abi.PREC_FP64:
        for _ in range(args.warmup):
            process(abi.PREC_FP64)
        ph64 = timed_steps(abi.PREC_FP64, args.steps)
        ref64 = download()
        ms64 = ph64[4] / args.steps
        ms64_max, = allreduce([ms64], torch.distributed.ReduceOp.MAX) if world > 1 else [ms64]
        tiers["fp64"] = {"value": total_nnz / (ms64_max * 1e-3), "ms_per_step": ms64_max}
        tiers[args.precision] = {"value": value, "ms_per_step": dev_ms_max, "rel_fro_err_vs_fp64": rel_fro(mine, ref64),
                                 "speedup_vs_fp64": ms64_max / dev_ms_max}
        if prec != abi.PREC_FP32:
            for _ in range(args.warmup):
                process(abi.PREC_FP32)
            ph32 = timed_steps(abi.PREC_FP32, args.steps)
            ms32 = ph32[4] / args.steps
            tiers["fp32"] = {"value": total_nnz / (ms32 * 1e-3), "ms_per_step": ms32,
                             "rel_fro_err_vs_fp64": rel_fro(download(), ref64), "speedup_vs_fp64": ms64_max / ms32}
        del ref64
    del mine

    # ---- per-kernel and per-phase events: the same steps again with timers on
    # (after warm-up steps that capture the graph with its event nodes), for
    # this precision and for the FP64 path
    lib.slgpu_ctx_set_kernel_timers(ctx, 1)
    for _ in range(args.warmup):
        process()
    phase = np.zeros(5)
    with ClockSampler(local) as clk_k:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            phase += process()
            kernel_stats(lib, ctx, stats)
    if "fp64" in tiers:
        st64 = {}
        for _ in range(min(args.warmup, 2)):
            process(abi.PREC_FP64)
        for _ in range(min(args.steps, 5)):
            flush.zero_()
            torch.cuda.synchronize()
            process(abi.PREC_FP64)
            kernel_stats(lib, ctx, st64)
        tiers["fp64"]["kernels"] = st64
        c = st64.get("contract_fp64")
        if c:
            tiers["fp64"]["contract_fp64_tflops"] = c["work"] / (c["ms"] * 1e-3) / 1e12
    lib.slgpu_ctx_set_kernel_timers(ctx, 0)
    ph = phase / args.steps
    roof = roofline_of(stats, args.workload, n, int8_tops)
    tb = ctypes.create_string_buffer(8192)
    lib.slgpu_tuned_tiles(ctx, tb, 8192)
    tuned = [x for x in tb.value.decode().splitlines() if x]

    # ---- end to end through sparselizard's API: warm generate() + A() + b()
    # of the resident problem (one untimed warm repetition first)
    e2e_reps = max(1, min(args.steps, args.e2e_steps))
    tt = (ctypes.c_double * (3 * (e2e_reps + 1)))()
    lib.slgpu_transfer_bytes(ctx, ctypes.byref(h2d0), ctypes.byref(d2h0))
    torch.cuda.synchronize()
    if lib.slz_bench_reassemble(1, tt, info4) != 0:
        raise RuntimeError("reassemble failed: " + lib.slz_last_error().decode(errors="replace"))
    h2d1, d2h1 = ctypes.c_int64(), ctypes.c_int64()
    lib.slgpu_transfer_bytes(ctx, ctypes.byref(h2d1), ctypes.byref(d2h1))
    if lib.slz_bench_reassemble(e2e_reps, tt, info4) != 0:
        raise RuntimeError("reassemble failed: " + lib.slz_last_error().decode(errors="replace"))
    torch.cuda.synchronize()
    h2d2, d2h2 = ctypes.c_int64(), ctypes.c_int64()
    lib.slgpu_transfer_bytes(ctx, ctypes.byref(h2d2), ctypes.byref(d2h2))
    et = np.ctypeslib.as_array(tt, (3 * (e2e_reps + 1),))[: 3 * e2e_reps].reshape(e2e_reps, 3)
    e2e_s = float(et.sum(axis=1).mean())
    e2e_s_max, = allreduce([e2e_s], torch.distributed.ReduceOp.MAX) if world > 1 else [e2e_s]
    e2e = {"value": total_nnz / e2e_s_max, "unit": "nnz/s", "ms_per_step": e2e_s_max * 1e3, "steps": e2e_reps,
           "phases_s": {"generate": float(et[:, 0].mean()), "A": float(et[:, 1].mean()), "b": float(et[:, 2].mean())},
           "h2d_bytes_per_step": int((h2d2.value - h2d1.value) / e2e_reps),
           "d2h_bytes_per_step": int((d2h2.value - d2h1.value) / e2e_reps),
           "what": "warm generate()+A()+b() through sparselizard's API with the drop-in: host lowering and DOF "
                   "addresses, uploads, assembly on the resident pattern, download of the CSR values into a new "
                   "rawmat, which shares the row pointers and column indices downloaded for the same pattern before "
                   "(one untimed warm repetition first; first_assembly downloads all CSR arrays)"}
    lib.slz_bench_release()
    del flush
    torch.cuda.empty_cache()

    cpu, ref_arrays = cpu_baseline(args, spec, rank, world)
    parity = None
    if ref_arrays is not None:
        parity = parity_vs_reference(spec, spec["ref_n"], ref_arrays, args.precision)
        del ref_arrays
    per_config = run_per_config(args) if (rank == 0 and world == 1 and args.workload == "c2" and not args.no_per_config) else None

    if rank == 0:
        line = {
            "metric": "assembled_nnz_per_s", "value": value, "unit": "nnz/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered mesh)",
            "config": headline_config(spec, n, world),
            "workload_detail": {"precision": args.precision, "ndofs": ndofs, "nnz": nnz, "ncoo": int(work.ncoo),
                                "groups": int(work.ngroups), "l2": l2_rule,
                                "timing": "ms_per_step from steps without per-kernel events; phases_ms, kernels and "
                                          "roofline from as many steps with them"},
            "phases_ms": {"geometry_coef": ph[0], "contraction": ph[1], "values": ph[3], "total": ph[4]},
            "kernels": stats,
            "tiers": tiers,
            "first_assembly": first,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "graph_replays": int(graph_replays),
            "roofline": roof,
            "tuned": tuned,
            "int8_peak_tops": {"burst": int8_tops[0], "sustained": int8_tops[1]},
            "cpu_baseline": cpu,
            "parity": parity,
            "per_config": per_config,
            "clocks": clk.summary(),
            "clocks_kernel_steps": clk_k.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _child_line(argv, timeout):
    """Runs bench.py with argv in a child process; returns its JSON line."""
    t0 = time.perf_counter()
    r = subprocess.run([sys.executable, os.path.abspath(__file__)] + argv, capture_output=True, text=True, timeout=timeout)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": (r.stdout + r.stderr)[-500:], "rc": r.returncode}
    d = json.loads(lines[-1])
    d["child_wall_s"] = round(time.perf_counter() - t0, 1)
    return d


def run_per_config(args):
    """The other workloads, each in a child process on this GPU after the
    headline's memory is released: their device and end-to-end nnz/s, the
    split and FP32-tier errors against FP64, C4's sweep and C5's served
    latencies.  Errors are reported in place of a line that failed."""
    out = {}
    k = ["--steps", "10", "--warmup", "3", "--no-cpu-baseline", "--no-per-config"]
    for name in ("c1", "c3"):
        d = _child_line(["--workload", name] + k, 900)
        out[name] = d if "error" in d else {
            "workload": d["config"]["workload"], "value": d["value"], "ms_per_step": d["ms_per_step"],
            "e2e": d["e2e"]["value"], "e2e_ms_per_step": d["e2e"]["ms_per_step"], "tiers": d.get("tiers"),
            "first_assembly": d.get("first_assembly"), "roofline": d.get("roofline"), "child_wall_s": d["child_wall_s"]}
    d = _child_line(["--workload", "c4", "--warmup", "3", "--no-cpu-baseline"], 900)
    out["c4"] = d if "error" in d else {
        "workload": d["config"]["workload"], "value": d["value"], "ms_per_frequency": d["ms_per_step"],
        "e2e": d["e2e"]["value"], "e2e_ms_per_frequency": d["e2e"]["ms_per_step"], "tiers": d.get("tiers"),
        "roofline": d.get("roofline"), "child_wall_s": d["child_wall_s"]}
    d = _child_line(["--workload", "c5", "--warmup", "3"], 1200)
    out["c5"] = d if "error" in d else {
        "workload": d["config"]["workload"], "serving": {
            p: {k2: v for k2, v in d["serving"][p].items() if k2 not in ("per_problem", "clocks")} for p in d["serving"]},
        "errors_vs_fp64": d.get("errors_vs_fp64"), "child_wall_s": d["child_wall_s"]}
    return out


def run_sweep(args, spec):
    """C4: the harmonic problem re-assembled at 64 log-spaced frequencies on its
    resident pattern (scales set per frequency, no generate())."""
    import torch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    os.environ["SLGPU_DEVICE"] = str(local)
    os.environ["SLGPU_PRECISION"] = args.precision
    prec = {"fp64": abi.PREC_FP64, "split": abi.PREC_SPLIT, "fp32": abi.PREC_FP32}[args.precision]
    tmpd = tempfile.mkdtemp(prefix=f"slsweep{rank}_")
    msh = os.path.join(tmpd, "m.msh")
    n = args.n or spec["n"]
    write_mesh(spec, n, msh)
    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slz_sweep_prepare.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                      ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_sweep_run.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    lib.slz_sweep_values.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.slz_sweep_values.restype = ctypes.c_longlong
    sig = (ctypes.c_double * 4)(*SIGMAS)
    info = (ctypes.c_longlong * 4)()
    t0 = time.perf_counter()
    if lib.slz_sweep_prepare(msh.encode(), 2, sig, 1.0e3, 1.0e5, info) != 0:
        raise RuntimeError("sweep prepare failed: " + lib.slz_last_error().decode(errors="replace"))
    prep_s = time.perf_counter() - t0
    nnz = int(info[2])
    nf = spec["sweep"]
    freqs = np.logspace(0.0, 6.0, nf)
    dev, host = np.zeros(nf), np.zeros(nf)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    for _ in range(args.warmup):
        lib.slz_sweep_run(min(nf, 3), abi.f64p(freqs), prec, abi.f64p(dev), abi.f64p(host))
    launches0, graphs0 = lib.slgpu_kernel_launches(ctx), lib.slgpu_graph_launches(ctx)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if lib.slz_sweep_run(nf, abi.f64p(freqs), prec, abi.f64p(dev), abi.f64p(host)) != 0:
            raise RuntimeError("sweep failed: " + lib.slz_last_error().decode(errors="replace"))
        torch.cuda.synchronize()
    launches = lib.slgpu_kernel_launches(ctx) - launches0
    graph_replays = lib.slgpu_graph_launches(ctx) - graphs0
    stats = kernel_stats(lib, ctx, {})  # the last frequency's process()
    dev_s = dev.sum() * 1e-3
    dev_s_max, = allreduce([dev_s], torch.distributed.ReduceOp.MAX) if world > 1 else [dev_s]
    total, = allreduce([float(nnz) * nf], torch.distributed.ReduceOp.SUM) if world > 1 else [float(nnz) * nf]
    # End to end: scale update, process and download of the values per frequency.
    nnzA = int(lib.slz_sweep_values(None, None))
    A = np.zeros(max(1, nnzA))
    D = np.zeros(max(1, nnz - nnzA))
    d1, h1 = np.zeros(1), np.zeros(1)
    t0 = time.perf_counter()
    for f in freqs:
        lib.slz_sweep_run(1, abi.f64p(np.array([f])), prec, abi.f64p(d1), abi.f64p(h1))
        lib.slz_sweep_values(abi.f64p(A), abi.f64p(D))
    e2e_s = time.perf_counter() - t0
    # Errors of the split and FP32-level tiers against the FP64 path at the
    # last frequency (values of A and D), and their device times there.
    tiers = {}
    vals = {}
    for name, p in (("fp64", abi.PREC_FP64), ("split", abi.PREC_SPLIT), ("fp32", abi.PREC_FP32)):
        last = np.ascontiguousarray(freqs[-1:])
        for _ in range(3):
            if lib.slz_sweep_run(1, abi.f64p(last), p, abi.f64p(d1), abi.f64p(h1)) != 0:
                raise RuntimeError("sweep failed: " + lib.slz_last_error().decode(errors="replace"))
        lib.slz_sweep_values(abi.f64p(A), abi.f64p(D))
        vals[name] = np.concatenate([A[:nnzA], D[: nnz - nnzA]])
        tiers[name] = {"ms_at_last_frequency": float(d1[0])}
    r64 = vals["fp64"]
    for name in ("split", "fp32"):
        tiers[name]["rel_fro_err_vs_fp64"] = float(np.linalg.norm(vals[name] - r64) / max(np.linalg.norm(r64), 1e-300))
    del vals, r64
    lib.slz_sweep_release()
    roof = roofline_of(stats, args.workload, n)
    cpu, _ = cpu_baseline(args, spec, rank, world)
    if rank == 0:
        line = {
            "metric": "assembled_nnz_per_s", "value": total / dev_s_max, "unit": "nnz/s", "n_gpus": world, "steps": nf,
            "warmup": args.warmup, "ms_per_step": dev_s_max * 1e3 / nf, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered tet mesh, random material regions)",
            "config": {"workload": spec["name"], "n": n, "precision": args.precision, "nnz": nnz, "frequencies": nf,
                       "prepare_s": prep_s, "parallelism": f"replicas{world}", "l2": "inputs larger than L2"},
            "e2e": {"value": total / e2e_s, "unit": "nnz/s", "ms_per_step": e2e_s * 1e3 / nf, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 * nnz},
            "kernels_last_frequency": stats,
            "tiers": tiers,
            "gpu_launches": int(launches),
            "graph_replays": int(graph_replays),
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_serving(args, spec):
    """C5: a pool of resident problems and a Poisson stream of requests with new
    per-element coefficient fields, served by the engine's request server."""
    import torch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    os.environ["SLGPU_DEVICE"] = str(local)
    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    lib.slz_serve_add.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_serve_run_warm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double)]
    lib.slz_serve_error.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    tmpd = tempfile.mkdtemp(prefix=f"slserve{rank}_")
    pool = []
    t0 = time.perf_counter()
    for i, (phys, mk, n, dim, order) in enumerate(SERVE_POOL):
        msh = os.path.join(tmpd, f"p{i}.msh")
        write_pool_mesh(mk, n, msh)
        info = (ctypes.c_longlong * 6)()
        idx = lib.slz_serve_add(phys, msh.encode(), dim, order, info)
        if idx < 0:
            raise RuntimeError("serve_add failed: " + lib.slz_last_error().decode(errors="replace"))
        pool.append(dict(physics=["poisson", "elasticity"][phys - 1], mesh=mk, n=n, order=order, nnz=int(info[1] + info[2]),
                         elements=int(info[3]), ndofs=int(info[5])))
        err2 = np.zeros(2)
        if lib.slz_serve_error(idx, abi.f64p(err2)) != 0:
            raise RuntimeError("serve_error failed: " + lib.slz_last_error().decode(errors="replace"))
        pool[-1]["rel_fro_err_vs_fp64"] = {"split": float(err2[0]), "fp32": float(err2[1])}
        os.remove(msh)
    setup_s = time.perf_counter() - t0
    nreq = args.requests or spec["requests"]
    nwarm = max(args.warmup, 0) * 50  # warm-up requests on the same server before the measured stream
    rate = spec["rate"]
    res = {}
    for name, prec in (("split", abi.PREC_SPLIT), ("fp64", abi.PREC_FP64)):
        lat = np.zeros(nreq)
        done = np.zeros(nreq)
        dev = np.zeros(nreq)
        prob = np.zeros(nreq, np.int32)
        detail = np.zeros((nreq, 6))
        summ = np.zeros(9)
        with ClockSampler(local) as clk:
            rc = lib.slz_serve_run_warm(nwarm, nreq, rate, args.slots, prec, 12345, min(8, os.cpu_count() or 4), abi.f64p(lat),
                                        abi.f64p(done), abi.f64p(dev), prob.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        abi.f64p(detail), abi.f64p(summ))
        if rc != 0:
            raise RuntimeError("serve_run failed: " + lib.slz_last_error().decode(errors="replace"))
        res[name] = dict(p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                         p90_ms=float(np.percentile(lat, 90) * 1e3), max_ms=float(lat.max() * 1e3), warmup_requests=nwarm,
                         mean_ms=float(lat.mean() * 1e3), matrices_per_s=nreq / summ[0], nnz_per_s=summ[1] / summ[0],
                         wall_s=float(summ[0]), device_busy=float(summ[2] * 1e-3 / summ[0]), late_submissions=int(summ[3]),
                         launch_ms=float(summ[4]), launch_parts_ms=[float(x) for x in summ[6:9]], queue_ms=float(summ[5]),
                         per_problem=serving_per_problem(pool, prob, lat, dev, detail), clocks=clk.summary())
    lib.slz_serve_release()
    if rank == 0:
        mixed, plain = res["split"], res["fp64"]
        line = {
            "metric": "assembled_nnz_per_s", "value": mixed["nnz_per_s"], "unit": "nnz/s", "n_gpus": world,
            "steps": nreq, "warmup": nwarm, "ms_per_step": mixed["mean_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded meshes, lognormal per-element coefficients)",
            "config": {"workload": spec["name"], "requests": nreq, "rate_per_s": rate, "slots": args.slots,
                       "pool": pool, "setup_s": setup_s, "parallelism": f"replicas{world}",
                       "l2": "per-request inputs and outputs cross PCIe; no L2 flush"},
            "serving": {"mixed_precision": mixed, "fp64": plain},
            "errors_vs_fp64": {"split_max": max(p["rel_fro_err_vs_fp64"]["split"] for p in pool),
                               "fp32_max": max(p["rel_fro_err_vs_fp64"]["fp32"] for p in pool),
                               "what": "relative Frobenius error of each pool problem's assembled values against the "
                                       "FP64 path on its resident pattern; max over the pool"},
            "e2e": {"value": mixed["nnz_per_s"], "unit": "nnz/s", "note": "the served stream is end to end (host inputs to host outputs)",
                    "h2d_bytes_per_step": int(np.mean([p["elements"] for p in pool]) * 8),
                    "d2h_bytes_per_step": int(np.mean([p["nnz"] for p in pool]) * 8)},
            "clocks": mixed["clocks"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="split", choices=["fp64", "split", "fp32"])
    ap.add_argument("--n", type=int, default=0, help="override the mesh size (elements per side)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-config", action="store_true", help="skip the per_config block of the default run")
    ap.add_argument("--e2e-steps", type=int, default=3, help="timed warm generate()+A()+b() repetitions (at most --steps)")
    ap.add_argument("--requests", type=int, default=0, help="serving: number of requests (default 2000)")
    ap.add_argument("--slots", type=int, default=4, help="serving: concurrent request slots")
    args = ap.parse_args()
    spec = WORKLOADS[args.workload]
    if spec["kind"] == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "serving has no counterpart in the reference"}), flush=True)
        else:
            run_serving(args, spec)
    elif args.impl == "reference":
        run_reference(args, spec)
    elif spec.get("sweep"):
        run_sweep(args, spec)
    else:
        run_ours(args, spec)


if __name__ == "__main__":
    main()

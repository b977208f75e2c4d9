#!/usr/bin/env python
"""Assembly benchmark: nnz/s of sparselizard's generate()/A()/b() path on B200.

A step is one assembly pass over the workload on its resident pattern:
geometry + coefficients + element contraction for every element group, then
the A/D CSR values (duplicates summed in a fixed order).  The first
generate()/A()/b() through the drop-in (lowering, upload, pattern build) is
reported separately as `first_assembly`.

value  : device throughput, inputs already in HBM (CUDA events on the engine's
         stream, summed over the K steps; max over ranks).
e2e    : the same metric through the C ABI with host buffers: every step
         uploads the mesh node coordinates from pinned memory, assembles and
         downloads the CSR values to pinned memory (host clock around
         synchronised calls).
--impl reference times stock sparselizard (built from its sources, CPU, all
host threads) on a bounded sample of the same workload.

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
    "c2": dict(kind=W.ELASTICITY_HEX, mesh="hex", n=64, params=[2, -2], ref_n=16,
               name="elasticity_hex_64^3_h1xyz_order2"),
    "c3": dict(kind=W.HELMHOLTZ_TET, mesh="tet_orders", n=32, params=[], ref_n=8,
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
    if spec["mesh"] == "quad":
        meshgen.quad_mesh(path, n, jitter=0.2, seed=1)
    elif spec["mesh"] == "hex":
        meshgen.hex_mesh(path, n, jitter=0.15, seed=1)
    elif spec["mesh"] == "tet_orders":
        rng = np.random.Generator(np.random.PCG64(1))
        tags = meshgen.ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
        meshgen.tet_mesh(path, n, jitter=0.1, seed=1, element_tags=tags)
    elif spec["mesh"] == "tet_sigma":
        rng = np.random.Generator(np.random.PCG64(1))
        tags = meshgen.MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
        meshgen.tet_mesh(path, n, jitter=0.1, seed=1, element_tags=tags)
    else:
        raise ValueError(spec["mesh"])


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
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
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
    # profiles/k_contract_split_elasticity_hex32.md, 32768 elements: a symmetric
    # launch reads 59.91 MB and writes 138.28 MB, a paired one 70.26 + 338.40 MB;
    # a step runs three of each, so a launch averages their mean.
    ("c2", "contract_split"): ((59.910656e6 + 138.279168e6) + (70.263296e6 + 338.402048e6)) / 2 / 32768,
    # profiles/k_row_values_elasticity_hex32.md: 2.859 GB read + 1.202 GB
    # written by the launch over all 9 groups of 32768 elements.
    ("c2", "row_values"): (2.858950e9 + 1.201917e9) / 32768,
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


def cpu_reference_run(spec, n, reps, warmup, threads):
    with tempfile.TemporaryDirectory() as d:
        msh = os.path.join(d, "m.msh")
        write_mesh(spec, n, msh)
        r = W.run(REF_LIB, spec["kind"], msh, spec["params"], reps=warmup + reps, threads=threads)
    per = r.times[warmup:].sum(axis=1)
    return r.nnz, per


def run_reference(args, spec):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(threads))
    nnz, per = cpu_reference_run(spec, spec["ref_n"], args.steps, args.warmup, threads)
    value = nnz / float(np.mean(per))
    sample = f"{spec['name']} at n={spec['ref_n']} ({nnz} nnz), generate()+A()+b() per step"
    line = {
        "impl": "reference", "metric": "assembled_nnz_per_s", "value": value, "unit": "nnz/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(per)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded jittered mesh)",
        "config": {"workload": spec["name"], "sample_n": spec["ref_n"], "precision": "fp64"},
        "cpu_baseline": {"value": value, "unit": "nnz/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


KERNEL_NAMES = {"coefficients": "slgpu_coef (runtime-compiled)", "contract_fp64": "k_contract_fp64 / k_contract_small",
                "slice_cols": "k_slice_cols", "contract_split": "k_contract_split<7,8>",
                "contract_split_fp32": "k_contract_split<5,6>", "row_values": "k_row_values / k_row_stream (chosen per pattern)"}


def roofline_of(stats, workload, n):
    """Roofline entry of the kernel family with the most device time in `stats`
    (CUDA-event times and algorithmic work summed over launches)."""
    hbm, bf16, peak_kind = peaks()
    dom = max(stats, key=lambda f: stats[f]["ms"])
    k = stats[dom]
    rate = k["work"] / (k["ms"] * 1e-3)
    if dom.startswith("contract_split"):
        peak = 2.0 * bf16
        roof = {"kernel": KERNEL_NAMES[dom], "bound": "tensor", "achieved": rate / 1e12, "peak": peak, "unit": "TFLOP/s",
                "peak_kind": f"INT8 dense = 2 x {peak_kind} bf16 burst ({bf16:.0f} TFLOP/s); achieved counts INT8 ops",
                "frac": rate / 1e12 / peak}
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


def cpu_baseline(args, spec, rank, world):
    """Stock sparselizard (oracle/_ref) on the host cores, on the workload's
    bounded sample size, rank 0 of a one-GPU run only."""
    if rank != 0 or world != 1 or args.no_cpu_baseline or not os.path.exists(REF_LIB):
        return None
    threads = os.cpu_count() or 1
    cnnz, per = cpu_reference_run(spec, spec["ref_n"], 2, 1, threads)
    return {"value": cnnz / float(np.mean(per)), "unit": "nnz/s", "cores": threads, "kind": "reference",
            "sample": f"stock sparselizard generate()+A()+b(), {spec['name']} at n={spec['ref_n']} ({cnnz} nnz), "
                      f"mean of 2 after 1 warm-up"}


def run_ours(args, spec):
    import torch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    os.environ["SLGPU_DEVICE"] = str(local)
    os.environ["SLGPU_PRECISION"] = args.precision
    prec = {"fp64": abi.PREC_FP64, "split": abi.PREC_SPLIT, "fp32": abi.PREC_FP32}[args.precision]
    tmpd = tempfile.mkdtemp(prefix=f"slbench{rank}_")
    msh = os.path.join(tmpd, "m.msh")
    n = args.n or spec["n"]
    write_mesh(spec, n, msh)

    lib = W.load(GPU_LIB)
    abi.bind(lib)
    lib.slgpu_adapter_ctx.restype = ctypes.c_void_p
    lib.slz_bench_prepare.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
    lib.slz_bench_constraints.restype = ctypes.POINTER(ctypes.c_uint8)
    lib.slz_bench_nodes.argtypes = [ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
    lib.slz_bench_nodes.restype = ctypes.c_longlong
    params = (ctypes.c_double * max(1, len(spec["params"])))(*spec["params"])
    t3 = (ctypes.c_double * 3)()
    info4 = (ctypes.c_longlong * 4)()
    rc = lib.slz_bench_prepare(spec["kind"], msh.encode(), params, t3, info4)
    if rc != 0:
        raise RuntimeError("prepare failed: " + lib.slz_last_error().decode(errors="replace"))
    first = dict(generate_s=t3[0], A_s=t3[1], b_s=t3[2])
    handle = int(info4[0])
    ctx = ctypes.c_void_p(lib.slgpu_adapter_ctx())
    ndofs = int(info4[1])
    cons = lib.slz_bench_constraints()
    info = abi.CsrInfo()

    def process():
        st = lib.slgpu_matrix_process(ctx, handle, cons, prec, ctypes.byref(info))
        if st != 0:
            buf = ctypes.create_string_buffer(2048)
            lib.slgpu_last_error(ctx, buf, 2048)
            raise RuntimeError(f"process failed ({st}): {buf.value.decode()}")
        ms = np.zeros(5)
        lib.slgpu_last_timings(ctx, abi.f64p(ms))
        return ms

    work = abi.Work()
    nnz = info4[2]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # Timed steps without per-kernel events (a replayed graph then holds only
    # the kernels); the per-kernel breakdown comes from separate steps below.
    lib.slgpu_ctx_set_kernel_timers(ctx, 0)
    for _ in range(args.warmup):
        process()
    lib.slgpu_matrix_work(ctx, handle, ctypes.byref(work))
    nnz = int(work.nnz)
    l2_rule = "inputs larger than L2" if work.nvalid * 8 > 126e6 else "L2 flushed between steps"

    # ---- device-resident steps
    phase = np.zeros(5)
    stats = {}
    launches0 = lib.slgpu_kernel_launches(ctx)
    graphs0 = lib.slgpu_graph_launches(ctx)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            phase += process()
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

    # ---- end-to-end steps through the C ABI with pinned host buffers
    xyzp = ctypes.POINTER(ctypes.c_double)()
    nnodes = lib.slz_bench_nodes(ctypes.byref(xyzp))
    host_xyz = torch.empty(3 * nnodes, dtype=torch.float64).pin_memory()
    host_xyz.numpy()[:] = np.ctypeslib.as_array(xyzp, (3 * nnodes,))
    avals = torch.empty(max(1, info.nnzA), dtype=torch.float64).pin_memory()
    dvals = torch.empty(max(1, info.nnzD), dtype=torch.float64).pin_memory()
    e2e_t = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = lib.slgpu_mesh_set_nodes(ctx, 0, nnodes, ctypes.cast(host_xyz.data_ptr(), ctypes.POINTER(ctypes.c_double)))
        assert st == 0
        process()
        st = lib.slgpu_matrix_download_values(ctx, handle, ctypes.cast(avals.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                              ctypes.cast(dvals.data_ptr(), ctypes.POINTER(ctypes.c_double)))
        assert st == 0
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_t))
    e2e_s_max, = allreduce([e2e_s], torch.distributed.ReduceOp.MAX) if world > 1 else [e2e_s]
    e2e_value = total_nnz / e2e_s_max

    # ---- the plain FP64 GPU path on the same resident pattern, and the
    # split path's error against it on the assembled matrix
    fp64 = None
    if prec != abi.PREC_FP64:
        split_vals = avals.numpy()[: info.nnzA].copy()
        prec_run = prec
        prec = abi.PREC_FP64
        for _ in range(args.warmup):
            process()
        ph64 = np.zeros(5)
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ph64 += process()
        st = lib.slgpu_matrix_download_values(ctx, handle, ctypes.cast(avals.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                              ctypes.cast(dvals.data_ptr(), ctypes.POINTER(ctypes.c_double)))
        assert st == 0
        ref = avals.numpy()[: info.nnzA]
        num = den = 0.0
        for a in range(0, ref.size, 1 << 26):
            d = split_vals[a:a + (1 << 26)] - ref[a:a + (1 << 26)]
            num += float(d @ d)
            den += float(ref[a:a + (1 << 26)] @ ref[a:a + (1 << 26)])
        del split_vals
        ms64 = ph64[4] / args.steps
        ms64_max, = allreduce([ms64], torch.distributed.ReduceOp.MAX) if world > 1 else [ms64]
        fp64 = {"value": total_nnz / (ms64_max * 1e-3), "ms_per_step": ms64_max,
                "rel_fro_err_vs_fp64": (num / den) ** 0.5 if den > 0 else 0.0,
                "speedup": ms64_max / dev_ms_max}
        prec = prec_run

    # ---- per-kernel and per-phase events: the same steps again with timers on
    # (after warm-up steps that capture the graph with its event nodes)
    lib.slgpu_ctx_set_kernel_timers(ctx, 1)
    for _ in range(args.warmup):
        process()
    phase = np.zeros(5)
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        phase += process()
        kernel_stats(lib, ctx, stats)
    # ---- roofline of the dominant kernel
    ph = phase / args.steps
    roof = roofline_of(stats, args.workload, n)
    cpu = cpu_baseline(args, spec, rank, world)

    if rank == 0:
        line = {
            "metric": "assembled_nnz_per_s", "value": value, "unit": "nnz/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered mesh)",
            "config": {"workload": spec["name"], "n": n, "precision": args.precision, "ndofs": ndofs, "nnz": nnz,
                       "ncoo": int(work.ncoo), "groups": int(work.ngroups), "l2": l2_rule,
                       "parallelism": f"replicas{world}",
                       "timing": "ms_per_step from steps without per-kernel events; phases_ms, kernels and roofline from "
                                 "as many steps with them"},
            "phases_ms": {"geometry_coef": ph[0], "contraction": ph[1], "values": ph[3], "total": ph[4]},
            "kernels": stats,
            "fp64_gpu": fp64,
            "first_assembly": first,
            "e2e": {"value": e2e_value, "unit": "nnz/s", "ms_per_step": e2e_s_max * 1e3,
                    "h2d_bytes_per_step": int(24 * nnodes), "d2h_bytes_per_step": int(8 * (info.nnzA + info.nnzD))},
            "gpu_launches": int(launches),
            "graph_replays": int(graph_replays),
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    lib.slz_bench_release()
    if world > 1:
        torch.distributed.destroy_process_group()


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
    lib.slz_sweep_release()
    roof = roofline_of(stats, args.workload, n)
    cpu = cpu_baseline(args, spec, rank, world)
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

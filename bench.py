#!/usr/bin/env python
"""Benchmark of the linear-static hot path on B200.

One step is one full linear-static solve of the 160 x 16 x 16 C3D8
cantilever (139,587 DOF, 10,393,929 nonzeros, seeded interior jitter): element
integration, CSR assembly, Dirichlet, FP64 Jacobi-PCG to a relative residual
of 1e-10 and von Mises / reaction recovery.

* ``value`` - PCG DOF.iterations per second of whole solves whose inputs are
  already resident in HBM (svx_op_reassemble + svx_op_solve on the device
  copy of the model), timed with CUDA events on the library's stream.
* ``e2e`` - the same metric through the public C ABI call a user makes
  (svx_solve_flat) from pinned host buffers: the model's H2D copy and the
  D2H read of u, displacements, von Mises and reactions are inside the
  timed region.
* ``roofline`` - the dominant kernel (the persistent PCG kernel) against
  the measured HBM copy peak, from its algorithmic bytes and its live
  CUDA-event duration.
* ``cpu_baseline`` - the oracle (the C++ restatement of the reference's
  Rust path) solving the same model on the host cores.
* ``precision_c3``, ``batched_c4``, ``served_c5`` - the metric's own
  comparisons, measured in the same single-GPU run after the plain line
  (skipped with ``--plain-only`` and under torchrun): FP64 against mixed on
  the 480x48x48 heterogeneous C3D8 model; the 4,096-plate mix batched in
  FP64 and mixed against one-at-a-time FP64 solves; a reduced served stream
  in mixed precision with p50/p95/p99 latency, the FP64 saturation beside
  it, and the 4,096-plate mix through the server.

``--form direct`` times the direct path (RCM-ordered band LDL^T on the
device, the reference's Method::Ldlt) on the mesh of the reference's own
LDL^T timing test, against the oracle's serial LDL^T.

``--impl reference`` times only the oracle port on the host cores (rank 0).
Multi-GPU runs (torchrun) solve independent replicas per GPU ("replicas
only": the plain solve does not shard); ``value`` sums all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PCG DOF-iters/s & solves/s: mixed/batched vs FP64 at 1e-8 err; p50/p99 ms"
UNIT = "DOF*iter/s"
HBM_FALLBACK_GBS = 6650.0
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "pcg_smem_fp64_c3d8_160x16x16.txt")
BATCH_TRAFFIC_FILE = os.path.join(ROOT, "profiles", "batch_pcg_fp64_plates4096_dram.txt")


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default=None,
                    help="plain, batched and served forms: fp64 (default) or the mixed form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-only", action="store_true",
                    help="plain form: skip the precision / batched / served blocks that the "
                         "default single-GPU line carries beside the plain solve")
    ap.add_argument("--form",
                    choices=["plain", "batched", "precision", "served", "thermal", "direct",
                             "kernels"],
                    default="plain",
                    help="plain: the 160x16x16 C3D8 solve (default); batched: 4,096 uneven "
                         "2D plates in one launch; precision: FP64, relaxed mixed and defect "
                         "correction on the 480x48x48 heterogeneous C3D8 model; served: Poisson request "
                         "stream through the continuous-batching server; thermal: steady "
                         "conduction in a 480x48x48 C3D8 block; direct: the band LDL^T "
                         "direct path; kernels: device times of single kernels on one "
                         "workload (the command the profiles are captured with)")
    ap.add_argument("--direct-workload", choices=["hex40", "c2"], default="hex40",
                    help="direct form: the 40x4x4 hex cantilever of the reference's LDL^T "
                         "test (default) or the 160x16x16 C3D8 cantilever")
    ap.add_argument("--requests", type=int, default=20000,
                    help="served form: requests per rate point")
    ap.add_argument("--workload", choices=sorted(KERNEL_WORKLOADS), default="c3d8_160",
                    help="kernels form: the model")
    ap.add_argument("--kernel-mode", choices=["iteration", "solve", "batch", "batch-3d",
                                              "direct", "defect"], default="iteration",
                    help="kernels form: the iteration kernels back to back (iteration), one "
                         "FP64 solve (solve), one batched solve of --batch-count plates or "
                         "C3D8 cantilevers of the served stream (batch, batch-3d), the direct "
                         "path (direct), an FP64 solve and one defect-correction solve per "
                         "--inner-tols value (defect)")
    ap.add_argument("--inner-tols", type=str, default="1e-1,1e-2,1e-3,1e-4,1e-5,1e-6",
                    help="kernels form, defect mode: comma-separated inner tolerances")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--reps", type=int, default=20, help="kernels form: launches per kernel")
    ap.add_argument("--rates", type=str, default="",
                    help="served form: comma-separated arrival rates (requests/s); default "
                         "fractions of the measured saturation throughput")
    return ap.parse_args()


def workload():
    from solvix_b200 import workloads
    return workloads.cantilever_c3d8(160, 16, 16)


WORKLOAD_NAME = ("C3D8 cantilever 160x16x16 over 2.0x0.2x0.2 m (46,529 nodes, 139,587 DOF, "
                 "10,393,929 nnz), jitter +-0.1h seed 2, E=70e9, nu=0.33, x=0 clamped, -5 kN "
                 "in z over the x=L face; FP64 assembly + Jacobi-PCG to 1e-10 + stress")


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def _profile_figure(path, key):
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith(key + ":"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def ncu_traffic():
    """DRAM bytes per iteration of the shared-memory persistent PCG kernel
    (ncu summary)."""
    return _profile_figure(TRAFFIC_FILE, "dram_bytes_per_iteration")


def batch_ncu_traffic():
    """DRAM bytes of the full 4,096-plate FP64 batch launch (ncu summary)."""
    return _profile_figure(BATCH_TRAFFIC_FILE, "dram_bytes_per_launch")


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_baseline(flat, iterations_hint=None):
    """The oracle's full solve of the same model on min(8, cores) threads."""
    from oracle import oracle
    threads = oracle.default_threads()
    t0 = time.perf_counter()
    ref = oracle.solve_flat(flat, threads=threads)
    dt = time.perf_counter() - t0
    n = flat.n_dof
    return {
        "value": n * ref.iterations / dt, "unit": UNIT, "cores": threads, "kind": "port",
        "sample": (f"one full oracle solve of the same model (assembly, {ref.iterations} "
                   f"PCG iterations, stress) on {threads} threads in {dt:.2f} s "
                   f"(host: {os.cpu_count()} cores)"),
        "solves_per_s": 1.0 / dt,
    }


def pinned_like(a):
    import numpy as np
    import torch
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    out = t.numpy().view(a.dtype).reshape(a.shape)
    np.copyto(out, a)
    return out, t


def run_reference(args, rank):
    """--impl reference: the oracle port on the host cores, rank 0 only."""
    if rank != 0:
        return None
    if args.form == "direct":
        return run_reference_direct(args)
    flat = workload()
    from oracle import oracle
    oracle.build()
    for _ in range(max(0, args.warmup)):
        cpu_baseline(flat)
    vals, times = [], []
    for _ in range(args.steps):
        cb = cpu_baseline(flat)
        vals.append(cb["value"])
        times.append(1.0 / cb["solves_per_s"])
    value = len(times) * flat.n_dof * (vals[0] * times[0] / flat.n_dof) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": {"workload": WORKLOAD_NAME, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solves_per_s": 1.0 / (sum(times) / len(times)),
        "note": ("the reference is Rust and no Rust toolchain exists here or on the GPU box; "
                 "the arm times the C++ restatement (oracle/) that reproduces the reference's "
                 "published iteration counts and residuals bit for bit"),
    }
    return line


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import numpy as np
    import torch

    from solvix_b200 import Context, abi
    from solvix_b200.marshal import FlatModel

    torch.cuda.set_device(local_rank)
    precision = abi.SVX_MIXED if args.precision == "mixed" else abi.SVX_FP64
    flat = workload()
    n = flat.n_dof
    ctx = Context(local_rank)
    lib = ctx.lib
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local_rank}")
    op = ctx.assemble(flat)
    nnz = op.nnz

    def step():
        op.reassemble()
        return op.solve_device(precision=precision, want_stress=True)

    # nvidia-smi starts before the warm-up, so that its start-up (driver and
    # NVML initialisation) does not fall into the timed steps
    clocks = ClockSampler(local_rank)
    clocks.start()
    for _ in range(max(args.warmup, 0)):
        step()
    # flush L2 before the timed region (the per-step working set, K + Ke
    # ~ 315 MB, is larger than the 126 MB L2 on its own)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    with torch.cuda.stream(stream):
        flush.fill_(1)
    del flush
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = lib.svx_launch_count()
    ev0.record(stream)
    iters = []
    ms_parts = np.zeros(3)
    for _ in range(args.steps):
        it, res, ms_s, ms_st, ms_a = step()
        iters.append(it)
        ms_parts += [ms_a, ms_s, ms_st]
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = lib.svx_launch_count() - launches0
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
    ms_max = float(ms_t.item())
    dof_iters = float(np.sum(iters)) * n
    value = world * dof_iters / (ms_max / 1000.0)

    # roofline of the dominant kernel, the persistent PCG kernel: its
    # algorithmic bytes per launch (CHUNK iterations) over its average
    # launch duration, from the PCG device time of the timed steps
    from solvix_b200.roofline import pcg_iteration_bytes, spmv_node_bytes
    # iterations per persistent launch (persistent_chunk in svx_pcg.cu)
    chunk = 64 if nnz > 100_000_000 else (256 if nnz > 10_000_000 else 1024)
    it_total = float(np.sum(iters))
    launches_pcg = float(sum(-(-i // chunk) for i in iters))
    iter_bytes = pcg_iteration_bytes(n, nnz, flat.ndof, flat.n_nodes)
    launch_ms = ms_parts[1] / launches_pcg
    launch_bytes = iter_bytes * it_total / launches_pcg
    achieved = launch_bytes / (launch_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peaks()
    traffic_it = ncu_traffic()
    traffic = traffic_it * it_total / launches_pcg if traffic_it else None
    # the node-block SpMV alone (spmv_node_dot), back-to-back launches
    kms = op.time_kernels(reps=50)
    spmv_bytes = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes)

    # e2e: the public C ABI call from pinned host memory
    keep = []
    pinned = {}
    for name in ("xyz", "kind", "conn_ptr", "conn", "youngs", "poisson", "fixed_row", "f",
                 "node_id", "elem_id"):
        a = getattr(flat, name)
        if a is None:
            continue
        pa, t = pinned_like(np.ascontiguousarray(a))
        keep.append(t)
        pinned[name] = pa
    pflat = FlatModel(thickness=flat.thickness, ndof=flat.ndof, **pinned)
    outs = {}
    for name, shape in (("u", (n,)), ("disp", (flat.n_nodes, 3)), ("vm", (flat.n_elem,)),
                        ("vmn", (flat.n_nodes,)), ("react", (flat.fixed_row.shape[0],))):
        pa, t = pinned_like(np.zeros(shape))
        keep.append(t)
        outs[name] = pa
    sol = abi.SvxSolution()
    sol.u = abi.ptr(outs["u"], C.c_double)
    sol.displacements = abi.ptr(outs["disp"], C.c_double)
    sol.von_mises = abi.ptr(outs["vm"], C.c_double)
    sol.nodal_von_mises = abi.ptr(outs["vmn"], C.c_double)
    sol.reactions = abi.ptr(outs["react"], C.c_double)
    opts = abi.default_opts(precision=precision)
    err = abi.SvxError()
    s = pflat.as_struct()
    h2d = pflat.nbytes()
    d2h = sum(a.nbytes for a in outs.values())

    def e2e_step():
        st = lib.svx_solve_flat(ctx.handle, C.byref(s), C.byref(opts), C.byref(sol),
                                C.byref(err))
        if st != abi.SVX_OK:
            raise RuntimeError(err.message.decode())
        return int(sol.iterations)

    e2e_step()
    e2e_steps = max(3, min(args.steps, 10))
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e_iters = 0
    for _ in range(e2e_steps):
        e_iters += e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local_rank}")
    if world > 1:
        torch.distributed.all_reduce(e_ms, op=torch.distributed.ReduceOp.MAX)
    e2e_value = world * e_iters * n / (float(e_ms.item()) / 1000.0)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == 0 else "f32/f64",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": {"workload": WORKLOAD_NAME, "n_dof": n, "nnz": nnz,
                   "precision": args.precision or "fp64",
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (K 125 MB + Ke 189 MB per step vs 126 MB L2); "
                         "L2 flushed before the timed region"},
        "solves_per_s": world * args.steps / (ms_max / 1000.0),
        "iterations": int(iters[-1]),
        "ms_breakdown": {"assemble": ms_parts[0] / args.steps, "pcg": ms_parts[1] / args.steps,
                         "stress": ms_parts[2] / args.steps},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                "solves_per_s": world * e2e_steps / (float(e_ms.item()) / 1000.0)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "pcg_smem_kernel<3,8,512,1,0,1> "
                                                 f"(FP64, {chunk} PCG iterations a launch)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": int(launch_bytes),
                     "algorithmic_bytes_per_iteration": int(iter_bytes),
                     "launch_ms": float(launch_ms),
                     "traffic": traffic,
                     "note": "K (87.7 MB in FP64 node blocks) fits the 126 MB L2; traffic "
                             "(ncu DRAM bytes) below the algorithmic bytes is K served from "
                             "L2 across iterations",
                     "spmv_node_dot_alone": {
                         "launch_ms": float(kms[0]), "bytes": int(spmv_bytes),
                         "gbs": spmv_bytes / (kms[0] / 1000.0) / 1e9,
                         "frac": spmv_bytes / (kms[0] / 1000.0) / 1e9 / peak},
                     "other_kernels_ms": {"update": float(kms[1]), "p_update": float(kms[2])}},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(flat)
        line["cpu_baseline"].pop("solves_per_s", None)
    op.free()
    ctx.close()
    return line



BATCH_NAME = ("4,096 independent 2D plates (nx~U{10..160}, ny~U{4..40}, h=1, CPS4 or CPS3 "
              "p=0.5, E=10^U(9,log10 3e11), nu~U(0.15,0.45), t~U(0.001,0.05), left edge "
              "clamped, one CLOAD U(100,1e4) N at a random right-edge node; seed 4), "
              "Jacobi-PCG to 1e-10 per model, centroid von Mises")


def mix_cpu_baseline(flats, what, max_seconds=20.0):
    """The oracle's full solves of the sampled models of a mix, one after
    another on min(8, cores) threads, stopping after max_seconds; the mix's
    CPU rate is extrapolated from the models solved."""
    from oracle import oracle
    oracle.build()
    threads = oracle.default_threads()
    dof_it, done, t_all = 0.0, 0, 0.0
    for f in flats:
        t0 = time.perf_counter()
        ref = oracle.solve_flat(f, threads=threads)
        t_all += time.perf_counter() - t0
        dof_it += f.n_dof * ref.iterations
        done += 1
        if t_all >= max_seconds:
            break
    return {"value": dof_it / t_all, "unit": UNIT, "cores": threads, "kind": "port",
            "solves_per_s": done / t_all, "extrapolated": True,
            "sample": (f"oracle full solves (assembly, PCG, stress) of {done} of the {what}, "
                       f"one after another on {threads} threads in {t_all:.2f} s; the mix's "
                       "CPU rate is extrapolated from them")}


def one_at_a_time(ctx, flats):
    """The one-at-a-time plain FP64 GPU path on a sample: every model through
    svx_solve_flat, one after another, wall clock.  Two passes over the
    sample (the first also warms the context's pool); the faster is kept.
    Returns (seconds per solve, device ms per solve of assembly + PCG +
    stress recovery in that pass)."""
    best = None
    for _ in range(2):
        dev = 0.0
        t0 = time.perf_counter()
        for f in flats:
            sol = ctx.solve_flat(f)
            dev += sol.ms_assemble + sol.ms_solve + sol.ms_stress
        per = (time.perf_counter() - t0) / len(flats)
        if best is None or per < best[0]:
            best = (per, dev / len(flats))
    return best


def run_batched(args, rank, world, local_rank):
    """C4: the whole plate mix per step through svx_batch_solve; models are
    sharded over ranks (greedy on estimated work, no collective)."""
    import numpy as np
    import torch

    from solvix_b200 import Context, abi, workloads
    from solvix_b200.roofline import pcg_iteration_bytes
    from solvix_b200.sharding import shard_instances

    torch.cuda.set_device(local_rank)
    flats = workloads.plate_batch(4096, seed=4)
    mine = shard_instances([f.n_dof for f in flats], world)[rank]
    sub = [flats[k] for k in mine]
    ctx = Context(local_rank)
    lib = ctx.lib
    prec = abi.SVX_MIXED if args.precision == "mixed" else abi.SVX_FP64
    for _ in range(max(args.warmup, 0)):
        ctx.solve_batch(sub, precision=prec)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = lib.svx_launch_count()
    dev_ms, wall_s, dof_it, bytes_alg = [], [], 0.0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        out, st = ctx.solve_batch(sub, precision=prec)
        wall_s.append(time.perf_counter() - t0)
        dev_ms.append(st["ms_assemble"] + st["ms_solve"] + st["ms_stress"])
        solve_ms = st["ms_solve"]
        dof_it = float(sum(f.n_dof * o["iterations"] for f, o in zip(sub, out)))
        # per iteration of each model: the node-block SpMV and the vector
        # streams of the update (pcg_iteration_bytes)
        bytes_alg = float(sum(o["iterations"] * pcg_iteration_bytes(f.n_dof, o["nnz"], f.ndof,
                                                                    f.n_nodes)
                              for f, o in zip(sub, out)))
    launches = lib.svx_launch_count() - launches0
    clk = clocks.stop()
    vals = torch.tensor([sum(dev_ms), sum(wall_s), dof_it], dtype=torch.float64,
                        device=f"cuda:{local_rank}")
    if world > 1:
        mx = vals[:2].clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        tot = vals[2:].clone()
        torch.distributed.all_reduce(tot, op=torch.distributed.ReduceOp.SUM)
        vals = torch.cat([mx, tot])
    ms_max, wall_max, dof_it_all = (float(v) for v in vals.tolist())
    value = args.steps * dof_it_all / (ms_max / 1000.0)
    e2e_value = args.steps * dof_it_all / wall_max
    peak, peak_kind = measured_peaks()
    achieved = bytes_alg / (solve_ms / 1000.0) / 1e9
    iters = np.array([o["iterations"] for o in out])
    line = {
        "metric": METRIC, "form": "batched", "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64" if prec == abi.SVX_FP64 else "f64+f32",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": {"workload": BATCH_NAME, "models": len(flats),
                   "precision": args.precision or "fp64",
                   "total_dof": int(sum(f.n_dof for f in flats)),
                   "parallelism": f"instances sharded over {world} GPU(s), no collective",
                   "autotuned": {"threads_per_cta": st["threads_per_cta"],
                                 "lanes_per_node": st["lanes_per_node"]}},
        "solves_per_s": world * len(sub) * args.steps / (ms_max / 1000.0),
        "iterations": {"min": int(iters.min()), "mean": float(iters.mean()),
                       "max": int(iters.max())},
        "ms_breakdown": {"assemble": st["ms_assemble"], "pcg": st["ms_solve"],
                         "stress": st["ms_stress"]},
        "cluster_members": st["cluster_members"], "fp32_iterations": st["fp32_iterations"],
        "e2e": {"value": e2e_value, "unit": UNIT,
                "solves_per_s": len(flats) * args.steps / wall_max,
                "h2d_bytes_per_step": int(sum(f.nbytes() for f in sub)),
                "d2h_bytes_per_step": int(sum(8 * (f.n_dof + f.n_elem) for f in sub)),
                "note": "svx_batch_solve from pageable host arrays, wall clock per call"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "batch_pcg_kernel (one CTA per member) beside "
                                                 "batch_pcg_cluster_kernel (one 8-CTA cluster "
                                                 "per large member), one launch each per step",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": int(bytes_alg),
                     "launch_ms": solve_ms,
                     # the ncu capture covers the whole 4,096-plate FP64 launch on one GPU
                     "traffic": (batch_ncu_traffic()
                                 if world == 1 and prec == abi.SVX_FP64 else None)},
        "clocks": clk,
    }
    if rank == 0:
        # the one-at-a-time plain GPU path on a sample of the same models
        rng = np.random.default_rng(0)
        idx = rng.choice(len(flats), 64, replace=False)
        per, dev_ms = one_at_a_time(ctx, [flats[int(k)] for k in idx])
        line["one_at_a_time"] = {
            "solves_per_s": 1.0 / per,
            "device_ms_per_solve": dev_ms,
            "sample": "64 models of the mix through svx_solve_flat one after another "
                      "(wall clock, faster of two passes), projected to the set",
            "speedup_device": line["solves_per_s"] * per,
            "speedup_e2e": line["e2e"]["solves_per_s"] * per}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = mix_cpu_baseline(
                [flats[int(k)] for k in idx], "64 sampled models of the plate mix")
    ctx.close()
    return line


PRECISION_NAME = ("C3D8 cantilever 480x48x48 over 2.0x0.2x0.2 m (1,154,881 nodes, 3,464,643 "
                  "DOF, 272,673,225 nnz), per-element E=10^U(9,11) seed 3, nu=0.3, x=0 "
                  "clamped, -5 kN in z over the x=L face; relative residual 1e-10")


def run_precision(args, rank, world, local_rank):
    """--form precision: the default line's precision_c3 block (FP64,
    relaxed mixed and defect-correction solves of the heterogeneous model,
    device-timed) as a line of its own, its value the FP64 solve's
    DOF-iterations per second."""
    import torch

    torch.cuda.set_device(local_rank)
    blk = precision_block(local_rank)
    f64 = blk["fp64"]
    peak, peak_kind = blk["peak_gbs"], blk["peak_source"]
    line = {
        "metric": METRIC, "form": "precision", "value": f64["dof_iter_per_s"],
        "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": f64["ms_per_solve"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": {"workload": PRECISION_NAME, "n_dof": blk["n_dof"], "nnz": blk["nnz"]},
        "precision_c3": blk,
        "roofline": {"bound": "hbm", "kernel": "node-block FP64 SpMV (spmv_node_dot)",
                     "achieved": blk["spmv_fp64"]["gbs"], "peak": peak, "unit": "GB/s",
                     "frac": blk["spmv_fp64"]["frac"], "peak_source": peak_kind,
                     "launch_ms": blk["spmv_fp64"]["ms"], "traffic": None},
        "clocks": blk["clocks"],
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = precision_cpu_baseline(f64["iterations"], blk["n_dof"])
    return line


def precision_cpu_baseline(gpu_fp64_iterations, n_c3, iterations=200):
    """The CPU leg of the precision form: a full oracle solve of C3 takes
    hours (and its triplet assembly about 20 GB of host memory), so this
    times `iterations` oracle PCG iterations on the 160x16x16 model of the
    same kind (heterogeneous C3D8, seed 3) for the CPU's DOF.iter/s, and
    projects C3's CPU solves/s from the GPU's FP64 iteration count."""
    from oracle import oracle
    from solvix_b200 import workloads
    flat = workloads.heterogeneous_c3d8(160, 16, 16, seed=3)
    threads = oracle.default_threads()
    k = oracle.assemble(flat, threads)
    f = flat.f.copy()
    oracle.apply_dirichlet(k, f, flat.fixed_row)
    t0 = time.perf_counter()
    _st, _u, it, _res = oracle.pcg(k, f, tol=1e-300, max_iter=iterations, threads=threads)
    dt = time.perf_counter() - t0
    rate = flat.n_dof * it / dt
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{it} oracle PCG iterations on the 160x16x16 heterogeneous C3D8 model "
                       f"({flat.n_dof} DOF, {k.nnz} nnz) on {threads} threads in {dt:.2f} s; "
                       "C3 itself is not solved on the CPU"),
            "projected_c3_solves_per_s": (rate / (n_c3 * gpu_fp64_iterations)
                                          if gpu_fp64_iterations else None),
            "projected": True}


SERVED_NAME = ("Poisson stream of solve requests: 70% 2D plates of the batched mix, 30% "
               "C3D8 cantilevers nx~U{20..120}, ny=nz~U{4..16}, E=70e9, nu=0.33, tip load "
               "U(1e3,1e4) N (seed 5); relative residual 1e-10; 40 GiB admission budget; "
               "2 lanes")


def _serve_run(srv, reqs, rate_scale, base_t):
    """Submit reqs at base_t * rate_scale seconds after the start (0 scale:
    all at once), collect every result; returns (results, wall_s)."""
    results = {}
    done = threading.Event()
    count = len(reqs)

    def collect():
        while len(results) < count:
            r = srv.poll(200)
            if r is not None:
                r.pop("u", None)
                r.pop("von_mises", None)
                results[r["tag"]] = r
        done.set()

    th = threading.Thread(target=collect, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for k, flat in enumerate(reqs):
        due = t0 + base_t[k] * rate_scale
        while True:
            now = time.perf_counter()
            if now >= due:
                break
            time.sleep(min(due - now, 0.002))
        st, msg = srv.submit(flat, k)
        if st != 0:
            raise RuntimeError(f"request {k} refused: {msg}")
    th.join()
    return results, time.perf_counter() - t0


def run_served(args, rank, world, local_rank):
    """C5: the request stream through svx_serve_* (continuous batching): all
    requests at saturation, then a sweep of Poisson rates on a prefix of the
    stream; latency from submit to result on the host.  The same
    saturation run in the other precision is reported beside it."""
    import numpy as np
    import torch

    from solvix_b200 import Context, abi, workloads
    from solvix_b200.roofline import pcg_iteration_bytes
    from solvix_b200.serve import Server

    torch.cuda.set_device(local_rank)
    prec_name = args.precision or "fp64"
    prec = abi.SVX_MIXED if prec_name == "mixed" else abi.SVX_FP64
    other_name = "fp64" if prec_name == "mixed" else "mixed"
    other = abi.SVX_FP64 if prec == abi.SVX_MIXED else abi.SVX_MIXED
    count = max(16, args.requests)
    stream = workloads.request_stream(count, 1.0, seed=5)  # unit-rate arrival times
    mine = list(range(rank, count, world))  # round-robin keeps each rank's arrivals Poisson
    reqs = [stream[k][1] for k in mine]
    base_t = np.array([stream[k][0] for k in mine])  # arrivals at a total rate of 1/s
    n_dof = {k: f.n_dof for k, f in enumerate(reqs)}
    sweep_n = min(len(reqs), max(200, len(reqs) // 10))

    def summarize(results, wall):
        lat = np.array([r["t_done_ms"] - r["t_submit_ms"] for r in results.values()])
        ok = [r for r in results.values() if r["status"] == 0]
        dof_it = float(sum(n_dof[r["tag"]] * r["iterations"] for r in results.values()))
        # algorithmic bytes of every member iteration (node-block SpMV and
        # vector streams), as in the batched form
        alg = float(sum(r["iterations"] * pcg_iteration_bytes(
            n_dof[r["tag"]], r["nnz"], reqs[r["tag"]].ndof, reqs[r["tag"]].n_nodes)
            for r in ok))
        return {"solves_per_s": len(ok) / wall, "dof_iter_per_s": dof_it / wall,
                "algorithmic_bytes": alg,
                "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
                "p99_ms": float(np.percentile(lat, 99)), "failed": len(results) - len(ok),
                "mean_batch": float(np.mean([r["batch_size"] for r in results.values()])),
                "requests": len(results), "wall_s": wall}

    def saturation(p):
        srv = Server(local_rank, precision=p)
        warm = reqs[:min(len(reqs), 512)]
        _serve_run(srv, warm, 0.0, np.zeros(len(warm)))
        s0 = srv.stats()
        l0 = srv.lib.svx_launch_count()
        res, wall = _serve_run(srv, reqs, 0.0, base_t)
        row = summarize(res, wall)
        row["rate_per_s"] = "all at t=0"
        s1 = srv.stats()
        row["phases_ms"] = {k: round(s1[k] - s0[k], 1) for k in (
            "prep_ms", "assemble_ms", "solve_ms", "output_ms", "device_solve_ms", "pool_ms")}
        row["pool_mallocs"] = int(s1["pool_mallocs"] - s0["pool_mallocs"])
        row["batches"] = int(s1["batches"] - s0["batches"])
        row["peak_bytes_admitted"] = int(s1["peak_bytes_admitted"])
        return srv, row, srv.lib.svx_launch_count() - l0

    clocks = ClockSampler(local_rank)
    clocks.start()
    srv, sat, launches = saturation(prec)
    cap = sat["solves_per_s"] * world
    rates = ([float(x) for x in args.rates.split(",") if x] if args.rates
             else [round(cap * f, 1) for f in (0.25, 0.5, 0.8)])
    sweep = []
    sub = reqs[:sweep_n]
    for rate in rates:
        res, wall = _serve_run(srv, sub, 1.0 / rate, base_t[:sweep_n])
        row = summarize(res, wall)
        row["rate_per_s"] = rate
        sweep.append(row)
    srv.close()
    srv2, sat_other, _ = saturation(other)
    srv2.close()
    clk = clocks.stop()
    # error against FP64 and the one-at-a-time plain FP64 GPU path on a sample
    ctx = Context(local_rank)
    rng = np.random.default_rng(1)
    idx = [int(i) for i in rng.choice(len(reqs), min(48, len(reqs)), replace=False)]
    with Server(local_rank, lanes=1, precision=prec) as one:
        for k in idx:
            one.submit(reqs[k], k)
        served_u = {}
        while len(served_u) < len(idx):
            r = one.poll(200)
            if r is not None:
                served_u[r["tag"]] = r["u"]
    errs = []
    for k in idx:
        ref = ctx.solve_flat(reqs[k])
        errs.append(float(np.linalg.norm(served_u[k] - ref.u) / np.linalg.norm(ref.u)))
    one_per, one_dev_ms = one_at_a_time(ctx, [reqs[k] for k in idx])
    ctx.close()
    cpu_leg = (mix_cpu_baseline([reqs[k] for k in idx],
                                f"{len(idx)} sampled requests of the served mix")
               if rank == 0 and not args.no_cpu_baseline else None)
    rows = [sat] + sweep
    if world > 1:
        gathered = [None] * world
        torch.distributed.all_gather_object(gathered, rows)
        rows = [{"solves_per_s": sum(g[i]["solves_per_s"] for g in gathered),
                 "dof_iter_per_s": sum(g[i]["dof_iter_per_s"] for g in gathered),
                 "algorithmic_bytes": sum(g[i]["algorithmic_bytes"] for g in gathered),
                 "p50_ms": max(g[i]["p50_ms"] for g in gathered),
                 "p95_ms": max(g[i]["p95_ms"] for g in gathered),
                 "p99_ms": max(g[i]["p99_ms"] for g in gathered),
                 "failed": sum(g[i]["failed"] for g in gathered),
                 "requests": sum(g[i]["requests"] for g in gathered),
                 "mean_batch": float(np.mean([g[i]["mean_batch"] for g in gathered])),
                 "wall_s": max(g[i]["wall_s"] for g in gathered),
                 "rate_per_s": rows[i]["rate_per_s"]} for i in range(len(rows))]
    sat = rows[0]
    head = rows[-1] if len(rows) > 1 else sat
    peak, peak_kind = measured_peaks()
    line = {
        "metric": METRIC, "form": "served", "value": sat["dof_iter_per_s"], "unit": UNIT,
        "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": 1000 * sat["wall_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == abi.SVX_FP64 else "f64+f32",
        "data": "synthetic (seeded generator; no public dataset exists for this path)",
        "config": {"workload": SERVED_NAME, "precision": prec_name, "requests": count,
                   "sweep_requests_per_rate": sweep_n,
                   "parallelism": f"requests round-robin over {world} GPU(s), no collective"},
        "solves_per_s": sat["solves_per_s"],
        "latency_ms": {"p50": head["p50_ms"], "p95": head["p95_ms"], "p99": head["p99_ms"],
                       "at_rate_per_s": head["rate_per_s"]},
        "sweep": rows,
        f"saturation_{other_name}": sat_other,
        "rel_err_vs_fp64": {"max": max(errs), "median": float(np.median(errs)),
                            "sample": len(errs)},
        "one_at_a_time": {"solves_per_s": 1.0 / one_per,
                          "device_ms_per_solve": one_dev_ms,
                          "sample": f"{len(idx)} requests through svx_solve_flat (FP64) one "
                                    "after another, wall clock, faster of two passes",
                          "speedup_served": sat["solves_per_s"] * one_per,
                          f"speedup_served_{other_name}": sat_other["solves_per_s"] * one_per},
        "e2e": {"value": sat["dof_iter_per_s"], "unit": UNIT,
                "note": "submit of host models to results on the host, wall clock",
                "h2d_bytes_per_step": int(sum(f.nbytes() for f in reqs)),
                "d2h_bytes_per_step": int(sum(8 * (f.n_dof + f.n_elem) for f in reqs))},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "batch_pcg_kernel / batch_pcg_cluster_kernel "
                     "of every lane's batches",
                     "achieved": sat["algorithmic_bytes"] / sat["wall_s"] / 1e9,
                     "peak": peak, "unit": "GB/s",
                     "frac": sat["algorithmic_bytes"] / sat["wall_s"] / 1e9 / peak,
                     "peak_source": peak_kind,
                     "algorithmic_bytes": sat["algorithmic_bytes"],
                     "note": "over the saturation run's wall clock, host phases included",
                     "traffic": None},
        "clocks": clk,
    }
    if cpu_leg is not None:
        line["cpu_baseline"] = cpu_leg
    return line


# ---------------------------------------------------------------------------
# The metric's own comparisons (mixed / batched / served against FP64), run
# after the plain line in the default single-GPU bench and reported beside it.
# ---------------------------------------------------------------------------
def _rel(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(b)), 1e-300))


def _device_timed(stream, fn):
    """fn() between two CUDA events on the library's stream; (result, ms)."""
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def precision_block(local_rank):
    """The 480x48x48 heterogeneous C3D8 cantilever: one FP64, one mixed and
    one defect-correction solve (reassembly + PCG + stress) of the same
    device-resident operator, each timed with CUDA events on the library's
    stream; the FP32 forms' iteration splits and their displacement errors
    against the FP64 solve (the oracle itself cannot solve this size: hours
    and ~20 GB of triplets).  The defect-correction form (SVX_MIXED_DEFECT)
    is the textbook one: an FP32 inner PCG (FP32 K, vectors and Jacobi;
    FP64 dots) to 1e-5 inside FP64 defect correction."""
    import numpy as np
    import torch

    from solvix_b200 import Context, abi, workloads
    from solvix_b200.model import NotConverged

    flat = workloads.heterogeneous_c3d8(480, 48, 48, seed=3)
    n = flat.n_dof
    with Context(local_rank) as ctx:
        stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local_rank}")
        op = ctx.assemble(flat)
        try:
            forms = (("fp64", abi.SVX_FP64), ("mixed", abi.SVX_MIXED),
                     ("defect", abi.SVX_MIXED_DEFECT))
            for _, prec in forms:  # graphs, pools, first launches
                try:
                    op.solve_device(precision=prec, max_iter=64, want_stress=False)
                except NotConverged:
                    pass
            clocks = ClockSampler(local_rank)
            clocks.start()
            res = {}
            for name, prec in forms:
                def one():
                    op.reassemble()
                    return op.solve_device(precision=prec, max_iter=200000, want_stress=True)
                try:
                    (it, r, ms_s, _ms_st, ms_a), ms = _device_timed(stream, one)
                except NotConverged as e:  # reported in the line, the other forms kept
                    if name == "fp64":
                        raise
                    res[name] = {"error": f"NotConverged: {e}"}
                    continue
                fp32_it = op.last_fp32_iterations
                outer = op.last_outer_iterations
                disp = op.stress()[3]
                res[name] = {"iterations": it, "fp32_iterations": fp32_it, "ms": ms,
                             "pcg_ms": ms_s, "residual": r, "outer": outer,
                             "u": np.asarray(disp).reshape(-1, 3)[:, :flat.ndof].ravel()}
            clk = clocks.stop()
            kms = op.time_kernels(reps=10)
            nnz = op.nnz
        finally:
            op.free()
    from solvix_b200.roofline import spmv_node_bytes
    spmv64 = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes)
    spmv32 = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes, value_bytes=4)
    peak, peak_kind = measured_peaks()
    f64, mx, dc = res["fp64"], res["mixed"], res["defect"]
    def form(d, **extra):
        return dict(row(d), **extra) if "error" not in d else d

    row = lambda d: {"iterations": d["iterations"], "ms_per_solve": d["ms"],
                     "pcg_ms": d["pcg_ms"], "solves_per_s": 1000.0 / d["ms"],
                     "dof_iter_per_s": n * d["iterations"] / (d["ms"] / 1000.0),
                     "residual": d["residual"]}
    out = {
        "workload": PRECISION_NAME, "n_dof": n, "nnz": nnz,
        "fp64": row(f64),
        "mixed": form(mx, fp32_iterations=mx.get("fp32_iterations"),
                      fp32_share=mx.get("fp32_iterations", 0) / max(1, mx.get("iterations", 1)),
                      rel_err_vs_fp64=_rel(mx["u"], f64["u"]) if "u" in mx else None),
        "ratio_mixed_over_fp64": f64["ms"] / mx["ms"] if "ms" in mx else None,
        "defect_correction": form(dc, fp32_iterations=dc.get("fp32_iterations"),
                                  fp64_iterations=dc.get("iterations", 0) -
                                  dc.get("fp32_iterations", 0),
                                  corrections=dc.get("outer"), inner_tol=1e-5,
                                  rel_err_vs_fp64=_rel(dc["u"], f64["u"]) if "u" in dc else None),
        "ratio_defect_over_fp64": f64["ms"] / dc["ms"] if "ms" in dc else None,
        "spmv_fp64": {"ms": float(kms[0]), "gbs": spmv64 / kms[0] / 1e6,
                      "frac": spmv64 / kms[0] / 1e6 / peak},
        "spmv_fp32": {"ms": float(kms[3]), "gbs": spmv32 / kms[3] / 1e6,
                      "frac": spmv32 / kms[3] / 1e6 / peak},
        "peak_gbs": peak, "peak_source": peak_kind,
        "timing": "CUDA events on the library stream around reassembly + PCG + stress of one "
                  "solve per precision, after a 64-iteration warm-up of each; K (2.3 GB FP64) "
                  "is larger than L2",
        "clocks": clk,
    }
    return out


def _serve_summary(results, wall, reqs):
    import numpy as np

    from solvix_b200.roofline import pcg_iteration_bytes
    lat = np.array([r["t_done_ms"] - r["t_submit_ms"] for r in results.values()])
    ok = [r for r in results.values() if r["status"] == 0]
    dof_it = float(sum(reqs[r["tag"]].n_dof * r["iterations"] for r in results.values()))
    alg = float(sum(r["iterations"] * pcg_iteration_bytes(
        reqs[r["tag"]].n_dof, r["nnz"], reqs[r["tag"]].ndof, reqs[r["tag"]].n_nodes)
        for r in ok))
    return {"requests": len(results), "failed": len(results) - len(ok),
            "solves_per_s": len(ok) / wall, "dof_iter_per_s": dof_it / wall,
            "algorithmic_gbs": alg / wall / 1e9,
            "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)),
            "mean_batch": float(np.mean([r["batch_size"] for r in results.values()])),
            "wall_s": wall}


def _served_saturation(local_rank, prec, reqs):
    """Every request submitted at once to a fresh server (after a warm-up of
    the first 256); returns (server, summary)."""
    import numpy as np

    from solvix_b200.serve import Server
    srv = Server(local_rank, precision=prec)
    warm = reqs[:min(len(reqs), 256)]
    _serve_run(srv, warm, 0.0, np.zeros(len(warm)))
    res, wall = _serve_run(srv, reqs, 0.0, np.zeros(len(reqs)))
    return srv, _serve_summary(res, wall, reqs)


def batched_block(local_rank):
    """The 4,096-plate mix through svx_batch_solve in FP64 and mixed, against
    the one-at-a-time plain FP64 GPU path (svx_solve_flat) on a sample."""
    import numpy as np
    import torch

    from solvix_b200 import Context, abi, workloads

    torch.cuda.set_device(local_rank)
    flats = workloads.plate_batch(4096, seed=4)
    total_dof = int(sum(f.n_dof for f in flats))
    out = {"workload": BATCH_NAME, "models": len(flats), "total_dof": total_dof}
    us = {}
    with Context(local_rank) as ctx:
        clocks = ClockSampler(local_rank)
        clocks.start()
        for name, prec in (("fp64", abi.SVX_FP64), ("mixed", abi.SVX_MIXED)):
            ctx.solve_batch(flats, precision=prec)  # warm-up (autotune, pools)
            best = None
            for _ in range(2):
                t0 = time.perf_counter()
                res, st = ctx.solve_batch(flats, precision=prec)
                wall = time.perf_counter() - t0
                dev_ms = st["ms_assemble"] + st["ms_solve"] + st["ms_stress"]
                if best is None or dev_ms < best[1]:
                    best = (wall, dev_ms, st, res)
            wall, dev_ms, st, res = best
            us[name] = [r["u"] for r in res]
            its = np.array([r["iterations"] for r in res])
            out[name] = {
                "solves_per_s_device": len(flats) / (dev_ms / 1000.0),
                "solves_per_s_e2e": len(flats) / wall,
                "dof_iter_per_s_device": float(sum(f.n_dof * int(r["iterations"])
                                                   for f, r in zip(flats, res))) /
                (dev_ms / 1000.0),
                "ms_device": dev_ms, "ms_pcg": st["ms_solve"], "wall_s": wall,
                "iterations_mean": float(its.mean()), "not_converged": int(st["not_converged"]),
                "fp32_iterations": int(st["fp32_iterations"])}
        rng = np.random.default_rng(0)
        idx = [int(k) for k in rng.choice(len(flats), 64, replace=False)]
        per, dev_one = one_at_a_time(ctx, [flats[k] for k in idx])
        clk = clocks.stop()
    out["one_at_a_time"] = {"solves_per_s": 1.0 / per, "device_ms_per_solve": dev_one,
                            "sample": "64 models of the mix through svx_solve_flat (FP64), one "
                                      "after another, wall clock, faster of two passes"}
    for name in ("fp64", "mixed"):
        out[name]["ratio_device_vs_one_at_a_time"] = out[name]["solves_per_s_device"] * per
        out[name]["ratio_e2e_vs_one_at_a_time"] = out[name]["solves_per_s_e2e"] * per
    errs = [_rel(a, b) for a, b in zip(us["mixed"], us["fp64"])]
    out["mixed"]["rel_err_vs_fp64"] = {"max": max(errs), "median": float(np.median(errs))}
    out["timing"] = ("device = the call's CUDA-event times (assembly + batched PCG + von "
                     "Mises), e2e = wall clock of the svx_batch_solve call from host arrays; "
                     "best of 2 after a warm-up")
    out["clocks"] = clk
    return out, per


def served_block(local_rank, c4_one_at_a_time_s=None, count=2000):
    """A reduced C5 stream (the first `count` requests: 70% plates, 30% C3D8
    cantilevers) served in mixed precision as C5 specifies, at saturation
    and as a Poisson stream at half the saturation rate (p50/p95/p99), the
    FP64 saturation beside it, against one-at-a-time FP64 solves of a
    sample; then the 4,096-plate mix through the same server."""
    import numpy as np

    from solvix_b200 import Context, abi, workloads
    from solvix_b200.serve import Server

    stream = workloads.request_stream(count, 1.0, seed=5)
    reqs = [m for _, m in stream]
    base_t = np.array([t for t, _ in stream])
    out = {"workload": SERVED_NAME.replace("2 lanes", f"2 lanes; first {count} requests"),
           "requests": count}
    clocks = ClockSampler(local_rank)
    clocks.start()
    srv, sat = _served_saturation(local_rank, abi.SVX_MIXED, reqs)
    rate = round(0.5 * sat["solves_per_s"], 1)
    res, wall = _serve_run(srv, reqs, 1.0 / rate, base_t)
    poisson = _serve_summary(res, wall, reqs)
    poisson["rate_per_s"] = rate
    srv.close()
    srv64, sat64 = _served_saturation(local_rank, abi.SVX_FP64, reqs)
    srv64.close()
    # error of the served mixed results against one-at-a-time FP64 solves
    rng = np.random.default_rng(1)
    idx = [int(i) for i in rng.choice(len(reqs), 48, replace=False)]
    with Server(local_rank, lanes=1, precision=abi.SVX_MIXED) as one:
        for k in idx:
            one.submit(reqs[k], k)
        served_u = {}
        while len(served_u) < len(idx):
            r = one.poll(200)
            if r is not None:
                served_u[r["tag"]] = r["u"]
    with Context(local_rank) as ctx:
        errs = [_rel(served_u[k], ctx.solve_flat(reqs[k]).u) for k in idx]
        per, dev_one = one_at_a_time(ctx, [reqs[k] for k in idx])
    out["mixed_saturation"] = sat
    out["mixed_poisson"] = poisson
    out["fp64_saturation"] = sat64
    out["latency_ms"] = {"p50": poisson["p50_ms"], "p95": poisson["p95_ms"],
                         "p99": poisson["p99_ms"], "at_rate_per_s": rate,
                         "precision": "mixed"}
    out["one_at_a_time"] = {"solves_per_s": 1.0 / per, "device_ms_per_solve": dev_one,
                            "sample": "48 requests through svx_solve_flat (FP64), one after "
                                      "another, wall clock, faster of two passes"}
    out["ratio_mixed_vs_one_at_a_time"] = sat["solves_per_s"] * per
    out["ratio_fp64_vs_one_at_a_time"] = sat64["solves_per_s"] * per
    out["mixed_rel_err_vs_fp64"] = {"max": max(errs), "median": float(np.median(errs)),
                                    "sample": len(errs)}
    # the 4,096-plate mix through the same server (the batched form's mix)
    plates = workloads.plate_batch(4096, seed=4)
    c4 = {}
    for name, prec in (("mixed", abi.SVX_MIXED), ("fp64", abi.SVX_FP64)):
        s, row = _served_saturation(local_rank, prec, plates)
        s.close()
        if c4_one_at_a_time_s:
            row["ratio_vs_one_at_a_time"] = row["solves_per_s"] * c4_one_at_a_time_s
        c4[name] = row
    out["plates4096_saturation"] = c4
    out["clocks"] = clocks.stop()
    out["timing"] = ("wall clock from the first submit to the last result on the host; "
                     "latency from each submit to its result")
    return out


def metric_forms(local_rank):
    """precision_c3, batched_c4 and served_c5 blocks of the default line."""
    blocks = {}
    t0 = time.perf_counter()

    def guarded(name, fn):
        # a failing block is reported in the line, never loses the line
        try:
            return fn()
        except Exception as e:  # noqa: BLE001
            blocks[name] = {"error": f"{type(e).__name__}: {e}"}
            return None

    out = guarded("precision_c3", lambda: precision_block(local_rank))
    if out is not None:
        blocks["precision_c3"] = out
    per_c4 = None
    out = guarded("batched_c4", lambda: batched_block(local_rank))
    if out is not None:
        blocks["batched_c4"], per_c4 = out
    out = guarded("served_c5", lambda: served_block(local_rank, c4_one_at_a_time_s=per_c4))
    if out is not None:
        blocks["served_c5"] = out
    blocks["metric_forms_wall_s"] = time.perf_counter() - t0
    return blocks


THERMAL_NAME = ("steady conduction in a C3D8 block 480x48x48 over 2.0x0.2x0.2 m (1,154,881 "
                "nodes = DOF, 30,297,025 nnz), k=45, uniform source 1e5, T=20 on x=0 and T=80 "
                "on x=L; relative residual 1e-10")


def thermal_block(nx, ny, nz, lx, ly, lz, k=45.0, source=1e5):
    """Structured C3D8 conduction block (k-major node order) with fixed
    temperatures on the x = 0 and x = L faces."""
    import numpy as np

    from solvix_b200.marshal import ThermalModel

    i, j, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                           indexing="ij")
    i, j, kk = (a.transpose(2, 1, 0).ravel() for a in (i, j, kk))
    xyz = np.stack([lx * i / nx, ly * j / ny, lz * kk / nz], axis=1)
    p = (ny + 1) * (nx + 1)
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = (ek * p + ej * (nx + 1) + ei).transpose(2, 1, 0).ravel()
    offs = np.array([0, 1, nx + 2, nx + 1, p, p + 1, p + nx + 2, p + nx + 1])
    conn = (base[:, None] + offs[None, :]).ravel()
    ne = nx * ny * nz
    cold = np.flatnonzero(i == 0)
    hot = np.flatnonzero(i == nx)
    return ThermalModel(xyz, np.full(ne, 5, dtype=np.uint8), np.arange(ne + 1) * 8, conn, k,
                        source=source, temp_node=np.concatenate([cold, hot]),
                        temp_value=np.concatenate([np.full(cold.size, 20.0),
                                                   np.full(hot.size, 80.0)]))


def run_thermal(args, rank, world, local_rank):
    """Steady conduction (svx_solve_thermal_flat) on one GPU: each step one
    full solve from the host model to host temperatures (upload, conduction
    matrices, pattern, assembly, loads, temperature rows, PCG, download),
    wall clock.  The CPU leg times the oracle on a 120x12x12 block."""
    import numpy as np
    import torch

    from oracle import oracle
    from solvix_b200 import Context
    from solvix_b200.roofline import pcg_iteration_bytes

    torch.cuda.set_device(local_rank)
    nx, ny, nz = 480, 48, 48
    tm = thermal_block(nx, ny, nz, 2.0, 0.2, 0.2)
    n = tm.n_nodes
    nnz = (3 * (nx + 1) - 2) * (3 * (ny + 1) - 2) * (3 * (nz + 1) - 2)
    ctx = Context(local_rank)
    lib = ctx.lib
    for _ in range(max(args.warmup, 0)):
        ctx.solve_thermal(tm)
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = lib.svx_launch_count()
    walls, iters = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, it, res = ctx.solve_thermal(tm)
        walls.append(time.perf_counter() - t0)
        iters.append(it)
    launches = lib.svx_launch_count() - launches0
    clk = clocks.stop()
    ctx.close()
    wall = float(sum(walls))
    dof_it = float(n * sum(iters))
    value = dof_it / wall
    peak, peak_kind = measured_peaks()
    bytes_it = pcg_iteration_bytes(n, nnz, 1, n)
    achieved = bytes_it * sum(iters) / wall / 1e9
    line = {
        "metric": METRIC, "form": "thermal", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (structured block; no public dataset exists for this path)",
        "config": {"workload": THERMAL_NAME, "n_dof": n, "nnz": nnz,
                   "l2": "K 256 MB per solve vs 126 MB L2"},
        "solves_per_s": args.steps / wall, "iterations": int(np.median(iters)),
        "residual": res,
        "e2e": {"value": value, "unit": UNIT,
                "note": "svx_solve_thermal_flat from host arrays to host temperatures; the "
                        "value is this same wall-clock figure",
                "h2d_bytes_per_step": int(tm.xyz.nbytes + tm.conn.nbytes + tm.conn_ptr.nbytes
                                          + tm.kind.nbytes + tm.temp_node.nbytes
                                          + tm.temp_value.nbytes),
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "pcg_persistent2_kernel<1, 16, double> and the "
                     "assembly kernels, whole solve",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "algorithmic_bytes_per_iteration": bytes_it,
                     "note": "PCG algorithmic bytes over the whole solve's wall clock (assembly "
                             "and copies included): a lower bound of the kernel's rate",
                     "traffic": None},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        small = thermal_block(120, 12, 12, 0.5, 0.05, 0.05)
        threads = max(1, min(8, os.cpu_count() or 1))
        t0 = time.perf_counter()
        _, it_c, _ = oracle.solve_thermal(small, threads=threads)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": small.n_nodes * it_c / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one full oracle conduction solve of a 120x12x12 block ({small.n_nodes} "
                      f"DOF, {it_c} PCG iterations) on {threads} threads in {dt:.2f} s"}
    return line


DIRECT_NAMES = {
    "hex40": ("C3D8 hex cantilever 40x4x4 over 2.0x0.1x0.1 m (the mesh of the reference's LDLT "
              "timing test, ldl.rs:361-434; 1,025 nodes, 3,075 DOF), E=210e9, nu=0.3, tip-face "
              "load; direct path (Method::Ldlt)"),
    "c2": ("C3D8 cantilever 160x16x16 over 2.0x0.2x0.2 m (139,587 DOF, 10,393,929 nnz), "
           "seeded jitter; direct path (Method::Ldlt)"),
}


def direct_workload(which):
    from solvix_b200 import workloads
    if which == "c2":
        return workload()
    return workloads.cantilever_c3d8(40, 4, 4, lx=2.0, ly=0.1, lz=0.1, jitter=0.0, E=210e9,
                                     nu=0.3)


def direct_cpu(flat, min_seconds=2.0, max_solves=20):
    """The oracle's full direct solve (assembly, RCM, up-looking LDL^T,
    solve, residual, stress) repeated until min_seconds or max_solves
    (exactly max_solves when min_seconds <= 0)."""
    from oracle import oracle
    oracle.build()
    threads = oracle.default_threads()
    times = []
    while len(times) < max_solves and (min_seconds <= 0 or sum(times) < min_seconds):
        t0 = time.perf_counter()
        ref = oracle.solve_flat(flat, threads=threads, method="ldlt")
        times.append(time.perf_counter() - t0)
    return len(times) / sum(times), times, threads, ref


def run_reference_direct(args):
    flat = direct_workload(args.direct_workload)
    for _ in range(max(0, args.warmup)):
        direct_cpu(flat, min_seconds=0.0, max_solves=1)
    value, times, threads, _ = direct_cpu(flat, min_seconds=0.0, max_solves=args.steps)
    sample = (f"{len(times)} full oracle direct solves (assembly on {threads} threads, serial "
              f"RCM + up-looking LDLT as in ldl.rs) of the same model")
    return {
        "impl": "reference", "metric": "direct solves/s (Method::Ldlt)", "form": "direct",
        "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": 1000.0 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (structured mesh; no public dataset exists for this path)",
        "config": {"workload": DIRECT_NAMES[args.direct_workload], "parallelism": "host"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_direct(args, rank, world, local_rank):
    """The direct path on one GPU.  value: svx_op_solve with SVX_METHOD_LDLT
    on the assembled operator (host RCM ordering, band fill, factorization,
    solves, residual), CUDA events on the library's stream around the steps;
    e2e: svx_solve_flat with the same method from host arrays (upload,
    assembly, direct solve, stress, download), wall clock."""
    import torch

    from solvix_b200 import Context, abi

    torch.cuda.set_device(local_rank)
    flat = direct_workload(args.direct_workload)
    ctx = Context(local_rank)
    lib = ctx.lib
    op = ctx.assemble(flat)
    for _ in range(max(args.warmup, 0)):
        op.solve(method=abi.SVX_METHOD_LDLT)
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local_rank}")
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = lib.svx_launch_count()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        _u, _it, res, cond = op.solve(method=abi.SVX_METHOD_LDLT)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = lib.svx_launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    # the factorization's own device time and bandwidth, from one more solve
    sol = ctx.solve_flat(flat, method=abi.SVX_METHOD_LDLT, want_stress=False)
    for _ in range(max(args.warmup, 0)):
        ctx.solve_flat(flat, method=abi.SVX_METHOD_LDLT)
    walls = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.solve_flat(flat, method=abi.SVX_METHOD_LDLT)
        walls.append(time.perf_counter() - t0)
    clk = clocks.stop()
    op.free()
    ctx.close()
    n, bw = flat.n_dof, sol.factor_bandwidth
    band_bytes = 8 * 1024 * ((n + 31) // 32) * ((bw + 31) // 32 + 1)
    value = args.steps / (ms * 1e-3)
    flops = float(n) * bw * bw
    line = {
        "metric": "direct solves/s (Method::Ldlt)", "form": "direct", "value": value,
        "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (structured mesh; no public dataset exists for this path)",
        "config": {"workload": DIRECT_NAMES[args.direct_workload], "n_dof": n,
                   "half_bandwidth_rcm": bw,
                   "band_bytes": band_bytes,
                   "l2": ("band resident in the 126 MB L2" if band_bytes < 126e6 else
                          "band larger than the 126 MB L2")},
        "residual": res, "cond_estimate": cond,
        "e2e": {"value": args.steps / sum(walls), "unit": "solves/s",
                "note": "svx_solve_flat (method LDLT, stress on) from host arrays, wall clock",
                "h2d_bytes_per_step": int(flat.xyz.nbytes + flat.conn.nbytes +
                                          flat.conn_ptr.nbytes + flat.kind.nbytes +
                                          flat.youngs.nbytes + flat.poisson.nbytes +
                                          flat.fixed_row.nbytes + flat.f.nbytes),
                "d2h_bytes_per_step": int(8 * (2 * n + 3 * flat.n_nodes + flat.n_elem +
                                               flat.n_nodes + flat.fixed_row.shape[0]))},
        "gpu_launches": int(launches),
        "roofline": {"bound": "fp64", "kernel": "ldlt_update_kernel + ldlt_panel_kernel "
                     "(whole direct solve)", "achieved": flops / (sol.ms_factor * 1e-3) / 1e12,
                     "peak": None, "unit": "TFLOP/s", "frac": None, "traffic": None,
                     "device_ms": sol.ms_factor,
                     "note": "n * bandwidth^2 flops (the band LDLT's leading term) over the "
                             "device time from band fill to residual; no measured FP64 peak "
                             "exists for this pool, so no fraction is given"},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        if args.direct_workload == "c2":
            # one serial LDLT of the full cantilever takes about two minutes;
            # time a 60x6x6 cantilever of the same kind instead
            from solvix_b200 import workloads
            small = workloads.cantilever_c3d8(60, 6, 6, lx=0.75, ly=0.075, lz=0.075)
            cps, times, threads, _ = direct_cpu(small, min_seconds=2.0, max_solves=3)
            what = f"a 60x6x6 C3D8 cantilever ({small.n_dof} DOF), not the same model"
        else:
            cps, times, threads, _ = direct_cpu(flat)
            what = "the same model"
        line["cpu_baseline"] = {
            "value": cps, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} full oracle direct solves of {what} "
                      f"(assembly on {threads} threads, serial up-looking LDLT) in "
                      f"{sum(times):.2f} s"}
    return line


KERNEL_WORKLOADS = {
    "c3d8_160": ("C3D8 cantilever 160x16x16 (C2)",
                 lambda w: w.cantilever_c3d8(160, 16, 16)),
    "c3d8_480": ("heterogeneous C3D8 cantilever 480x48x48 (C3)",
                 lambda w: w.heterogeneous_c3d8(480, 48, 48)),
    "c3d8_240": ("heterogeneous C3D8 cantilever 240x24x24",
                 lambda w: w.heterogeneous_c3d8(240, 24, 24)),
    "hetero_160": ("heterogeneous C3D8 cantilever 160x16x16",
                   lambda w: w.heterogeneous_c3d8(160, 16, 16)),
    "cps4_200": ("CPS4 cantilever 200x20 (C1)", lambda w: w.cantilever_cps4(200, 20)),
    "c3d8_40x4x4": ("C3D8 cantilever 40x4x4",
                    lambda w: w.cantilever_c3d8(40, 4, 4, lx=2.0, ly=0.1, lz=0.1)),
}


def run_kernels(args, local_rank):
    """--form kernels: device times of single kernels on one workload, small
    and self-contained so that ncu can capture one kernel of it.

    * iteration: the FP64 node-block SpMV + p.Kp, the u/r update, the p
      update and the FP32 difference-form SpMV, each over --reps
      back-to-back launches (CUDA events);
    * solve: one full FP64 solve (the persistent kernel while K fits in L2);
    * batch / batch-3d: one batched solve of the first --batch-count plates
      of the 4,096-plate mix / C3D8 cantilevers of the served stream;
    * direct: the direct path twice, the second run's device time;
    * defect: one FP64 solve, then one SVX_MIXED_DEFECT solve per inner
      tolerance of --inner-tols, each with its iteration split, its device
      PCG time against the FP64 one and its error against the FP64 u."""
    from solvix_b200 import Context, abi, workloads
    from solvix_b200.roofline import pcg_iteration_bytes, spmv_node_bytes

    out = {"form": "kernels", "mode": args.kernel_mode}
    prec = abi.SVX_MIXED if args.precision == "mixed" else abi.SVX_FP64
    with Context(local_rank) as ctx:
        if args.kernel_mode in ("batch", "batch-3d"):
            if args.kernel_mode == "batch":
                flats = workloads.plate_batch(4096, seed=4)[:args.batch_count]
            else:
                stream = workloads.request_stream(max(64, 4 * args.batch_count), 1.0, seed=5)
                flats = [m for _, m in stream if m.ndof == 3][:args.batch_count]
            res, st = ctx.solve_batch(flats, precision=prec)
            b = sum(r["iterations"] * pcg_iteration_bytes(f.n_dof, r["nnz"], f.ndof, f.n_nodes)
                    for f, r in zip(flats, res))
            out.update({"models": len(flats), "total_dof": int(st["total_dof"]),
                        "iterations": int(sum(r["iterations"] for r in res)),
                        "pcg_ms": st["ms_solve"], "threads_per_cta": st["threads_per_cta"],
                        "lanes_per_node": st["lanes_per_node"],
                        "cluster_members": st["cluster_members"], "algorithmic_bytes": b,
                        "gbs": b / (st["ms_solve"] * 1e-3) / 1e9})
            return out
        name, make = KERNEL_WORKLOADS[args.workload]
        flat = make(workloads)
        out["workload"] = name
        if args.kernel_mode == "direct":
            for _ in range(2):
                sol = ctx.solve_flat(flat, want_stress=False, method=abi.SVX_METHOD_LDLT)
            n, bw = flat.n_dof, sol.factor_bandwidth
            out.update({"n": n, "bandwidth": bw, "direct_ms": sol.ms_factor,
                        "residual": sol.final_residual,
                        "band_gflops": n * bw * bw / (sol.ms_factor * 1e-3) / 1e9})
            return out
        op = ctx.assemble(flat)
        try:
            n, nnz = op.n, op.nnz
            out.update({"n": n, "nnz": nnz})
            if args.kernel_mode == "defect":
                import numpy as np

                from solvix_b200.model import NotConverged
                u64, it64, _, _ = op.solve(max_iter=200000)
                _, _, ms64, _, _ = op.solve_device(max_iter=200000, want_stress=False)
                rows = []
                for itol in (float(t) for t in args.inner_tols.split(",") if t):
                    try:
                        u, it, res, _ = op.solve(precision=abi.SVX_MIXED_DEFECT,
                                                 inner_tol=itol, max_iter=200000)
                    except NotConverged as e:
                        rows.append({"inner_tol": itol, "error": f"NotConverged: {e}"})
                        continue
                    row = {"inner_tol": itol, "iterations": it,
                           "fp32_iterations": op.last_fp32_iterations,
                           "corrections": op.last_outer_iterations, "residual": res,
                           "rel_err_vs_fp64": float(np.linalg.norm(u - u64) /
                                                    np.linalg.norm(u64))}
                    _, _, ms, _, _ = op.solve_device(precision=abi.SVX_MIXED_DEFECT,
                                                     inner_tol=itol, max_iter=200000,
                                                     want_stress=False)
                    row.update({"pcg_ms": ms, "ms_per_iteration": ms / it,
                                "vs_fp64": ms64 / ms})
                    rows.append(row)
                out.update({"fp64": {"iterations": it64, "pcg_ms": ms64,
                                     "ms_per_iteration": ms64 / it64},
                            "defect": rows})
            elif args.kernel_mode == "solve":
                runs = []
                for _ in range(max(1, args.reps)):
                    runs.append(op.solve_device(precision=prec, want_stress=False,
                                                max_iter=200000))
                it, res, _, _, _ = runs[-1]
                ms_solve = sorted(r[2] for r in runs)[len(runs) // 2]  # median
                b = pcg_iteration_bytes(n, nnz, flat.ndof, flat.n_nodes)
                out.update({"iterations": it, "residual": res, "pcg_ms": ms_solve,
                            "solves": len(runs),
                            "fp32_iterations": op.last_fp32_iterations,
                            "us_per_iteration": 1000.0 * ms_solve / max(1, it),
                            "bytes_per_iteration": b,
                            "gbs": b * it / (ms_solve * 1e-3) / 1e9})
            else:
                ms = op.time_kernels(reps=args.reps)
                b64 = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes)
                b32 = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes, value_bytes=4)
                out.update({"reps": args.reps, "spmv_ms": ms[0], "update_ms": ms[1],
                            "p_update_ms": ms[2], "spmv_fp32_ms": ms[3],
                            "spmv_bytes": b64, "spmv_gbs": b64 / (ms[0] * 1e-3) / 1e9,
                            "spmv_fp32_bytes": b32,
                            "spmv_fp32_gbs": b32 / (ms[3] * 1e-3) / 1e9})
        finally:
            op.free()
    return out


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.form == "batched":
            line = run_batched(args, rank, world, local_rank)
        elif args.form == "served":
            line = run_served(args, rank, world, local_rank)
        elif args.form == "precision":
            line = run_precision(args, rank, world, local_rank) if rank == 0 else None
        elif args.form == "thermal":
            line = run_thermal(args, rank, world, local_rank) if rank == 0 else None
        elif args.form == "direct":
            line = run_direct(args, rank, world, local_rank) if rank == 0 else None
        elif args.form == "kernels":
            line = run_kernels(args, local_rank) if rank == 0 else None
        else:
            line = run_ours(args, rank, world, local_rank)
            if world == 1 and not args.plain_only:
                line.update(metric_forms(local_rank))
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

"""Device timing of the PCG iteration kernels on a synthetic workload.

    python -m solvix_b200.kernel_timer [--workload c3d8_160|c3d8_480|cps4_200] [--reps N]
                                       [--solve | --direct] [--batch N | --batch-3d N]

Assembles the workload on cuda:0, then times the three FP64 iteration
kernels (node-block SpMV + p.Kp, u/r update + dots, p update) with CUDA
events over ``--reps`` back-to-back launches each and prints their average
duration and the SpMV's HBM throughput from its algorithmic bytes.  With
``--solve`` it runs one full FP64 solve instead (the persistent cooperative
PCG kernel, one launch per chunk of iterations) and prints its device time
and per-iteration algorithmic bytes.  With ``--batch N`` it runs one
batched FP64 solve of the first N plates of the 4,096-plate mix, with
``--batch-3d N`` of the first N C3D8 cantilevers of the served request
stream (the cluster kernel's members).  With ``--direct`` it runs the
direct path (RCM-ordered band LDL^T on the device) twice and prints the
second run's device time, half-bandwidth and band arithmetic rate
(n * bandwidth^2 flops, the leading term of a band LDL^T).  Small and
self-contained, so it is also the command to profile a single kernel with
ncu.
"""
from __future__ import annotations

import argparse
import json

from . import abi, workloads
from .core import Context

WORKLOADS = {
    "c3d8_160": lambda: workloads.cantilever_c3d8(160, 16, 16),
    "c3d8_480": lambda: workloads.heterogeneous_c3d8(480, 48, 48),
    "c3d8_240": lambda: workloads.heterogeneous_c3d8(240, 24, 24),
    "cps4_200": lambda: workloads.cantilever_cps4(200, 20),
    "c3d8_40x4x4": lambda: workloads.cantilever_c3d8(40, 4, 4, lx=2.0, ly=0.1, lz=0.1),
    "c3d8_80x8x8": lambda: workloads.cantilever_c3d8(80, 8, 8, lx=2.0, ly=0.2, lz=0.2),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description="time the PCG iteration kernels")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3d8_160")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--solve", action="store_true", help="one full persistent FP64 solve")
    ap.add_argument("--direct", action="store_true",
                    help="the direct path (band LDL^T) instead of the PCG")
    ap.add_argument("--batch", type=int, default=0,
                    help="instead: one batched solve of this many plates of the 4,096-plate mix")
    ap.add_argument("--batch-3d", type=int, default=0,
                    help="instead: one batched solve of the first this many C3D8 cantilevers "
                         "of the served request stream")
    ap.add_argument("--repeat", type=int, default=1, help="batched solves (the last is printed)")
    ap.add_argument("--mixed", action="store_true",
                    help="with --batch/--batch-3d: the mixed form instead of FP64")
    ap.add_argument("--solo", action="store_true",
                    help="with --batch/--batch-3d: also solve each model alone (svx_solve_flat) "
                         "and print the summed device PCG time")
    args = ap.parse_args(argv)
    if args.batch > 0 or args.batch_3d > 0:
        if args.batch > 0:
            flats = workloads.plate_batch(4096, seed=4)[:args.batch]
        else:
            stream = workloads.request_stream(max(64, 4 * args.batch_3d), 1.0, seed=5)
            flats = [m for _, m in stream if m.ndof == 3][:args.batch_3d]
        with Context(0) as ctx:
            for _ in range(max(1, args.repeat)):
                out, st = ctx.solve_batch(
                    flats, precision=abi.SVX_MIXED if args.mixed else abi.SVX_FP64)
            its = sum(o["iterations"] for o in out)
            b = sum(o["iterations"] * pcg_iteration_bytes(f.n_dof, o["nnz"], f.ndof, f.n_nodes)
                    for f, o in zip(flats, out))
            print(json.dumps({"batch": len(flats), "total_dof": st["total_dof"],
                              "iterations": its, "pcg_ms": st["ms_solve"],
                              "threads_per_cta": st["threads_per_cta"],
                              "lanes_per_node": st["lanes_per_node"],
                              "cluster_members": st["cluster_members"],
                              "algorithmic_bytes": b,
                              "gbs": b / (st["ms_solve"] * 1e-3) / 1e9}))
            if args.solo:
                ms = its_solo = 0
                for f in flats:
                    sol = ctx.solve_flat(f, want_stress=False)
                    ms += sol.ms_solve
                    its_solo += sol.iterations
                print(json.dumps({"solo_pcg_ms": ms, "solo_iterations": its_solo,
                                  "batched_speedup": ms / st["ms_solve"]}))
        return
    flat = WORKLOADS[args.workload]()
    if args.direct:
        with Context(0) as ctx:
            for _ in range(2):
                sol = ctx.solve_flat(flat, want_stress=False, method=abi.SVX_METHOD_LDLT)
            n, bw = flat.n_dof, sol.factor_bandwidth
            print(json.dumps({"workload": args.workload, "n": n, "bandwidth": bw,
                              "direct_ms": sol.ms_factor, "residual": sol.final_residual,
                              "cond_estimate": sol.cond_estimate,
                              "band_gflops": n * bw * bw / (sol.ms_factor * 1e-3) / 1e9}))
        return
    with Context(0) as ctx:
        op = ctx.assemble(flat)
        n, nnz = op.n, op.nnz
        if args.solve:
            it, res, ms_solve, _, _ = op.solve_device(want_stress=False)
            b = pcg_iteration_bytes(n, nnz, flat.ndof, flat.n_nodes)
            out = {"workload": args.workload, "n": n, "nnz": nnz, "iterations": it,
                   "residual": res, "pcg_ms": ms_solve, "bytes_per_iteration": b,
                   "gbs": b * it / (ms_solve * 1e-3) / 1e9}
        else:
            ms = op.time_kernels(reps=args.reps)
            spmv_bytes = spmv_node_bytes(n, nnz, flat.ndof, flat.n_nodes)
            out = {"workload": args.workload, "n": n, "nnz": nnz, "reps": args.reps,
                   "spmv_ms": ms[0], "update_ms": ms[1], "p_update_ms": ms[2],
                   "spmv_bytes": spmv_bytes, "spmv_gbs": spmv_bytes / (ms[0] * 1e-3) / 1e9,
                   "spmv_fp32_ms": ms[3],
                   "spmv_fp32_gbs": (spmv_bytes - 4 * nnz) / (ms[3] * 1e-3) / 1e9}
        op.free()
    print(json.dumps(out))


def spmv_node_bytes(n: int, nnz: int, ndof: int, n_nodes: int) -> int:
    """Algorithmic bytes of one node-block SpMV + p.Kp (spmv_node_dot): K
    values, one 4-byte column index per ndof x ndof block, adj_ptr and
    node_base, p gathered once, q written, p read for the dot."""
    return int(8 * nnz + 4 * nnz // (ndof * ndof) + 16 * (n_nodes + 1) + 24 * n)


def pcg_iteration_bytes(n: int, nnz: int, ndof: int, n_nodes: int) -> int:
    """Algorithmic bytes of one persistent PCG iteration: the node-block
    SpMV with p.Kp, then u/r update (u r/w, p, r r/w, q, inv_diag) and the
    p update (p r/w, r, inv_diag)."""
    return spmv_node_bytes(n, nnz, ndof, n_nodes) + 8 * n * 11


if __name__ == "__main__":
    main()

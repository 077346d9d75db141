"""Device timing of the PCG iteration kernels on a synthetic workload.

    python -m solvix_b200.kernel_timer [--workload c3d8_160|c3d8_480|cps4_200] [--reps N]

Assembles the workload on cuda:0, then times the three FP64 iteration
kernels (SpMV + p.Kp, u/r update + dots, p update) with CUDA events over
``--reps`` back-to-back launches each and prints their average duration
and the SpMV's HBM throughput from its algorithmic bytes.  Small and
self-contained, so it is also the command to profile a single kernel with
ncu.
"""
from __future__ import annotations

import argparse
import json

from . import workloads
from .core import Context

WORKLOADS = {
    "c3d8_160": lambda: workloads.cantilever_c3d8(160, 16, 16),
    "c3d8_480": lambda: workloads.heterogeneous_c3d8(480, 48, 48),
    "c3d8_240": lambda: workloads.heterogeneous_c3d8(240, 24, 24),
    "cps4_200": lambda: workloads.cantilever_cps4(200, 20),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description="time the PCG iteration kernels")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3d8_160")
    ap.add_argument("--reps", type=int, default=20)
    args = ap.parse_args(argv)
    flat = WORKLOADS[args.workload]()
    with Context(0) as ctx:
        op = ctx.assemble(flat)
        ms = op.time_kernels(reps=args.reps)
        n, nnz = op.n, op.nnz
        spmv_bytes = nnz * 12 + 4 * (n + 1) + 16 * n
        out = {"workload": args.workload, "n": n, "nnz": nnz, "reps": args.reps,
               "spmv_ms": ms[0], "update_ms": ms[1], "p_update_ms": ms[2],
               "spmv_bytes": spmv_bytes, "spmv_gbs": spmv_bytes / (ms[0] * 1e-3) / 1e9}
        op.free()
    print(json.dumps(out))


if __name__ == "__main__":
    main()

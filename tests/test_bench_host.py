"""bench.py's host side (no GPU): the reference arm's JSON line and the
readers of the peak and ncu-traffic figures that the GPU arm's roofline
uses."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_reader_takes_the_profile_figure():
    per_iteration = bench.ncu_traffic()
    assert per_iteration is not None
    with open(bench.TRAFFIC_FILE) as fh:
        line = next(l for l in fh if l.startswith("dram_bytes_per_iteration:"))
    assert per_iteration == float(line.split(":", 1)[1].split()[0])
    # DRAM bytes of an L2-resident iteration stay below its algorithmic bytes
    assert 0 < per_iteration < 104149180


def test_batch_traffic_reader_takes_the_full_launch_figure():
    traffic = bench.batch_ncu_traffic()
    assert traffic is not None
    with open(bench.BATCH_TRAFFIC_FILE) as fh:
        alg = next(float(l.split(":", 1)[1].split()[0]) for l in fh
                   if l.startswith("algorithmic_bytes_per_launch:"))
    assert 0.5 * alg < traffic < 1.5 * alg


def test_peak_reader_falls_back_or_reads_the_measured_file():
    peak, kind = bench.measured_peaks()
    assert kind in ("measured", "fallback")
    if kind == "fallback":
        assert peak == bench.HBM_FALLBACK_GBS
    assert peak > 1000.0


@pytest.mark.timeout(600)
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


@pytest.mark.timeout(600)
def test_reference_arm_of_the_direct_form():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--form", "direct", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["form"] == "direct" and d["unit"] == "solves/s"
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["workload"] == bench.DIRECT_NAMES["hex40"]
    assert d["cpu_baseline"]["value"] == d["value"]


def test_direct_workload_is_the_reference_test_mesh():
    flat = bench.direct_workload("hex40")
    assert (flat.n_nodes, flat.n_elem, flat.n_dof) == (1025, 640, 3075)
    assert float(flat.youngs[0]) == 210e9 and float(flat.poisson[0]) == 0.3


def test_precision_cpu_sample_is_bounded_and_labelled():
    import time
    t0 = time.perf_counter()
    cb = bench.precision_cpu_baseline(7688, 3464643, iterations=20)
    assert time.perf_counter() - t0 < 120
    assert cb["kind"] == "port" and cb["unit"] == bench.UNIT and cb["value"] > 0
    assert cb["projected"] is True and cb["projected_c3_solves_per_s"] > 0
    assert "not solved on the CPU" in cb["sample"]


def test_mix_cpu_sample_is_bounded_and_labelled():
    import numpy as np
    from solvix_b200 import workloads
    rng = np.random.Generator(np.random.PCG64(4))
    flats = [workloads.plate(rng) for _ in range(6)]
    cb = bench.mix_cpu_baseline(flats, "6 plates", max_seconds=5.0)
    assert cb["kind"] == "port" and cb["unit"] == bench.UNIT and cb["value"] > 0
    assert cb["extrapolated"] is True and cb["solves_per_s"] > 0
    assert "extrapolated" in cb["sample"]


def test_algorithmic_bytes_of_the_160x16x16_cantilever():
    """The roofline numerators: K values, one column index per 3 x 3 block,
    adj_ptr and node_base, p gathered once, q written, p read for the dot;
    then the two vector updates (11 doubles a row)."""
    from solvix_b200.roofline import pcg_iteration_bytes, spmv_node_bytes
    n, nnz, nodes = 139_587, 10_393_929, 46_529
    spmv = spmv_node_bytes(n, nnz, 3, nodes)
    assert spmv == 8 * nnz + 4 * nnz // 9 + 16 * (nodes + 1) + 24 * n
    assert pcg_iteration_bytes(n, nnz, 3, nodes) == spmv + 88 * n == 104_149_180
    # the FP32 operator streams 4-byte values and the same indices
    assert spmv_node_bytes(n, nnz, 3, nodes, value_bytes=4) == spmv - 4 * nnz


def test_precision_form_line_carries_the_block(monkeypatch):
    """--form precision wraps the default line's precision_c3 block in a
    contract line of its own (the block itself is device-timed on a GPU)."""
    import types

    import torch
    blk = {"workload": bench.PRECISION_NAME, "n_dof": 3464643, "nnz": 272673225,
           "fp64": {"iterations": 7688, "ms_per_solve": 4400.0, "pcg_ms": 4300.0,
                    "solves_per_s": 1000.0 / 4400.0,
                    "dof_iter_per_s": 3464643 * 7688 / 4.4, "residual": 9.9e-11},
           "mixed": {}, "defect_correction": {},
           "ratio_mixed_over_fp64": 0.93, "ratio_defect_over_fp64": 0.46,
           "spmv_fp64": {"ms": 0.451, "gbs": 5330.0, "frac": 0.815},
           "spmv_fp32": {"ms": 0.271, "gbs": 4850.0, "frac": 0.74},
           "peak_gbs": 6537.3, "peak_source": "measured", "timing": "t",
           "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 9}}
    monkeypatch.setattr(bench, "precision_block", lambda rank: blk)
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    args = types.SimpleNamespace(no_cpu_baseline=True)
    line = bench.run_precision(args, 0, 1, 0)
    assert line["form"] == "precision" and line["metric"] == bench.METRIC
    assert line["unit"] == bench.UNIT and line["higher_is_better"] is True
    assert line["value"] == blk["fp64"]["dof_iter_per_s"]
    assert line["ms_per_step"] == blk["fp64"]["ms_per_solve"]
    assert line["precision_c3"] is blk
    assert line["roofline"]["frac"] == blk["spmv_fp64"]["frac"]
    assert line["config"]["workload"] == bench.PRECISION_NAME
    assert json.loads(json.dumps(line)) == line

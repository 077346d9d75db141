"""The served form (continuous batching) and the mixed batched form (GPU).

Each served result must be the same alone and in a mix of concurrently
arriving requests (within 1e-10 in FP64, the default, and within the mixed
form's 1e-8 bar against FP64 in the mixed form), a bad
request must come back as its own failure without touching the others, and
admission must keep the admitted device bytes under the budget.
"""
import time

import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi, workloads
from solvix_b200.serve import Server

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def mix(count, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        if rng.random() < 0.7:
            out.append(workloads.plate(rng, nx=int(rng.integers(6, 30)),
                                       ny=int(rng.integers(3, 9))))
        else:
            nx, nyz = int(rng.integers(6, 16)), int(rng.integers(2, 4))
            out.append(workloads.cantilever_c3d8(nx, nyz, nyz, lx=nx / nyz * 0.1, ly=0.1,
                                                 lz=0.1, jitter=0.0, E=70e9, nu=0.33,
                                                 total_load=-2e3,
                                                 seed=int(rng.integers(1 << 20))))
    return out


def drain(srv, count, timeout_s=120.0):
    got = {}
    t0 = time.time()
    while len(got) < count:
        assert time.time() - t0 < timeout_s, "served results did not arrive"
        r = srv.poll(100)
        if r is not None:
            got[r["tag"]] = r
    return got


def test_mixed_batch_matches_fp64_and_is_the_same_alone(ctx):
    flats = [workloads.plate(np.random.Generator(np.random.PCG64(60 + k)),
                             nx=12 + k, ny=4 + k % 5) for k in range(12)]
    fp64, _ = ctx.solve_batch(flats)
    mixed, stats = ctx.solve_batch(flats, precision=abi.SVX_MIXED)
    assert stats["not_converged"] == 0
    for k in range(len(flats)):
        assert mixed[k]["converged"] and mixed[k]["residual"] <= 1e-10
        assert rel(mixed[k]["u"], fp64[k]["u"]) <= 1e-8
    for k in (0, 5, 11):
        alone, _ = ctx.solve_batch([flats[k]], precision=abi.SVX_MIXED)
        assert np.array_equal(alone[0]["u"].view(np.int64), mixed[k]["u"].view(np.int64))


def test_mixed_single_solve_meets_fp64_bar(ctx):
    flat = workloads.cantilever_c3d8(24, 4, 4, lx=0.6, ly=0.1, lz=0.1, seed=9)
    ref = ctx.solve_flat(flat)
    op = ctx.assemble(flat)
    u, it, res, _ = op.solve(precision=abi.SVX_MIXED)
    op.free()
    assert res <= 1e-10
    assert rel(u, ref.u) <= 1e-8


@pytest.mark.parametrize("precision,bar", [(abi.SVX_FP64, 1e-10), (abi.SVX_MIXED, 1e-8)])
def test_served_results_are_the_same_alone_and_in_the_mix(precision, bar):
    flats = mix(40, seed=71)
    with Server(lanes=3, precision=precision) as srv:
        for k, f in enumerate(flats):
            st, msg = srv.submit(f, k)
            assert st == abi.SVX_OK, msg
            if k % 7 == 0:
                time.sleep(0.002)  # arrivals while earlier batches are on the device
        in_mix = drain(srv, len(flats))
        stats = srv.stats()
    assert stats["completed"] == len(flats) and stats["batches"] >= 2
    assert max(r["batch_size"] for r in in_mix.values()) > 1
    with Server(lanes=1, precision=precision) as srv:
        for k in (0, 3, 17, 39):
            srv.submit(flats[k], 1000 + k)
            alone = drain(srv, 1)[1000 + k]
            assert alone["batch_size"] == 1
            assert alone["status"] == abi.SVX_OK and in_mix[k]["status"] == abi.SVX_OK
            assert rel(in_mix[k]["u"], alone["u"]) <= bar
    for k in (1, 2):
        ref = oracle.solve_flat(flats[k])
        assert rel(in_mix[k]["u"], ref.u) <= 1e-8


def test_served_bad_request_does_not_affect_the_others():
    flats = [workloads.plate(np.random.Generator(np.random.PCG64(80 + k)), nx=10, ny=4)
             for k in range(6)]
    bad = workloads.plate(np.random.Generator(np.random.PCG64(89)), nx=10, ny=4)  # CPS4
    conn = bad.conn.copy()
    nn = int(bad.conn_ptr[1])
    conn[3 * nn:4 * nn] = conn[3 * nn:4 * nn][::-1]  # element 4 turned inside out
    bad.conn = conn
    alone = {}
    with Server(lanes=1, precision=abi.SVX_FP64) as srv:
        for k, f in enumerate(flats):
            srv.submit(f, k)
            alone[k] = drain(srv, 1)[k]
    with Server(lanes=1, max_batch=64, precision=abi.SVX_FP64) as srv:
        for k, f in enumerate(flats[:3]):
            srv.submit(f, k)
        srv.submit(bad, 99)
        for k, f in enumerate(flats[3:], start=3):
            srv.submit(f, k)
        got = drain(srv, 7)
    assert got[99]["status"] == abi.SVX_INVALID_MODEL
    assert got[99]["message"].startswith("element 4:")
    assert got[99]["elem_index"] == 3
    for k in range(6):
        assert got[k]["status"] == abi.SVX_OK
        assert rel(got[k]["u"], alone[k]["u"]) <= 1e-12
        # the member's own nonzero count, the same alone and in the batch
        assert got[k]["nnz"] == alone[k]["nnz"] > 0


def test_served_admission_keeps_within_the_budget():
    flats = mix(12, seed=73)
    with Server(lanes=2, precision=abi.SVX_FP64) as probe:
        sizes = [probe.estimate_bytes(f) for f in flats]
    budget = 2 * max(sizes)
    with Server(hbm_budget_bytes=budget, lanes=4, precision=abi.SVX_FP64) as srv:
        for k, f in enumerate(flats):
            assert srv.submit(f, k)[0] == abi.SVX_OK
        got = drain(srv, len(flats))
        stats = srv.stats()
        huge = workloads.cantilever_c3d8(40, 8, 8, lx=0.5, ly=0.1, lz=0.1, seed=3)
        st, msg = srv.submit(huge, 500)
        assert st == abi.SVX_OOM and "budget" in msg
    assert all(r["status"] == abi.SVX_OK for r in got.values())
    assert 0 < stats["peak_bytes_admitted"] <= budget
    assert stats["rejected"] == 0


def test_served_rejects_host_checkable_decks_at_submit():
    good = workloads.plate(np.random.Generator(np.random.PCG64(5)), nx=8, ny=3)
    unconstrained = workloads.plate(np.random.Generator(np.random.PCG64(6)), nx=8, ny=3)
    unconstrained.fixed_row = np.zeros(0, dtype=np.int64)
    with Server(lanes=1) as srv:
        st, msg = srv.submit(unconstrained, 1)
        assert st == abi.SVX_NO_CONSTRAINTS and msg == "no constraints"
        assert srv.submit(good, 2)[0] == abi.SVX_OK
        got = drain(srv, 1)
        assert got[2]["status"] == abi.SVX_OK
        assert srv.stats()["rejected"] == 1

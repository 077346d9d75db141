"""The batched form: many independent models in one launch (GPU).

Each model of a batch must match its own plain solve (svx_solve_flat) and
the oracle within the plain form's bars, converge on its own iteration
count, and give a bitwise identical result alone and inside a mix.
"""
import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import workloads

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def small_plates(count, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return [workloads.plate(rng, nx=int(rng.integers(4, 24)), ny=int(rng.integers(2, 8)))
            for _ in range(count)]


def test_batch_matches_individual_solves_and_oracle(ctx):
    flats = small_plates(24, seed=41)
    out, stats = ctx.solve_batch(flats)
    assert stats["not_converged"] == 0 and stats["total_dof"] == sum(f.n_dof for f in flats)
    its = set()
    for k, f in enumerate(flats):
        single = ctx.solve_flat(f)
        assert out[k]["converged"] and out[k]["residual"] <= 1e-10
        assert rel(out[k]["u"], single.u) <= 1e-10
        np.testing.assert_allclose(out[k]["von_mises"], single.von_mises, rtol=1e-8,
                                   atol=1e-8 * np.abs(single.von_mises).max())
        assert out[k]["cond_estimate"] == pytest.approx(single.cond_estimate, rel=1e-14)
        its.add(out[k]["iterations"])
        if k < 4:
            ref = oracle.solve_flat(f)
            assert rel(out[k]["u"], ref.u) <= 1e-10
    assert len(its) > 1  # per-instance convergence, not a shared count


def test_batch_result_is_the_same_alone_and_in_a_mix(ctx):
    flats = small_plates(16, seed=42)
    mix, _ = ctx.solve_batch(flats)
    for k in (0, 7, 15):
        alone, _ = ctx.solve_batch([flats[k]])
        assert np.array_equal(alone[0]["u"].view(np.int64), mix[k]["u"].view(np.int64))
        assert alone[0]["iterations"] == mix[k]["iterations"]


def test_batch_c3d8_models(ctx):
    rng = np.random.Generator(np.random.PCG64(5))
    flats = [workloads.cantilever_c3d8(int(rng.integers(6, 14)), 2, 3, lx=1.0, ly=0.2, lz=0.3,
                                       seed=int(rng.integers(1 << 20))) for _ in range(6)]
    out, _ = ctx.solve_batch(flats)
    for k, f in enumerate(flats):
        single = ctx.solve_flat(f)
        assert rel(out[k]["u"], single.u) <= 1e-10


def test_batch_budget_is_per_model(ctx):
    flats = small_plates(8, seed=43)
    out, stats = ctx.solve_batch(flats, max_iter=5)
    assert stats["not_converged"] == 8
    assert all(o["iterations"] == 5 and not o["converged"] for o in out)

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


def test_batch_large_members_run_on_clusters(ctx):
    """Large members (3D >= 4096 rows, 2D >= 16384 rows) are solved by an
    8-CTA cluster each, beside the CTA-per-member kernel; both classes meet
    the plain bars and a large member is bitwise the same alone and in the
    mix."""
    rng = np.random.Generator(np.random.PCG64(44))
    big = [workloads.plate(rng, nx=150, ny=60), workloads.plate(rng, nx=130, ny=70)]
    small = small_plates(10, seed=45)
    flats = [big[0]] + small[:5] + [big[1]] + small[5:]
    assert sum(f.n_dof >= 16384 for f in flats) == 2
    out, stats = ctx.solve_batch(flats)
    assert stats["cluster_members"] == 2 and stats["not_converged"] == 0
    for k, f in enumerate(flats):
        single = ctx.solve_flat(f)
        assert rel(out[k]["u"], single.u) <= 1e-10
    alone, st1 = ctx.solve_batch([flats[6]])
    assert st1["cluster_members"] == 1
    assert np.array_equal(alone[0]["u"].view(np.int64), out[6]["u"].view(np.int64))
    hexes = [workloads.cantilever_c3d8(40, 8, 8, lx=1.0, ly=0.2, lz=0.2, seed=46),
             workloads.cantilever_c3d8(8, 2, 2, lx=0.4, ly=0.1, lz=0.1, seed=47)]
    out3, st3 = ctx.solve_batch(hexes)
    assert st3["cluster_members"] == 1
    for k, f in enumerate(hexes):
        assert rel(out3[k]["u"], ctx.solve_flat(f).u) <= 1e-10
    from solvix_b200 import abi
    mixed, stm = ctx.solve_batch(flats, precision=abi.SVX_MIXED)
    assert stm["cluster_members"] == 2 and stm["fp32_iterations"] > 0
    for k in range(len(flats)):
        assert mixed[k]["converged"]
        assert rel(mixed[k]["u"], out[k]["u"]) <= 1e-8

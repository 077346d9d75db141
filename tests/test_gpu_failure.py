"""Failure detection on the device without a GPU fault (GPU).

Every inter-block wait in the library's kernels polls a bounded number of
times.  Here a grid barrier is given one block where it expects two, so
nothing ever releases it: the wait must run out, raise the barrier's error
flag and return, and the context must stay usable for the next solve.
Host-side failures (a device error code reported as SVX_CUDA_ERROR, a
budget overrun as NotConverged) are covered by the parity and batch tests.
"""
import ctypes as C

import numpy as np
import pytest

from solvix_b200 import abi, workloads

pytestmark = pytest.mark.gpu


def test_grid_barrier_wait_runs_out_and_reports(ctx):
    lib = abi.load()
    ok, flag = C.c_int(-1), C.c_int(-1)
    st = lib.svx_diag_barrier_timeout(0, 100000, C.byref(ok), C.byref(flag))
    assert st == abi.SVX_OK
    assert ok.value == 0 and flag.value == 1
    # the context is still usable afterwards
    flat = workloads.cantilever_c3d8(6, 2, 2, lx=0.6, ly=0.2, lz=0.2, seed=3)
    sol = ctx.solve_flat(flat)
    assert sol.iterations > 0 and np.isfinite(sol.u).all()


def test_barrier_diagnostic_rejects_unbounded_spins():
    lib = abi.load()
    ok, flag = C.c_int(), C.c_int()
    assert lib.svx_diag_barrier_timeout(0, 0, C.byref(ok), C.byref(flag)) == abi.SVX_BAD_ARGUMENT
    assert lib.svx_diag_barrier_timeout(0, 1 << 40, C.byref(ok),
                                        C.byref(flag)) == abi.SVX_BAD_ARGUMENT

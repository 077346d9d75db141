"""ctypes mirror of ``include/solvix_gpu.h`` and the loader of the native library.

The structures below are field-for-field copies of the C structs; the
functions of ``libsolvix_b200.so`` get explicit argtypes so that a wrong call
fails in Python instead of corrupting memory.  There is no fallback: when the
shared library is missing, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libsolvix_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

# enum svx_status
SVX_OK = 0
SVX_EMPTY_MESH = 1
SVX_NO_CONSTRAINTS = 2
SVX_INVALID_MODEL = 3
SVX_NOT_CONVERGED = 4
SVX_OOM = 5
SVX_CUDA_ERROR = 6
SVX_BAD_ARGUMENT = 7
SVX_QUEUE_EMPTY = 8
SVX_IO_ERROR = 9
SVX_PARSE_ERROR = 10
SVX_UNSUPPORTED = 11

# enum svx_elem_kind (order of ElemKind, crates/solvix-core/src/lib.rs:54-73)
SVX_CPS3, SVX_CPS4, SVX_CPS8, SVX_CPE4, SVX_CPE8, SVX_C3D8, SVX_C3D4, SVX_B31 = range(8)

SVX_KEEP_ORIGINAL = 1
SVX_NOALLOC_MAX_DOF = 262144

# enum svx_precision
SVX_FP64 = 0
SVX_MIXED = 1
SVX_MIXED_DEFECT = 2
SVX_METHOD_PCG = 0
SVX_METHOD_LDLT = 1
SVX_METHOD_AUTO = 2

c_double_p = C.POINTER(C.c_double)
c_int64_p = C.POINTER(C.c_int64)
c_int32_p = C.POINTER(C.c_int32)
c_uint32_p = C.POINTER(C.c_uint32)
c_uint8_p = C.POINTER(C.c_uint8)
c_char_pp = C.POINTER(C.c_char_p)


class SvxError(C.Structure):
    _fields_ = [
        ("code", C.c_int32),
        ("reason", C.c_int32),
        ("elem_index", C.c_int64),
        ("iterations", C.c_int64),
        ("residual", C.c_double),
        ("message", C.c_char * 512),
    ]


class SvxModelDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("node_ids", c_uint32_p),
        ("node_coords", c_double_p),
        ("n_elems", C.c_int64),
        ("elem_ids", c_uint32_p),
        ("elem_kinds", c_uint8_p),
        ("elem_conn_ptr", c_int64_p),
        ("elem_conn", c_uint32_p),
        ("n_materials", C.c_int32),
        ("material_names", c_char_pp),
        ("youngs_modulus", c_double_p),
        ("poisson_ratio", c_double_p),
        ("n_elsets", C.c_int32),
        ("elset_names", c_char_pp),
        ("elset_ptr", c_int64_p),
        ("elset_elem_ids", c_uint32_p),
        ("n_assignments", C.c_int32),
        ("assign_elset", c_char_pp),
        ("assign_material", c_char_pp),
        ("thickness", C.c_double),
        ("n_bcs", C.c_int32),
        ("bc_node_ptr", c_int64_p),
        ("bc_node_ids", c_uint32_p),
        ("bc_dof_ptr", c_int64_p),
        ("bc_dofs", c_int64_p),
        ("n_cloads", C.c_int64),
        ("cload_node_ids", c_uint32_p),
        ("cload_dofs", c_int64_p),
        ("cload_values", c_double_p),
        ("density", C.c_double),
        ("n_dloads", C.c_int64),
        ("dload_elem_ids", c_uint32_p),
        ("dload_faces", c_int64_p),
        ("dload_values", c_double_p),
        ("has_gravity", C.c_int32),
        ("gravity_magnitude", C.c_double),
        ("gravity_dir", C.c_double * 3),
    ]


class SvxFlatModel(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("xyz", c_double_p),
        ("node_id", c_uint32_p),
        ("n_elem", C.c_int64),
        ("kind", c_uint8_p),
        ("conn_ptr", c_int64_p),
        ("conn", c_int32_p),
        ("youngs", c_double_p),
        ("poisson", c_double_p),
        ("no_material", c_uint8_p),
        ("elem_id", c_uint32_p),
        ("thickness", C.c_double),
        ("ndof", C.c_int32),
        ("n_fixed", C.c_int64),
        ("fixed_row", c_int64_p),
        ("f", c_double_p),
    ]


class SvxFlatModelRaw(C.Structure):
    """svx_flat_model_t with untyped pointers: the same layout, filled from
    integer addresses (cheap for thousands of batch members)."""
    _fields_ = [(name, C.c_void_p if issubclass(t, C._Pointer) else t)
                for name, t in SvxFlatModel._fields_]


class SvxSolveOpts(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("max_iter", C.c_int64),
        ("precision", C.c_int32),
        ("inner_tol", C.c_double),
        ("check_every", C.c_int32),
        ("want_stress", C.c_int32),
        ("method", C.c_int32),
    ]


class SvxSolution(C.Structure):
    _fields_ = [
        ("u", c_double_p),
        ("displacements", c_double_p),
        ("von_mises", c_double_p),
        ("nodal_von_mises", c_double_p),
        ("reactions", c_double_p),
        ("iterations", C.c_int64),
        ("outer_iterations", C.c_int64),
        ("final_residual", C.c_double),
        ("cond_estimate", C.c_double),
        ("ms_assemble", C.c_double),
        ("ms_solve", C.c_double),
        ("ms_stress", C.c_double),
        ("fp32_iterations", C.c_int64),
        ("solver_method", C.c_int32),
        ("factor_bandwidth", C.c_int64),
        ("ms_factor", C.c_double),
    ]


class SvxBatchResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("residual", C.c_double),
        ("status", C.c_int32),
        ("reason", C.c_int32),
        ("cond_estimate", C.c_double),
        ("nnz", C.c_int64),
        ("elem_index", C.c_int64),
    ]


class SvxBatchStats(C.Structure):
    _fields_ = [
        ("ms_assemble", C.c_double),
        ("ms_solve", C.c_double),
        ("ms_stress", C.c_double),
        ("threads_per_cta", C.c_int32),
        ("lanes_per_node", C.c_int32),
        ("total_iterations", C.c_int64),
        ("total_dof", C.c_int64),
        ("not_converged", C.c_int32),
        ("cluster_members", C.c_int32),
        ("fp32_iterations", C.c_int64),
    ]


class SvxThermalModel(C.Structure):
    """svx_thermal_model_t (steady conduction, heat.rs:52-98)."""
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("xyz", c_double_p),
        ("n_elem", C.c_int64),
        ("kind", c_uint8_p),
        ("conn_ptr", c_int64_p),
        ("conn", c_int32_p),
        ("elem_id", c_uint32_p),
        ("thickness", C.c_double),
        ("conductivity", C.c_double),
        ("has_source", C.c_int32),
        ("source", C.c_double),
        ("n_temp", C.c_int64),
        ("temp_node", c_int64_p),
        ("temp_value", c_double_p),
        ("n_flux", C.c_int64),
        ("flux_elem", c_int64_p),
        ("flux_face", c_int32_p),
        ("flux_value", c_double_p),
    ]


class SvxVtuData(C.Structure):
    """svx_vtu_data_t (what vtu.rs's writers read)."""
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("xyz", c_double_p),
        ("n_elem", C.c_int64),
        ("kind", c_uint8_p),
        ("conn_ptr", c_int64_p),
        ("conn", c_int32_p),
        ("n_disp", C.c_int64),
        ("displacements", c_double_p),
        ("n_von_mises", C.c_int64),
        ("von_mises", c_double_p),
        ("n_extra", C.c_int32),
        ("extra_names", C.POINTER(C.c_char_p)),
        ("extra_values", C.POINTER(c_double_p)),
        ("extra_len", c_int64_p),
    ]


class SvxServeOpts(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_int64),
        ("lanes", C.c_int32),
        ("max_batch", C.c_int32),
        ("solve", SvxSolveOpts),
        ("max_batch_bytes", C.c_int64),
    ]


class SvxServeResult(C.Structure):
    _fields_ = [
        ("tag", C.c_uint64),
        ("status", C.c_int32),
        ("ndof", C.c_int32),
        ("n_nodes", C.c_int64),
        ("n_elem", C.c_int64),
        ("iterations", C.c_int64),
        ("residual", C.c_double),
        ("cond_estimate", C.c_double),
        ("t_submit_ms", C.c_double),
        ("t_start_ms", C.c_double),
        ("t_done_ms", C.c_double),
        ("batch_size", C.c_int32),
        ("lane", C.c_int32),
        ("u", C.POINTER(C.c_double)),
        ("von_mises", C.POINTER(C.c_double)),
        ("error", SvxError),
        ("nnz", C.c_int64),
    ]


class SvxServeStats(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "submitted", "rejected", "completed", "batches", "pending", "in_flight",
        "bytes_admitted", "peak_bytes_admitted", "device_bytes", "peak_device_bytes")] + \
        [(name, C.c_double) for name in (
            "prep_ms", "assemble_ms", "solve_ms", "output_ms", "device_solve_ms", "pool_ms")] + \
        [("pool_mallocs", C.c_int64)]


def ptr(a: np.ndarray | None, ctype):
    """Pointer to a contiguous numpy array (or NULL)."""
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


# Every symbol include/solvix_gpu.h declares, with (restype, argtypes).
_VP = C.c_void_p
SIGNATURES = {
    "svx_version": (C.c_char_p, []),
    "svx_default_opts": (None, [C.POINTER(SvxSolveOpts)]),
    "svx_ctx_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "svx_ctx_destroy": (C.c_int, [_VP]),
    "svx_ctx_stream": (C.c_void_p, [_VP]),
    "svx_op_reassemble": (C.c_int, [_VP, C.POINTER(SvxError)]),
    "svx_launch_count": (C.c_int64, []),
    "svx_diag_barrier_timeout": (C.c_int, [C.c_int, C.c_longlong, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int)]),
    "svx_op_time_kernels": (C.c_int, [_VP, C.c_int, c_double_p]),
    "svx_pcg_solve_noalloc": (C.c_int, [C.c_int64, _VP, _VP, _VP, _VP, C.c_double, C.c_int64,
                                        _VP, c_int64_p, c_double_p, _VP]),
    "svx_last_error": (C.c_int, [_VP, C.c_char_p, C.c_size_t]),
    "svx_resolve": (C.c_int, [C.POINTER(SvxModelDesc), C.POINTER(_VP), C.POINTER(SvxError)]),
    "svx_resolved_flat": (C.POINTER(SvxFlatModel), [_VP]),
    "svx_resolved_pending": (C.c_int, [_VP, C.POINTER(SvxError)]),
    "svx_resolved_free": (C.c_int, [_VP]),
    "svx_assemble_mass": (C.c_int, [_VP, C.POINTER(SvxFlatModel), C.c_double, C.POINTER(_VP),
                                    C.POINTER(SvxError)]),
    "svx_assemble": (C.c_int, [_VP, C.POINTER(SvxFlatModel), C.c_uint32, C.POINTER(_VP),
                               C.POINTER(SvxError)]),
    "svx_op_free": (C.c_int, [_VP]),
    "svx_op_dims": (C.c_int, [_VP, c_int64_p, c_int64_p]),
    "svx_op_get_csr": (C.c_int, [_VP, C.c_int, c_int64_p, c_int32_p, c_double_p]),
    "svx_op_get_vectors": (C.c_int, [_VP, C.c_int, c_double_p, c_double_p]),
    "svx_op_spmv": (C.c_int, [_VP, c_double_p, c_double_p]),
    "svx_op_set_solution": (C.c_int, [_VP, c_double_p]),
    "svx_order_rcm": (C.c_int, [C.c_int64, c_int64_p, c_int32_p, c_int32_p, c_int64_p]),
    "svx_op_solve": (C.c_int, [_VP, C.POINTER(SvxSolveOpts), C.POINTER(SvxSolution),
                               C.POINTER(SvxError)]),
    "svx_op_stress": (C.c_int, [_VP, C.POINTER(SvxSolution)]),
    "svx_batch_solve": (C.c_int, [_VP, C.c_int32, C.POINTER(SvxFlatModel),
                                  C.POINTER(SvxSolveOpts), C.POINTER(c_double_p),
                                  C.POINTER(c_double_p), C.POINTER(SvxBatchResult),
                                  C.POINTER(SvxBatchStats), C.POINTER(SvxError)]),
    "svx_serve_default_opts": (None, [C.POINTER(SvxServeOpts)]),
    "svx_serve_create": (C.c_int, [C.c_int, C.POINTER(SvxServeOpts), C.POINTER(_VP),
                                   C.POINTER(SvxError)]),
    "svx_serve_submit": (C.c_int, [_VP, C.POINTER(SvxFlatModel), C.c_uint64,
                                   C.POINTER(SvxError)]),
    "svx_serve_estimate_bytes": (C.c_int64, [C.POINTER(SvxFlatModel)]),
    "svx_serve_poll": (C.c_int, [_VP, C.c_int32, C.POINTER(C.POINTER(SvxServeResult))]),
    "svx_serve_result_free": (None, [C.POINTER(SvxServeResult)]),
    "svx_serve_stats": (C.c_int, [_VP, C.POINTER(SvxServeStats)]),
    "svx_serve_now_ms": (C.c_double, [_VP]),
    "svx_serve_destroy": (C.c_int, [_VP]),
    "svx_solve_flat": (C.c_int, [_VP, C.POINTER(SvxFlatModel), C.POINTER(SvxSolveOpts),
                                 C.POINTER(SvxSolution), C.POINTER(SvxError)]),
    "svx_solve_resolved": (C.c_int, [_VP, _VP, C.POINTER(SvxSolveOpts), C.POINTER(SvxSolution),
                                     C.POINTER(SvxError)]),
    "svx_write_vtu": (C.c_int, [C.c_char_p, C.POINTER(SvxVtuData), C.c_int32, C.c_int32,
                                C.POINTER(SvxError)]),
    "svx_inp_parse": (C.c_int, [C.c_char_p, C.c_int64, C.POINTER(_VP), C.POINTER(SvxError)]),
    "svx_inp_model": (C.POINTER(SvxModelDesc), [_VP]),
    "svx_inp_step_count": (C.c_int32, [_VP]),
    "svx_inp_warning_count": (C.c_int32, [_VP]),
    "svx_inp_warning": (C.c_char_p, [_VP, C.c_int32]),
    "svx_inp_free": (None, [_VP]),
    "svx_solve_thermal_flat": (C.c_int, [_VP, C.POINTER(SvxThermalModel),
                                         C.POINTER(SvxSolveOpts), c_double_p, c_int64_p,
                                         c_double_p, C.POINTER(SvxError)]),
}

_lib = None
_lock = threading.Lock()


def load(path: str | None = None):
    """Load ``libsolvix_b200.so`` (built in-tree) and bind every symbol.

    Raises ``OSError`` when the library is missing: the package has no
    pure-Python or CPU path to fall back to.
    """
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            raise OSError(
                f"{p} is missing: build the CUDA library first "
                "(python -c 'import __graft_entry__ as g; g.build()')")
        lib = C.CDLL(p)
        bind(lib, SIGNATURES)
        if path is None:
            _lib = lib
        return lib


def bind(lib, signatures):
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def default_opts(**kw) -> SvxSolveOpts:
    o = SvxSolveOpts()
    o.tol = 1e-10
    o.max_iter = 0
    o.precision = SVX_FP64
    o.inner_tol = 1e-5
    o.check_every = 0
    o.want_stress = 1
    o.method = SVX_METHOD_PCG
    for k, v in kw.items():
        setattr(o, k, v)
    return o

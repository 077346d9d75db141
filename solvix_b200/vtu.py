"""VTU output through svx_write_vtu: the reference's ASCII and appended
binary UnstructuredGrid writers (crates/solvix-io/src/vtu.rs), byte for
byte, with the ASCII lines formatted on the host cores."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


def write_vtu(path: str, xyz, kind, conn_ptr, conn, displacements=None, von_mises=None,
              extra=(), binary: bool = False, threads: int = 0) -> None:
    """Write a .vtu file.  ``conn`` holds 0-based node indices;
    ``displacements`` ([n, 3]) and ``von_mises`` ([n_elem]) may be shorter
    than the mesh (the rest prints 0, like the reference); ``extra`` is a
    sequence of (name, per-node values) written as scalar PointData arrays
    (ASCII form only, vtu.rs:14-19)."""
    lib = abi.load()
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    kind = np.ascontiguousarray(kind, dtype=np.uint8)
    conn_ptr = np.ascontiguousarray(conn_ptr, dtype=np.int64)
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    disp = (np.zeros((0, 3)) if displacements is None else
            np.ascontiguousarray(displacements, dtype=np.float64).reshape(-1, 3))
    vm = (np.zeros(0) if von_mises is None else
          np.ascontiguousarray(von_mises, dtype=np.float64).ravel())
    names = [str(n).encode() for n, _ in extra]
    values = [np.ascontiguousarray(v, dtype=np.float64).ravel() for _, v in extra]
    d = abi.SvxVtuData()
    d.n_nodes = xyz.shape[0]
    d.xyz = abi.ptr(xyz, C.c_double)
    d.n_elem = kind.shape[0]
    d.kind = abi.ptr(kind, C.c_uint8)
    d.conn_ptr = abi.ptr(conn_ptr, C.c_int64)
    d.conn = abi.ptr(conn, C.c_int32)
    d.n_disp = disp.shape[0]
    d.displacements = abi.ptr(disp, C.c_double) if disp.size else None
    d.n_von_mises = vm.shape[0]
    d.von_mises = abi.ptr(vm, C.c_double) if vm.size else None
    d.n_extra = len(extra)
    if extra:
        c_names = (C.c_char_p * len(names))(*names)
        c_vals = (abi.c_double_p * len(values))(
            *[abi.ptr(v, C.c_double) if v.size else None for v in values])
        lens = np.array([v.shape[0] for v in values], dtype=np.int64)
        d.extra_names = C.cast(c_names, C.POINTER(C.c_char_p))
        d.extra_values = C.cast(c_vals, C.POINTER(abi.c_double_p))
        d.extra_len = abi.ptr(lens, C.c_int64)
    err = abi.SvxError()
    st = lib.svx_write_vtu(str(path).encode(), C.byref(d), int(bool(binary)), int(threads),
                           C.byref(err))
    if st == abi.SVX_BAD_ARGUMENT:
        raise ValueError(err.message.decode())
    if st != abi.SVX_OK:
        raise OSError(err.message.decode())

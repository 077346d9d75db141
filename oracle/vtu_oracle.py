"""Python restatement of the reference's VTU writers (TEST INFRASTRUCTURE
ONLY): crates/solvix-io/src/vtu.rs:14-115 (ASCII, write_vtu_ex) and
:148-288 (appended raw binary, write_vtu_binary), producing the file bytes.
f64 values print as Rust's `{}` Display: the shortest round-trip digits in
positional notation (numpy's Dragon4 ``unique`` mode), "NaN", "inf"."""
from __future__ import annotations

import math
import struct

import numpy as np

VTK_TYPES = [5, 9, 23, 9, 23, 12, 10, 3]  # vtu.rs:62-70 in ElemKind order


def rust_f64(v: float) -> str:
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return np.format_float_positional(v, unique=True, trim="-")


def ascii_bytes(xyz, kind, conn_ptr, conn, disp, vm, extra=()) -> bytes:
    nn, ne = len(xyz), len(kind)
    s = ['<?xml version="1.0"?>\n',
         '<VTKFile type="UnstructuredGrid" version="0.1" byte_format="ascii">\n',
         "  <UnstructuredGrid>\n",
         f'    <Piece NumberOfPoints="{nn}" NumberOfCells="{ne}">\n',
         "      <Points>\n",
         '        <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n']
    for p in xyz:
        s.append(f"          {rust_f64(p[0])} {rust_f64(p[1])} {rust_f64(p[2])}\n")
    s.append("        </DataArray>\n      </Points>\n")
    s.append("      <Cells>\n")
    s.append('        <DataArray type="Int64" Name="connectivity" format="ascii">\n          ')
    for e in range(ne):
        for q in range(conn_ptr[e], conn_ptr[e + 1]):
            s.append(f"{conn[q]} ")
    s.append("\n        </DataArray>\n")
    s.append('        <DataArray type="Int64" Name="offsets" format="ascii">\n          ')
    off = 0
    for e in range(ne):
        off += conn_ptr[e + 1] - conn_ptr[e]
        s.append(f"{off} ")
    s.append("\n        </DataArray>\n")
    s.append('        <DataArray type="Int64" Name="types" format="ascii">\n          ')
    for e in range(ne):
        s.append(f"{VTK_TYPES[kind[e]]} ")
    s.append("\n        </DataArray>\n      </Cells>\n")
    s.append('      <PointData>\n        <DataArray type="Float64" Name="Displacement" '
             'NumberOfComponents="3" format="ascii">\n')
    for i in range(nn):
        d = disp[i] if i < len(disp) else (0.0, 0.0, 0.0)
        s.append(f"          {rust_f64(d[0])} {rust_f64(d[1])} {rust_f64(d[2])}\n")
    s.append("        </DataArray>\n      </PointData>\n")
    for name, values in extra:
        s.append(f'      <PointData>\n        <DataArray type="Float64" Name="{name}" '
                 'format="ascii">\n')
        for i in range(nn):
            s.append(f"          {rust_f64(values[i] if i < len(values) else 0.0)}\n")
        s.append("        </DataArray>\n      </PointData>\n")
    s.append('      <CellData>\n        <DataArray type="Float64" Name="VonMises" '
             'format="ascii">\n')
    for e in range(ne):
        s.append(f"          {rust_f64(vm[e] if e < len(vm) else 0.0)}\n")
    s.append("        </DataArray>\n      </CellData>\n")
    s.append("    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n")
    return "".join(s).encode()


def binary_bytes(xyz, kind, conn_ptr, conn, disp, vm) -> bytes:
    nn, ne = len(xyz), len(kind)
    pts = b"".join(struct.pack("<d", float(c)) for p in xyz for c in p)
    con = b"".join(struct.pack("<q", int(conn[q])) for q in range(conn_ptr[0], conn_ptr[ne]))
    offs = b"".join(struct.pack("<q", int(conn_ptr[e + 1] - conn_ptr[0])) for e in range(ne))
    typ = b"".join(struct.pack("<q", VTK_TYPES[kind[e]]) for e in range(ne))
    dsp = b"".join(struct.pack("<d", float(disp[i][c]) if i < len(disp) else 0.0)
                   for i in range(nn) for c in range(3))
    vms = b"".join(struct.pack("<d", float(vm[e]) if e < len(vm) else 0.0) for e in range(ne))
    blob, at = b"", []
    for block in (pts, con, offs, typ, dsp, vms):
        at.append(len(blob))
        blob += struct.pack("<i", len(block)) + block
    x = ('<?xml version="1.0"?>\n'
         '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n'
         "  <UnstructuredGrid>\n"
         f'    <Piece NumberOfPoints="{nn}" NumberOfCells="{ne}">\n'
         '      <Points>\n        <DataArray type="Float64" NumberOfComponents="3" '
         f'format="appended" offset="{at[0]}"/>\n      </Points>\n'
         '      <Cells>\n        <DataArray type="Int64" Name="connectivity" '
         f'format="appended" offset="{at[1]}"/>\n'
         f'        <DataArray type="Int64" Name="offsets" format="appended" offset="{at[2]}"/>\n'
         f'        <DataArray type="Int64" Name="types" format="appended" offset="{at[3]}"/>\n'
         "      </Cells>\n"
         '      <PointData>\n        <DataArray type="Float64" Name="Displacement" '
         f'NumberOfComponents="3" format="appended" offset="{at[4]}"/>\n      </PointData>\n'
         '      <CellData>\n        <DataArray type="Float64" Name="VonMises" '
         f'format="appended" offset="{at[5]}"/>\n      </CellData>\n'
         '    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding="raw">_')
    return x.encode() + blob + b"\n  </AppendedData>\n</VTKFile>\n"

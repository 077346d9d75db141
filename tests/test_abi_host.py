"""CPU tests of the C ABI library: it loads, exports every symbol the public
header declares, and its host-side model resolution (svx_resolve, no GPU
needed) matches the oracle's restatement of the reference's lookups and
error order."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle
from solvix_b200 import abi
from solvix_b200.marshal import FlatModel, model_desc
from solvix_b200.model import (BoundaryCondition, ConcentratedLoad, DistributedLoad, ElemKind,
                               Element, ElementSet, InvalidModel, Material, Mesh, Model, Node,
                               NoConstraints, SolveError, Step)
from svx_cases import (cantilever_deck, hex_cantilever, hex_mesh, load_golden, patch_deck,
                       quad_mesh, steel_model)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "solvix_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(svx_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    syms = header_symbols()
    assert len(syms) >= 19
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and the ctypes signature table covers the same set
    assert sorted(abi.SIGNATURES) == syms


def test_version_string():
    assert b"sm_100a" in abi.load().svx_version()


def test_no_device_is_a_loud_error():
    """Without a CUDA device the compute entry points refuse (no CPU path)."""
    lib = abi.load()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert lib.svx_ctx_create(0, C.byref(h)) == abi.SVX_CUDA_ERROR
    buf = C.create_string_buffer(512)
    lib.svx_last_error(None, buf, 512)
    assert buf.value


def product_resolve(model, pending=None):
    """svx_resolve -> (FlatModel, status, message); the error raised after
    the element loop, if any, goes into the `pending` list as
    (code, message)."""
    lib = abi.load()
    desc, keep = model_desc(model)
    res = C.c_void_p()
    err = abi.SvxError()
    st = lib.svx_resolve(C.byref(desc), C.byref(res), C.byref(err))
    if st != abi.SVX_OK:
        return None, st, err.message.decode()
    try:
        flat = FlatModel.from_struct(lib.svx_resolved_flat(res).contents)
        if pending is not None:
            perr = abi.SvxError()
            code = lib.svx_resolved_pending(res, C.byref(perr))
            if code != abi.SVX_OK:
                pending.append((code, perr.message.decode()))
    finally:
        lib.svx_resolved_free(res)
    return flat, st, ""


def oracle_resolve(model):
    try:
        flat, pending = oracle.resolve(model)
    except SolveError as e:
        code = abi.SVX_NO_CONSTRAINTS if isinstance(e, NoConstraints) else abi.SVX_INVALID_MODEL
        return None, code, str(e)
    return flat, pending, None


def assert_same_flat(a: FlatModel, b: FlatModel):
    assert a.ndof == b.ndof and a.thickness == b.thickness
    for name in ("xyz", "kind", "conn_ptr", "conn", "youngs", "poisson", "f", "no_material",
                 "node_id", "elem_id"):
        x, y = getattr(a, name), getattr(b, name)
        assert np.array_equal(np.asarray(x), np.asarray(y)), name


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_resolve_matches_oracle_on_golden_decks(name):
    model, _ = load_golden(name)
    fp, st, _ = product_resolve(model)
    fo, pending, _ = oracle_resolve(model)
    assert st == abi.SVX_OK and pending is None
    assert_same_flat(fp, fo)
    assert np.array_equal(fp.fixed_row, fo.fixed_row)


def test_resolve_duplicate_ids_and_first_assignment_wins():
    """node_index takes the first node with an id (lib.rs:106-108); the first
    assignment whose set holds the element decides, even with no material
    of that name (lib.rs:357-367)."""
    m = steel_model(quad_mesh(3, 1, 3.0, 1.0))
    m.materials = [Material("a", 1e9, 0.2), Material("b", 2e9, 0.3), Material("a", 5e9, 0.1)]
    m.elsets = [ElementSet("s1", [2]), ElementSet("s2", [1, 2, 3]), ElementSet("s1", [3]),
                ElementSet("ghost", [1])]
    m.mat_assignments = [("s1", "missing"), ("s2", "b"), ("nope", "a")]
    m.boundary_conditions = [BoundaryCondition([1, 5], [1, 2])]
    m.cloads = [ConcentratedLoad(4, 2, -1.0), ConcentratedLoad(4, 2, -2.0)]
    fp, st, _ = product_resolve(m)
    fo, pending, _ = oracle_resolve(m)
    assert st == abi.SVX_OK and pending is None
    assert_same_flat(fp, fo)
    assert list(fp.no_material) == [0, 1, 0]
    assert fp.f[(4 - 1) * 2 + 1] == -3.0


ERROR_CASES = []


def _case(fn):
    ERROR_CASES.append(fn)
    return fn


@_case
def free_body():
    return steel_model(quad_mesh(2, 1, 2.0, 1.0))


@_case
def empty_mesh():
    m = Model(materials=[Material("s", 1.0, 0.3)])
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def no_material():
    m = steel_model(quad_mesh(2, 1, 2.0, 1.0))
    m.materials = []
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def malformed_element():
    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (1, 1, 0))],
                [Element(7, ElemKind.Cps4, [1, 2, 3])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def unknown_node():
    mesh = Mesh([Node(1, (0, 0, 0)), Node(2, (1, 0, 0)), Node(3, (1, 1, 0))],
                [Element(1, ElemKind.Cps3, [1, 2, 42])])
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def bad_thickness():
    m = steel_model(quad_mesh(1, 1, 1.0, 1.0), thickness=0.0)
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def mixed_dimensionality():
    mesh = hex_mesh(1, 1, 1, 1, 1, 1)
    quad = Mesh([Node(100, (0, 0, 5)), Node(101, (1, 0, 5)), Node(102, (1, 1, 5)),
                 Node(103, (0, 1, 5))], [Element(50, ElemKind.Cps4, [100, 101, 102, 103])])
    mesh = Mesh(mesh.nodes + quad.nodes, mesh.elements + quad.elements)
    m = steel_model(mesh)
    m.boundary_conditions = [BoundaryCondition([1], [1])]
    return m


@_case
def cload_bad_dof():
    m = cantilever_deck(4, 1)
    m.cloads = [ConcentratedLoad(5, 3, 1.0)]
    return m


@_case
def cload_unknown_node():
    m = cantilever_deck(4, 1)
    m.cloads = [ConcentratedLoad(500, 1, 1.0)]
    return m


@_case
def bc_unknown_node():
    m = cantilever_deck(4, 1)
    m.boundary_conditions = [BoundaryCondition([1, 600], [1])]
    return m


@_case
def bc_bad_dof():
    m = cantilever_deck(4, 1)
    m.boundary_conditions = [BoundaryCondition([1], [1, 0])]
    return m


def _pressure_model(kind_mix=True):
    """A jittered 4 x 2 plate (thickness 0.02, density 2700) whose last quad
    is split into two CPS3, with edge pressures on every kind of face and a
    slanted gravity in its one step."""
    mesh = quad_mesh(4, 2, 2.0, 1.0)
    rng = np.random.default_rng(12)
    nodes = [Node(n.id, (n.coords[0] + rng.uniform(-0.05, 0.05),
                         n.coords[1] + rng.uniform(-0.05, 0.05), 0.0)) for n in mesh.nodes]
    elems = list(mesh.elements)
    if kind_mix:
        last = elems.pop()
        a, b, c, d = last.connectivity
        elems += [Element(last.id, ElemKind.Cps3, [a, b, c]),
                  Element(last.id + 1, ElemKind.Cps3, [a, c, d])]
    m = steel_model(Mesh(nodes, elems), thickness=0.02)
    m.density = 2700.0
    bcs = [BoundaryCondition([1, 6, 11], [1, 2])]
    m.steps = [Step(boundary_conditions=bcs, cloads=[ConcentratedLoad(15, 2, -300.0)],
                    dloads=[DistributedLoad(4, 2, 2.5e5), DistributedLoad(1, 1, -1.0e5),
                            DistributedLoad(8, 3, 7.0e4), DistributedLoad(9, 1, 3.3e4),
                            DistributedLoad(4, 2, 1.5e4)],
                    gravity=(9.81, (0.3, -1.0, 0.7)))]
    return m


def test_pressure_and_gravity_load_vector_bit_exact():
    """edge_pressure_forces and gravity_forces (assembly.rs:382-539) after
    the CLOADs, in the reference's order and operation order: the load
    vector is bit-identical to the oracle's, and its resultant is the
    pressures' and the weight's."""
    m = _pressure_model()
    fp, st, _ = product_resolve(m)
    fo, pending, _ = oracle_resolve(m)
    assert st == abi.SVX_OK and pending is None
    assert_same_flat(fp, fo)
    assert np.array_equal(fp.fixed_row, fo.fixed_row)
    # the weight: rho * t * area * g along the in-plane direction
    xy = np.array([n.coords[:2] for n in m.mesh.nodes])
    area = 0.0
    for e in m.mesh.elements:
        p = xy[[i - 1 for i in e.connectivity]]
        area += 0.5 * abs(np.dot(p[:, 0], np.roll(p[:, 1], -1)) -
                          np.dot(np.roll(p[:, 0], -1), p[:, 1]))
    weight = 2700.0 * 0.02 * area * 9.81
    no_grav = _pressure_model()
    no_grav.steps[0].gravity = None
    fg, _, _ = product_resolve(no_grav)
    diff = (fp.f - fg.f).reshape(-1, 2).sum(axis=0)
    assert np.allclose(diff, [0.3 * weight, -1.0 * weight], rtol=1e-12)


@_case
def dload_unknown_element():
    m = _pressure_model()
    m.steps[0].dloads.append(DistributedLoad(99, 1, 1.0))
    return m


@_case
def dload_no_face():
    m = _pressure_model()
    m.steps[0].dloads.append(DistributedLoad(8, 4, 1.0))  # a CPS3 has edges 1..3
    return m


@_case
def dload_face_zero():
    m = _pressure_model()
    m.steps[0].dloads.insert(0, DistributedLoad(2, 0, 1.0))
    return m


@_case
def dload_zero_length_edge():
    m = _pressure_model(kind_mix=False)
    first = m.mesh.elements[0]
    a, b, c, _d = first.connectivity
    m.mesh = Mesh(m.mesh.nodes, [Element(first.id, ElemKind.Cps4, [a, b, c, c])] +
                  list(m.mesh.elements[1:]))
    m.steps[0].dloads = [DistributedLoad(first.id, 3, 5.0)]
    return m


@_case
def dload_on_a_solid():
    m = hex_cantilever(2, 1, 1)
    m.steps = [Step(boundary_conditions=m.boundary_conditions, cloads=m.cloads,
                    dloads=[DistributedLoad(1, 1, 1.0)])]
    return m


@_case
def gravity_out_of_plane():
    m = _pressure_model()
    m.steps[0].gravity = (9.81, (0.0, 0.0, -1.0))
    return m


@_case
def gravity_on_a_solid():
    m = hex_cantilever(2, 1, 1)
    m.steps = [Step(boundary_conditions=m.boundary_conditions, cloads=m.cloads,
                    gravity=(9.81, (0.0, -1.0, 0.0)))]
    return m


@_case
def cload_error_before_dload_error():
    m = _pressure_model()
    m.steps[0].cloads.append(ConcentratedLoad(777, 1, 1.0))
    m.steps[0].dloads.append(DistributedLoad(99, 1, 1.0))
    return m


@_case
def dload_error_before_gravity_and_bc_errors():
    m = _pressure_model()
    m.steps[0].dloads.append(DistributedLoad(8, 4, 1.0))
    m.steps[0].gravity = (9.81, (0.0, 0.0, 1.0))
    m.steps[0].boundary_conditions.append(BoundaryCondition([888], [1]))
    return m


@_case
def gravity_error_before_bc_error():
    m = _pressure_model()
    m.steps[0].gravity = (9.81, (0.0, 0.0, 1.0))
    m.steps[0].boundary_conditions.append(BoundaryCondition([888], [1]))
    return m


@pytest.mark.parametrize("case", ERROR_CASES, ids=[f.__name__ for f in ERROR_CASES])
def test_resolve_errors_match_oracle(case):
    model = case()
    pend = []
    fp, st, msg = product_resolve(model, pend)
    fo, ost, omsg = oracle_resolve(model)
    if fo is None:  # raised before assembly
        assert st == ost and msg == omsg
    else:
        assert st == abi.SVX_OK
        if ost is None:
            assert_same_flat(fp, fo)
            assert pend == []
    if fo is not None and ost is not None:
        # pending error, raised by the reference after the element loop
        assert pend == [(abi.SVX_INVALID_MODEL, str(ost.err))]
        with pytest.raises(InvalidModel) as ei:
            oracle.solve(model)
        assert str(ei.value) == str(ost.err)


def test_patch_deck_resolves():
    fp, st, _ = product_resolve(patch_deck())
    assert st == abi.SVX_OK and list(fp.fixed_row) == [0, 14, 6, 1]


def test_raw_flat_struct_is_byte_identical_to_the_typed_one():
    """Batches marshal svx_flat_model_t from integer addresses; the bytes
    must be the typed struct's."""
    import ctypes as C
    import numpy as np
    from solvix_b200 import abi, workloads
    rng = np.random.Generator(np.random.PCG64(8))
    flats = [workloads.plate(rng, nx=5, ny=3),
             workloads.cantilever_c3d8(3, 2, 2, lx=0.3, ly=0.2, lz=0.2, seed=1)]
    size = C.sizeof(abi.SvxFlatModel)
    assert C.sizeof(abi.SvxFlatModelRaw) == size
    for f in flats:
        typed = f.as_struct()
        raw = abi.SvxFlatModelRaw(*f.raw_fields())
        assert C.string_at(C.addressof(typed), size) == C.string_at(C.addressof(raw), size)


# every ctypes mirror against the C compiler's own layout of the public header
STRUCTS = [("svx_error_t", abi.SvxError), ("svx_model_desc_t", abi.SvxModelDesc),
           ("svx_flat_model_t", abi.SvxFlatModel), ("svx_solve_opts_t", abi.SvxSolveOpts),
           ("svx_solution_t", abi.SvxSolution), ("svx_batch_result_t", abi.SvxBatchResult),
           ("svx_batch_stats_t", abi.SvxBatchStats), ("svx_serve_opts_t", abi.SvxServeOpts),
           ("svx_serve_result_t", abi.SvxServeResult), ("svx_serve_stats_t", abi.SvxServeStats),
           ("svx_thermal_model_t", abi.SvxThermalModel)]


def test_ctypes_mirrors_match_the_c_header_layout(tmp_path):
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "solvix_gpu.h"',
             "int main(void) {"]
    for cname, cls in STRUCTS:
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}
    for cname, cls in STRUCTS:
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)

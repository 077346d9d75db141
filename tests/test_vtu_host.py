"""svx_write_vtu (host, no GPU) against the Python restatement of the
reference's writers (crates/solvix-io/src/vtu.rs): the same bytes for the
ASCII and the appended binary forms, whatever the thread count, and the
reference's own checks of vtu.rs:382-700 (well-formed XML, exact round
trips of the appended values, VTK types per element kind, extra PointData,
binary smaller than ASCII)."""
import os
import re
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from oracle import vtu_oracle
from solvix_b200.vtu import write_vtu


def mesh(nx=7, ny=3, seed=0, specials=False):
    rng = np.random.Generator(np.random.PCG64(seed))
    xs, ys = np.meshgrid(np.linspace(0, 2.5, nx + 1), np.linspace(0, 0.7, ny + 1))
    xyz = np.zeros(((nx + 1) * (ny + 1), 3))
    xyz[:, 0] = xs.ravel() + rng.uniform(-0.01, 0.01, xs.size)
    xyz[:, 1] = ys.ravel()
    conn, kind = [], []
    for j in range(ny):
        for i in range(nx):
            a = j * (nx + 1) + i
            if (i + j) % 3 == 0:
                conn += [a, a + 1, a + nx + 2]
                kind.append(0)
            else:
                conn += [a, a + 1, a + nx + 2, a + nx + 1]
                kind.append(1)
    cp = np.zeros(len(kind) + 1, dtype=np.int64)
    cp[1:] = np.cumsum([3 if k == 0 else 4 for k in kind])
    scale = 10.0 ** rng.integers(-12, 6, (xyz.shape[0], 1))
    disp = rng.normal(0, 1e-3, (xyz.shape[0], 3)) * scale
    vm = rng.uniform(0, 3e8, len(kind))
    if specials:
        disp[0] = [0.0, -0.0, 1e21]
        disp[1] = [5e-324, -1.7976931348623157e308, 0.1]
        disp[2] = [float("nan"), float("inf"), -float("inf")]
        vm[0] = 1e-7
    return xyz, np.array(kind, dtype=np.uint8), cp, np.array(conn, dtype=np.int32), disp, vm


@pytest.mark.parametrize("threads", [1, 3, 0])
def test_ascii_bytes_match_the_reference_writer(tmp_path, threads):
    xyz, kind, cp, conn, disp, vm = mesh(specials=True)
    extra = [("Temperature", np.linspace(-5, 5, xyz.shape[0])), ("Short", [1.5, -2.25])]
    path = tmp_path / "a.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp, vm, extra=extra, threads=threads)
    assert path.read_bytes() == vtu_oracle.ascii_bytes(xyz, kind, cp, conn, disp, vm, extra)


def test_ascii_is_thread_count_independent_on_a_larger_mesh(tmp_path):
    xyz, kind, cp, conn, disp, vm = mesh(120, 60, seed=3)
    a, b = tmp_path / "1.vtu", tmp_path / "8.vtu"
    write_vtu(a, xyz, kind, cp, conn, disp, vm, threads=1)
    write_vtu(b, xyz, kind, cp, conn, disp, vm, threads=8)
    assert a.read_bytes() == b.read_bytes() == vtu_oracle.ascii_bytes(xyz, kind, cp, conn, disp,
                                                                      vm)


def test_short_solution_arrays_print_zero(tmp_path):
    # vtu.rs:79-84, :104-109: .get(i).unwrap_or(0)
    xyz, kind, cp, conn, disp, vm = mesh(4, 2)
    path = tmp_path / "s.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp[:3], vm[:2])
    assert path.read_bytes() == vtu_oracle.ascii_bytes(xyz, kind, cp, conn, disp[:3], vm[:2])


def test_binary_bytes_match_and_round_trip_exactly(tmp_path):
    # vtu.rs:560-673
    xyz, kind, cp, conn, disp, vm = mesh(9, 4, seed=2, specials=True)
    path = tmp_path / "b.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp, vm, binary=True)
    data = path.read_bytes()
    assert data == vtu_oracle.binary_bytes(xyz, kind, cp, conn, disp, vm)
    marker = b'<AppendedData encoding="raw">_'
    start = data.index(marker) + len(marker)
    xml = data[:start].decode()
    offsets = [int(x) for x in re.findall(r'offset="(\d+)"', xml)]

    def block(k):
        at = start + offsets[k]
        (n,) = struct.unpack("<i", data[at:at + 4])
        return data[at + 4:at + 4 + n]

    pts = np.frombuffer(block(0), dtype="<f8")
    assert np.array_equal(pts.view(np.int64), xyz.ravel().view(np.int64))
    assert np.array_equal(np.frombuffer(block(1), dtype="<i8"), conn.astype(np.int64))
    assert np.array_equal(np.frombuffer(block(2), dtype="<i8"), cp[1:])
    d = np.frombuffer(block(4), dtype="<f8")
    assert np.array_equal(d.view(np.int64), disp.ravel().view(np.int64))
    assert np.array_equal(np.frombuffer(block(5), dtype="<f8").view(np.int64),
                          vm.view(np.int64))


def test_vtk_types_per_element_kind(tmp_path):
    # vtu.rs:515-558 (every ElemKind)
    xyz = np.zeros((8, 3))
    sizes = [3, 4, 8, 4, 8, 8, 4, 2]
    cp = np.concatenate([[0], np.cumsum(sizes)])
    conn = np.concatenate([np.arange(s) for s in sizes]).astype(np.int32)
    kind = np.arange(8, dtype=np.uint8)
    path = tmp_path / "t.vtu"
    write_vtu(path, xyz, kind, cp, conn)
    root = ET.parse(path).getroot()
    types = next(a for a in root.iter("DataArray") if a.get("Name") == "types")
    assert [int(t) for t in types.text.split()] == [5, 9, 23, 9, 23, 12, 10, 3]


def test_well_formed_with_extra_point_data(tmp_path):
    # vtu.rs:382-513
    xyz, kind, cp, conn, disp, vm = mesh(5, 2)
    path = tmp_path / "w.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp, vm, extra=[("Mode1", np.ones(xyz.shape[0]))])
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    assert int(piece.get("NumberOfPoints")) == xyz.shape[0]
    assert int(piece.get("NumberOfCells")) == len(kind)
    names = [a.get("Name") for a in root.iter("DataArray")]
    assert names == [None, "connectivity", "offsets", "types", "Displacement", "Mode1",
                     "VonMises"]


def test_binary_is_smaller_than_ascii_for_a_large_mesh(tmp_path):
    # vtu.rs:675-700
    xyz, kind, cp, conn, disp, vm = mesh(80, 40, seed=7)
    a, b = tmp_path / "a.vtu", tmp_path / "b.vtu"
    write_vtu(a, xyz, kind, cp, conn, disp, vm)
    write_vtu(b, xyz, kind, cp, conn, disp, vm, binary=True)
    assert os.path.getsize(b) < os.path.getsize(a)


def test_errors(tmp_path):
    xyz, kind, cp, conn, disp, vm = mesh(2, 1)
    with pytest.raises(ValueError):
        write_vtu(tmp_path / "x.vtu", xyz, kind, cp, conn, extra=[("T", [1.0])], binary=True)
    bad = conn.copy()
    bad[0] = 999
    with pytest.raises(ValueError):
        write_vtu(tmp_path / "x.vtu", xyz, kind, cp, bad)
    with pytest.raises(OSError):
        write_vtu(tmp_path / "no" / "such" / "dir.vtu", xyz, kind, cp, conn)


def test_f64_text_matches_rust_display_on_random_bit_patterns(tmp_path):
    # every finite binade, subnormals and integers above 2^53 included
    rng = np.random.Generator(np.random.PCG64(11))
    bits = rng.integers(0, 2**63, 30000, dtype=np.int64) | \
        (rng.integers(0, 2, 30000, dtype=np.int64) << 63)
    vals = bits.view(np.float64)
    vals = vals[np.isfinite(vals)]
    ints = rng.integers(2**53, 2**62, 2000).astype(np.float64) * rng.choice([1.0, 1e3], 2000)
    vals = np.concatenate([vals, ints, [2.0**-1074, 2.0**-1022, 0.5, 1e23, 9007199254740993.0]])
    n = vals.shape[0] // 3
    disp = vals[:3 * n].reshape(n, 3)
    xyz = np.zeros((n, 3))
    path = tmp_path / "r.vtu"
    write_vtu(path, xyz, np.zeros(0, np.uint8), [0], np.zeros(0, np.int32), disp, threads=4)
    text = path.read_text()
    body = text.split('Name="Displacement" NumberOfComponents="3" format="ascii">\n')[1]
    lines = body.split("        </DataArray>")[0].splitlines()
    got = [tok for ln in lines for tok in ln.split()]
    want = [vtu_oracle.rust_f64(v) for v in disp.ravel()]
    assert got == want
    assert all(float(t) == v or (v == 0.0) for t, v in zip(got, disp.ravel()))


# ---- the reference's own fixtures and literal expectations (vtu.rs:382-738)
def _ref_quad_tri():
    """vtu.rs:382-430: a unit square as one CPS4 (1 2 3 4) and one CPS3
    (2 4 3), with its solution."""
    xyz = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 1.0, 0.0], [0.0, 1.0, 0.0]])
    kind = np.array([1, 0], dtype=np.uint8)
    cp = np.array([0, 4, 7], dtype=np.int64)
    conn = np.array([0, 1, 2, 3, 1, 3, 2], dtype=np.int32)
    disp = np.array([[0.1, 0.2, 0.0], [0.0, -0.5, 0.0], [-0.3, 0.0, 0.5], [0.0, 0.0, 0.0]])
    vm = np.array([42.5, 7.25])
    return xyz, kind, cp, conn, disp, vm


def test_reference_fixture_is_well_formed_and_round_trips(tmp_path):
    # vtu.rs:382-451 (vtu_is_well_formed_and_round_trips)
    xyz, kind, cp, conn, disp, vm = _ref_quad_tri()
    path = tmp_path / "r.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp, vm)
    xml = path.read_text()
    for literal in ('type="UnstructuredGrid"', 'byte_format="ascii"', 'NumberOfPoints="4"',
                    'NumberOfCells="2"', "0 1 2 3 1 3 2", "4 7", "9 5", 'Name="Displacement"',
                    "0.1 0.2 0", "-0.3 0 0.5", 'Name="VonMises"', "42.5", "7.25"):
        assert literal in xml, literal
    assert xml.rstrip().endswith("</VTKFile>")


def test_reference_fixture_extra_point_data_arrays(tmp_path):
    # vtu.rs:453-513 (vtu_extra_point_data_arrays): one B31 on two nodes,
    # an empty solution, two extra PointData arrays read back; with no extra
    # arrays the file is byte-identical to the stock writer's
    xyz = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    kind = np.array([7], dtype=np.uint8)
    cp = np.array([0, 2], dtype=np.int64)
    conn = np.array([0, 1], dtype=np.int32)
    empty = np.zeros((0, 3))
    path = tmp_path / "x.vtu"
    arrays = [("Mode1", [0.25, 1.0]), ("Temperature", [100.0, 0.5])]
    write_vtu(path, xyz, kind, cp, conn, empty, np.zeros(0),
              extra=[(n, np.array(v)) for n, v in arrays])
    xml = path.read_text()
    for name, values in arrays:
        after = xml.split(f'Name="{name}"')[1]
        body = after[:after.index("</DataArray>")]
        nums = []
        for line in body.splitlines():
            try:
                nums.append(float(line.strip()))
            except ValueError:
                pass
        assert nums == values, name
    plain, stock = tmp_path / "p.vtu", tmp_path / "s.vtu"
    write_vtu(plain, xyz, kind, cp, conn, empty, np.zeros(0), extra=[])
    write_vtu(stock, xyz, kind, cp, conn, empty, np.zeros(0))
    assert plain.read_bytes() == stock.read_bytes()


def test_reference_fixture_types_for_new_kinds(tmp_path):
    # vtu.rs:515-558 (vtu_types_for_new_kinds): CPS8, CPE8 -> 23, CPE4 -> 9,
    # B31 -> 3 on nodes x = 1..11
    xyz = np.array([[float(i), 0.0, 0.0] for i in range(1, 12)])
    kind = np.array([2, 4, 3, 7], dtype=np.uint8)
    cp = np.array([0, 8, 16, 20, 22], dtype=np.int64)
    conn = np.array(list(range(8)) + list(range(8)) + [0, 1, 2, 3] + [8, 9], dtype=np.int32)
    path = tmp_path / "k.vtu"
    write_vtu(path, xyz, kind, cp, conn, np.zeros((0, 3)), np.zeros(0))
    assert "23 23 9 3" in path.read_text()


def test_reference_fixture_binary_round_trips_exact_appended_values(tmp_path):
    # vtu.rs:560-673 (binary_vtu_round_trips_exact_appended_values): its bit
    # patterns, the extremes of f64 and signed zeros; nodes 10 20 30 40,
    # CPS4 (20 40 10 30) and CPS3 (20 30 40)
    bits = lambda b: struct.unpack("<d", struct.pack("<Q", b))[0]  # noqa: E731
    coordinate, displacement, stress = bits(0x3FF3C0D6E2F4B0D1), bits(0x3FDD555555555555), \
        bits(0x404ACCCCCCCCCCCC)
    tiny, big = 2.2250738585072014e-308, 1.7976931348623157e308
    xyz = np.array([[tiny, -0.0, coordinate], [big, coordinate, 0.0],
                    [-coordinate, tiny, -0.0], [0.0, -coordinate, big]])
    kind = np.array([1, 0], dtype=np.uint8)
    cp = np.array([0, 4, 7], dtype=np.int64)
    conn = np.array([1, 3, 0, 2, 1, 2, 3], dtype=np.int32)
    disp = np.array([[displacement, big, -tiny], [-0.0, coordinate, -displacement],
                     [tiny, -coordinate, 0.0], [-big, displacement, coordinate]])
    vm = np.array([stress, -stress])
    path = tmp_path / "e.vtu"
    write_vtu(path, xyz, kind, cp, conn, disp, vm, binary=True)
    data = path.read_bytes()
    marker = b'<AppendedData encoding="raw">_'
    start = data.index(marker) + len(marker)
    xml = data[:start].decode()
    assert ('<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">'
            in xml)
    assert '<Piece NumberOfPoints="4" NumberOfCells="2">' in xml

    def block(name_or_section):
        section, name = name_or_section
        s = xml[xml.index(f"<{section}>"):xml.index(f"</{section}>")]
        arrays = re.findall(r"<DataArray[^>]*/>", s)
        arr = next(a for a in arrays if name is None or f'Name="{name}"' in a)
        assert 'format="appended"' in arr
        at = start + int(re.search(r'offset="(\d+)"', arr).group(1))
        (n,) = struct.unpack("<i", data[at:at + 4])
        return data[at + 4:at + 4 + n]

    def same_bits(raw, expected):
        got = np.frombuffer(raw, dtype="<f8")
        return np.array_equal(got.view(np.int64), np.asarray(expected).view(np.int64))

    pts = block(("Points", None))
    assert len(pts) == 4 * 3 * 8 and same_bits(pts, xyz.ravel())
    assert list(np.frombuffer(block(("Cells", "connectivity")), "<i8")) == [1, 3, 0, 2, 1, 2, 3]
    assert list(np.frombuffer(block(("Cells", "offsets")), "<i8")) == [4, 7]
    assert list(np.frombuffer(block(("Cells", "types")), "<i8")) == [9, 5]
    d = block(("PointData", "Displacement"))
    assert len(d) == 4 * 3 * 8 and same_bits(d, disp.ravel())
    v = block(("CellData", "VonMises"))
    assert len(v) == 2 * 8 and list(np.frombuffer(v, "<f8")) == [stress, -stress]


def test_reference_fixture_binary_smaller_than_ascii(tmp_path):
    # vtu.rs:675-737 (binary_vtu_is_smaller_than_ascii_for_a_large_mesh):
    # 300 nodes on a line of B31 elements with its values
    bits = lambda b: struct.unpack("<d", struct.pack("<Q", b))[0]  # noqa: E731
    coordinate, displacement, stress = bits(0x3FF3C0D6E2F4B0D1), bits(0x3FDD555555555555), \
        bits(0x404ACCCCCCCCCCCC)
    ids = np.arange(1, 301, dtype=np.float64)
    xyz = np.stack([ids * coordinate, -ids * coordinate, coordinate / ids], axis=1)
    kind = np.full(299, 7, dtype=np.uint8)
    cp = np.arange(0, 600, 2, dtype=np.int64)
    conn = np.stack([np.arange(299), np.arange(1, 300)], axis=1).ravel().astype(np.int32)
    disp = np.stack([np.full(300, displacement), np.full(300, -displacement),
                     displacement / ids], axis=1)
    vm = stress * np.arange(1, 300, dtype=np.float64)
    a, b = tmp_path / "a.vtu", tmp_path / "b.vtu"
    write_vtu(a, xyz, kind, cp, conn, disp, vm)
    write_vtu(b, xyz, kind, cp, conn, disp, vm, binary=True)
    assert os.path.getsize(b) < os.path.getsize(a)

"""The linear-static .inp reader (svx_inp_parse, host) against the
reference's parser tests (crates/solvix-io/src/parser.rs:1507-2058) for the
keywords it covers, and end to end: decks written from the golden models
parse back to the same models, which reproduce the reference's published
iteration counts and residuals through the oracle."""
import json
import os

import pytest

from oracle import oracle
from solvix_b200.inp import ParseError, UnsupportedDeck, parse_inp
from solvix_b200.model import ElemKind
from svx_cases import GOLDEN_DIR, fmt_e3

DECK = """
** full-coverage smoke deck
*HEADING
    smoke deck
*NODE
1, 0.0, 0.0
2, 1.0, 0.0, 0.0
3, 2.0, 0.5
4, 0.0, 1.0
5, 1.0, 1.0
6, 2.0, 1.5
*ELEMENT, TYPE=CPS4, ELSET=QUADS
1, 1, 2, 5, 4
*ELEMENT, TYPE=CPS3, ELSET=TRIS
2, 2, 3, 5
*ELSET, ELSET=ALLELM
1, 2
*ELSET, ELSET=TOP, GENERATE
4, 6, 2
*NSET, NSET=FIX
1, 4
*NSET, NSET=TIP, GENERATE
5, 6, 1
*MATERIAL, NAME=steel
*ELASTIC
210.0E9, 0.3
*SOLID SECTION, ELSET=ALLELM, MATERIAL=steel
0.05
{dload}*STEP
*STATIC
*BOUNDARY
FIX, 1, 2
7, 1, 1, 2.5
*CLOAD
TIP, 2, -50.0
1, 1, 10.0
*END STEP
"""


def elset(m, name):
    return next(s for s in m.elsets if s.name == name).element_ids


def test_full_deck_parses_all_keywords():
    # parser.rs:1554-1617 without its *DLOAD block (outside this reader)
    m, w, steps = parse_inp(DECK.format(dload=""))
    assert list(m.mesh.node_ids) == [1, 2, 3, 4, 5, 6]
    assert list(m.mesh.coords[1]) == [1.0, 0.0, 0.0]
    assert list(m.mesh.coords[2]) == [2.0, 0.5, 0.0]
    assert [ElemKind(k) for k in m.mesh.elem_kinds] == [ElemKind.Cps4, ElemKind.Cps3]
    assert list(m.mesh.conn) == [1, 2, 5, 4, 2, 3, 5]
    assert elset(m, "QUADS") == [1] and elset(m, "TRIS") == [2]
    assert elset(m, "ALLELM") == [1, 2] and elset(m, "TOP") == [4, 6]
    assert m.thickness == 0.05
    assert [(x.name, x.youngs_modulus, x.poisson_ratio) for x in m.materials] == \
        [("STEEL", 210.0e9, 0.3)]
    assert m.mat_assignments == [("ALLELM", "STEEL")]
    assert [(b.node_ids, b.dofs) for b in m.boundary_conditions] == \
        [([1, 4], [1, 2]), ([7], [1])]
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == \
        [(5, 2, -50.0), (6, 2, -50.0), (1, 1, 10.0)]
    assert steps == 1
    assert len(w) == 1 and "nonzero prescribed displacement 2.5 ignored" in w[0]
    assert w[0].startswith("line 33: ")


def test_full_deck_with_its_dload_block_outside_the_step():
    # parser.rs:1554-1617 with its *DLOAD block, which sits before *STEP:
    # skipped with a warning, then the prescribed-displacement warning
    m, w, steps = parse_inp(DECK.format(dload="*DLOAD\nALLSIDES, P, 1.0\n"))
    assert len(w) == 2 and steps == 1
    assert w[0] == ("line 29: *DLOAD outside *STEP — ignored (distributed loads live in "
                    "steps)")
    assert "nonzero prescribed displacement" in w[1]
    assert m.load_state()[2] == [] and m.load_state()[3] is None


def test_keywords_outside_the_reader_send_the_deck_to_the_reference_parser():
    with pytest.raises(UnsupportedDeck, match="NLGEOM"):
        parse_inp("*NODE\n1,0,0\n*STEP, NLGEOM=YES\n*STATIC\n*END STEP\n")
    for kw in ("PLASTIC", "DYNAMIC", "TEMPERATURE", "CONTACT PAIR", "BEAM SECTION"):
        with pytest.raises(UnsupportedDeck):
            parse_inp(f"*NODE\n1,0,0\n*{kw}\n1.0\n")


def test_lowercase_keywords_crlf_generate_and_default_thickness():
    # parser.rs:1620-1658
    deck = ("*node\r\n1, 0.0, 0.0\r\n2, 1.0, 0.0\r\n3, 0.0, 1.0\r\n"
            "*element, type=cps3, elset=e1\r\n1, 1, 2, 3\r\n"
            "*nset, nset=load, generate\r\n1, 3, 1\r\n"
            "*material, name=m\r\n*elastic\r\n1.0e5, 0.0\r\n"
            "*solid section, elset=e1, material=m\r\n"
            "*boundary\r\nload, 1, 2\r\n*cload\r\n2, 2, 7.0\r\n")
    m, w, _ = parse_inp(deck)
    assert len(m.mesh.node_ids) == 3
    assert m.elsets[0].name == "E1" and m.elsets[0].element_ids == [1]
    assert m.boundary_conditions[0].node_ids == [1, 2, 3]
    assert m.boundary_conditions[0].dofs == [1, 2]
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == [(2, 2, 7.0)]
    assert m.materials[0].name == "M" and m.materials[0].youngs_modulus == 1.0e5
    assert m.thickness == 1.0
    assert w == []


def test_element_connectivity_continues_on_next_line():
    # parser.rs:1661-1670
    m, w, _ = parse_inp("*NODE\n1,0,0\n2,1,0\n3,1,1\n4,0,1\n"
                        "*ELEMENT, TYPE=CPS4\n1, 1, 2,\n3, 4\n")
    assert list(m.mesh.conn) == [1, 2, 3, 4] and w == []


def test_unsupported_element_type_and_missing_type_warn_and_skip():
    # parser.rs:1672-1684
    m, w, _ = parse_inp("*NODE\n1,0,0\n2,1,0\n3,0,1\n*ELEMENT, TYPE=S4R\n1, 1, 2, 3, 1\n"
                        "*ELEMENT\n5, 1, 2, 3\n")
    assert len(m.mesh.elem_ids) == 0
    assert len(w) == 2 and "TYPE=S4R" in w[0] and "TYPE-less" in w[1]
    assert w[0] == ("line 5: unsupported element TYPE=S4R — block skipped (supported: "
                    "CPS3/CPS4/CPS8/CPE4/CPE8/C3D8/C3D4/B31)")


def test_c3d8_and_c3d4_element_types_parse():
    # parser.rs:1686-1699
    m, w, _ = parse_inp("*NODE\n1,0,0,0\n2,1,0,0\n3,1,1,0\n4,0,1,0\n5,0,0,1\n6,1,0,1\n7,1,1,1\n"
                        "8,0,1,1\n*ELEMENT, TYPE=C3D8\n1, 1, 2, 3, 4, 5, 6, 7, 8\n"
                        "*ELEMENT, TYPE=C3D4\n2, 1, 2, 3, 5\n")
    assert w == []
    assert [ElemKind(k) for k in m.mesh.elem_kinds] == [ElemKind.C3d8, ElemKind.C3d4]
    assert list(m.mesh.conn_ptr) == [0, 8, 12]


@pytest.mark.parametrize("deck,line,text", [
    # parser.rs:1778-1810
    ("*NODE\n1, 0.0\n", 2, "*NODE expects id, x, y[, z]; got 2 field(s)"),
    ("*NODE\n1, abc, 0.0\n", 2, "malformed coordinate 'abc'"),
    ("*NODE\n1,0,0\n1,1,1\n", 3, "duplicate node id 1"),
    ("*NODE\n1,0,0\n2,1,0\n3,0,1\n*ELEMENT, TYPE=CPS3\n1,1,2,3\n1,2,3,1\n", 7,
     "duplicate element id 1"),
    ("*BOUNDARY\nNOPE, 1, 2\n", 2, "unknown node set 'NOPE'"),
    ("*CLOAD\nNOPE, 1, 1.0\n", 2, "unknown node set 'NOPE'"),
    ("*MATERIAL, NAME=M\n*ELASTIC\n1.0\n", 3,
     "*ELASTIC expects youngs_modulus, poisson_ratio; got 1 field(s)"),
    ("*SOLID SECTION, ELSET=NOPE, MATERIAL=M\n", 1,
     "*SOLID SECTION references unknown ELSET 'NOPE'"),
    # the same rules on other fields
    ("*NODE\n-1, 0, 0\n", 2, "malformed node id '-1'"),
    ("*NODE\n1, 1e, 0\n", 2, "malformed coordinate '1e'"),
    ("*NODE\n1,0,0\n*ELEMENT, TYPE=CPS3\n1, 1, 2\n", 4,
     "*ELEMENT Cps3 expects 4 field(s) (id + 3 nodes); got 3"),
    ("*NSET, NSET=A, GENERATE\n1, 5, 0\n", 2, "GENERATE step must be >= 1"),
    ("*NSET, NSET=A\n1\n*CLOAD\nA, x, 1.0\n", 4, "malformed dof 'x'"),
])
def test_fatal_errors_carry_line_numbers(deck, line, text):
    with pytest.raises(ParseError) as e:
        parse_inp(deck)
    assert e.value.line == line and e.value.message == text


def test_rust_number_grammar():
    # f64: [+-] digits [. digits] [e [+-] digits], inf / nan; u32: [+] digits
    m, _, _ = parse_inp("*NODE\n+7, .5, 1., -2e-3\n8, +1E+2, inf, -NaN\n")
    assert list(m.mesh.node_ids) == [7, 8]
    assert list(m.mesh.coords[0]) == [0.5, 1.0, -0.002]
    assert m.mesh.coords[1][0] == 100.0 and m.mesh.coords[1][1] == float("inf")
    for bad in ("0x10", "1e5.0", ".", "1..2", "1 2"):
        with pytest.raises(ParseError):
            parse_inp(f"*NODE\n1, {bad}, 0\n")
    with pytest.raises(ParseError, match="malformed node id '4294967296'"):
        parse_inp("*NODE\n4294967296, 0, 0\n")


def plate_deck(pre, steps):
    # parser.rs:1837-1857
    return ("*NODE\n1, 0.0, 0.0\n2, 0.5, 0.0\n3, 1.0, 0.0\n4, 0.0, 0.5\n5, 0.5, 0.5\n"
            "6, 1.0, 0.5\n7, 0.0, 1.0\n8, 0.5, 1.0\n9, 1.0, 1.0\n"
            "*ELEMENT, TYPE=CPS4, ELSET=ALL\n1, 1, 2, 5, 4\n2, 2, 3, 6, 5\n3, 4, 5, 8, 7\n"
            "4, 5, 6, 9, 8\n*NSET, NSET=BASE\n1, 2, 3\n*MATERIAL, NAME=STEEL\n"
            "*ELASTIC\n210.0E9, 0.3\n" + pre +
            "*SOLID SECTION, ELSET=ALL, MATERIAL=STEEL\n0.01\n" + steps)


def test_dload_edges_grav_and_density_parse():
    # parser.rs:1858-1898
    m, w, steps = parse_inp(plate_deck("*DENSITY\n7850.,\n", (
        "*STEP, NAME=PRESS\n*STATIC\n*DLOAD\nALL, P1, 1.5e6\n3, P3, 2.5e5\n"
        "GRAV, 9.81, 0.0, -1.0\n*BOUNDARY\nBASE, 1, 2\n*END STEP\n")))
    assert w == [] and steps == 1
    assert m.density == 7850.0
    bcs, _cl, dloads, gravity = m.load_state()
    assert len(dloads) == 5  # ALL expands to the 4 quads, then element 3
    assert [(d.element_id, d.face, d.magnitude) for d in dloads] == \
        [(1, 1, 1.5e6), (2, 1, 1.5e6), (3, 1, 1.5e6), (4, 1, 1.5e6), (3, 3, 2.5e5)]
    assert gravity == (9.81, (0.0, -1.0, 0.0))
    assert [(b.node_ids, b.dofs) for b in bcs] == [([1, 2, 3], [1, 2])]


def test_dload_unsupported_types_and_targets_warn():
    # parser.rs:1900-1919
    m, w, _ = parse_inp(plate_deck("", (
        "*STEP\n*STATIC\n*DLOAD\nNOSUCHSET, P1, 1.0\nALL, P5, 2.0\nALL, TRVEC, 3.0\n"
        "3, P4, 4.0\nALL, P3, 5.0\n*BOUNDARY\nBASE, 1, 2\n*END STEP\n")))
    assert w == [
        "line 26: *DLOAD target 'NOSUCHSET' is not a known element or ELSET — line ignored",
        "line 27: *DLOAD type 'P5' unsupported (v0.3: P1|P2|P3|P4, GRAV) — line ignored",
        "line 28: *DLOAD type 'TRVEC' unsupported (v0.3: P1|P2|P3|P4, GRAV) — line ignored",
    ]
    assert len(m.load_state()[2]) == 5


def test_density_after_elastic_and_overwrite_warning():
    # parser.rs:1921-1931
    m, w, _ = parse_inp(plate_deck("*DENSITY\n2500.,\n", (
        "*STEP\n*STATIC\n*BOUNDARY\nBASE, 1, 2\n*CLOAD\n9, 2, -1.0\n*END STEP\n")))
    assert w == [] and m.density == 2500.0
    assert [(x.name, x.youngs_modulus) for x in m.materials] == [("STEEL", 210.0e9)]


def test_density_and_dload_warnings_errors_and_op_new():
    """parser.rs:332-365 and :846-950: the density default, its overwrite,
    extra-field, extra-row and outside-material warnings; GRAV and Pn field
    counts; a face beyond the element's edges and an unknown element warn;
    *DLOAD, OP=NEW clears the pressures and gravity the step inherited."""
    m, w, _ = parse_inp(plate_deck("", "*STEP\n*STATIC\n*BOUNDARY\nBASE, 1, 2\n*END STEP\n"))
    assert w == [] and m.density == 7850.0
    deck = ("*NODE\n1, 0, 0\n2, 1, 0\n3, 0, 1\n*DENSITY\n1.0\n"
            "*ELEMENT, TYPE=CPS3, ELSET=T\n7, 1, 2, 3\n*MATERIAL, NAME=M\n*ELASTIC\n1e9, 0.3\n"
            "*DENSITY\n2000., 20.\n3000.\n*DENSITY\n2500.\n"
            "*SOLID SECTION, ELSET=T, MATERIAL=M\n*STEP\n*STATIC\n"
            "*DLOAD\nT, P4, 5.0\n8, P1, 1.0\nT, P2, 6.0\nGRAV, 9.8, 1.0\n*BOUNDARY\n1, 1, 2\n"
            "*END STEP\n*STEP\n*STATIC\n*DLOAD\nT, P1, 2.0\n*END STEP\n"
            "*STEP\n*STATIC\n*DLOAD, OP=NEW\nT, P3, 3.0\n*END STEP\n")
    m, w, steps = parse_inp(deck)
    assert w == [
        "line 6: *DENSITY outside *MATERIAL — ignored",
        "line 13: extra *DENSITY fields ignored (temperature dependence is v0.2)",
        "line 14: extra *DENSITY row ignored (temperature dependence is v0.2)",
        "line 16: *DENSITY overwrites an earlier value (per-material density is v0.4)",
        "line 21: element 7 (cps3) has no face 4 — ignored",
        "line 22: *DLOAD on unknown element 8 — ignored",
    ]
    assert m.density == 2500.0 and steps == 3
    _b, _c, dloads, gravity = m.load_state()
    assert [(d.element_id, d.face, d.magnitude) for d in dloads] == [(7, 3, 3.0)]
    assert gravity is None
    for bad, text in (("GRAV, 9.8\n", "*DLOAD GRAV expects GRAV, magnitude, dir1[, dir2][, "
                                      "dir3]; got 2 field(s)"),
                      ("GRAV, 9.8, 1, 2, 3, 4\n", "got 6 field(s)"),
                      ("T, P1\n", "*DLOAD expects element/elset, P1..P4, magnitude; got 2 "
                                  "field(s)"),
                      ("T, P1, x\n", "malformed pressure magnitude 'x'")):
        with pytest.raises(ParseError) as ei:
            parse_inp(plate_deck("", "*STEP\n*STATIC\n*DLOAD\n" + bad))
        assert text in str(ei.value)


def two_step_deck(op_new):
    op = ", OP=NEW" if op_new else ""
    return plate_deck("", "*STEP\n*STATIC\n*BOUNDARY\nBASE, 1, 2\n*CLOAD\n8, 2, -100.0\n"
                          "*END STEP\n*STEP\n*STATIC\n*CLOAD" + op + "\n8, 2, -250.0\n*END STEP\n")


def test_two_step_mod_accumulates():
    # parser.rs:1977-2012: the last step carries the accumulated state
    m, w, steps = parse_inp(two_step_deck(False))
    assert w == [] and steps == 2
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == [(8, 2, -100.0), (8, 2, -250.0)]
    assert [(b.node_ids, b.dofs) for b in m.boundary_conditions] == [([1, 2, 3], [1, 2])]
    single, _, _ = parse_inp(plate_deck("", "*STEP\n*STATIC\n*BOUNDARY\nBASE, 1, 2\n*CLOAD\n"
                                            "8, 2, -350.0\n*END STEP\n"))
    (a, _), (b, _) = oracle.solve(m), oracle.solve(single)
    assert abs(a.displacements - b.displacements).max() < 1e-9


def test_two_step_op_new_replaces_previous_loads():
    # parser.rs:2014-2036
    m, w, steps = parse_inp(two_step_deck(True))
    assert w == [] and steps == 2
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == [(8, 2, -250.0)]


def test_step_op_new_clears_bcs_and_loads_static_params_warn():
    # parser.rs:2038-2058
    m, w, steps = parse_inp(plate_deck("", (
        "*STEP\n*STATIC, INITIAL\n*BOUNDARY\nBASE, 1, 2\n*CLOAD\n8, 2, -1.0\n*END STEP\n"
        "*STEP, OP=NEW\n*STATIC\n*BOUNDARY\nBASE, 1, 2\n*CLOAD\n9, 2, -5.0\n*END STEP\n")))
    assert len(w) == 1 and "*STATIC parameters ignored" in w[0] and steps == 2
    assert len(m.boundary_conditions) == 1
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == [(9, 2, -5.0)]


def test_warnings_of_the_keyword_loop():
    deck = ("1, 2, 3\n*NODE\n1,0,0\n*OUTPUT, FIELD\n*NODE OUTPUT\nU\n*MATERIAL, NAME=A\n"
            "*SOLID SECTION\n*ELASTIC\n1.0, 0.3\n*MATERIAL\n*BOUNDARY, OP=NEW\n1, 1\n"
            "*STEP, OP=KEEP\n*END STEP\n*CLOAD\n1, 1, 2.0\n*MATERIAL, NAME=B\n")
    _, w, steps = parse_inp(deck)
    assert w == [
        "line 1: data line outside any keyword block ignored",
        "line 4: unsupported keyword '*OUTPUT' — block skipped",
        "line 5: unsupported keyword '*NODE OUTPUT' — block skipped",
        "line 8: material 'A' has no *ELASTIC block",
        "line 8: *SOLID SECTION needs ELSET and MATERIAL — block skipped",
        "line 10: *ELASTIC outside *MATERIAL — block ignored",
        "line 11: *MATERIAL without NAME — block ignored",
        "line 12: OP=NEW outside *STEP ignored",
        "line 14: unsupported OP='keep' on *STEP — treated as MOD",
        "line 16: *CLOAD between steps — ignored",
        "material 'B' has no *ELASTIC block",
    ]
    assert steps == 1


def deck_from_model(m: dict) -> str:
    """A deck in the examples' keyword style, written from a golden model."""
    out = ["*HEADING\n golden model\n*NODE\n"]
    out += [f"{i}, {c[0]!r}, {c[1]!r}, {c[2]!r}\n" for i, c in m["nodes"]]
    names = {int(ElemKind.Cps4): "CPS4", int(ElemKind.Cps3): "CPS3", int(ElemKind.C3d8): "C3D8"}
    for k in sorted({e[1] for e in m["elements"]}):
        out.append(f"*ELEMENT, TYPE={names[k]}\n")
        out += [", ".join(str(x) for x in [i] + conn) + "\n" for i, kk, conn in m["elements"]
                if kk == k]
    for s in m["elsets"]:
        out.append(f"*ELSET, ELSET={s['name']}\n")
        ids = s["element_ids"]
        out += [", ".join(str(x) for x in ids[q:q + 16]) + "\n" for q in range(0, len(ids), 16)]
    for mat in m["materials"]:
        out.append(f"*MATERIAL, NAME={mat['name']}\n*ELASTIC\n{mat['E']!r}, {mat['nu']!r}\n")
    for e, mat in m["mat_assignments"]:
        out.append(f"*SOLID SECTION, ELSET={e}, MATERIAL={mat}\n{m['thickness']!r}\n")
    for b, bc in enumerate(m["boundary_conditions"]):
        out.append(f"*NSET, NSET=BC{b}\n" + ", ".join(str(x) for x in bc["node_ids"]) + "\n")
    out.append("*STEP\n*STATIC\n*BOUNDARY\n")
    for b, bc in enumerate(m["boundary_conditions"]):
        d = bc["dofs"]
        assert d == list(range(d[0], d[-1] + 1))
        out.append(f"BC{b}, {d[0]}, {d[-1]}\n")
    out.append("*CLOAD\n")
    out += [f"{c['node_id']}, {c['dof']}, {c['value']!r}\n" for c in m["cloads"]]
    out.append("*END STEP\n")
    return "".join(out)


@pytest.mark.parametrize("name", ["cantilever", "cantilever3d", "plate_hole"])
def test_golden_models_round_trip_and_reproduce_the_published_solve(name):
    with open(os.path.join(GOLDEN_DIR, f"{name}.json")) as fh:
        g = json.load(fh)
    m, w, steps = parse_inp(deck_from_model(g["model"]))
    assert w == [] and steps == 1
    gm = g["model"]
    assert [int(i) for i in m.mesh.node_ids] == [i for i, _ in gm["nodes"]]
    assert m.mesh.coords.tolist() == [c for _, c in gm["nodes"]]
    assert [s.element_ids for s in m.elsets] == [s["element_ids"] for s in gm["elsets"]]
    assert [(c.node_id, c.dof, c.value) for c in m.cloads] == \
        [(c["node_id"], c["dof"], c["value"]) for c in gm["cloads"]]
    sol, _ = oracle.solve(m)
    assert sol.iterations == g["golden"]["iterations"]
    assert fmt_e3(sol.final_residual) == g["golden"]["residual"]

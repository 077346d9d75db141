"""Host side of the served form (no GPU): the JSON-lines front end, the
admission estimate and the instance sharding of the batched and served
forms.

The front end's framing follows the reference's MCP loop
(crates/solvix-cli/src/mcp.rs:549-592): a bad line is answered and the loop
keeps serving (mcp.rs:1228 tests the same), EOF ends it with exit code 0.
"""
import ctypes as C
import io
import json

import numpy as np
import pytest

from solvix_b200 import abi, workloads
from solvix_b200.serve import fmt_e, flat_from_json, serve_json, solve_error_message
from solvix_b200.sharding import estimated_work, shard_instances


class FakeServer:
    """Duck-typed stand-in for serve.Server: answers every submit with a
    canned result (tag 3 fails as InvalidModel)."""

    def __init__(self):
        self.queue = []

    def submit(self, flat, tag):
        if flat.n_elem == 0:
            return abi.SVX_EMPTY_MESH, "empty mesh"
        n = flat.n_dof
        u = np.zeros(n)
        u[-1] = 1e-3 * tag
        ok = tag != 3
        self.queue.append({
            "tag": tag, "status": abi.SVX_OK if ok else abi.SVX_INVALID_MODEL,
            "ndof": flat.ndof, "iterations": 10 * tag, "residual": 5e-11,
            "cond_estimate": 12345.0, "t_submit_ms": 1.0, "t_start_ms": 2.0,
            "t_done_ms": 4.5, "batch_size": 2, "u": u,
            "von_mises": np.full(flat.n_elem, 2e6),
            "message": "" if ok else "element 2: non-positive Jacobian determinant at a "
                                     "Gauss point"})
        return abi.SVX_OK, ""

    def poll(self, wait_ms):
        return self.queue.pop(0) if self.queue else None


def request_line(ident, flat):
    loads = [[int(r), float(flat.f[r])] for r in np.flatnonzero(flat.f)]
    conn = [flat.conn[flat.conn_ptr[e]:flat.conn_ptr[e + 1]].tolist()
            for e in range(flat.n_elem)]
    return json.dumps({"id": ident, "model": {
        "ndof": flat.ndof, "xyz": flat.xyz.tolist(), "kind": flat.kind.tolist(),
        "conn": conn, "youngs": flat.youngs.tolist(), "poisson": float(flat.poisson[0]),
        "thickness": flat.thickness, "fixed_rows": flat.fixed_row.tolist(), "loads": loads}})


def test_json_request_round_trips_a_flat_model():
    flat = workloads.plate(np.random.Generator(np.random.PCG64(3)), nx=6, ny=3)
    back = flat_from_json(json.loads(request_line("a", flat))["model"])
    for name in ("xyz", "kind", "conn_ptr", "conn", "youngs", "poisson", "fixed_row", "f"):
        np.testing.assert_array_equal(getattr(back, name), getattr(flat, name))
    assert back.thickness == flat.thickness and back.ndof == flat.ndof


def test_serve_json_framing_keeps_serving_after_bad_lines():
    rng = np.random.Generator(np.random.PCG64(4))
    flats = [workloads.plate(rng, nx=5, ny=2) for _ in range(3)]
    lines = [request_line("first", flats[0]), "{not json", "",
             json.dumps({"id": "no-model"}), request_line("second", flats[1]),
             request_line("third", flats[2])]
    out = io.StringIO()
    code = serve_json(io.StringIO("\n".join(lines) + "\n"), out, FakeServer())
    assert code == 0
    replies = [json.loads(x) for x in out.getvalue().splitlines()]
    assert len(replies) == 5
    parse_errors = [r for r in replies if r.get("stage") == "parse"]
    assert len(parse_errors) == 2 and all(r["ok"] is False for r in parse_errors)
    by_id = {r["id"]: r for r in replies if r["id"] is not None}
    assert by_id["first"]["ok"] and by_id["first"]["iterations"] == 10
    assert by_id["first"]["max_disp_mm"] == 1.0
    assert by_id["first"]["max_von_mises_mpa"] == 2.0
    assert by_id["first"]["latency_ms"] == 3.5 and by_id["first"]["solve_ms"] == 2.5
    assert by_id["third"] == {"id": "third", "ok": False, "stage": "solve",
                              "error": "invalid model: element 2: non-positive Jacobian "
                                       "determinant at a Gauss point"}


def test_solve_error_texts_follow_the_reference():
    # crates/solvix-cli/src/main.rs:1150-1163
    assert solve_error_message(abi.SVX_EMPTY_MESH, "") == "empty mesh"
    assert solve_error_message(abi.SVX_NO_CONSTRAINTS, "") == "no constraints"
    assert solve_error_message(abi.SVX_NOT_CONVERGED, "", 1000, 3.25e-7) == \
        "not converged after 1000 iterations (residual 3.250e-7)"
    assert fmt_e(6.933e-11) == "6.933e-11" and fmt_e(12345.0) == "1.234e4"


def test_admission_estimate_grows_with_the_model():
    lib = abi.load()
    small = workloads.cantilever_c3d8(4, 2, 2, lx=0.4, ly=0.1, lz=0.1, seed=1)
    big = workloads.cantilever_c3d8(16, 4, 4, lx=0.4, ly=0.1, lz=0.1, seed=1)
    s_small, s_big = small.as_struct(), big.as_struct()
    b_small = lib.svx_serve_estimate_bytes(C.byref(s_small))
    b_big = lib.svx_serve_estimate_bytes(C.byref(s_big))
    # at least K in FP64 plus its FP32 copy (24^2 slots per hex element)
    assert b_small >= small.n_elem * 576 * 12
    assert b_big > 8 * b_small
    assert lib.svx_serve_estimate_bytes(None) == -1


def test_server_without_a_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from solvix_b200.model import DeviceError
    from solvix_b200.serve import Server
    with pytest.raises(DeviceError):
        Server(lanes=2)


def test_sharding_is_a_balanced_partition():
    n_dof = [f.n_dof for f in workloads.plate_batch(256, seed=4)]
    for world in (1, 2, 3, 8):
        shards = shard_instances(n_dof, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(n_dof)))
        loads = [sum(estimated_work(n_dof[i]) for i in s) for s in shards]
        assert max(loads) <= 1.05 * (sum(loads) / world) + max(estimated_work(n) for n in n_dof)
        assert shards == shard_instances(n_dof, world)  # deterministic


def small_deck(cload_node=10, bcs=True, bad_line=None):
    """A 4x1 CPS4 strip of my own: nodes 1-10 row-major, clamped at x = 0."""
    lines = ["*HEADING", " strip"]
    lines.append("*NODE")
    for j in range(2):
        for i in range(5):
            lines.append(f"{j * 5 + i + 1}, {0.25 * i}, {0.1 * j}")
    if bad_line is not None:
        lines[bad_line - 1] = "3, x.y, 0.0"
    lines.append("*ELEMENT, TYPE=CPS4, ELSET=ALL")
    for i in range(4):
        lines.append(f"{i + 1}, {i + 1}, {i + 2}, {i + 7}, {i + 6}")
    lines += ["*MATERIAL, NAME=STEEL", "*ELASTIC", "210e9, 0.3",
              "*SOLID SECTION, ELSET=ALL, MATERIAL=STEEL", "0.01", "*STEP", "*STATIC"]
    if bcs:
        lines += ["*BOUNDARY", "1, 1, 2", "6, 1, 2"]
    lines += ["*CLOAD", f"{cload_node}, 2, -100.0", "*END STEP"]
    return "\n".join(lines) + "\n"


def run_lines(lines):
    out = io.StringIO()
    assert serve_json(io.StringIO("\n".join(lines) + "\n"), out, FakeServer()) == 0
    return [json.loads(l) for l in out.getvalue().splitlines()]


def test_deck_requests_are_read_resolved_and_solved():
    from oracle import oracle
    from solvix_b200.inp import parse_inp
    from solvix_b200.serve import flat_from_deck
    flat, late = flat_from_deck(small_deck())
    assert late is None and flat.ndof == 2 and flat.n_elem == 4
    want, _ = oracle.resolve(parse_inp(small_deck())[0])
    for name in ("xyz", "kind", "conn_ptr", "conn", "youngs", "poisson", "fixed_row", "f"):
        assert np.array_equal(getattr(flat, name), getattr(want, name)), name
    out = run_lines([json.dumps({"id": "a", "deck": small_deck()})])
    assert out == [dict(out[0], id="a", ok=True)] and out[0]["iterations"] == 10


def test_deck_errors_follow_the_reference_stages_and_order():
    out = run_lines([json.dumps({"id": 1, "deck": small_deck(bad_line=5)}),
                     json.dumps({"id": 2, "deck": small_deck(bcs=False)}),
                     json.dumps({"id": "x", "deck": small_deck(cload_node=99)})])
    by_id = {o["id"]: o for o in out}
    assert by_id[1] == {"id": 1, "ok": False, "stage": "parse",
                        "error": "line 5: malformed coordinate 'x.y'"}
    assert by_id[2] == {"id": 2, "ok": False, "stage": "solve", "error": "no constraints"}
    # the CLOAD error is raised after the element loop: reported once the
    # solve found no failing element
    assert by_id["x"] == {"id": "x", "ok": False, "stage": "solve",
                          "error": "invalid model: load on unknown node 99"}
    # ... and an element failure wins over it (the fake server fails the
    # third submitted request, tag 3)
    out = run_lines([json.dumps({"id": "g1", "deck": small_deck()}),
                     json.dumps({"id": "g2", "deck": small_deck()}),
                     json.dumps({"id": "y", "deck": small_deck(cload_node=99)})])
    by_id = {o["id"]: o for o in out}
    assert by_id["g1"]["ok"] and by_id["g2"]["ok"]
    assert by_id["y"]["ok"] is False and by_id["y"]["stage"] == "solve"
    assert by_id["y"]["error"].startswith("invalid model: element 2")

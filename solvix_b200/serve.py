"""Served solves: continuous batching behind ``solvix serve --json``.

``Server`` wraps the library's request loop (``svx_serve_*``): ``submit``
queues a copy of a flat model and returns at once; the library's lanes
solve whatever is waiting in batches on their own CUDA streams while more
requests arrive, and ``poll`` hands back results in completion order.

``python -m solvix_b200.serve --json`` is the line-oriented front end.  Its
framing follows the reference's only request loop, the MCP server
(crates/solvix-cli/src/mcp.rs:549-592): one JSON object per input line,
one JSON object per output line, a malformed line answered with an error
object and the loop kept alive, EOF ends the loop (after the admitted work
has finished) with exit code 0.  A request line is

    {"id": <any>, "model": {"ndof": 2|3, "xyz": [[x, y, z], ...],
     "kind": [k, ...], "conn": [[n0, n1, ...], ...], "youngs": [...] | E,
     "poisson": [...] | nu, "thickness": t, "fixed_rows": [...],
     "loads": [[row, value], ...]}}

(0-based node indices, element kinds in the reference's ElemKind order,
rows = node * ndof + dof), or a deck as it arrives:

    {"id": <any>, "deck": "<.inp text>"}

read by the linear-static .inp reader (svx_inp_parse) and resolved on the
host (svx_resolve): a parse error answers {"ok": false, "stage": "parse",
"error": "line 7: ..."} as the reference's CLI does (main.rs:1150-1163),
and a CLOAD / BC error the reference raises after the element loop is
reported only when the solve finds no failing element.  A result line carries the fields of the
reference's success envelope (crates/solvix-cli/src/main.rs:889-938:
iterations, solver_method, cond_estimate, residual, solve_ms, max_disp_mm,
max_von_mises_mpa) plus latency_ms and batch_size; a failed request gets
the reference's error envelope {"ok": false, "stage", "error"} (main.rs:
334-340) with the request's id.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import threading

import numpy as np

from . import abi
from .marshal import FlatModel
from .model import DeviceError


class Server:
    """A served-solve loop on one device (svx_serve_create)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 40 << 30, lanes: int = 2,
                 max_batch: int = 4096, tol: float = 1e-10, precision: int = abi.SVX_FP64,
                 max_iter: int = 0, want_stress: bool = True, max_batch_bytes: int = 0):
        self.lib = abi.load()
        opts = abi.SvxServeOpts()
        self.lib.svx_serve_default_opts(C.byref(opts))
        opts.hbm_budget_bytes = int(hbm_budget_bytes)
        opts.lanes = int(lanes)
        opts.max_batch = int(max_batch)
        opts.max_batch_bytes = int(max_batch_bytes)
        opts.solve = abi.default_opts(tol=tol, precision=precision, max_iter=max_iter,
                                      want_stress=int(want_stress))
        self.opts = opts
        h = C.c_void_p()
        err = abi.SvxError()
        st = self.lib.svx_serve_create(int(device), C.byref(opts), C.byref(h), C.byref(err))
        if st != abi.SVX_OK:
            raise DeviceError(err.message.decode() or f"svx_serve_create failed ({st})")
        self.handle = h

    def submit(self, flat: FlatModel, tag: int):
        """Queue a model; returns (status, message).  A refusal (status != 0)
        means no result will come back for this tag."""
        s = flat.as_struct()
        err = abi.SvxError()
        st = self.lib.svx_serve_submit(self.handle, C.byref(s), C.c_uint64(tag), C.byref(err))
        return int(st), err.message.decode() if st != abi.SVX_OK else ""

    def estimate_bytes(self, flat: FlatModel) -> int:
        s = flat.as_struct()
        return int(self.lib.svx_serve_estimate_bytes(C.byref(s)))

    def poll(self, wait_ms: int = -1):
        """Next completed result as a dict, or None when none arrived."""
        out = C.POINTER(abi.SvxServeResult)()
        st = self.lib.svx_serve_poll(self.handle, int(wait_ms), C.byref(out))
        if st == abi.SVX_QUEUE_EMPTY:
            return None
        if st != abi.SVX_OK:
            raise DeviceError(f"svx_serve_poll failed ({st})")
        r = out.contents
        try:
            n = int(r.n_nodes) * int(r.ndof)
            res = {
                "tag": int(r.tag), "status": int(r.status), "ndof": int(r.ndof),
                "n_nodes": int(r.n_nodes), "n_elem": int(r.n_elem),
                "iterations": int(r.iterations), "residual": float(r.residual),
                "cond_estimate": float(r.cond_estimate),
                "t_submit_ms": float(r.t_submit_ms), "t_start_ms": float(r.t_start_ms),
                "t_done_ms": float(r.t_done_ms), "batch_size": int(r.batch_size),
                "lane": int(r.lane),
                "u": np.ctypeslib.as_array(r.u, shape=(n,)).copy() if n else np.zeros(0),
                "von_mises": (np.ctypeslib.as_array(r.von_mises, shape=(int(r.n_elem),)).copy()
                              if r.von_mises and r.n_elem else None),
                "message": r.error.message.decode() if r.status != abi.SVX_OK else "",
                "reason": int(r.error.reason), "elem_index": int(r.error.elem_index),
                "nnz": int(r.nnz),
            }
        finally:
            self.lib.svx_serve_result_free(out)
        return res

    def stats(self) -> dict:
        st = abi.SvxServeStats()
        self.lib.svx_serve_stats(self.handle, C.byref(st))
        return {name: getattr(st, name) for name, _ in abi.SvxServeStats._fields_}

    def now_ms(self) -> float:
        return float(self.lib.svx_serve_now_ms(self.handle))

    def close(self):
        """Finish every submitted request, then free the server."""
        if getattr(self, "handle", None):
            self.lib.svx_serve_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ JSON front end
def flat_from_json(m: dict) -> FlatModel:
    ndof = int(m["ndof"])
    xyz = np.asarray(m["xyz"], dtype=np.float64).reshape(-1, 3)
    conn_lists = [list(map(int, c)) for c in m["conn"]]
    kind = np.asarray(m["kind"], dtype=np.uint8)
    if kind.shape[0] != len(conn_lists):
        raise ValueError("kind and conn differ in length")
    conn_ptr = np.zeros(len(conn_lists) + 1, dtype=np.int64)
    conn_ptr[1:] = np.cumsum([len(c) for c in conn_lists])
    conn = np.asarray([i for c in conn_lists for i in c], dtype=np.int32)
    f = np.zeros(xyz.shape[0] * ndof)
    for row, val in m.get("loads", []):
        f[int(row)] += float(val)
    n_elem = kind.shape[0]
    return FlatModel(xyz=xyz, kind=kind, conn_ptr=conn_ptr, conn=conn,
                     youngs=np.broadcast_to(np.asarray(m["youngs"], dtype=np.float64), (n_elem,)),
                     poisson=np.broadcast_to(np.asarray(m["poisson"], dtype=np.float64),
                                             (n_elem,)),
                     thickness=float(m.get("thickness", 1.0)), ndof=ndof,
                     fixed_row=np.asarray(m.get("fixed_rows", []), dtype=np.int64), f=f)


def fmt_e(x: float) -> str:
    """3-significant-digit scientific notation as Rust's ``{:.3e}`` writes it
    (no exponent sign for positive exponents, no zero padding)."""
    m, e = f"{x:.3e}".split("e")
    return f"{m}e{int(e)}"


def solve_error_message(code: int, message: str, iterations: int = 0,
                        residual: float = 0.0) -> str:
    """The reference's text for a SolveError (crates/solvix-cli/src/main.rs:1150-1163)."""
    if code == abi.SVX_EMPTY_MESH:
        return "empty mesh"
    if code == abi.SVX_NO_CONSTRAINTS:
        return "no constraints"
    if code == abi.SVX_INVALID_MODEL:
        return f"invalid model: {message}"
    if code == abi.SVX_NOT_CONVERGED:
        return f"not converged after {iterations} iterations (residual {fmt_e(residual)})"
    return message


def error_json(ident, stage: str, message: str) -> dict:
    """The reference's error envelope (main.rs:334-340) with the request id;
    stage "parse" for an unreadable request, "solve" for a SolveError (the
    stages behind exit codes 2 and 3, main.rs:91-116)."""
    return {"id": ident, "ok": False, "stage": stage, "error": message}


class DeckError(Exception):
    """A deck request that fails before it reaches the device."""

    def __init__(self, stage: str, message: str):
        super().__init__(message)
        self.stage = stage


def flat_from_deck(text: str):
    """.inp text -> (FlatModel, pending error message or None), through
    svx_inp_parse and svx_resolve; raises DeckError("parse" | "solve")."""
    lib = abi.load()
    raw = text.encode()
    h = C.c_void_p()
    err = abi.SvxError()
    st = lib.svx_inp_parse(raw, len(raw), C.byref(h), C.byref(err))
    if st == abi.SVX_PARSE_ERROR:
        raise DeckError("parse", f"line {int(err.elem_index)}: {err.message.decode()}")
    if st != abi.SVX_OK:
        raise DeckError("parse", err.message.decode() or f"deck rejected ({st})")
    res = C.c_void_p()
    try:
        st = lib.svx_resolve(lib.svx_inp_model(h), C.byref(res), C.byref(err))
        if st != abi.SVX_OK:
            raise DeckError("solve", solve_error_message(st, err.message.decode()))
        try:
            d = lib.svx_resolved_flat(res).contents
            nn, ne, nf = int(d.n_nodes), int(d.n_elem), int(d.n_fixed)
            ndof = int(d.ndof)

            def arr(p, n, dt):
                return np.ctypeslib.as_array(p, shape=(n,)).astype(dt) if n else \
                    np.zeros(0, dt)
            conn_ptr = arr(d.conn_ptr, ne + 1, np.int64)
            flat = FlatModel(
                xyz=arr(d.xyz, 3 * nn, np.float64).reshape(nn, 3), kind=arr(d.kind, ne, np.uint8),
                conn_ptr=conn_ptr, conn=arr(d.conn, int(conn_ptr[-1]), np.int32),
                youngs=arr(d.youngs, ne, np.float64), poisson=arr(d.poisson, ne, np.float64),
                thickness=float(d.thickness), ndof=ndof,
                fixed_row=arr(d.fixed_row, nf, np.int64), f=arr(d.f, nn * ndof, np.float64),
                node_id=arr(d.node_id, nn, np.uint32), elem_id=arr(d.elem_id, ne, np.uint32),
                no_material=arr(d.no_material, ne, np.uint8) if d.no_material else None)
            pst = lib.svx_resolved_pending(res, C.byref(err))
            pending = solve_error_message(pst, err.message.decode()) if pst else None
        finally:
            lib.svx_resolved_free(res)
    finally:
        lib.svx_inp_free(h)
    return flat, pending


def result_json(ident, r: dict) -> dict:
    if r["status"] != abi.SVX_OK:
        return error_json(ident, "solve", solve_error_message(
            r["status"], r["message"], r["iterations"], r["residual"]))
    u = r["u"].reshape(-1, r["ndof"])
    vm = r["von_mises"]
    return {
        "id": ident,
        "ok": True,
        "iterations": r["iterations"],
        "solver_method": "pcg-mixed" if SOLVER_PRECISION[0] == abi.SVX_MIXED else "pcg",
        "cond_estimate": float(f"{r['cond_estimate']:.3e}"),
        "residual": float(f"{r['residual']:.3e}"),
        "solve_ms": round(r["t_done_ms"] - r["t_start_ms"], 3),
        "max_disp_mm": round(float(np.linalg.norm(u, axis=1).max()) * 1e3, 3) if u.size else 0.0,
        "max_von_mises_mpa": round(float(vm.max()) / 1e6, 3) if vm is not None else 0.0,
        "latency_ms": round(r["t_done_ms"] - r["t_submit_ms"], 3),
        "batch_size": r["batch_size"],
    }


SOLVER_PRECISION = [abi.SVX_FP64]


def serve_json(inp, out, server: Server) -> int:
    """Read request lines from ``inp`` until EOF, write result lines to
    ``out``; returns the process exit code (0)."""
    lock = threading.Lock()
    ids = {}
    late_errors = {}
    pending = [0]
    eof = threading.Event()

    def emit(obj):
        with lock:
            out.write(json.dumps(obj) + "\n")
            out.flush()

    def drain():
        while True:
            with lock:
                if eof.is_set() and pending[0] == 0:
                    return
            r = server.poll(50)
            if r is None:
                continue
            with lock:
                ident = ids.pop(r["tag"], None)
                late = late_errors.pop(r["tag"], None)
                pending[0] -= 1
            if late is not None and r["status"] == abi.SVX_OK:
                emit(error_json(ident, "solve", late))
            else:
                emit(result_json(ident, r))

    t = threading.Thread(target=drain, daemon=True)
    t.start()
    tag = 0
    for line in inp:
        line = line.strip()
        if not line:
            continue
        late = None
        try:
            req = json.loads(line)
            ident = req.get("id")
            if "deck" in req:
                flat, late = flat_from_deck(req["deck"])
            else:
                flat = flat_from_json(req["model"])
        except DeckError as e:
            emit(error_json(ident, e.stage, str(e)))
            continue
        except Exception as e:  # malformed request: answer and keep serving
            emit(error_json(None, "parse", f"bad request: {e}"))
            continue
        tag += 1
        with lock:
            ids[tag] = ident
            if late is not None:
                late_errors[tag] = late
            pending[0] += 1
        st, msg = server.submit(flat, tag)
        if st != abi.SVX_OK:
            with lock:
                ids.pop(tag, None)
                late_errors.pop(tag, None)
                pending[0] -= 1
            emit(error_json(ident, "solve", solve_error_message(st, msg)))
    eof.set()
    t.join()
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="solvix serve",
                                 description="served linear-static solves (JSON lines)")
    ap.add_argument("--json", action="store_true", required=True,
                    help="JSON-lines requests on stdin, results on stdout")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--hbm-budget-gb", type=float, default=40.0)
    ap.add_argument("--lanes", type=int, default=2)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--tol", type=float, default=1e-10)
    args = ap.parse_args(argv)
    prec = abi.SVX_MIXED if args.precision == "mixed" else abi.SVX_FP64
    SOLVER_PRECISION[0] = prec
    with Server(args.device, int(args.hbm_budget_gb * (1 << 30)), args.lanes,
                tol=args.tol, precision=prec) as srv:
        return serve_json(sys.stdin, sys.stdout, srv)


if __name__ == "__main__":
    sys.exit(main())

// svx_resolve.cpp - a1: resolution of a reference-shaped model (ids,
// element sets, material assignments, BCs and loads by node id) into the
// flat index arrays of the device path, in O(N) with hash maps.
//
// Restates, with the reference's error order and texts:
//   solve_with_thermal's checks   crates/solvix-core/src/lib.rs:596-612
//   Model::validate               lib.rs:406-436 (InvalidModel("{:?}"))
//   ndof_per_node                 lib.rs:725-752
//   Mesh::node_index              lib.rs:106-108 (first node with the id)
//   Model::material_for_element   lib.rs:357-367 (first assignment whose
//                                 first-named elset holds the id decides)
//   CLOAD loop of assemble_with   crates/solvix-core/src/assembly.rs:365-380
//   edge_pressure_forces          assembly.rs:382, :393-452 (*DLOAD Pn)
//   gravity_forces                assembly.rs:383, :458-539 (*DLOAD GRAV)
//   constrained_dofs              crates/solvix-core/src/solver.rs:15-41
// The reference's lookups are linear scans (O(N^2) over a mesh); the
// results here are identical.  CLOAD, DLOAD, gravity and BC errors are
// raised by the reference only after the element loop (in that order), so
// they are kept pending and reported by svx_solve_resolved when no element
// fails first.  The load vector is summed in the reference's order with
// its operation order (CLOADs, then pressures, then gravity per element).

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "svx_internal.h"

struct svx_resolved {
    std::vector<double> xyz;
    std::vector<uint32_t> node_id;
    std::vector<uint8_t> kind;
    std::vector<int64_t> conn_ptr;
    std::vector<int32_t> conn;
    std::vector<double> youngs, poisson;
    std::vector<uint8_t> no_material;
    std::vector<uint32_t> elem_id;
    std::vector<int64_t> fixed_row;
    std::vector<double> f;
    svx_flat_model_t flat{};
    int pending_code = SVX_OK;
    std::string pending_msg;
};

namespace {

int node_count(int kind) {
    static const int nc[8] = {3, 4, 8, 4, 8, 8, 4, 2};
    return (kind >= 0 && kind < 8) ? nc[kind] : -1;
}

struct Fail {
    int code;
    std::string msg;
};

void set_err(svx_error_t* err, int code, const std::string& msg) {
    if (!err) return;
    err->code = code;
    err->reason = 0;
    err->elem_index = -1;
    err->iterations = 0;
    err->residual = 0.0;
    std::snprintf(err->message, sizeof(err->message), "%s", msg.c_str());
}

// ElemKind's Debug names, as the reference's "{:?}" prints them.
const char* kind_debug(int kind) {
    static const char* names[8] = {"Cps3", "Cps4", "Cps8", "Cpe4", "Cpe8", "C3d8", "C3d4", "B31"};
    return (kind >= 0 && kind < 8) ? names[kind] : "?";
}

void pend(svx_resolved* r, const std::string& msg) {
    r->pending_code = SVX_INVALID_MODEL;
    r->pending_msg = msg;
}

// edge_pressure_forces (assembly.rs:393-452): the total pressure *
// thickness * edge length splits half and half over the edge's two end
// nodes, along the inward normal of a counter-clockwise element.
void edge_pressure(const svx_model_desc_t* d,
                   const std::unordered_map<uint32_t, int32_t>& node_index, int ndof,
                   svx_resolved* r) {
    if (d->n_dloads <= 0) return;
    std::unordered_map<uint32_t, int64_t> first_elem;  // the first element with an id
    first_elem.reserve(size_t(d->n_elems) * 2);
    for (int64_t e = 0; e < d->n_elems; ++e) first_elem.emplace(d->elem_ids[e], e);
    for (int64_t k = 0; k < d->n_dloads; ++k) {
        const uint32_t id = d->dload_elem_ids[k];
        const auto it = first_elem.find(id);
        if (it == first_elem.end()) {
            pend(r, "distributed load on unknown element " + std::to_string(id));
            return;
        }
        const int64_t e = it->second;
        const int kind = d->elem_kinds[e];
        int max_face = 0;
        if (kind == SVX_CPS3) max_face = 3;
        else if (kind == SVX_CPS4 || kind == SVX_CPE4) max_face = 4;
        else {
            pend(r, "edge pressure on element " + std::to_string(id) + " (" + kind_debug(kind) +
                        ") unsupported (linear quad/tri edges only)");
            return;
        }
        const int64_t face = d->dload_faces[k];
        if (face <= 0 || face > max_face) {
            pend(r, "element " + std::to_string(id) + " (" + kind_debug(kind) +
                        ") has no face " + std::to_string(face));
            return;
        }
        const int64_t c0 = d->elem_conn_ptr[e];
        const int64_t nn = d->elem_conn_ptr[e + 1] - c0;
        const int32_t ia = node_index.at(d->elem_conn[c0 + face - 1]);
        const int32_t ib = node_index.at(d->elem_conn[c0 + face % nn]);
        const double pax = d->node_coords[3 * int64_t(ia)], pay = d->node_coords[3 * int64_t(ia) + 1];
        const double pbx = d->node_coords[3 * int64_t(ib)], pby = d->node_coords[3 * int64_t(ib) + 1];
        const double dx = pbx - pax, dy = pby - pay;
        const double len = std::sqrt(dx * dx + dy * dy);
        if (len == 0.0) {
            pend(r, "zero-length pressure edge on element " + std::to_string(id));
            return;
        }
        const double nx = -dy / len, ny = dx / len;
        const double fmag = d->dload_values[k] * d->thickness * len / 2.0;
        for (const int32_t i : {ia, ib}) {
            r->f[size_t(int64_t(i) * ndof)] += fmag * nx;
            r->f[size_t(int64_t(i) * ndof + 1)] += fmag * ny;
        }
    }
}

// gravity_forces (assembly.rs:458-539) for the element kinds this path
// assembles: rho * t * area * g lumped in equal thirds (CPS3) or quarters
// (CPS4, CPE4) along the in-plane direction; solid elements are rejected
// with the reference's text.  Kinds the element loop rejects anyway
// (CPS8, CPE8, B31) add nothing here: their element error comes first.
void gravity(const svx_model_desc_t* d, const std::unordered_map<uint32_t, int32_t>& node_index,
             int ndof, svx_resolved* r) {
    if (!d->has_gravity) return;
    const double g = d->gravity_magnitude;
    const double dir0 = d->gravity_dir[0], dir1 = d->gravity_dir[1];
    if (dir0 == 0.0 && dir1 == 0.0) {
        pend(r, "gravity direction has no in-plane component");
        return;
    }
    for (int64_t e = 0; e < d->n_elems; ++e) {
        const int kind = d->elem_kinds[e];
        const int64_t c0 = d->elem_conn_ptr[e];
        int32_t idx[4];
        double px[4], py[4];
        int nn = 0;
        double per = 0.0;
        if (kind == SVX_CPS3 || kind == SVX_CPS4 || kind == SVX_CPE4) {
            nn = kind == SVX_CPS3 ? 3 : 4;
            for (int q = 0; q < nn; ++q) {
                idx[q] = node_index.at(d->elem_conn[c0 + q]);
                px[q] = d->node_coords[3 * int64_t(idx[q])];
                py[q] = d->node_coords[3 * int64_t(idx[q]) + 1];
            }
            if (nn == 3) {
                const double cross =
                    (px[1] - px[0]) * (py[2] - py[0]) - (py[1] - py[0]) * (px[2] - px[0]);
                per = d->density * d->thickness * std::fabs(cross) / 2.0 * g / 3.0;
            } else {
                double shoelace = 0.0;
                for (int q = 0; q < 4; ++q) {
                    const int b = (q + 1) % 4;
                    shoelace += px[q] * py[b] - px[b] * py[q];
                }
                per = d->density * d->thickness * std::fabs(shoelace) / 2.0 * g / 4.0;
            }
        } else if (kind == SVX_C3D8 || kind == SVX_C3D4) {
            pend(r, "gravity on solid elements unsupported (plane and beam only)");
            return;
        } else {
            continue;
        }
        for (int q = 0; q < nn; ++q) {
            r->f[size_t(int64_t(idx[q]) * ndof)] += per * dir0;
            r->f[size_t(int64_t(idx[q]) * ndof + 1)] += per * dir1;
        }
    }
}

svx_resolved* resolve(const svx_model_desc_t* d) {
    if (!d) throw Fail{SVX_BAD_ARGUMENT, "null model"};
    if (d->n_nodes < 0 || d->n_elems < 0 || d->n_materials < 0 || d->n_elsets < 0 ||
        d->n_assignments < 0 || d->n_bcs < 0 || d->n_cloads < 0 || d->n_dloads < 0)
        throw Fail{SVX_BAD_ARGUMENT, "negative size"};
    // lib.rs:597-599: a free body is NoConstraints before anything else
    if (d->n_bcs == 0) throw Fail{SVX_NO_CONSTRAINTS, "no constraints"};
    // validate (lib.rs:406-436)
    if (d->n_nodes == 0 || d->n_elems == 0) throw Fail{SVX_INVALID_MODEL, "EmptyMesh"};
    if (d->n_materials == 0) throw Fail{SVX_INVALID_MODEL, "NoMaterial"};
    std::unordered_map<uint32_t, int32_t> node_index;
    node_index.reserve(size_t(d->n_nodes) * 2);
    for (int64_t i = 0; i < d->n_nodes; ++i) node_index.emplace(d->node_ids[i], int32_t(i));
    for (int64_t e = 0; e < d->n_elems; ++e) {
        int nc = node_count(d->elem_kinds[e]);
        if (nc < 0) throw Fail{SVX_BAD_ARGUMENT, "unknown element kind"};
        int64_t a = d->elem_conn_ptr[e], b = d->elem_conn_ptr[e + 1];
        if (b - a != nc)
            throw Fail{SVX_INVALID_MODEL, "MalformedElement(" + std::to_string(d->elem_ids[e]) + ")"};
        for (int64_t q = a; q < b; ++q)
            if (!node_index.count(d->elem_conn[q]))
                throw Fail{SVX_INVALID_MODEL,
                           "UnknownNode(" + std::to_string(d->elem_conn[q]) + ")"};
    }
    if (d->thickness <= 0.0 || std::isnan(d->thickness))
        throw Fail{SVX_INVALID_MODEL, "thickness must be positive"};
    // ndof_per_node
    bool plane = false, solid = false, beam = false;
    for (int64_t e = 0; e < d->n_elems; ++e) {
        int k = d->elem_kinds[e];
        if (k == SVX_C3D8 || k == SVX_C3D4) solid = true;
        else if (k == SVX_B31) beam = true;
        else plane = true;
    }
    if (beam && (plane || solid))
        throw Fail{SVX_INVALID_MODEL, "mixed beam and continuum elements (v1: B31-only models)"};
    if (plane && solid) throw Fail{SVX_INVALID_MODEL, "mixed dimensionality"};
    const int ndof = (beam || solid) ? 3 : 2;

    std::unique_ptr<svx_resolved> r(new svx_resolved());
    r->xyz.assign(d->node_coords, d->node_coords + 3 * d->n_nodes);
    r->node_id.assign(d->node_ids, d->node_ids + d->n_nodes);
    r->kind.assign(d->elem_kinds, d->elem_kinds + d->n_elems);
    r->conn_ptr.assign(d->elem_conn_ptr, d->elem_conn_ptr + d->n_elems + 1);
    const int64_t n_conn = d->elem_conn_ptr[d->n_elems];
    r->conn.resize(size_t(n_conn));
    for (int64_t q = 0; q < n_conn; ++q) r->conn[q] = node_index.at(d->elem_conn[q]);
    r->elem_id.assign(d->elem_ids, d->elem_ids + d->n_elems);

    // material_for_element: first deciding assignment per element id
    std::unordered_map<std::string, int32_t> set_first, mat_first;
    for (int32_t s = 0; s < d->n_elsets; ++s) set_first.emplace(d->elset_names[s], s);
    for (int32_t m = 0; m < d->n_materials; ++m) mat_first.emplace(d->material_names[m], m);
    std::unordered_map<uint32_t, int32_t> decided;  // elem id -> material (-1: none)
    decided.reserve(size_t(d->n_elems) * 2);
    for (int32_t a = 0; a < d->n_assignments; ++a) {
        auto sit = set_first.find(d->assign_elset[a]);
        if (sit == set_first.end()) continue;
        auto mit = mat_first.find(d->assign_material[a]);
        int32_t mat = (mit == mat_first.end()) ? -1 : mit->second;
        int32_t s = sit->second;
        for (int64_t q = d->elset_ptr[s]; q < d->elset_ptr[s + 1]; ++q)
            decided.emplace(d->elset_elem_ids[q], mat);
    }
    r->youngs.assign(size_t(d->n_elems), 0.0);
    r->poisson.assign(size_t(d->n_elems), 0.0);
    r->no_material.assign(size_t(d->n_elems), 0);
    for (int64_t e = 0; e < d->n_elems; ++e) {
        auto it = decided.find(d->elem_ids[e]);
        if (it == decided.end() || it->second < 0) {
            r->no_material[e] = 1;
        } else {
            r->youngs[e] = d->youngs_modulus[it->second];
            r->poisson[e] = d->poisson_ratio[it->second];
        }
    }

    // loads (assembly.rs:365-380)
    const int64_t n = d->n_nodes * ndof;
    r->f.assign(size_t(n), 0.0);
    for (int64_t c = 0; c < d->n_cloads; ++c) {
        int64_t dof = d->cload_dofs[c];
        uint32_t nid = d->cload_node_ids[c];
        if (dof <= 0 || dof > ndof) {
            r->pending_code = SVX_INVALID_MODEL;
            r->pending_msg = "load on node " + std::to_string(nid) + " has unsupported dof " +
                             std::to_string(dof);
            break;
        }
        auto it = node_index.find(nid);
        if (it == node_index.end()) {
            r->pending_code = SVX_INVALID_MODEL;
            r->pending_msg = "load on unknown node " + std::to_string(nid);
            break;
        }
        r->f[size_t(int64_t(it->second) * ndof + dof - 1)] += d->cload_values[c];
    }
    if (r->pending_code == SVX_OK) edge_pressure(d, node_index, ndof, r.get());
    if (r->pending_code == SVX_OK) gravity(d, node_index, ndof, r.get());
    // constrained_dofs (solver.rs:15-41)
    if (r->pending_code == SVX_OK) {
        for (int32_t b = 0; b < d->n_bcs && r->pending_code == SVX_OK; ++b) {
            for (int64_t q = d->bc_node_ptr[b]; q < d->bc_node_ptr[b + 1]; ++q) {
                uint32_t nid = d->bc_node_ids[q];
                auto it = node_index.find(nid);
                if (it == node_index.end()) {
                    r->pending_code = SVX_INVALID_MODEL;
                    r->pending_msg = "boundary condition on unknown node " + std::to_string(nid);
                    break;
                }
                bool bad = false;
                for (int64_t k = d->bc_dof_ptr[b]; k < d->bc_dof_ptr[b + 1]; ++k) {
                    int64_t dof = d->bc_dofs[k];
                    if (dof <= 0 || dof > ndof) {
                        r->pending_code = SVX_INVALID_MODEL;
                        r->pending_msg = "boundary condition on node " + std::to_string(nid) +
                                         " has unsupported dof " + std::to_string(dof);
                        bad = true;
                        break;
                    }
                    r->fixed_row.push_back(int64_t(it->second) * ndof + dof - 1);
                }
                if (bad) break;
            }
        }
    }
    if (r->pending_code != SVX_OK) r->fixed_row.clear();

    svx_flat_model_t& fl = r->flat;
    fl.n_nodes = d->n_nodes;
    fl.xyz = r->xyz.data();
    fl.node_id = r->node_id.data();
    fl.n_elem = d->n_elems;
    fl.kind = r->kind.data();
    fl.conn_ptr = r->conn_ptr.data();
    fl.conn = r->conn.data();
    fl.youngs = r->youngs.data();
    fl.poisson = r->poisson.data();
    fl.no_material = r->no_material.data();
    fl.elem_id = r->elem_id.data();
    fl.thickness = d->thickness;
    fl.ndof = ndof;
    fl.n_fixed = int64_t(r->fixed_row.size());
    fl.fixed_row = r->fixed_row.data();
    fl.f = r->f.data();
    return r.release();
}

}  // namespace

extern "C" {

int svx_resolve(const svx_model_desc_t* desc, svx_resolved_t** out, svx_error_t* err) {
    if (!out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    try {
        *out = resolve(desc);
        set_err(err, SVX_OK, "");
        return SVX_OK;
    } catch (const Fail& f) {
        set_err(err, f.code, f.msg);
        return f.code;
    } catch (const std::bad_alloc&) {
        set_err(err, SVX_OOM, "host allocation failed");
        return SVX_OOM;
    }
}

int svx_resolved_pending(const svx_resolved_t* res, svx_error_t* err) {
    if (!res) return SVX_BAD_ARGUMENT;
    if (err) {
        std::memset(err, 0, sizeof(*err));
        err->code = res->pending_code;
        err->elem_index = -1;
        std::snprintf(err->message, sizeof(err->message), "%s", res->pending_msg.c_str());
    }
    return res->pending_code;
}

const svx_flat_model_t* svx_resolved_flat(const svx_resolved_t* res) {
    return res ? &res->flat : nullptr;
}

int svx_resolved_free(svx_resolved_t* res) {
    delete res;
    return SVX_OK;
}

int svx_solve_resolved(svx_ctx_t* ctx, const svx_resolved_t* res, const svx_solve_opts_t* opts,
                       svx_solution_t* sol, svx_error_t* err) {
    if (!ctx || !res) return SVX_BAD_ARGUMENT;
    if (res->pending_code == SVX_OK) return svx_solve_flat(ctx, &res->flat, opts, sol, err);
    // a pending CLOAD / BC error loses only to an element error
    svx_op_t* op = nullptr;
    int st = svx_assemble(ctx, &res->flat, 0, &op, err);
    if (op) svx_op_free(op);
    if (st != SVX_OK) return st;
    set_err(err, res->pending_code, res->pending_msg);
    return res->pending_code;
}

}  // extern "C"

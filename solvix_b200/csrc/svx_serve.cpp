// Served solves: the request loop behind `solvix serve --json`.
//
// The reference has no server for the solve path; its CLI solves one deck
// per process (crates/solvix-cli/src/main.rs:1165-1224, do_run) and its only
// line-oriented request loop is the MCP server (crates/solvix-cli/src/
// mcp.rs:549-592, handle_message / serve), which answers one request at a
// time.  This file is the device side of a served form of the same solve:
// requests are queued as they arrive and solved in batches while later ones
// keep arriving (continuous batching).
//
// Design.  `lanes` dispatcher threads each own a context (CUDA streams and
// a device memory pool of their own: a block a lane frees may still be read
// by that lane's queued kernels, so it is reused only on that lane's
// streams).  Each lane's pool reserves budget / lanes as its arena.  A free
// lane takes every waiting request, in arrival order, that has the ndof of
// the oldest one, until max_batch, until its batch would exceed
// max_batch_bytes (default 4/5 of its arena), or until the next one's
// estimated device bytes do not fit what is left of the admission budget;
// it then solves them as one
// block-diagonal batch (run_batch: per-model checks, per-model convergence,
// a failed member isolated from the others) and publishes one result per
// request.  While one lane's batch runs, other lanes start the requests
// that arrived meanwhile on their own streams, so batches overlap on the
// device.  Admission is FIFO: when the oldest request does not fit, later
// ones wait too (no starvation of large requests).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "svx_internal.h"

using namespace svx;

namespace {

// Owning copy of a flat model (the caller's arrays may be freed after
// svx_serve_submit returns).
struct ModelCopy {
    std::vector<double> xyz, youngs, poisson, f;
    std::vector<uint8_t> kind, no_material;
    std::vector<int64_t> conn_ptr, fixed_row;
    std::vector<int32_t> conn;
    std::vector<uint32_t> node_id, elem_id;
    svx_flat_model_t view{};

    explicit ModelCopy(const svx_flat_model_t& m) {
        const size_t nn = size_t(m.n_nodes), ne = size_t(m.n_elem);
        xyz.assign(m.xyz, m.xyz + 3 * nn);
        kind.assign(m.kind, m.kind + ne);
        conn_ptr.assign(m.conn_ptr, m.conn_ptr + ne + 1);
        conn.assign(m.conn, m.conn + conn_ptr[ne]);
        youngs.assign(m.youngs, m.youngs + ne);
        poisson.assign(m.poisson, m.poisson + ne);
        fixed_row.assign(m.fixed_row, m.fixed_row + m.n_fixed);
        if (m.f) f.assign(m.f, m.f + nn * size_t(m.ndof));
        if (m.node_id) node_id.assign(m.node_id, m.node_id + nn);
        if (m.elem_id) elem_id.assign(m.elem_id, m.elem_id + ne);
        if (m.no_material) no_material.assign(m.no_material, m.no_material + ne);
        view = m;
        view.xyz = xyz.data();
        view.kind = kind.data();
        view.conn_ptr = conn_ptr.data();
        view.conn = conn.data();
        view.youngs = youngs.data();
        view.poisson = poisson.data();
        view.fixed_row = fixed_row.data();
        view.f = f.empty() ? nullptr : f.data();
        view.node_id = node_id.empty() ? nullptr : node_id.data();
        view.elem_id = elem_id.empty() ? nullptr : elem_id.data();
        view.no_material = no_material.empty() ? nullptr : no_material.data();
    }
};

struct Request {
    uint64_t tag = 0;
    std::unique_ptr<ModelCopy> model;
    int64_t bytes = 0;
    double t_submit = 0.0;
};

int element_nodes(int kind) {
    switch (kind) {
        case SVX_CPS3: return 3;
        case SVX_CPS4: return 4;
        case SVX_C3D8: return 8;
        default: return 8;
    }
}

}  // namespace

struct svx_server {
    svx_serve_opts_t opts{};
    int device = 0;
    std::vector<svx_ctx*> lane_ctx;
    std::vector<std::thread> lanes;
    std::mutex mu;
    std::condition_variable cv_work;   // new request, memory freed, or stop
    std::condition_variable cv_done;   // a result was published
    std::deque<Request> pending;
    std::deque<svx_serve_result_t*> done;
    bool stopping = false;
    int64_t bytes_admitted = 0, peak_bytes_admitted = 0, peak_device_bytes = 0;
    int64_t submitted = 0, rejected = 0, completed = 0, batches = 0, in_flight = 0;
    double prep_ms = 0.0, assemble_ms = 0.0, solve_ms = 0.0, output_ms = 0.0,
           device_solve_ms = 0.0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
            .count();
    }
    void lane_loop(int lane);
};

namespace {

// Upper bound of the device bytes one model occupies while it is assembled
// and solved inside a batch: its model arrays, the element matrices of K1
// (freed after assembly, counted anyway), the pattern and slot map, K, the
// PCG vectors and the stress outputs.
int64_t estimate_bytes(const svx_flat_model_t& m) {
    const int64_t nd = m.ndof;
    int64_t ke = 0, conn = 0;
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int64_t nn = element_nodes(m.kind[e]);
        ke += nn * nd * nn * nd;
        conn += nn;
    }
    const int64_t n = m.n_nodes * nd;
    // a node's row block spans at most its 9 (2D) or 27 (3D) grid neighbours
    const int64_t nnz = m.n_nodes * nd * nd * (nd == 3 ? 27 : 9);
    int64_t b = 0;
    b += ke * 8;                         // element matrices (freed after assembly)
    b += nnz * (8 + 4 + 4);              // K, its column indices, FP32 copy
    b += n * 8 * 17 + m.n_fixed * 16;    // PCG, mixed-form rollback and output vectors,
                                         // constraints
    b += m.n_nodes * (24 + 40) + m.n_elem * 64 + conn * (4 + 1 + 4 + 2 * 8);
    return b + 64 * 1024;
}

void fill_result_error(svx_serve_result_t& r, int code, int reason, int64_t elem,
                       const std::string& msg) {
    r.status = code;
    r.error.code = code;
    r.error.reason = reason;
    r.error.elem_index = elem;
    std::snprintf(r.error.message, sizeof(r.error.message), "%s", msg.c_str());
}

}  // namespace

void svx_server::lane_loop(int lane) {
    svx_ctx* ctx = lane_ctx[lane];
    DevicePool* pool = ctx->pool;
    // a batch takes at most 4/5 of the lane's arena in estimated bytes: the
    // rest absorbs fragmentation, so that no block falls back to cudaMalloc
    // and the device-synchronising cudaFree of the trim below.  Measured on
    // 6,000 requests of the serving mix (FP64, solves/s): 2 lanes with 4/5
    // arena batches 1,078 (no pool time), whole-arena 969 (0.8 s in the
    // driver's allocator), half-arena 650; 3 lanes whole-arena 939, 4 lanes
    // 725 / 537 (whole / half): large batches on two lanes fill the device
    // best.  With 4/5 batches and the faster batched kernels: 2 lanes 1,116,
    // 3 lanes 1,106, 4 lanes 1,008.
    const int64_t lane_cap =
        opts.max_batch_bytes > 0
            ? opts.max_batch_bytes
            : std::max<int64_t>(1, opts.hbm_budget_bytes / opts.lanes / 5 * 4);
    cudaSetDevice(device);
    for (;;) {
        std::vector<Request> batch;
        int64_t batch_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] {
                if (pending.empty()) return stopping;
                return bytes_admitted + pending.front().bytes <= opts.hbm_budget_bytes ||
                       bytes_admitted == 0;
            });
            if (pending.empty() && stopping) return;
            const int ndof = pending.front().model->view.ndof;
            for (auto it = pending.begin(); it != pending.end() &&
                                            int32_t(batch.size()) < opts.max_batch;) {
                if (it->model->view.ndof != ndof) {
                    ++it;
                    continue;
                }
                // the oldest request always fits here (see the wait above)
                if (bytes_admitted + it->bytes > opts.hbm_budget_bytes && bytes_admitted > 0)
                    break;
                if (!batch.empty() && batch_bytes + it->bytes > lane_cap) break;
                bytes_admitted += it->bytes;
                batch_bytes += it->bytes;
                batch.push_back(std::move(*it));
                it = pending.erase(it);
            }
            peak_bytes_admitted = std::max(peak_bytes_admitted, bytes_admitted);
            in_flight += int64_t(batch.size());
            ++batches;
        }
        if (batch.empty()) continue;
        const double t_start = now_ms();
        const int32_t count = int32_t(batch.size());
        // each result owns its arrays (freed by svx_serve_result_free)
        std::vector<svx_serve_result_t*> boxes(static_cast<size_t>(count));
        std::vector<const svx_flat_model_t*> models(static_cast<size_t>(count));
        std::vector<double*> u(static_cast<size_t>(count)), vm(static_cast<size_t>(count));
        const bool want_vm = opts.solve.want_stress != 0;
        for (int32_t k = 0; k < count; ++k) {
            const svx_flat_model_t& m = batch[k].model->view;
            svx_serve_result_t* r = new svx_serve_result_t();
            u[k] = new double[size_t(std::max<int64_t>(m.n_nodes * m.ndof, 1))]();
            vm[k] = want_vm ? new double[size_t(std::max<int64_t>(m.n_elem, 1))]() : nullptr;
            r->u = u[k];
            r->von_mises = vm[k];
            boxes[k] = r;
            models[k] = &m;
        }
        std::vector<BatchModelOut> out;
        BatchRun run;
        int code = SVX_OK;
        std::string msg;
        try {
            run_batch(ctx, count, models.data(), opts.solve, u.data(),
                      want_vm ? vm.data() : nullptr, out, run);
        } catch (const ModelFail& f) {
            code = f.code;
            msg = f.message;
        } catch (const CudaFail& c) {
            cudaGetLastError();
            code = SVX_CUDA_ERROR;
            msg = std::string("CUDA error: ") + cudaGetErrorString(c.code) + " (" + c.where + ")";
        } catch (const std::bad_alloc&) {
            code = SVX_OOM;
            msg = "host allocation failed";
        }
        const double t_done = now_ms();
        for (int32_t k = 0; k < count; ++k) {
            svx_serve_result_t& r = *boxes[k];
            const svx_flat_model_t& m = *models[k];
            r.tag = batch[k].tag;
            r.ndof = m.ndof;
            r.n_nodes = m.n_nodes;
            r.n_elem = m.n_elem;
            r.t_submit_ms = batch[k].t_submit;
            r.t_start_ms = t_start;
            r.t_done_ms = t_done;
            r.batch_size = count;
            r.lane = lane;
            r.error.elem_index = -1;
            if (code != SVX_OK) {
                fill_result_error(r, code, 0, -1, msg);
                continue;
            }
            const BatchModelOut& o = out[k];
            r.status = o.status;
            r.iterations = o.iterations;
            r.residual = o.residual;
            r.cond_estimate = o.cond;
            r.nnz = o.nnz;
            if (o.status != SVX_OK) {
                fill_result_error(r, o.status, o.reason, o.elem_index, o.message);
                r.error.iterations = o.iterations;
                r.error.residual = o.residual;
            }
        }
        batch.clear();  // the model copies go before the budget is returned
        // blocks beyond the arena (admission estimates are upper bounds, so
        // rarely) go back to the driver once the lane exceeds its share
        if (int64_t(pool->bytes_in_use() + pool->bytes_cached()) >
            opts.hbm_budget_bytes / opts.lanes)
            pool->trim();
        int64_t dev = 0;
        for (svx_ctx* c : lane_ctx)
            dev += int64_t(std::max(c->pool->arena_bytes(),
                                    c->pool->bytes_in_use() + c->pool->bytes_cached()));
        {
            std::lock_guard<std::mutex> lk(mu);
            peak_device_bytes = std::max(peak_device_bytes, dev);
            prep_ms += run.wall_prep;
            assemble_ms += run.wall_assemble;
            solve_ms += run.wall_solve;
            output_ms += run.wall_output;
            device_solve_ms += run.ms_solve;
            bytes_admitted -= batch_bytes;
            in_flight -= count;
            completed += count;
            for (svx_serve_result_t* b : boxes) done.push_back(b);
        }
        cv_work.notify_all();
        cv_done.notify_all();
    }
}

extern "C" {

void svx_serve_default_opts(svx_serve_opts_t* opts) {
    if (!opts) return;
    std::memset(opts, 0, sizeof(*opts));
    opts->hbm_budget_bytes = int64_t(40) << 30;
    opts->lanes = 2;
    opts->max_batch = 4096;
    svx_default_opts(&opts->solve);
}

int64_t svx_serve_estimate_bytes(const svx_flat_model_t* model) {
    if (!model || model->n_elem < 0 || model->n_nodes < 0 || (model->n_elem && !model->kind))
        return -1;
    return estimate_bytes(*model);
}

int svx_serve_create(int device, const svx_serve_opts_t* opts, svx_server_t** out,
                     svx_error_t* err) {
    if (!out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<svx_server> srv(new svx_server());
    svx_serve_default_opts(&srv->opts);
    if (opts) {
        srv->opts = *opts;
        if (srv->opts.hbm_budget_bytes <= 0) srv->opts.hbm_budget_bytes = int64_t(40) << 30;
        if (srv->opts.lanes <= 0) srv->opts.lanes = 2;
        if (srv->opts.max_batch <= 0) srv->opts.max_batch = 4096;
    }
    if (srv->opts.lanes > 64) srv->opts.lanes = 64;
    srv->device = device;
    for (int l = 0; l < srv->opts.lanes; ++l) {
        svx_ctx_t* c = nullptr;
        const int st = svx_ctx_create(device, &c);
        if (st != SVX_OK) {
            if (err) {
                err->code = st;
                err->reason = 0;
                err->elem_index = -1;
                svx_last_error(nullptr, err->message, sizeof(err->message));
            }
            for (svx_ctx* x : srv->lane_ctx) svx_ctx_destroy(x);
            return st;
        }
        srv->lane_ctx.push_back(c);
    }
    // the admission budget is reserved up front as the lanes' arenas:
    // steady-state batches make no cudaMalloc / cudaFree calls
    try {
        cudaSetDevice(device);
        for (svx_ctx* c : srv->lane_ctx)
            c->pool->reserve(size_t(srv->opts.hbm_budget_bytes / srv->opts.lanes));
    } catch (const ModelFail& f) {
        if (err) {
            err->code = f.code;
            err->reason = 0;
            err->elem_index = -1;
            std::snprintf(err->message, sizeof(err->message), "%s", f.message.c_str());
        }
        for (svx_ctx* x : srv->lane_ctx) svx_ctx_destroy(x);
        return f.code;
    }
    svx_server* s = srv.get();
    for (int l = 0; l < s->opts.lanes; ++l) s->lanes.emplace_back([s, l] { s->lane_loop(l); });
    if (err) {
        err->code = SVX_OK;
        err->message[0] = 0;
    }
    *out = srv.release();
    return SVX_OK;
}

int svx_serve_submit(svx_server_t* srv, const svx_flat_model_t* model, uint64_t tag,
                     svx_error_t* err) {
    if (!srv || !model) return SVX_BAD_ARGUMENT;
    auto refuse = [&](int code, int reason, int64_t elem, const std::string& msg) {
        if (err) {
            err->code = code;
            err->reason = reason;
            err->elem_index = elem;
            err->iterations = 0;
            err->residual = 0.0;
            std::snprintf(err->message, sizeof(err->message), "%s", msg.c_str());
        }
        std::lock_guard<std::mutex> lk(srv->mu);
        ++srv->submitted;
        ++srv->rejected;
        return code;
    };
    try {
        check_batch_member(model);
    } catch (const ModelFail& f) {
        return refuse(f.code, f.reason, f.elem_index, f.message);
    }
    Request r;
    r.tag = tag;
    r.bytes = estimate_bytes(*model);
    if (r.bytes > srv->opts.hbm_budget_bytes)
        return refuse(SVX_OOM, 0, -1,
                      "request needs about " + std::to_string(r.bytes) +
                          " device bytes, above the server's budget of " +
                          std::to_string(srv->opts.hbm_budget_bytes));
    try {
        r.model.reset(new ModelCopy(*model));
    } catch (const std::bad_alloc&) {
        return refuse(SVX_OOM, 0, -1, "host allocation failed");
    }
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stopping) return SVX_BAD_ARGUMENT;
        r.t_submit = srv->now_ms();
        ++srv->submitted;
        srv->pending.push_back(std::move(r));
    }
    srv->cv_work.notify_one();
    if (err) {
        err->code = SVX_OK;
        err->message[0] = 0;
    }
    return SVX_OK;
}

int svx_serve_poll(svx_server_t* srv, int32_t wait_ms, svx_serve_result_t** out) {
    if (!srv || !out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto ready = [&] { return !srv->done.empty(); };
    if (wait_ms < 0)
        srv->cv_done.wait(lk, ready);
    else if (wait_ms > 0)
        srv->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
    if (srv->done.empty()) return SVX_QUEUE_EMPTY;
    *out = srv->done.front();
    srv->done.pop_front();
    return SVX_OK;
}

void svx_serve_result_free(svx_serve_result_t* res) {
    if (!res) return;
    delete[] const_cast<double*>(res->u);
    delete[] const_cast<double*>(res->von_mises);
    delete res;
}

int svx_serve_stats(svx_server_t* srv, svx_serve_stats_t* st) {
    if (!srv || !st) return SVX_BAD_ARGUMENT;
    std::lock_guard<std::mutex> lk(srv->mu);
    st->submitted = srv->submitted;
    st->rejected = srv->rejected;
    st->completed = srv->completed;
    st->batches = srv->batches;
    st->pending = int64_t(srv->pending.size());
    st->in_flight = srv->in_flight;
    st->bytes_admitted = srv->bytes_admitted;
    st->peak_bytes_admitted = srv->peak_bytes_admitted;
    st->device_bytes = 0;
    st->pool_ms = 0.0;
    st->pool_mallocs = 0;
    for (svx_ctx* c : srv->lane_ctx) {
        st->device_bytes += int64_t(std::max(c->pool->arena_bytes(),
                                             c->pool->bytes_in_use() + c->pool->bytes_cached()));
        st->pool_ms += c->pool->malloc_ms();
        st->pool_mallocs += c->pool->mallocs();
    }
    st->peak_device_bytes = std::max(srv->peak_device_bytes, st->device_bytes);
    st->prep_ms = srv->prep_ms;
    st->assemble_ms = srv->assemble_ms;
    st->solve_ms = srv->solve_ms;
    st->output_ms = srv->output_ms;
    st->device_solve_ms = srv->device_solve_ms;
    return SVX_OK;
}

double svx_serve_now_ms(const svx_server_t* srv) { return srv ? srv->now_ms() : 0.0; }

int svx_serve_destroy(svx_server_t* srv) {
    if (!srv) return SVX_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
    }
    srv->cv_work.notify_all();
    for (auto& t : srv->lanes) t.join();
    for (svx_serve_result_t* b : srv->done) svx_serve_result_free(b);
    for (svx_ctx* c : srv->lane_ctx) svx_ctx_destroy(c);
    delete srv;
    return SVX_OK;
}

}  // extern "C"

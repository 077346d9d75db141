// svx_api.cpp - the C ABI of libsolvix_b200: contexts, operators and the
// one-call linear-static pipeline that replaces the body of
// solve_with_thermal (crates/solvix-core/src/lib.rs:614-703).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <exception>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "svx_internal.h"

namespace svx {

// ------------------------------------------------------------ DevicePool
DevicePool::~DevicePool() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    for (auto& kv : sizes_)
        if (!in_arena(kv.first)) cudaFree(kv.first);
    if (arena_) cudaFree(arena_);
    cudaSetDevice(prev);
}

static size_t round_bytes(size_t b) {
    // 512 B granules below 2 MiB; above, four size classes per octave
    // (at most 25% slack), so that batches of varying size reuse the cached
    // blocks instead of calling cudaMalloc for every new size.
    if (b < (size_t(1) << 21)) return (b + 511) & ~size_t(511);
    int top = 63 - __builtin_clzll(static_cast<unsigned long long>(b));
    const size_t step = size_t(1) << (top - 2);
    return (b + step - 1) & ~(step - 1);
}

void DevicePool::reserve(size_t bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    if (arena_ || bytes == 0) return;
    bytes = (bytes + (size_t(1) << 21) - 1) & ~((size_t(1) << 21) - 1);
    const auto t0 = std::chrono::steady_clock::now();
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    malloc_ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw ModelFail{SVX_OOM, 0, -1,
                        "could not reserve a device arena of " + std::to_string(bytes) + " bytes"};
    }
    ++mallocs_;
    arena_ = static_cast<char*>(p);
    arena_size_ = bytes;
    ranges_[0] = bytes;
}

void* DevicePool::carve(size_t bytes) {
    for (auto it = ranges_.begin(); it != ranges_.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t off = it->first, len = it->second;
        ranges_.erase(it);
        if (len > bytes) ranges_[off + bytes] = len - bytes;
        return arena_ + off;
    }
    return nullptr;
}

void DevicePool::give_back(void* p, size_t bytes) {
    size_t off = size_t(static_cast<char*>(p) - arena_), len = bytes;
    auto next = ranges_.lower_bound(off);
    if (next != ranges_.end() && off + len == next->first) {
        len += next->second;
        next = ranges_.erase(next);
    }
    if (next != ranges_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            prev->second += len;
            return;
        }
    }
    ranges_[off] = len;
}

void DevicePool::flush_arena_cache() {
    for (auto it = free_.begin(); it != free_.end();) {
        if (in_arena(it->second)) {
            cached_ -= it->first;
            sizes_.erase(it->second);
            give_back(it->second, it->first);
            it = free_.erase(it);
        } else {
            ++it;
        }
    }
}

void* DevicePool::alloc(size_t bytes) {
    // cached blocks up to 25% larger are reused; the arena is carved at the
    // 512 B-aligned size (a size class's slack there would make a batch that
    // the admission estimate fits overflow the arena); a driver allocation
    // takes the size class, so that later sizes of the class reuse it
    const size_t exact = (std::max<size_t>(bytes, 1) + 511) & ~size_t(511);
    const size_t want = round_bytes(bytes);
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.lower_bound(exact);
        if (it != free_.end() && it->first <= exact + exact / 4) {
            void* p = it->second;
            free_.erase(it);
            cached_ -= sizes_[p];
            in_use_ += sizes_[p];
            return p;
        }
        if (arena_) {
            void* p = carve(exact);
            if (!p) {  // cached arena blocks of other sizes go back, coalesced
                flush_arena_cache();
                p = carve(exact);
            }
            if (p) {
                sizes_[p] = exact;
                in_use_ += exact;
                return p;
            }
        }
    }
    // the driver call runs outside the lock: other streams' allocations
    // that hit the cache do not wait for it
    const auto t0 = std::chrono::steady_clock::now();
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        // drop the cache and retry once
        cudaGetLastError();
        trim();
        e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw ModelFail{SVX_OOM, 0, -1,
                            "device allocation of " + std::to_string(want) + " bytes failed"};
        }
    }
    std::lock_guard<std::mutex> lk(mu_);
    malloc_ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
    ++mallocs_;
    sizes_[p] = want;
    in_use_ += want;
    return p;
}

void DevicePool::release(void* p) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = sizes_.find(p);
    if (it == sizes_.end()) return;
    in_use_ -= it->second;
    cached_ += it->second;
    free_.emplace(it->second, p);
}

void DevicePool::trim() {
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    flush_arena_cache();
    for (auto& kv : free_) {
        cudaFree(kv.second);
        sizes_.erase(kv.second);
    }
    free_.clear();
    cached_ = 0;
    malloc_ms_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
}

}  // namespace svx

using namespace svx;

namespace {

thread_local std::string g_thread_error;

void fill_error(svx_error_t* err, int code, int reason, int64_t elem, const std::string& msg) {
    if (!err) return;
    err->code = code;
    err->reason = reason;
    err->elem_index = elem;
    err->iterations = 0;
    err->residual = 0.0;
    std::snprintf(err->message, sizeof(err->message), "%s", msg.c_str());
}

void clear_error(svx_error_t* err) { fill_error(err, SVX_OK, 0, -1, ""); }

// Runs fn, mapping exceptions to status codes and error records.
template <class F>
int guarded(svx_ctx* ctx, svx_error_t* err, F&& fn) {
    try {
        return fn();
    } catch (const ModelFail& m) {
        fill_error(err, m.code, m.reason, m.elem_index, m.message);
        if (ctx) ctx->last_error = m.message;
        g_thread_error = m.message;
        return m.code;
    } catch (const CudaFail& c) {
        std::string msg = std::string("CUDA error: ") + cudaGetErrorString(c.code) + " (" +
                          c.where + ")";
        cudaGetLastError();
        fill_error(err, SVX_CUDA_ERROR, 0, -1, msg);
        if (ctx) ctx->last_error = msg;
        g_thread_error = msg;
        return SVX_CUDA_ERROR;
    } catch (const std::bad_alloc&) {
        fill_error(err, SVX_OOM, 0, -1, "host allocation failed");
        g_thread_error = "host allocation failed";
        return SVX_OOM;
    }
}

int node_count(int kind) {
    switch (kind) {
        case SVX_CPS3: return 3;
        case SVX_CPS4: return 4;
        case SVX_CPS8: return 8;
        case SVX_CPE4: return 4;
        case SVX_CPE8: return 8;
        case SVX_C3D8: return 8;
        case SVX_C3D4: return 4;
        case SVX_B31: return 2;
        default: return -1;
    }
}

const char* kind_name(int kind) {
    static const char* names[] = {"CPS3", "CPS4", "CPS8", "CPE4", "CPE8", "C3D8", "C3D4", "B31"};
    return (kind >= 0 && kind < 8) ? names[kind] : "unknown";
}

const char* reason_text(int reason) {
    switch (reason) {
        case SVX_REASON_NO_MATERIAL: return "no material assigned";
        case SVX_REASON_BAD_MATERIAL: return "invalid material constants";
        case SVX_REASON_SOLID_POISSON:
            return "poisson ratio must be < 0.5 for solids and plane strain";
        case SVX_REASON_DEGENERATE_TRI: return "degenerate (zero-area) triangle";
        case SVX_REASON_BAD_JACOBIAN: return "non-positive Jacobian determinant at a Gauss point";
        default: return "element kind outside the linear-static GPU path (CPS3, CPS4, C3D8)";
    }
}

uint32_t elem_id_of(const svx_flat_model_t* m, int64_t e) {
    return m->elem_id ? m->elem_id[e] : uint32_t(e + 1);
}

// element_entry's checks that precede the geometry (assembly.rs:143-160),
// plus the kinds this path integrates.
int material_reason(const svx_flat_model_t* m, int64_t e) {
    if (m->no_material && m->no_material[e]) return SVX_REASON_NO_MATERIAL;
    double E = m->youngs[e], nu = m->poisson[e];
    if (E <= 0.0 || std::fabs(nu) >= 1.0) return SVX_REASON_BAD_MATERIAL;
    int k = m->kind[e];
    bool solid = (k == SVX_C3D8 || k == SVX_C3D4);
    bool plane_strain = (k == SVX_CPE4 || k == SVX_CPE8);
    if ((solid || plane_strain) && nu >= 0.5) return SVX_REASON_SOLID_POISSON;
    if (!(k == SVX_CPS3 || k == SVX_CPS4 || k == SVX_C3D8)) return SVX_REASON_UNSUPPORTED_KIND;
    return 0;
}

std::string element_message(const svx_flat_model_t* m, int64_t e, int reason) {
    std::string msg = "element " + std::to_string(elem_id_of(m, e)) + ": ";
    if (reason == SVX_REASON_UNSUPPORTED_KIND)
        msg += std::string("element kind ") + kind_name(m->kind[e]) +
               " is outside the linear-static GPU path (CPS3, CPS4, C3D8)";
    else
        msg += reason_text(reason);
    return msg;
}

void check_flat(const svx_flat_model_t* m) {
    auto bad = [](const std::string& s) { throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, s}; };
    if (!m) bad("null model");
    if (m->n_nodes < 0 || m->n_elem < 0 || m->n_fixed < 0) bad("negative size");
    if (m->ndof != 2 && m->ndof != 3) bad("ndof must be 2 or 3");
    if (m->n_nodes > 0 && !m->xyz) bad("null xyz");
    if (m->n_elem > 0 && (!m->kind || !m->conn_ptr || !m->conn || !m->youngs || !m->poisson))
        bad("null element array");
    if (m->n_fixed > 0 && !m->fixed_row) bad("null fixed_row");
    if (m->n_nodes >= (int64_t(1) << 31) / 3) bad("too many nodes for int32 indices");
    if (m->n_elem > 0 && m->conn_ptr[0] != 0) bad("conn_ptr[0] must be 0");
    for (int64_t e = 0; e < m->n_elem; ++e) {
        int64_t a = m->conn_ptr[e], b = m->conn_ptr[e + 1];
        int nn = node_count(m->kind[e]);
        if (nn < 0) bad("unknown element kind " + std::to_string(int(m->kind[e])));
        if (b - a != nn)
            bad("element " + std::to_string(elem_id_of(m, e)) + " has " + std::to_string(b - a) +
                " nodes, kind needs " + std::to_string(nn));
        for (int64_t q = a; q < b; ++q)
            if (m->conn[q] < 0 || m->conn[q] >= m->n_nodes)
                bad("element " + std::to_string(elem_id_of(m, e)) + " references node index " +
                    std::to_string(m->conn[q]) + " out of range");
    }
    const int64_t n = m->n_nodes * m->ndof;
    for (int64_t k = 0; k < m->n_fixed; ++k)
        if (m->fixed_row[k] < 0 || m->fixed_row[k] >= n)
            bad("fixed row " + std::to_string(m->fixed_row[k]) + " out of range");
}

// fn(0..count-1) on up to 16 host threads (members of a batch are
// independent); the first exception is rethrown on the calling thread.
template <class F>
void parallel_for(int32_t count, F&& fn) {
    const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
    const int threads = std::min({hw, 16, int(count / 8) + 1});
    if (threads <= 1) {
        for (int32_t k = 0; k < count; ++k) fn(k);
        return;
    }
    std::atomic<int32_t> next{0};
    std::exception_ptr first;
    std::mutex mu;
    auto work = [&] {
        try {
            for (int32_t k = next.fetch_add(1); k < count; k = next.fetch_add(1)) fn(k);
        } catch (...) {
            std::lock_guard<std::mutex> lk(mu);
            if (!first) first = std::current_exception();
            next.store(count);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (first) std::rethrow_exception(first);
}

template <class T>
void upload(svx_ctx* ctx, DBuf<T>& dst, const T* src, size_t count) {
    dst.alloc(ctx->pool, count + 1);
    if (count)
        SVX_CUDA(cudaMemcpyAsync(dst.p, src, count * sizeof(T), cudaMemcpyHostToDevice,
                                 ctx->stream));
}

float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    SVX_CUDA(cudaEventSynchronize(b));
    SVX_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

// The consistent mass matrix from the operator's device-resident model:
// element mass matrices, pattern, fixed-order assembly (no Dirichlet rows;
// assemble_mass, modal.rs:203-271, has none).
void mass_assemble(svx_ctx* ctx, svx_op* op) {
    cudaStream_t st = ctx->stream;
    SVX_CUDA(cudaEventRecord(ctx->ev[2], st));
    DBuf<double> ke;
    ke.alloc(ctx->pool, size_t(op->n_elem) * op->pat.ke_stride + 1);
    const uint64_t g = integrate_mass(ctx, op, op->mass_rho, ke.p, op->pat.ke_stride);
    if (g != ~uint64_t(0)) {
        const int64_t g_fail = int64_t(g >> 8);
        const int g_reason = int(g & 0xff);
        throw ModelFail{SVX_INVALID_MODEL, g_reason, g_fail,
                        "element " + std::to_string(op->h_elem_id[g_fail]) + ": " +
                            reason_text(g_reason)};
    }
    if (!op->pat.row_ptr.p) build_pattern(ctx, op);
    op->vals.alloc(ctx->pool, op->pat.nnz + 1);
    assemble_values(ctx, op, ke.p, op->pat.ke_stride, op->vals.p);
    ke.reset();
    op->spmv_group = choose_spmv_group(op);
    SVX_CUDA(cudaEventRecord(ctx->ev[3], st));
    op->ms_assemble = elapsed_ms(ctx->ev[2], ctx->ev[3]);
}

// K1-K4 from the operator's device-resident model: element integration,
// pattern, fixed-order assembly and Dirichlet.  Needs no host model.
void device_assemble(svx_ctx* ctx, svx_op* op) {
    if (op->mass_rho >= 0.0) {
        mass_assemble(ctx, op);
        return;
    }
    cudaStream_t st = ctx->stream;
    SVX_CUDA(cudaEventRecord(ctx->ev[2], st));
    DBuf<double> ke;
    ke.alloc(ctx->pool, size_t(op->n_elem) * op->pat.ke_stride + 1);
    uint64_t g = integrate_elements(ctx, op, ke.p, op->pat.ke_stride);
    if (g != ~uint64_t(0)) {
        int64_t g_fail = int64_t(g >> 8);
        int g_reason = int(g & 0xff);
        throw ModelFail{SVX_INVALID_MODEL, g_reason, g_fail,
                        "element " + std::to_string(op->h_elem_id[g_fail]) + ": " +
                            reason_text(g_reason)};
    }
    if (!op->pat.row_ptr.p) build_pattern(ctx, op);
    op->vals.alloc(ctx->pool, op->pat.nnz + 1);
    assemble_values(ctx, op, ke.p, op->pat.ke_stride, op->vals.p);
    ke.reset();
    if (op->flags & SVX_KEEP_ORIGINAL) {
        op->vals_orig.alloc(ctx->pool, op->pat.nnz + 1);
        SVX_CUDA(cudaMemcpyAsync(op->vals_orig.p, op->vals.p, op->pat.nnz * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st));
    }
    op->vals32.reset();
    op->vals32q.reset();
    op->valsT.reset();
    apply_dirichlet(ctx, op);
    op->spmv_group = choose_spmv_group(op);
    SVX_CUDA(cudaEventRecord(ctx->ev[3], st));
    op->ms_assemble = elapsed_ms(ctx->ev[2], ctx->ev[3]);
}

// K1-K4 for a validated flat model; throws ModelFail for element errors.
svx_op* assemble_impl(svx_ctx* ctx, const svx_flat_model_t* m, uint32_t flags,
                      const double* thick_elem = nullptr, bool prechecked = false) {
    SVX_CUDA(cudaSetDevice(ctx->device));
    if (!prechecked) check_flat(m);
    // ndof_per_node (lib.rs:725-752) runs before assembly
    // first element failing a material / kind check (host, O(n_elem));
    // members of a batch were checked one by one already
    int64_t m_fail = -1;
    int m_reason = 0;
    if (!prechecked) {
        bool solid = false, plane = false, beam = false;
        for (int64_t e = 0; e < m->n_elem; ++e) {
            int k = m->kind[e];
            if (k == SVX_C3D8 || k == SVX_C3D4) solid = true;
            else if (k == SVX_B31) beam = true;
            else plane = true;
        }
        if (beam && (plane || solid))
            throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                            "mixed beam and continuum elements (v1: B31-only models)"};
        if (solid && plane) throw ModelFail{SVX_INVALID_MODEL, 0, -1, "mixed dimensionality"};
        if (m->ndof != ((solid || beam) ? 3 : 2))
            throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "ndof does not match the element kinds"};
        for (int64_t e = 0; e < m->n_elem; ++e) {
            int r = material_reason(m, e);
            if (r) {
                m_fail = e;
                m_reason = r;
                break;
            }
        }
    }

    std::unique_ptr<svx_op> op(new svx_op());
    op->ctx = ctx;
    op->n_nodes = m->n_nodes;
    op->n_elem = (m_fail >= 0) ? m_fail : m->n_elem;  // elements before a material failure
    op->ndof = m->ndof;
    op->n = m->n_nodes * m->ndof;
    op->thickness = m->thickness;
    op->flags = flags;
    cudaStream_t st = ctx->stream;
    SVX_CUDA(cudaEventRecord(ctx->ev[6], st));
    upload(ctx, op->xyz, m->xyz, size_t(3 * m->n_nodes));
    upload(ctx, op->kind, m->kind, size_t(op->n_elem));
    upload(ctx, op->conn_ptr, m->conn_ptr, size_t(op->n_elem + 1));
    upload(ctx, op->conn, m->conn, size_t(op->n_elem > 0 ? m->conn_ptr[op->n_elem] : 0));
    upload(ctx, op->youngs, m->youngs, size_t(op->n_elem));
    upload(ctx, op->poisson, m->poisson, size_t(op->n_elem));
    if (thick_elem) upload(ctx, op->thick_elem, thick_elem, size_t(op->n_elem));
    int max_nn = 0;
    for (int64_t e = 0; e < op->n_elem; ++e) max_nn = std::max(max_nn, node_count(m->kind[e]));
    op->pat.max_nn = std::max(max_nn, 1);
    const int max_N = max_nn * m->ndof;
    op->pat.ke_stride = std::max(1, max_N * max_N);
    op->h_elem_id.resize(size_t(op->n_elem));
    for (int64_t e = 0; e < op->n_elem; ++e) op->h_elem_id[e] = elem_id_of(m, e);
    if (m_fail >= 0) {
        // only the elements before the first material failure can fail first
        DBuf<double> ke;
        ke.alloc(ctx->pool, size_t(op->n_elem) * op->pat.ke_stride + 1);
        uint64_t g = integrate_elements(ctx, op.get(), ke.p, op->pat.ke_stride);
        if (g != ~uint64_t(0)) {
            int64_t g_fail = int64_t(g >> 8);
            int g_reason = int(g & 0xff);
            throw ModelFail{SVX_INVALID_MODEL, g_reason, g_fail,
                            element_message(m, g_fail, g_reason)};
        }
        throw ModelFail{SVX_INVALID_MODEL, m_reason, m_fail, element_message(m, m_fail, m_reason)};
    }
    // loads and constraints
    if (m->f) {
        upload(ctx, op->f_orig, m->f, size_t(op->n));
    } else {
        op->f_orig.alloc(ctx->pool, size_t(op->n) + 1);
        SVX_CUDA(cudaMemsetAsync(op->f_orig.p, 0, sizeof(double) * size_t(op->n), st));
    }
    op->n_fixed = m->n_fixed;
    op->h_fixed_row.assign(m->fixed_row, m->fixed_row + m->n_fixed);
    upload(ctx, op->fixed_row, op->h_fixed_row.data(), size_t(m->n_fixed));
    op->h_node_id.resize(size_t(m->n_nodes));
    for (int64_t i = 0; i < m->n_nodes; ++i)
        op->h_node_id[i] = m->node_id ? m->node_id[i] : uint32_t(i + 1);
    device_assemble(ctx, op.get());
    SVX_CUDA(cudaEventRecord(ctx->ev[7], st));
    op->ms_upload_assemble = elapsed_ms(ctx->ev[6], ctx->ev[7]);
    return op.release();
}

// svx_assemble_mass: the model's geometry on the device and its consistent
// mass matrix; no material, load or constraint data is read.
svx_op* assemble_mass_impl(svx_ctx* ctx, const svx_flat_model_t* m, double rho) {
    SVX_CUDA(cudaSetDevice(ctx->device));
    check_flat(m);
    if (!(rho >= 0.0) || std::isinf(rho))
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "density must be finite and >= 0"};
    bool solid = false, plane = false, beam = false;
    for (int64_t e = 0; e < m->n_elem; ++e) {
        const int k = m->kind[e];
        if (k == SVX_C3D8 || k == SVX_C3D4) solid = true;
        else if (k == SVX_B31) beam = true;
        else plane = true;
    }
    if (beam && (plane || solid))
        throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                        "mixed beam and continuum elements (v1: B31-only models)"};
    if (solid && plane) throw ModelFail{SVX_INVALID_MODEL, 0, -1, "mixed dimensionality"};
    if (m->ndof != ((solid || beam) ? 3 : 2))
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "ndof does not match the element kinds"};
    std::unique_ptr<svx_op> op(new svx_op());
    op->ctx = ctx;
    op->n_nodes = m->n_nodes;
    op->n_elem = m->n_elem;
    op->ndof = m->ndof;
    op->n = m->n_nodes * m->ndof;
    op->thickness = m->thickness;
    op->mass_rho = rho;
    cudaStream_t st = ctx->stream;
    SVX_CUDA(cudaEventRecord(ctx->ev[6], st));
    upload(ctx, op->xyz, m->xyz, size_t(3 * m->n_nodes));
    upload(ctx, op->kind, m->kind, size_t(op->n_elem));
    upload(ctx, op->conn_ptr, m->conn_ptr, size_t(op->n_elem + 1));
    upload(ctx, op->conn, m->conn, size_t(op->n_elem > 0 ? m->conn_ptr[op->n_elem] : 0));
    int max_nn = 0;
    for (int64_t e = 0; e < op->n_elem; ++e) max_nn = std::max(max_nn, node_count(m->kind[e]));
    op->pat.max_nn = std::max(max_nn, 1);
    const int max_N = max_nn * m->ndof;
    op->pat.ke_stride = std::max(1, max_N * max_N);
    op->h_elem_id.resize(size_t(op->n_elem));
    for (int64_t e = 0; e < op->n_elem; ++e) op->h_elem_id[e] = elem_id_of(m, e);
    op->h_node_id.resize(size_t(m->n_nodes));
    for (int64_t i = 0; i < m->n_nodes; ++i)
        op->h_node_id[i] = m->node_id ? m->node_id[i] : uint32_t(i + 1);
    mass_assemble(ctx, op.get());
    SVX_CUDA(cudaEventRecord(ctx->ev[7], st));
    op->ms_upload_assemble = elapsed_ms(ctx->ev[6], ctx->ev[7]);
    return op.release();
}

void refuse_mass(const svx_op* op, const char* what) {
    if (op->mass_rho >= 0.0)
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1,
                        std::string("the operator holds a consistent mass matrix; ") + what};
}

void stress_to_device(svx_op* op) {
    svx_ctx* ctx = op->ctx;
    if (!op->vm_elem.p) op->vm_elem.alloc(ctx->pool, op->n_elem + 1);
    if (!op->vm_node.p) op->vm_node.alloc(ctx->pool, op->n_nodes + 1);
    if (!op->react.p) op->react.alloc(ctx->pool, op->n_fixed + 1);
    if (!op->disp3.p) op->disp3.alloc(ctx->pool, 3 * op->n_nodes + 1);
    recover_stress(ctx, op, op->u.p, op->vm_elem.p, op->vm_node.p, op->react.p, op->disp3.p);
}

void copy_stress_out(svx_op* op, svx_solution_t* sol) {
    cudaStream_t st = op->ctx->stream;
    if (sol->von_mises && op->n_elem)
        SVX_CUDA(cudaMemcpyAsync(sol->von_mises, op->vm_elem.p, op->n_elem * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    if (sol->nodal_von_mises && op->n_nodes)
        SVX_CUDA(cudaMemcpyAsync(sol->nodal_von_mises, op->vm_node.p,
                                 op->n_nodes * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (sol->reactions && op->n_fixed)
        SVX_CUDA(cudaMemcpyAsync(sol->reactions, op->react.p, op->n_fixed * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    if (sol->displacements && op->n_nodes)
        SVX_CUDA(cudaMemcpyAsync(sol->displacements, op->disp3.p,
                                 3 * op->n_nodes * sizeof(double), cudaMemcpyDeviceToHost, st));
}

long long default_max_iter(int64_t n) { return std::max<long long>(1000, 10 * (long long)n); }

int solve_impl(svx_op* op, const svx_solve_opts_t* o, svx_solution_t* sol, svx_error_t* err) {
    svx_ctx* ctx = op->ctx;
    SVX_CUDA(cudaSetDevice(ctx->device));
    svx_solve_opts_t opts;
    svx_default_opts(&opts);
    if (o) opts = *o;
    long long max_iter = opts.max_iter > 0 ? opts.max_iter : default_max_iter(op->n);
    if (opts.method < SVX_METHOD_PCG || opts.method > SVX_METHOD_AUTO)
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "unknown solver method"};
    if (opts.precision != SVX_FP64 && opts.precision != SVX_MIXED &&
        opts.precision != SVX_MIXED_DEFECT)
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "unknown precision"};
    op->u.alloc(ctx->pool, op->n + 1);
    PcgResult r{PCG_CONVERGED, 0, 0.0, 0.0};
    long long outer = 0;
    if (opts.method != SVX_METHOD_LDLT) {
        if (opts.precision == SVX_MIXED)
            r = pcg_mixed(ctx, op, opts.tol, max_iter, opts.inner_tol, opts.check_every,
                          op->u.p, &outer);
        else if (opts.precision == SVX_MIXED_DEFECT)
            r = pcg_defect_correction(ctx, op, opts.tol, max_iter, opts.inner_tol,
                                      opts.check_every, op->u.p, &outer);
        else
            r = pcg_fp64(ctx, op, opts.tol, max_iter, opts.check_every, op->u.p);
    }
    // lib.rs:664-686: Ldlt factorizes; Auto factorizes when the PCG returns
    // NotConverged (budget overrun or breakdown).
    const bool direct = opts.method == SVX_METHOD_LDLT ||
                        (opts.method == SVX_METHOD_AUTO && r.status != PCG_CONVERGED);
    LdltOutcome dres;
    if (direct) {
        op->has_solution = false;
        dres = ldlt_direct(ctx, op, op->u.p);
        r = PcgResult{PCG_CONVERGED, 0, dres.residual, dres.ms};
        outer = 0;
    }
    op->has_solution = true;
    if (sol) {
        sol->iterations = r.iterations;
        sol->outer_iterations = outer;
        sol->fp32_iterations =
            (opts.precision != SVX_FP64 && !direct) ? op->mixed_sloppy_iters : 0;
        sol->final_residual = r.residual;
        sol->cond_estimate = direct ? dres.cond : op->cond_estimate;
        sol->solver_method = direct ? SVX_METHOD_LDLT : SVX_METHOD_PCG;
        sol->factor_bandwidth = direct ? dres.bandwidth : 0;
        sol->ms_factor = direct ? dres.ms : 0.0;
        sol->ms_assemble = op->ms_assemble;
        sol->ms_solve = r.ms;
        if (sol->u)
            SVX_CUDA(cudaMemcpyAsync(sol->u, op->u.p, op->n * sizeof(double),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (r.status != PCG_CONVERGED) {
        SVX_CUDA(cudaStreamSynchronize(ctx->stream));
        std::string msg = "not converged after " + std::to_string(r.iterations) + " iterations";
        fill_error(err, SVX_NOT_CONVERGED, 0, -1, msg);
        if (err) {
            err->iterations = r.iterations;
            err->residual = r.residual;
        }
        ctx->last_error = msg;
        return SVX_NOT_CONVERGED;
    }
    if (opts.want_stress) {
        SVX_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
        stress_to_device(op);
        SVX_CUDA(cudaEventRecord(ctx->ev[5], ctx->stream));
        if (sol) {
            copy_stress_out(op, sol);
            sol->ms_stress = elapsed_ms(ctx->ev[4], ctx->ev[5]);
        }
    }
    SVX_CUDA(cudaStreamSynchronize(ctx->stream));
    clear_error(err);
    return SVX_OK;
}

}  // namespace

namespace svx {

// Host checks of one batch member, in the reference's order: empty mesh,
// no constraints (lib.rs:600-606), flat-model consistency, the element
// kinds against ndof (lib.rs:725-752), then the first element failing a
// material check (assembly.rs:143-160).
void check_batch_member(const svx_flat_model_t* m) {
    check_flat(m);
    if (m->n_elem == 0) throw ModelFail{SVX_EMPTY_MESH, 0, -1, "empty mesh"};
    if (m->n_fixed == 0) throw ModelFail{SVX_NO_CONSTRAINTS, 0, -1, "no constraints"};
    bool solid = false, plane = false, beam = false;
    for (int64_t e = 0; e < m->n_elem; ++e) {
        const int k = m->kind[e];
        if (k == SVX_C3D8 || k == SVX_C3D4) solid = true;
        else if (k == SVX_B31) beam = true;
        else plane = true;
    }
    if (beam && (plane || solid))
        throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                        "mixed beam and continuum elements (v1: B31-only models)"};
    if (solid && plane) throw ModelFail{SVX_INVALID_MODEL, 0, -1, "mixed dimensionality"};
    if (m->ndof != ((solid || beam) ? 3 : 2))
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "ndof does not match the element kinds"};
    for (int64_t e = 0; e < m->n_elem; ++e) {
        const int r = material_reason(m, e);
        if (r) throw ModelFail{SVX_INVALID_MODEL, r, e, element_message(m, e, r)};
    }
}


// One block-diagonal batch.  Every member is checked on its own; a member
// that fails (host checks, or a non-positive Jacobian found by the element
// kernel) gets its own status and message and the batch is re-assembled
// without it, so no member's failure reaches another member.  The members
// that pass are concatenated (node, element and row offsets), assembled as
// one operator and solved by one batched PCG launch.
void run_batch(svx_ctx* ctx, int32_t count, const svx_flat_model_t* const* models,
               const svx_solve_opts_t& o, double* const* u, double* const* vm,
               std::vector<BatchModelOut>& out, BatchRun& run) {
    SVX_CUDA(cudaSetDevice(ctx->device));
    if (o.precision != SVX_FP64 && o.precision != SVX_MIXED)
        throw ModelFail{SVX_BAD_ARGUMENT, 0, -1,
                        "the batched and served forms run SVX_FP64 or SVX_MIXED"};
    out.assign(static_cast<size_t>(count), BatchModelOut{});
    run = BatchRun{};
    using clock = std::chrono::steady_clock;
    auto since = [](clock::time_point t) {
        return std::chrono::duration<double, std::milli>(clock::now() - t).count();
    };
    clock::time_point t_phase = clock::now();
    int ndof = 0;
    std::vector<int32_t> live;
    for (int32_t k = 0; k < count; ++k)
        if (!models[k]) throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "null model"};
    // the members' host checks are independent: run them on the host cores
    parallel_for(count, [&](int32_t k) {
        try {
            check_batch_member(models[k]);
        } catch (const ModelFail& f) {
            out[k].status = f.code;
            out[k].reason = f.reason;
            out[k].elem_index = f.elem_index;
            out[k].message = f.message;
        }
    });
    for (int32_t k = 0; k < count; ++k) {
        if (out[k].status != SVX_OK) continue;
        if (ndof == 0) ndof = models[k]->ndof;
        if (models[k]->ndof != ndof)
            throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "models of one batch share ndof"};
        live.push_back(k);
    }
    while (!live.empty()) {
        const int32_t L = int32_t(live.size());
        int64_t nn = 0, ne = 0, nc = 0, nf = 0;
        for (int32_t k : live) {
            const svx_flat_model_t& m = *models[k];
            nn += m.n_nodes;
            ne += m.n_elem;
            nc += m.conn_ptr[m.n_elem];
            nf += m.n_fixed;
        }
        // the concatenated model is written straight into the context's
        // page-locked staging buffer, so assembly uploads it by DMA
        const size_t une = static_cast<size_t>(ne), unn = static_cast<size_t>(nn);
        size_t off = 0;
        auto carve = [&](size_t bytes) {
            const size_t at = off;
            off += (bytes + 15) & ~size_t(15);
            return at;
        };
        const size_t o_xyz = carve(24 * unn), o_f = carve(8 * unn * ndof), o_E = carve(8 * une),
                     o_nu = carve(8 * une), o_th = carve(8 * une), o_cp = carve(8 * (une + 1)),
                     o_fix = carve(8 * static_cast<size_t>(nf)), o_eid = carve(4 * une),
                     o_conn = carve(4 * static_cast<size_t>(nc)), o_kind = carve(une);
        char* base = static_cast<char*>(ctx->staging.get(std::max<size_t>(off, 16)));
        double* xyz = reinterpret_cast<double*>(base + o_xyz);
        double* f = reinterpret_cast<double*>(base + o_f);
        double* E = reinterpret_cast<double*>(base + o_E);
        double* nu = reinterpret_cast<double*>(base + o_nu);
        double* th = reinterpret_cast<double*>(base + o_th);
        int64_t* conn_ptr = reinterpret_cast<int64_t*>(base + o_cp);
        int64_t* fixed = reinterpret_cast<int64_t*>(base + o_fix);
        uint32_t* eid = reinterpret_cast<uint32_t*>(base + o_eid);
        int32_t* conn = reinterpret_cast<int32_t*>(base + o_conn);
        uint8_t* kind = reinterpret_cast<uint8_t*>(base + o_kind);
        std::vector<int64_t> node_off(static_cast<size_t>(L) + 1, 0);
        std::vector<int64_t> elem_off(static_cast<size_t>(L) + 1, 0);
        std::vector<int64_t> conn_off(static_cast<size_t>(L) + 1, 0);
        std::vector<int64_t> fix_off(static_cast<size_t>(L) + 1, 0);
        for (int32_t j = 0; j < L; ++j) {
            const svx_flat_model_t& m = *models[live[j]];
            node_off[j + 1] = node_off[j] + m.n_nodes;
            elem_off[j + 1] = elem_off[j] + m.n_elem;
            conn_off[j + 1] = conn_off[j] + m.conn_ptr[m.n_elem];
            fix_off[j + 1] = fix_off[j] + m.n_fixed;
        }
        const int64_t n_fixed = fix_off[L];
        conn_ptr[0] = 0;
        // every member fills its own ranges: copy them on the host cores
        parallel_for(L, [&](int32_t j) {
            const svx_flat_model_t& m = *models[live[j]];
            const int64_t n0 = node_off[j], e0 = elem_off[j], c0 = conn_off[j];
            std::memcpy(xyz + 3 * n0, m.xyz, sizeof(double) * 3 * m.n_nodes);
            if (m.f)
                std::memcpy(f + n0 * ndof, m.f, sizeof(double) * m.n_nodes * ndof);
            else
                std::memset(f + n0 * ndof, 0, sizeof(double) * m.n_nodes * ndof);
            std::memcpy(kind + e0, m.kind, size_t(m.n_elem));
            std::memcpy(E + e0, m.youngs, sizeof(double) * m.n_elem);
            std::memcpy(nu + e0, m.poisson, sizeof(double) * m.n_elem);
            for (int64_t e = 0; e < m.n_elem; ++e) {
                th[e0 + e] = m.thickness;
                eid[e0 + e] = elem_id_of(&m, e);
                conn_ptr[e0 + e + 1] = c0 + m.conn_ptr[e + 1];
            }
            const int32_t shift = int32_t(n0);
            for (int64_t q = 0; q < m.conn_ptr[m.n_elem]; ++q) conn[c0 + q] = m.conn[q] + shift;
            for (int64_t q = 0; q < m.n_fixed; ++q)
                fixed[fix_off[j] + q] = m.fixed_row[q] + n0 * ndof;
        });
        svx_flat_model_t all{};
        all.n_nodes = nn;
        all.xyz = xyz;
        all.n_elem = ne;
        all.kind = kind;
        all.conn_ptr = conn_ptr;
        all.conn = conn;
        all.youngs = E;
        all.poisson = nu;
        all.elem_id = eid;
        all.thickness = 1.0;
        all.ndof = ndof;
        all.n_fixed = n_fixed;
        all.fixed_row = fixed;
        all.f = f;
        run.wall_prep += since(t_phase);
        t_phase = clock::now();
        std::unique_ptr<svx_op> op;
        try {
            op.reset(assemble_impl(ctx, &all, 0, th, true));
        } catch (const ModelFail& fail) {
            if (fail.code != SVX_INVALID_MODEL || fail.elem_index < 0 || fail.elem_index >= ne)
                throw;
            // the element kernel found a bad element: drop its model, retry
            const int32_t j = int32_t(std::upper_bound(elem_off.begin(), elem_off.end(),
                                                       fail.elem_index) -
                                      elem_off.begin()) - 1;
            BatchModelOut& bad = out[live[j]];
            bad.status = SVX_INVALID_MODEL;
            bad.reason = fail.reason;
            bad.elem_index = fail.elem_index - elem_off[j];
            bad.message = fail.message;
            live.erase(live.begin() + j);
            run.wall_assemble += since(t_phase);
            t_phase = clock::now();
            continue;
        }
        run.wall_assemble += since(t_phase);
        t_phase = clock::now();
        std::vector<double> tol(static_cast<size_t>(L), o.tol);
        std::vector<int64_t> mi(static_cast<size_t>(L));
        for (int32_t j = 0; j < L; ++j)
            mi[j] = o.max_iter > 0 ? o.max_iter
                                   : default_max_iter((node_off[j + 1] - node_off[j]) * ndof);
        std::vector<int64_t> it;
        std::vector<double> res, cond;
        std::vector<int32_t> status;
        BatchStats bs;
        batch_pcg(ctx, op.get(), L, node_off, tol, mi, it, res, status, cond, &bs,
                  o.precision == SVX_MIXED);
        run.wall_solve += since(t_phase);
        t_phase = clock::now();
        cudaStream_t st = ctx->stream;
        const bool want_vm = vm && o.want_stress;
        if (want_vm) {
            SVX_CUDA(cudaEventRecord(ctx->ev[4], st));
            if (!op->vm_elem.p) op->vm_elem.alloc(ctx->pool, op->n_elem + 1);
            recover_stress(ctx, op.get(), op->u.p, op->vm_elem.p, nullptr, nullptr, nullptr);
            SVX_CUDA(cudaEventRecord(ctx->ev[5], st));
        }
        // u and the von Mises field come back in two DMA copies through the
        // staging buffer (the uploads of this batch are complete), then are
        // split per member on the host
        const size_t nu_rows = static_cast<size_t>(nn * ndof);
        double* host = static_cast<double*>(
            ctx->staging.get(sizeof(double) * (nu_rows + (want_vm ? une : 0) + 1)));
        if (u) SVX_CUDA(cudaMemcpyAsync(host, op->u.p, sizeof(double) * nu_rows,
                                        cudaMemcpyDeviceToHost, st));
        if (want_vm)
            SVX_CUDA(cudaMemcpyAsync(host + nu_rows, op->vm_elem.p, sizeof(double) * une,
                                     cudaMemcpyDeviceToHost, st));
        SVX_CUDA(cudaStreamSynchronize(st));
        if (want_vm) run.ms_stress = elapsed_ms(ctx->ev[4], ctx->ev[5]);
        parallel_for(L, [&](int32_t j) {
            const int32_t k = live[j];
            if (u && u[k])
                std::memcpy(u[k], host + node_off[j] * ndof,
                            sizeof(double) * (node_off[j + 1] - node_off[j]) * ndof);
            if (want_vm && vm[k])
                std::memcpy(vm[k], host + nu_rows + elem_off[j],
                            sizeof(double) * (elem_off[j + 1] - elem_off[j]));
        });
        for (int32_t j = 0; j < L; ++j) {
            BatchModelOut& m = out[live[j]];
            m.iterations = it[j];
            m.residual = res[j];
            m.status = status[j] == PCG_CONVERGED ? SVX_OK : SVX_NOT_CONVERGED;
            if (m.status != SVX_OK)
                m.message = "not converged after " + std::to_string(it[j]) + " iterations";
            m.cond = cond[j];
            m.nnz = bs.member_nnz[j];
        }
        run.wall_output += since(t_phase);
        run.ms_assemble = op->ms_assemble;
        run.ms_solve = bs.ms_solve;
        run.threads_per_cta = bs.threads_per_cta;
        run.lanes_per_node = bs.lanes_per_node;
        run.cluster_members = bs.cluster_members;
        run.fp32_iterations = bs.fp32_iterations;
        break;
    }
}

}  // namespace svx

extern "C" {

const char* svx_version(void) { return "solvix_b200 0.1.0 (sm_100a)"; }

void svx_default_opts(svx_solve_opts_t* opts) {
    if (!opts) return;
    opts->tol = 1e-10;
    opts->max_iter = 0;
    opts->precision = SVX_FP64;
    opts->inner_tol = 1e-5;
    opts->check_every = 0;
    opts->want_stress = 1;
    opts->method = SVX_METHOD_PCG;
}

int svx_ctx_create(int device, svx_ctx_t** out) {
    if (!out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    return guarded(nullptr, nullptr, [&]() -> int {
        int count = 0;
        SVX_CUDA(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count)
            throw ModelFail{SVX_CUDA_ERROR, 0, -1,
                            "CUDA device " + std::to_string(device) + " is not available"};
        SVX_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        SVX_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            throw ModelFail{SVX_CUDA_ERROR, 0, -1,
                            std::string("device ") + prop.name +
                                " is not sm_100 (B200); this library is built for sm_100a only"};
        std::unique_ptr<svx_ctx> ctx(new svx_ctx());
        ctx->device = device;
        ctx->sm_count = prop.multiProcessorCount;
        ctx->l2_bytes = prop.l2CacheSize;
        if (const char* e = std::getenv("SVX_SHARED_ADJ_MAX")) {
            char* end = nullptr;
            const long long v = std::strtoll(e, &end, 10);
            if (end != e && v >= 0) ctx->shared_adj_max = v;
        }
        if (const char* e = std::getenv("SVX_GRAPH_MIN_NNZ")) {
            char* end = nullptr;
            const long long v = std::strtoll(e, &end, 10);
            if (end != e && v >= 0) ctx->graph_min_nnz = v;
        }
        if (const char* e = std::getenv("SVX_PCG_SMEM")) ctx->pcg_smem = (e[0] != '0');
        if (const char* e = std::getenv("SVX_PCG_ALG")) ctx->pcg_alg = (e[0] == '0') ? 0 : 1;
        if (const char* e = std::getenv("SVX_PCG_STAGE")) ctx->pcg_stage = (e[0] != '0');
        if (const char* e = std::getenv("SVX_FP32_QUADS")) ctx->fp32_quads = (e[0] != '0');
        if (const char* e = std::getenv("SVX_PCG_LANES")) ctx->pcg_lanes = std::atoi(e);
        if (const char* e = std::getenv("SVX_PCG_UNROLL")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v == 1 || v == 2 || v == 4) ctx->pcg_unroll = int(v);
        }
        // the main stream (uploads, assembly, stress, plain solves) has the
        // highest priority; the long batched PCG kernels run on the lowest,
        // so a served lane's assembly gets SMs while another lane's batch
        // is being solved
        int least = 0, greatest = 0;
        SVX_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        SVX_CUDA(cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, greatest));
        SVX_CUDA(cudaStreamCreateWithPriority(&ctx->pcg_stream, cudaStreamNonBlocking, least));
        SVX_CUDA(cudaStreamCreateWithPriority(&ctx->aux_stream, cudaStreamNonBlocking, least));
        for (auto& e : ctx->ev) SVX_CUDA(cudaEventCreate(&e));
        SVX_CUDA(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
        SVX_CUDA(cudaMallocHost(&ctx->h_scalars, 256));
        SVX_CUDA(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming));
        ctx->pool = new DevicePool(device);
        *out = ctx.release();
        return SVX_OK;
    });
}

int svx_ctx_destroy(svx_ctx_t* ctx) {
    if (!ctx) return SVX_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete ctx->pool;
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    for (cudaStream_t x : {ctx->pcg_stream, ctx->aux_stream})
        if (x) {
            cudaStreamSynchronize(x);
            cudaStreamDestroy(x);
        }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SVX_OK;
}

int svx_last_error(const svx_ctx_t* ctx, char* buf, size_t len) {
    if (!buf || len == 0) return SVX_BAD_ARGUMENT;
    const std::string& s = ctx ? ctx->last_error : g_thread_error;
    std::snprintf(buf, len, "%s", s.c_str());
    return SVX_OK;
}

int svx_assemble_mass(svx_ctx_t* ctx, const svx_flat_model_t* model, double density,
                      svx_op_t** out, svx_error_t* err) {
    if (!ctx || !out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    return guarded(ctx, err, [&]() -> int {
        *out = assemble_mass_impl(ctx, model, density);
        clear_error(err);
        return SVX_OK;
    });
}

int svx_assemble(svx_ctx_t* ctx, const svx_flat_model_t* model, uint32_t flags, svx_op_t** out,
                 svx_error_t* err) {
    if (!ctx || !out) return SVX_BAD_ARGUMENT;
    *out = nullptr;
    return guarded(ctx, err, [&]() -> int {
        *out = assemble_impl(ctx, model, flags);
        clear_error(err);
        return SVX_OK;
    });
}

void* svx_ctx_stream(svx_ctx_t* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t svx_launch_count(void) { return int64_t(g_launches.load()); }

int svx_op_time_kernels(svx_op_t* op, int reps, double* ms4) {
    if (!op || !ms4 || reps <= 0) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        time_iteration_kernels(ctx, op, reps, ms4);
        return SVX_OK;
    });
}

int svx_op_reassemble(svx_op_t* op, svx_error_t* err) {
    if (!op) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, err, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        device_assemble(ctx, op);
        clear_error(err);
        return SVX_OK;
    });
}

int svx_op_free(svx_op_t* op) {
    if (!op) return SVX_OK;
    cudaSetDevice(op->ctx->device);
    cudaStreamSynchronize(op->ctx->stream);
    delete op;
    return SVX_OK;
}

int svx_op_dims(const svx_op_t* op, int64_t* n_rows, int64_t* nnz) {
    if (!op) return SVX_BAD_ARGUMENT;
    if (n_rows) *n_rows = op->n;
    if (nnz) *nnz = op->pat.nnz;
    return SVX_OK;
}

int svx_op_get_csr(const svx_op_t* op, int which, int64_t* row_ptr, int32_t* col_idx,
                   double* vals) {
    if (!op) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        if (row_ptr) {
            std::vector<int32_t> rp(size_t(op->n + 1));
            SVX_CUDA(cudaMemcpyAsync(rp.data(), op->pat.row_ptr.p, (op->n + 1) * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, st));
            SVX_CUDA(cudaStreamSynchronize(st));
            for (int64_t i = 0; i <= op->n; ++i) row_ptr[i] = rp[i];
        }
        if (col_idx && op->pat.nnz)
            SVX_CUDA(cudaMemcpyAsync(col_idx, op->pat.col_idx.p, op->pat.nnz * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, st));
        if (vals && op->pat.nnz) {
            const double* src = which == 1 ? op->vals_orig.p : op->vals.p;
            if (!src)
                throw ModelFail{SVX_BAD_ARGUMENT, 0, -1,
                                "K before Dirichlet was not kept (assemble with SVX_KEEP_ORIGINAL)"};
            SVX_CUDA(cudaMemcpyAsync(vals, src, op->pat.nnz * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        }
        SVX_CUDA(cudaStreamSynchronize(st));
        return SVX_OK;
    });
}

int svx_op_get_vectors(const svx_op_t* op, int which, double* f, double* inv_diag) {
    if (!op) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        if (f || inv_diag) refuse_mass(op, "it has no load vector or Jacobi diagonal");
        SVX_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        if (f && op->n)
            SVX_CUDA(cudaMemcpyAsync(f, which == 1 ? op->f_orig.p : op->f.p, op->n * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        if (inv_diag && op->n)
            SVX_CUDA(cudaMemcpyAsync(inv_diag, op->inv_diag.p, op->n * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        SVX_CUDA(cudaStreamSynchronize(st));
        return SVX_OK;
    });
}

int svx_op_spmv(svx_op_t* op, const double* x, double* y) {
    if (!op || !x || !y) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        DBuf<double> dx, dy;
        dx.alloc(ctx->pool, op->n + 1);
        dy.alloc(ctx->pool, op->n + 1);
        SVX_CUDA(cudaMemcpyAsync(dx.p, x, op->n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        spmv_fp64(ctx, op, op->vals.p, dx.p, dy.p);
        SVX_CUDA(cudaMemcpyAsync(y, dy.p, op->n * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        SVX_CUDA(cudaStreamSynchronize(ctx->stream));
        return SVX_OK;
    });
}

int svx_op_set_solution(svx_op_t* op, const double* u) {
    if (!op || !u) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        op->u.alloc(ctx->pool, op->n + 1);
        SVX_CUDA(cudaMemcpyAsync(op->u.p, u, op->n * sizeof(double), cudaMemcpyHostToDevice,
                                 ctx->stream));
        SVX_CUDA(cudaStreamSynchronize(ctx->stream));
        op->has_solution = true;
        return SVX_OK;
    });
}

int svx_op_solve(svx_op_t* op, const svx_solve_opts_t* opts, svx_solution_t* sol,
                 svx_error_t* err) {
    if (!op) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, err, [&]() -> int {
        refuse_mass(op, "it is not solved");
        return solve_impl(op, opts, sol, err);
    });
}

int svx_op_stress(svx_op_t* op, svx_solution_t* sol) {
    if (!op || !sol) return SVX_BAD_ARGUMENT;
    svx_ctx* ctx = op->ctx;
    return guarded(ctx, nullptr, [&]() -> int {
        refuse_mass(op, "it has no stresses");
        if (!op->has_solution)
            throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, "operator has no solution yet"};
        SVX_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t st = ctx->stream;
        SVX_CUDA(cudaEventRecord(ctx->ev[4], st));
        stress_to_device(op);
        SVX_CUDA(cudaEventRecord(ctx->ev[5], st));
        copy_stress_out(op, sol);
        if (sol->u)
            SVX_CUDA(cudaMemcpyAsync(sol->u, op->u.p, op->n * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        sol->ms_stress = elapsed_ms(ctx->ev[4], ctx->ev[5]);
        SVX_CUDA(cudaStreamSynchronize(st));
        return SVX_OK;
    });
}

int svx_batch_solve(svx_ctx_t* ctx, int32_t count, const svx_flat_model_t* models,
                    const svx_solve_opts_t* opts, double* const* u, double* const* von_mises,
                    svx_batch_result_t* results, svx_batch_stats_t* stats, svx_error_t* err) {
    if (!ctx || count <= 0 || !models) return SVX_BAD_ARGUMENT;
    return guarded(ctx, err, [&]() -> int {
        svx_solve_opts_t o;
        svx_default_opts(&o);
        if (opts) o = *opts;
        std::vector<const svx_flat_model_t*> ptrs(static_cast<size_t>(count));
        for (int32_t k = 0; k < count; ++k) ptrs[k] = &models[k];
        std::vector<BatchModelOut> out;
        BatchRun run;
        run_batch(ctx, count, ptrs.data(), o, u, von_mises, out, run);
        int64_t total_it = 0, total_dof = 0;
        int failed = 0;
        for (int32_t k = 0; k < count; ++k) {
            const BatchModelOut& m = out[k];
            if (results) {
                results[k].iterations = m.iterations;
                results[k].residual = m.residual;
                results[k].status = m.status;
                results[k].reason = m.reason;
                results[k].cond_estimate = m.cond;
                results[k].nnz = m.nnz;
                results[k].elem_index = m.elem_index;
            }
            total_it += m.iterations;
            if (m.status == SVX_OK || m.status == SVX_NOT_CONVERGED)
                total_dof += models[k].n_nodes * models[k].ndof;
            failed += m.status != SVX_OK;
        }
        if (stats) {
            stats->ms_assemble = run.ms_assemble;
            stats->ms_solve = run.ms_solve;
            stats->ms_stress = run.ms_stress;
            stats->threads_per_cta = run.threads_per_cta;
            stats->lanes_per_node = run.lanes_per_node;
            stats->total_iterations = total_it;
            stats->total_dof = total_dof;
            stats->not_converged = failed;
            stats->cluster_members = run.cluster_members;
            stats->fp32_iterations = run.fp32_iterations;
        }
        clear_error(err);
        return SVX_OK;
    });
}

int svx_solve_flat(svx_ctx_t* ctx, const svx_flat_model_t* model, const svx_solve_opts_t* opts,
                   svx_solution_t* sol, svx_error_t* err) {
    if (!ctx) return SVX_BAD_ARGUMENT;
    return guarded(ctx, err, [&]() -> int {
        std::unique_ptr<svx_op> op(assemble_impl(ctx, model, 0));
        return solve_impl(op.get(), opts, sol, err);
    });
}

// heat::solve_thermal (heat.rs:52-98) on the device: the checks in the
// reference's order, conduction matrices (K1 form), the pattern and the
// fixed-order assembly at one dof per node (K3, K2), source and flux loads,
// temperature rows, the Jacobi diagonal and the FP64 PCG.
int svx_solve_thermal_flat(svx_ctx_t* ctx, const svx_thermal_model_t* m,
                           const svx_solve_opts_t* o, double* temperatures, int64_t* iterations,
                           double* residual, svx_error_t* err) {
    if (!ctx || !m) return SVX_BAD_ARGUMENT;
    return guarded(ctx, err, [&]() -> int {
        SVX_CUDA(cudaSetDevice(ctx->device));
        auto bad = [](const std::string& msg) { throw ModelFail{SVX_BAD_ARGUMENT, 0, -1, msg}; };
        if (m->n_nodes < 0 || m->n_elem < 0 || m->n_temp < 0 || m->n_flux < 0)
            bad("negative size");
        if (m->n_nodes > 0 && !m->xyz) bad("null xyz");
        if (m->n_elem > 0 && (!m->kind || !m->conn_ptr || !m->conn)) bad("null element array");
        if (m->n_temp > 0 && (!m->temp_node || !m->temp_value)) bad("null temperature array");
        if (m->n_flux > 0 && (!m->flux_elem || !m->flux_face || !m->flux_value))
            bad("null flux array");
        if (m->n_elem > 0 && m->conn_ptr[0] != 0) bad("conn_ptr[0] must be 0");
        auto eid = [&](int64_t e) { return m->elem_id ? m->elem_id[e] : uint32_t(e + 1); };
        int max_nn = 1;
        for (int64_t e = 0; e < m->n_elem; ++e) {
            const int nn = node_count(m->kind[e]);
            if (nn < 0) bad("unknown element kind " + std::to_string(int(m->kind[e])));
            if (m->conn_ptr[e + 1] - m->conn_ptr[e] != nn)
                bad("element " + std::to_string(eid(e)) + " has " +
                    std::to_string(m->conn_ptr[e + 1] - m->conn_ptr[e]) + " nodes, kind needs " +
                    std::to_string(nn));
            for (int64_t q = m->conn_ptr[e]; q < m->conn_ptr[e + 1]; ++q)
                if (m->conn[q] < 0 || m->conn[q] >= m->n_nodes)
                    bad("element " + std::to_string(eid(e)) + " references node index " +
                        std::to_string(m->conn[q]) + " out of range");
            max_nn = std::max(max_nn, nn);
        }
        for (int64_t q = 0; q < m->n_temp; ++q)
            if (m->temp_node[q] < 0 || m->temp_node[q] >= m->n_nodes)
                bad("temperature node index out of range");
        for (int64_t q = 0; q < m->n_flux; ++q)
            if (m->flux_elem[q] < 0 || m->flux_elem[q] >= m->n_elem)
                bad("flux element index out of range");
        // heat.rs:53-79
        if (m->n_nodes == 0 || m->n_elem == 0) throw ModelFail{SVX_EMPTY_MESH, 0, -1, "empty mesh"};
        for (int64_t e = 0; e < m->n_elem; ++e)
            if (m->kind[e] == SVX_B31)
                throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                                "beam elements have no conduction formulation (v1: plane and "
                                "solid only)"};
        if (m->n_temp == 0) throw ModelFail{SVX_NO_CONSTRAINTS, 0, -1, "no constraints"};
        if (!(m->thickness > 0.0) || !(m->conductivity > 0.0))
            throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                            "thickness and conductivity must be positive"};
        svx_solve_opts_t opts;
        svx_default_opts(&opts);
        if (o) opts = *o;
        if (opts.precision != SVX_FP64) bad("the conduction solve runs in FP64 only");

        std::unique_ptr<svx_op> op(new svx_op());
        op->ctx = ctx;
        op->n_nodes = m->n_nodes;
        op->n_elem = m->n_elem;
        op->ndof = 1;
        op->n = m->n_nodes;
        op->thickness = m->thickness;
        cudaStream_t st = ctx->stream;
        SVX_CUDA(cudaEventRecord(ctx->ev[6], st));
        upload(ctx, op->xyz, m->xyz, size_t(3 * m->n_nodes));
        upload(ctx, op->kind, m->kind, size_t(m->n_elem));
        upload(ctx, op->conn_ptr, m->conn_ptr, size_t(m->n_elem + 1));
        upload(ctx, op->conn, m->conn, size_t(m->conn_ptr[m->n_elem]));
        op->pat.max_nn = max_nn;
        op->pat.ke_stride = max_nn * max_nn;
        DBuf<double> ke, fe;
        ke.alloc(ctx->pool, size_t(m->n_elem) * op->pat.ke_stride + 1);
        fe.alloc(ctx->pool, size_t(m->n_elem) * max_nn + 1);
        // conduction_element runs first: its errors precede the flux checks
        const uint64_t g = integrate_conduction(ctx, op.get(), m->conductivity, m->has_source,
                                                m->source, ke.p, op->pat.ke_stride, fe.p);
        if (g != ~uint64_t(0)) {
            const int64_t e = int64_t(g >> 8);
            const int reason = int(g & 0xff);
            throw ModelFail{SVX_INVALID_MODEL, reason, e,
                            "element " + std::to_string(eid(e)) + ": " + reason_text(reason)};
        }
        // heat.rs:300-338: kinds, faces, edge lengths (host, flux order)
        static const char* debug_names[] = {"Cps3", "Cps4", "Cps8", "Cpe4",
                                            "Cpe8", "C3d8", "C3d4", "B31"};
        for (int64_t q = 0; q < m->n_flux; ++q) {
            const int64_t e = m->flux_elem[q];
            const int kd = m->kind[e];
            const int max_face = kd == SVX_CPS3 ? 3 : (kd == SVX_CPS4 || kd == SVX_CPE4) ? 4 : 0;
            if (!max_face)
                throw ModelFail{SVX_INVALID_MODEL, 0, e,
                                "heat flux on element " + std::to_string(eid(e)) + " (" +
                                    debug_names[kd] + ") unsupported (plane edges only)"};
            const int face = m->flux_face[q];
            if (face <= 0 || face > max_face)
                throw ModelFail{SVX_INVALID_MODEL, 0, e,
                                "element " + std::to_string(eid(e)) + " (" + debug_names[kd] +
                                    ") has no face " + std::to_string(face)};
            const int32_t* cn = m->conn + m->conn_ptr[e];
            const double* pa = m->xyz + 3 * int64_t(cn[face - 1]);
            const double* pb = m->xyz + 3 * int64_t(cn[face % max_face]);
            const double dx = pb[0] - pa[0], dy = pb[1] - pa[1];
            if (std::sqrt(dx * dx + dy * dy) == 0.0)
                throw ModelFail{SVX_INVALID_MODEL, 0, e,
                                "zero-length flux edge on element " + std::to_string(eid(e))};
        }
        build_pattern(ctx, op.get());
        op->vals.alloc(ctx->pool, op->pat.nnz + 1);
        assemble_values(ctx, op.get(), ke.p, op->pat.ke_stride, op->vals.p);
        ke.reset();
        DBuf<int64_t> d_fe_elem;
        DBuf<int32_t> d_face;
        DBuf<double> d_flux;
        if (m->n_flux > 0) {
            upload(ctx, d_fe_elem, m->flux_elem, size_t(m->n_flux));
            upload(ctx, d_face, m->flux_face, size_t(m->n_flux));
            upload(ctx, d_flux, m->flux_value, size_t(m->n_flux));
        }
        op->f.alloc(ctx->pool, size_t(op->n) + 1);
        thermal_loads(ctx, op.get(), fe.p, m->has_source, m->n_flux, d_fe_elem.p, d_face.p,
                      d_flux.p, op->f.p);
        fe.reset();
        // heat.rs:367-375: prescribed temperature per node, the last wins
        std::vector<double> pres(size_t(op->n), std::nan(""));
        for (int64_t q = 0; q < m->n_temp; ++q) pres[m->temp_node[q]] = m->temp_value[q];
        DBuf<double> d_pres;
        upload(ctx, d_pres, pres.data(), pres.size());
        apply_temperatures(ctx, op.get(), d_pres.p);
        jacobi_diagonal(ctx, op.get());
        SVX_CUDA(cudaEventRecord(ctx->ev[7], st));
        op->ms_assemble = elapsed_ms(ctx->ev[6], ctx->ev[7]);
        const long long max_iter = opts.max_iter > 0 ? opts.max_iter : default_max_iter(op->n);
        op->u.alloc(ctx->pool, size_t(op->n) + 1);
        const PcgResult r = pcg_fp64(ctx, op.get(), opts.tol, max_iter, opts.check_every, op->u.p);
        if (temperatures)
            SVX_CUDA(cudaMemcpyAsync(temperatures, op->u.p, sizeof(double) * size_t(op->n),
                                     cudaMemcpyDeviceToHost, st));
        SVX_CUDA(cudaStreamSynchronize(st));
        if (iterations) *iterations = r.iterations;
        if (residual) *residual = r.residual;
        if (r.status != PCG_CONVERGED) {
            std::string msg = "not converged after " + std::to_string(r.iterations) + " iterations";
            fill_error(err, SVX_NOT_CONVERGED, 0, -1, msg);
            if (err) {
                err->iterations = r.iterations;
                err->residual = r.residual;
            }
            ctx->last_error = msg;
            return SVX_NOT_CONVERGED;
        }
        clear_error(err);
        return SVX_OK;
    });
}

}  // extern "C"

// svx_internal.h - internal types shared by the host and device translation
// units of libsolvix_b200 (not part of the public C ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "solvix_gpu.h"

namespace svx {

// ------------------------------------------------------------------ errors
struct CudaFail {
    cudaError_t code;
    std::string where;
};

#define SVX_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) throw ::svx::CudaFail{e_, std::string(#call) + " @ " \
                                                         __FILE__ ":" + std::to_string(__LINE__)}; \
    } while (0)

// Kernels launched by this process through the library (graph nodes are
// counted when their graph is launched).
extern std::atomic<long long> g_launches;

#define SVX_LAUNCH_CHECK()                                     \
    do {                                                       \
        ::svx::g_launches.fetch_add(1, std::memory_order_relaxed); \
        SVX_CUDA(cudaGetLastError());                          \
    } while (0)

// Error thrown for model / argument problems (carries the svx_error_t).
struct ModelFail {
    int code;
    int reason;
    int64_t elem_index;
    std::string message;
};

// ------------------------------------------------------------------ memory
// Caching device allocator owned by a context: freed blocks are kept and
// reused by later requests of the same rounded size, so repeated solves on
// one context do not call cudaMalloc.
// Caching device allocator.  Freed blocks are kept by size class and handed
// out again; an optional arena (one cudaMalloc reserved up front, e.g. a
// server's whole budget) is carved first-fit with coalescing free ranges, so
// a steady stream of batches of varying size makes no driver calls.
class DevicePool {
public:
    explicit DevicePool(int device) : device_(device) {}
    ~DevicePool();
    void reserve(size_t bytes);  // the arena; throws ModelFail on failure
    void* alloc(size_t bytes);
    void release(void* p);
    void trim();  // return cached blocks to the driver (arena blocks to the arena)
    size_t bytes_in_use() const { return in_use_; }
    size_t bytes_cached() const { return cached_; }
    size_t arena_bytes() const { return arena_size_; }
    double malloc_ms() const { return malloc_ms_; }  // wall clock in cudaMalloc / cudaFree
    long long mallocs() const { return mallocs_; }

private:
    bool in_arena(void* p) const {
        return arena_ && static_cast<char*>(p) >= arena_ &&
               static_cast<char*>(p) < arena_ + arena_size_;
    }
    void* carve(size_t bytes);        // under mu_
    void give_back(void* p, size_t bytes);  // under mu_
    void flush_arena_cache();         // under mu_
    int device_;
    std::mutex mu_;
    std::multimap<size_t, void*> free_;      // size -> cached block
    std::map<void*, size_t> sizes_;          // live + cached blocks
    char* arena_ = nullptr;
    size_t arena_size_ = 0;
    std::map<size_t, size_t> ranges_;        // arena offset -> free length
    size_t in_use_ = 0, cached_ = 0;
    double malloc_ms_ = 0.0;
    long long mallocs_ = 0;
};

// Typed device buffer returned to the pool on destruction.
template <class T>
struct DBuf {
    DevicePool* pool = nullptr;
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : pool(o.pool), p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        reset();
        pool = o.pool; p = o.p; n = o.n;
        o.p = nullptr; o.n = 0;
        return *this;
    }
    ~DBuf() { reset(); }
    void alloc(DevicePool* pl, size_t count) {
        reset();
        pool = pl;
        n = count;
        p = count ? static_cast<T*>(pl->alloc(count * sizeof(T))) : nullptr;
    }
    void reset() {
        if (p && pool) pool->release(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Growable page-locked host buffer (one per context) that stages batched
// uploads and downloads, so they run as single DMA copies.  Contents are
// valid until the next get(); callers synchronise their stream first.
class PinnedBuffer {
public:
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() {
        if (p_) cudaFreeHost(p_);
    }
    void* get(size_t bytes) {
        if (bytes > cap_) {
            if (p_) cudaFreeHost(p_);
            p_ = nullptr;
            cap_ = 0;
            const size_t want = std::max(bytes, cap_ + cap_ / 2);
            cudaError_t e = cudaHostAlloc(&p_, want, cudaHostAllocDefault);
            if (e != cudaSuccess) {
                cudaGetLastError();
                p_ = nullptr;
                throw ModelFail{SVX_OOM, 0, -1, "page-locked host allocation failed"};
            }
            cap_ = want;
        }
        return p_;
    }

private:
    void* p_ = nullptr;
    size_t cap_ = 0;
};

}  // namespace svx

// ------------------------------------------------------------------ context
struct svx_ctx {
    int device = 0;
    int sm_count = 0;
    int64_t l2_bytes = 0;  // the device's L2 cache size
    int batch_choice[4] = {-1, -1, -1, -1};  // autotuned batched-PCG shape: FP64 (2D, 3D),
                                             // mixed (2D, 3D)
    cudaStream_t stream = nullptr;
    cudaStream_t pcg_stream = nullptr;  // batched PCG (lowest priority)
    cudaStream_t aux_stream = nullptr;  // its cluster kernel (lowest priority)
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    svx::DevicePool* pool = nullptr;
    svx::PinnedBuffer staging;  // batched host<->device staging
    std::string last_error;
    cudaEvent_t ev[8] = {};
    void* h_scalars = nullptr;  // page-locked PcgScalars of the context's solves
    // largest per-block shared-memory adjacency of the persistent PCG kernels
    // (bytes; 0 keeps it in global memory); SVX_SHARED_ADJ_MAX in the
    // environment at svx_ctx_create overrides the build's default
    long long shared_adj_max = -1;
    // systems with more nonzeros than this iterate with the standalone
    // kernels in a CUDA graph instead of the persistent kernel (-1: the
    // build's default); SVX_GRAPH_MIN_NNZ in the environment at
    // svx_ctx_create overrides it
    long long graph_min_nnz = -1;
    // plain FP64 solves below the graph threshold run the shared-memory
    // persistent kernel (1) or the register-vector one (0); SVX_PCG_SMEM in
    // the environment at svx_ctx_create overrides it
    int pcg_smem = 1;
    // the shared-memory kernel's form (-1: by size; 1 = two grid barriers an
    // iteration, neighbours forming p from z and the previous p; 0 = three,
    // p stored); SVX_PCG_ALG in the environment at svx_ctx_create sets it
    int pcg_alg = -1;
    // its nodes per warp step with all loads in flight (0: 1);
    // SVX_PCG_UNROLL sets it
    int pcg_unroll = 0;
    // lanes per node of the shared-memory kernel: 0 (or 8) eight, 32 (3D)
    // or 16 (2D) the degree-covering groups; SVX_PCG_LANES (measurements)
    int pcg_lanes = 0;
    // 1: the three-barrier form stages the gathered p window in shared
    // memory; SVX_PCG_STAGE=0 gathers from L2 (measurements)
    int pcg_stage = 1;
    // 1: the graph form's FP32 SpMV runs on the quad copy of the operator,
    // 0: on the node-block layout; SVX_FP32_QUADS (measurements)
    int fp32_quads = 1;
};

namespace svx {

// Device scalars of one PCG run (one 128-byte line).
struct PcgScalars {
    double rz;       // r . z of the current iterate
    double pap;      // p . Kp of the current iteration
    double alpha;
    double beta;
    double rr;       // r . r of the current iterate
    double bnorm;    // ||f||
    double tol;
    double res;      // ||r|| / ||f|| of the current iterate
    double rr_stop;  // stop with PCG_RELIABLE once r.r <= rr_stop (< 0: never)
    long long it;        // iterations completed
    long long max_iter;
    int status;          // PCG_RUNNING / PCG_CONVERGED / PCG_BREAKDOWN / PCG_MAXITER
    unsigned int count_a;  // last-block-done counters
    unsigned int count_b;
    unsigned int count_c;
};

enum { PCG_RUNNING = 0, PCG_CONVERGED = 1, PCG_BREAKDOWN = 2, PCG_MAXITER = 3,
       PCG_RELIABLE = 4 };

// State of the bounded grid-wide barrier of the persistent PCG kernel.
struct GridBarrier {
    unsigned int count;  // arrivals in this launch (zeroed by the host before each launch)
    unsigned int gen;    // unused
    int error;           // 1 after a bounded spin gave up
    int pad;
};

// Mesh pattern: node -> incident element slots and node adjacency.
struct Pattern {
    int64_t n_nodes = 0, n_elem = 0;
    int ndof = 0;
    int max_nn = 0;            // max nodes per element in the model
    int ke_stride = 0;         // doubles per element in the Ke buffer (max N^2)
    int64_t n_slots = 0;       // sum of nodes over elements
    int max_deg = 0;           // max node degree (adjacency incl. itself)
    int max_slots = 0;         // max incident slots of a node
    int64_t nnz = 0;
    int64_t n = 0;             // rows = n_nodes * ndof
    DBuf<int64_t> slot_ptr;    // [n_nodes + 1]
    DBuf<int32_t> slot_elem;   // [n_slots] element index, ascending per node
    DBuf<uint8_t> slot_local;  // [n_slots] local node position in the element
    DBuf<uint16_t> slot_map;   // [n_slots * max_nn] adjacency position of each element node
    DBuf<int64_t> adj_ptr;     // [n_nodes + 1]
    DBuf<int32_t> adj;         // sorted neighbour node indices
    DBuf<int64_t> node_base;   // [n_nodes + 1] first nnz of the node's rows
    DBuf<int32_t> row_ptr;     // [n + 1]
    DBuf<int32_t> col_idx;     // [nnz]
    DBuf<int32_t> diag_pos;    // [n] nnz index of the diagonal
};

}  // namespace svx

// ------------------------------------------------------------------ operator
struct svx_op {
    svx_ctx* ctx = nullptr;
    // model on the device
    int64_t n_nodes = 0, n_elem = 0, n = 0;
    int ndof = 0;
    double thickness = 1.0;
    svx::DBuf<double> xyz;
    svx::DBuf<uint8_t> kind;
    svx::DBuf<int64_t> conn_ptr;
    svx::DBuf<int32_t> conn;
    svx::DBuf<double> youngs, poisson;
    svx::DBuf<double> thick_elem;  // per-element thickness (batched models), else empty
    svx::Pattern pat;
    // assembled system
    svx::DBuf<double> vals;        // K after Dirichlet (the PCG operator)
    // K again with each node's values ordered (da, db, neighbour slot), the
    // slot fastest: the shared-memory PCG kernel's operand (ndof >= 2)
    svx::DBuf<double> valsT;
    svx::DBuf<float> vals32;       // FP32 copy (mixed precision)
    // the FP32 copy in quads (3D operators, graph-form SpMV): node i's 9
    // (da, db) rows over its neighbour slots, slot fastest, padded to a
    // multiple of 4 slots, from baseq[i]; adjq its neighbours padded with
    // the node itself, from baseq[i] / 9
    svx::DBuf<float> vals32q;
    svx::DBuf<int64_t> baseq;
    svx::DBuf<int32_t> adjq;
    int64_t n32q = 0;
    svx::DBuf<double> f;           // load vector after Dirichlet
    svx::DBuf<double> f_orig;      // load vector before Dirichlet
    svx::DBuf<double> inv_diag;
    svx::DBuf<uint8_t> is_fixed;
    // constrained rows of the unmodified K (reactions)
    int64_t n_fixed = 0;
    int64_t n_fixed_rows = 0;
    svx::DBuf<int64_t> fixed_row;      // [n_fixed] BC order
    svx::DBuf<int32_t> fixed_slot;     // [n_fixed] -> compact row
    svx::DBuf<int32_t> kc_ptr;         // [n_fixed_rows + 1]
    svx::DBuf<int32_t> kc_col;
    svx::DBuf<double> kc_val;
    std::vector<int64_t> h_fixed_row;
    std::vector<uint32_t> h_node_id;
    std::vector<uint32_t> h_elem_id;
    uint32_t flags = 0;
    double ms_upload_assemble = 0.0;
    // recovered fields (device)
    svx::DBuf<double> vm_elem, vm_node, react, disp3;
    // solution state
    svx::DBuf<double> u;
    bool has_solution = false;
    double cond_estimate = 0.0;
    double ms_assemble = 0.0;
    // K before Dirichlet is reconstructable only for the constrained rows;
    // svx_op_get_csr / svx_op_spmv use this copy when kept.
    svx::DBuf<double> vals_orig;
    // PCG tuning picked for this operator
    int spmv_group = 8;
    long long mixed_sloppy_iters = 0;  // FP32-operator iterations of the last mixed solve
    // >= 0: the operator holds the consistent mass matrix of this density
    // (svx_assemble_mass) instead of a stiffness
    double mass_rho = -1.0;
    int spmv_block = 256;
};

namespace svx {

// ---- host entry points implemented in the .cu files -------------------
// Pattern (svx_pattern.cu).
void build_pattern(svx_ctx* ctx, svx_op* op);
// Element integration into a Ke buffer; returns the first failing element
// as (index << 8 | reason) or UINT64_MAX (svx_element.cu).
uint64_t integrate_elements(svx_ctx* ctx, svx_op* op, double* ke, int ke_stride);
// Fixed-order gather of Ke into CSR values (svx_assemble.cu).
void assemble_values(svx_ctx* ctx, svx_op* op, const double* ke, int ke_stride, double* vals);
// Dirichlet + inverse diagonal + condition estimate (svx_assemble.cu).
void apply_dirichlet(svx_ctx* ctx, svx_op* op);
// Inverse diagonal and condition estimate of op->vals alone (svx_assemble.cu).
void jacobi_diagonal(svx_ctx* ctx, svx_op* op);
// The graph form's FP32 difference-form SpMV with p.q, for FP64 (V =
// double) or FP32 (V = float) vectors (svx_pcg.cu); at most `grid` blocks.
template <class V>
void launch_spmv_fp32(const svx_op* op, int G, unsigned grid, cudaStream_t st, const V* p, V* q,
                      double* partials, PcgScalars* s);
// Steady conduction (svx_element.cu): element conduction matrices into Ke
// slots and source loads into fe ([n_elem * max_nn]); returns the first
// failing element as (index << 8 | reason) or UINT64_MAX.
// consistent mass matrices (modal.rs:82-146) into ke; the first failing
// element as (index << 8 | reason), or all ones
uint64_t integrate_mass(svx_ctx* ctx, svx_op* op, double rho, double* ke, int ke_stride);
uint64_t integrate_conduction(svx_ctx* ctx, svx_op* op, double conductivity, int has_source,
                              double source, double* ke, int ke_stride, double* fe);
// f = element source loads (node order of the slots) + plane-edge fluxes.
void thermal_loads(svx_ctx* ctx, svx_op* op, const double* fe, int has_source, int64_t n_flux,
                   const int64_t* flux_elem, const int32_t* flux_face, const double* flux_value,
                   double* f);
// Nonhomogeneous temperature rows on op->vals / op->f (pres: NaN = free).
void apply_temperatures(svx_ctx* ctx, svx_op* op, const double* pres);
// Stress recovery (svx_element.cu).
void recover_stress(svx_ctx* ctx, svx_op* op, const double* u, double* vm_elem,
                    double* vm_node, double* reactions, double* disp3);

// PCG (svx_pcg.cu).
struct PcgResult {
    int status;
    long long iterations;
    double residual;
    double ms;
};
PcgResult pcg_fp64(svx_ctx* ctx, svx_op* op, double tol, long long max_iter, int check_every,
                   double* u_dev);
PcgResult pcg_mixed(svx_ctx* ctx, svx_op* op, double tol, long long max_iter, double inner_tol,
                    int check_every, double* u_dev, long long* outer_steps);
PcgResult pcg_defect_correction(svx_ctx* ctx, svx_op* op, double tol, long long max_iter,
                                double inner_tol, int check_every, double* u_dev,
                                long long* outer_steps);
void spmv_fp64(svx_ctx* ctx, const svx_op* op, const double* vals, const double* x, double* y);

// Direct path (svx_ldlt.cu): LDL^T of op->vals in the reverse Cuthill-McKee
// order, u_dev = K^-1 op->f.  Throws ModelFail with the reference's text on a
// failed pivot, SVX_OOM when the band does not fit on the device.
struct LdltOutcome {
    double residual = 0.0;   // ||f - K u|| / ||f|| (0 when f is zero)
    double cond = 0.0;       // max|D| / min|D|
    int64_t bandwidth = 0;   // half-bandwidth of K in the RCM order
    double ms = 0.0;         // device time: band fill, factorization, solves, residual
};
LdltOutcome ldlt_direct(svx_ctx* ctx, svx_op* op, double* u_dev);
int choose_spmv_group(const svx_op* op);
// Average device time (ms) of the three FP64 PCG iteration kernels
// (spmv_dot, update, p_update) over `reps` back-to-back launches each.
void time_iteration_kernels(svx_ctx* ctx, svx_op* op, int reps, double* ms4);

// Batched PCG over a block-diagonal concatenation of independent models
// (svx_pcg.cu).  node_off[count + 1] delimits each instance's nodes.
struct BatchStats {
    double ms_solve = 0.0;
    int64_t fp32_iterations = 0;  // mixed form: iterations on the FP32 operator
    int cluster_members = 0;      // members solved by the cluster kernel
    std::vector<int64_t> member_nnz;  // nonzeros of each member's K
    int threads_per_cta = 0;
    int lanes_per_node = 0;
};
// FP32 difference-form copy of the operator for the mixed forms (svx_pcg.cu).
void build_fp32_operator(svx_ctx* ctx, svx_op* op);
const double* transposed_values(svx_ctx* ctx, svx_op* op);
void batch_pcg(svx_ctx* ctx, svx_op* op, int count, const std::vector<int64_t>& node_off,
               const std::vector<double>& tol, const std::vector<int64_t>& max_iter,
               std::vector<int64_t>& it, std::vector<double>& res, std::vector<int32_t>& status,
               std::vector<double>& cond, BatchStats* stats, bool mixed = false);

// Per-member outcome of one batch (svx_api.cpp).
struct BatchModelOut {
    int64_t iterations = 0;
    double residual = 0.0;
    int32_t status = 0;      // svx_status
    int32_t reason = 0;      // svx_elem_reason for InvalidModel
    int64_t elem_index = -1;  // failing element (index within the member)
    double cond = 0.0;
    int64_t nnz = 0;
    std::string message;
};
struct BatchRun {
    double ms_assemble = 0.0, ms_solve = 0.0, ms_stress = 0.0;
    // host wall clock of the phases: checks + concatenation, upload +
    // assembly, batched PCG (incl. launch and result copies), outputs
    double wall_prep = 0.0, wall_assemble = 0.0, wall_solve = 0.0, wall_output = 0.0;
    int threads_per_cta = 0, lanes_per_node = 0, cluster_members = 0;
    int64_t fp32_iterations = 0;
};
void check_batch_member(const svx_flat_model_t* m);
void run_batch(svx_ctx* ctx, int32_t count, const svx_flat_model_t* const* models,
               const svx_solve_opts_t& o, double* const* u, double* const* vm,
               std::vector<BatchModelOut>& out, BatchRun& run);

// Generic device helpers (svx_pattern.cu).
void exclusive_scan_i64(svx_ctx* ctx, const int64_t* in, int64_t* out, int64_t n,
                        int64_t* total_host);

}  // namespace svx

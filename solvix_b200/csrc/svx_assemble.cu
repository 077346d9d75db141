// svx_assemble.cu - K2 fixed-order assembly and K4 Dirichlet / Jacobi
// diagonal.
//
// K2 replaces scatter + csr_from_triplets (crates/solvix-core/src/
// assembly.rs:87-133) without triplets and without float atomics.  One warp
// owns one node: its ndof CSR rows are a contiguous block of
// ndof * ndof * deg values (the pattern is node adjacency x dense ndof
// blocks).  The warp walks the node's incident (element, local position)
// slots in ascending order and adds the element's ndof rows of Ke into a
// shared-memory copy of the block, each value landing at the position the
// precomputed element-to-nonzero map gives.  Every CSR value is therefore
//   0.0 + Ke_e1 + Ke_e2 + ...   in ascending element order,
// which is the reference's triplet-stream order (diagonal seed first, then
// elements in enumeration order): deterministic run to run, and bit-equal to
// the oracle's stable-order assembly.
//
// K4 replaces apply_dirichlet (solver.rs:45-62), the inverse diagonal of
// pcg (solver.rs:96-107) and jacobi_cond (lib.rs:634-644).  The rows of the
// unmodified K at constrained dofs are kept in a compact CSR for reactions
// (stress.rs:103-118) instead of cloning all of K (lib.rs:623-628).

#include "svx_internal.h"

#include <algorithm>
#include <cmath>

namespace svx {

namespace {

constexpr int ASM_WARPS = 8;

__global__ void __launch_bounds__(ASM_WARPS * 32)
assemble_kernel(int64_t n_nodes, int ndof, int max_nn, int acc_stride,
                const int64_t* __restrict__ slot_ptr, const int32_t* __restrict__ slot_elem,
                const uint8_t* __restrict__ slot_local, const uint16_t* __restrict__ slot_map,
                const int64_t* __restrict__ conn_ptr, const int64_t* __restrict__ adj_ptr,
                const int64_t* __restrict__ node_base, const double* __restrict__ ke,
                int ke_stride, double* __restrict__ vals) {
    extern __shared__ double acc_all[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    double* acc = acc_all + size_t(w) * acc_stride;
    const int64_t warps_total = int64_t(gridDim.x) * ASM_WARPS;
    for (int64_t i = int64_t(blockIdx.x) * ASM_WARPS + w; i < n_nodes; i += warps_total) {
        const int64_t deg = adj_ptr[i + 1] - adj_ptr[i];
        const int64_t base = node_base[i];
        if (deg == 0) {  // unreferenced node: only the diagonal seeds
            if (lane < ndof) vals[base + lane] = 0.0;
            continue;
        }
        const int rowlen = int(ndof * deg);
        const int total = ndof * rowlen;
        for (int q = lane; q < total; q += 32) acc[q] = 0.0;
        __syncwarp();
        const int64_t s1 = slot_ptr[i + 1];
        for (int64_t s = slot_ptr[i]; s < s1; ++s) {
            const int64_t e = slot_elem[s];
            const int a = slot_local[s];
            const int nn = int(conn_ptr[e + 1] - conn_ptr[e]);
            const int N = nn * ndof;
            const uint16_t* map = slot_map + s * max_nn;
            const double* rows = ke + e * int64_t(ke_stride) + int64_t(a) * ndof * N;
            // an element that repeats a node maps two columns to one target
            bool dup = false;
            for (int c = 0; c < nn; ++c)
                for (int c2 = c + 1; c2 < nn; ++c2) dup |= (map[c] == map[c2]);
            if (!dup) {
                for (int t = lane; t < ndof * N; t += 32) {
                    int da = t / N, col = t - da * N;
                    int c = col / ndof, db = col - c * ndof;
                    acc[da * rowlen + int(map[c]) * ndof + db] += rows[t];
                }
            } else if (lane == 0) {
                for (int t = 0; t < ndof * N; ++t) {
                    int da = t / N, col = t - da * N;
                    int c = col / ndof, db = col - c * ndof;
                    acc[da * rowlen + int(map[c]) * ndof + db] += rows[t];
                }
            }
            __syncwarp();
        }
        for (int q = lane; q < total; q += 32) vals[base + q] = acc[q];
        __syncwarp();
    }
}

__global__ void mark_fixed_kernel(int64_t n_fixed, const int64_t* __restrict__ rows,
                                  uint8_t* __restrict__ is_fixed) {
    int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n_fixed) is_fixed[rows[k]] = 1;
}

// Row lengths of the compact constrained rows.
__global__ void fixed_len_kernel(int64_t m, const int64_t* __restrict__ rows,
                                 const int32_t* __restrict__ row_ptr, int32_t* __restrict__ len) {
    int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < m) len[k] = row_ptr[rows[k] + 1] - row_ptr[rows[k]];
}

// Copy the unmodified constrained rows (one warp per row).
__global__ void fixed_copy_kernel(int64_t m, const int64_t* __restrict__ rows,
                                  const int32_t* __restrict__ row_ptr,
                                  const int32_t* __restrict__ col_idx,
                                  const double* __restrict__ vals,
                                  const int32_t* __restrict__ kc_ptr, int32_t* __restrict__ kc_col,
                                  double* __restrict__ kc_val) {
    int64_t k = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (k >= m) return;
    int32_t a = row_ptr[rows[k]], len = row_ptr[rows[k] + 1] - a;
    int32_t o = kc_ptr[k];
    for (int j = lane; j < len; j += 32) {
        kc_col[o + j] = col_idx[a + j];
        kc_val[o + j] = vals[a + j];
    }
}

// Symmetric elimination: an entry dies if its row or column is constrained;
// a constrained diagonal becomes 1 (one warp per row).
__global__ void dirichlet_kernel(int64_t n, const int32_t* __restrict__ row_ptr,
                                 const int32_t* __restrict__ col_idx,
                                 const uint8_t* __restrict__ is_fixed, double* __restrict__ vals,
                                 double* __restrict__ f) {
    int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (r >= n) return;
    const bool fr = is_fixed[r] != 0;
    for (int32_t j = row_ptr[r] + lane; j < row_ptr[r + 1]; j += 32) {
        int32_t c = col_idx[j];
        if (fr || is_fixed[c]) vals[j] = (c == r) ? 1.0 : 0.0;
    }
    if (fr && lane == 0) f[r] = 0.0;
}

// inv_diag = 1/K_ii (0 when K_ii == 0) and the extreme |K_ii| per block.
__global__ void diag_kernel(int64_t n, const int32_t* __restrict__ diag_pos,
                            const double* __restrict__ vals, double* __restrict__ inv_diag,
                            double* __restrict__ block_hi, double* __restrict__ block_lo) {
    __shared__ double shi[256], slo[256];
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    double hi = 0.0, lo = INFINITY;
    if (i < n) {
        double d = vals[diag_pos[i]];
        inv_diag[i] = (d == 0.0) ? 0.0 : 1.0 / d;
        double a = fabs(d);
        hi = fmax(hi, a);
        lo = fmin(lo, a);
    }
    shi[threadIdx.x] = hi;
    slo[threadIdx.x] = lo;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            shi[threadIdx.x] = fmax(shi[threadIdx.x], shi[threadIdx.x + off]);
            slo[threadIdx.x] = fmin(slo[threadIdx.x], slo[threadIdx.x + off]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        block_hi[blockIdx.x] = shi[0];
        block_lo[blockIdx.x] = slo[0];
    }
}

inline unsigned blocks_for(int64_t n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace

void assemble_values(svx_ctx* ctx, svx_op* op, const double* ke, int ke_stride, double* vals) {
    const Pattern& P = op->pat;
    if (op->n_nodes == 0) return;
    const int acc_stride = op->ndof * op->ndof * std::max(1, P.max_deg);
    int warps = ASM_WARPS;
    size_t smem = size_t(warps) * acc_stride * sizeof(double);
    if (smem > 200 * 1024)
        throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                        "node degree " + std::to_string(P.max_deg) +
                            " exceeds the shared-memory block of the assembly kernel"};
    if (smem > 48 * 1024)
        SVX_CUDA(cudaFuncSetAttribute(assemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(smem)));
    int64_t blocks = (op->n_nodes + warps - 1) / warps;
    int64_t cap = int64_t(ctx->sm_count) * 32;
    if (blocks > cap) blocks = cap;
    assemble_kernel<<<unsigned(blocks), warps * 32, smem, ctx->stream>>>(
        op->n_nodes, op->ndof, P.max_nn, acc_stride, P.slot_ptr.p, P.slot_elem.p, P.slot_local.p,
        P.slot_map.p, op->conn_ptr.p, P.adj_ptr.p, P.node_base.p, ke, ke_stride, vals);
    SVX_LAUNCH_CHECK();
}

void apply_dirichlet(svx_ctx* ctx, svx_op* op) {
    cudaStream_t st = ctx->stream;
    const Pattern& P = op->pat;
    const int64_t n = op->n;
    op->is_fixed.alloc(ctx->pool, n + 1);
    SVX_CUDA(cudaMemsetAsync(op->is_fixed.p, 0, n + 1, st));
    if (op->n_fixed > 0) {
        mark_fixed_kernel<<<blocks_for(op->n_fixed, 256), 256, 0, st>>>(
            op->n_fixed, op->fixed_row.p, op->is_fixed.p);
        SVX_LAUNCH_CHECK();
    }
    // compact copy of the constrained rows of the unmodified K
    std::vector<int64_t> uniq(op->h_fixed_row);
    std::sort(uniq.begin(), uniq.end());
    uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
    const int64_t m = int64_t(uniq.size());
    op->n_fixed_rows = m;
    std::vector<int32_t> slot(op->n_fixed);
    for (int64_t k = 0; k < op->n_fixed; ++k)
        slot[k] = int32_t(std::lower_bound(uniq.begin(), uniq.end(), op->h_fixed_row[k]) -
                          uniq.begin());
    op->fixed_slot.alloc(ctx->pool, op->n_fixed + 1);
    op->kc_ptr.alloc(ctx->pool, m + 1);
    if (m > 0) {
        DBuf<int64_t> d_uniq;
        DBuf<int32_t> d_len;
        d_uniq.alloc(ctx->pool, m);
        d_len.alloc(ctx->pool, m);
        SVX_CUDA(cudaMemcpyAsync(d_uniq.p, uniq.data(), m * sizeof(int64_t),
                                 cudaMemcpyHostToDevice, st));
        SVX_CUDA(cudaMemcpyAsync(op->fixed_slot.p, slot.data(), op->n_fixed * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, st));
        fixed_len_kernel<<<blocks_for(m, 256), 256, 0, st>>>(m, d_uniq.p, P.row_ptr.p, d_len.p);
        SVX_LAUNCH_CHECK();
        std::vector<int32_t> len(m), ptr(m + 1, 0);
        SVX_CUDA(cudaMemcpyAsync(len.data(), d_len.p, m * sizeof(int32_t),
                                 cudaMemcpyDeviceToHost, st));
        SVX_CUDA(cudaStreamSynchronize(st));
        for (int64_t k = 0; k < m; ++k) ptr[k + 1] = ptr[k] + len[k];
        SVX_CUDA(cudaMemcpyAsync(op->kc_ptr.p, ptr.data(), (m + 1) * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, st));
        op->kc_col.alloc(ctx->pool, size_t(ptr[m]) + 1);
        op->kc_val.alloc(ctx->pool, size_t(ptr[m]) + 1);
        fixed_copy_kernel<<<blocks_for(m * 32, 256), 256, 0, st>>>(
            m, d_uniq.p, P.row_ptr.p, P.col_idx.p, op->vals.p, op->kc_ptr.p, op->kc_col.p,
            op->kc_val.p);
        SVX_LAUNCH_CHECK();
        SVX_CUDA(cudaStreamSynchronize(st));
    }
    // f_orig keeps the unmodified loads; f gets the eliminated copy
    op->f.alloc(ctx->pool, n + 1);
    SVX_CUDA(cudaMemcpyAsync(op->f.p, op->f_orig.p, n * sizeof(double), cudaMemcpyDeviceToDevice,
                             st));
    if (n > 0) {
        dirichlet_kernel<<<blocks_for(n * 32, 256), 256, 0, st>>>(
            n, P.row_ptr.p, P.col_idx.p, op->is_fixed.p, op->vals.p, op->f.p);
        SVX_LAUNCH_CHECK();
    }
    jacobi_diagonal(ctx, op);
}

// Jacobi inverse diagonal and cond estimate of the modified K
void jacobi_diagonal(svx_ctx* ctx, svx_op* op) {
    cudaStream_t st = ctx->stream;
    const Pattern& P = op->pat;
    const int64_t n = op->n;
    op->inv_diag.alloc(ctx->pool, n + 1);
    const int64_t nb = (n + 255) / 256;
    DBuf<double> bhi, blo;
    bhi.alloc(ctx->pool, nb + 1);
    blo.alloc(ctx->pool, nb + 1);
    if (n > 0) {
        diag_kernel<<<unsigned(nb), 256, 0, st>>>(n, P.diag_pos.p, op->vals.p, op->inv_diag.p,
                                                  bhi.p, blo.p);
        SVX_LAUNCH_CHECK();
    }
    std::vector<double> hhi(nb), hlo(nb);
    if (nb > 0) {
        SVX_CUDA(cudaMemcpyAsync(hhi.data(), bhi.p, nb * sizeof(double), cudaMemcpyDeviceToHost,
                                 st));
        SVX_CUDA(cudaMemcpyAsync(hlo.data(), blo.p, nb * sizeof(double), cudaMemcpyDeviceToHost,
                                 st));
    }
    SVX_CUDA(cudaStreamSynchronize(st));
    double hi = 0.0, lo = INFINITY;
    for (int64_t b = 0; b < nb; ++b) {
        hi = std::fmax(hi, hhi[b]);
        lo = std::fmin(lo, hlo[b]);
    }
    op->cond_estimate = hi / lo;
}

}  // namespace svx

// svx_pattern.cu - K3: the CSR pattern of the global stiffness, built on the
// device from the mesh connectivity.
//
// The reference builds its pattern implicitly: every element pushes all
// N x N (row, col) triplets of its node pairs, zeros included, and every
// dof gets a diagonal seed (crates/solvix-core/src/assembly.rs:120-133,
// :299-302); csr_from_triplets then sorts each row by column
// (assembly.rs:87-116).  The resulting pattern is exactly
//   row (i, a): columns (j, b) for every node j sharing an element with i
//               (i itself included) and every dof b, ascending;
//   a node used by no element keeps only its diagonal.
// This file computes that pattern without materialising triplets:
//   1. node -> incident (element, local position) slots, sorted ascending
//      (counting pass, scan, atomic fill, per-node insertion sort);
//   2. node adjacency = sorted union of the slots' element nodes;
//   3. row_ptr / col_idx / diagonal positions from the node blocks;
//   4. the element-to-nonzero map: for each slot and each node of the slot's
//      element, its position in the owner node's adjacency.
// All integer work; the result is bit-exact against the oracle's CSR.

#include "svx_internal.h"

#include <climits>

namespace svx {

namespace {

constexpr int SCAN_T = 512;
constexpr int SCAN_I = 8;
constexpr int64_t SCAN_TILE = int64_t(SCAN_T) * SCAN_I;

__global__ void scan_tile_kernel(const int64_t* __restrict__ in, int64_t* __restrict__ out,
                                 int64_t n, int64_t* __restrict__ tile_sums) {
    __shared__ int64_t s[SCAN_T];
    const int64_t base = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_I;
    int64_t v[SCAN_I];
    int64_t sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        int64_t idx = base + k;
        v[k] = idx < n ? in[idx] : 0;
        sum += v[k];
    }
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < SCAN_T; off <<= 1) {
        int64_t t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    int64_t run = s[threadIdx.x] - sum;
#pragma unroll
    for (int k = 0; k < SCAN_I; ++k) {
        int64_t idx = base + k;
        if (idx < n) out[idx] = run;
        run += v[k];
    }
    if (threadIdx.x == SCAN_T - 1) tile_sums[blockIdx.x] = s[SCAN_T - 1];
}

__global__ void scan_add_kernel(int64_t* __restrict__ out, int64_t n,
                                const int64_t* __restrict__ tile_offsets) {
    int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx < n) out[idx] += tile_offsets[idx / SCAN_TILE];
}

__global__ void scan_total_kernel(const int64_t* in, int64_t* out, int64_t n) {
    out[n] = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

void scan_rec(svx_ctx* ctx, const int64_t* in, int64_t* out, int64_t n) {
    if (n <= 0) return;
    int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    DBuf<int64_t> sums, offs;
    sums.alloc(ctx->pool, tiles + 1);
    scan_tile_kernel<<<unsigned(tiles), SCAN_T, 0, ctx->stream>>>(in, out, n, sums.p);
    SVX_LAUNCH_CHECK();
    if (tiles > 1) {
        offs.alloc(ctx->pool, tiles + 1);
        scan_rec(ctx, sums.p, offs.p, tiles);
        scan_add_kernel<<<unsigned((n + 255) / 256), 256, 0, ctx->stream>>>(out, n, offs.p);
        SVX_LAUNCH_CHECK();
    }
    // keep the temporaries alive until the stream has consumed them
    SVX_CUDA(cudaStreamSynchronize(ctx->stream));
}

// ---- 1. incidence ---------------------------------------------------------
__global__ void count_incidence_kernel(const int64_t* __restrict__ conn_ptr,
                                       const int32_t* __restrict__ conn, int64_t n_elem,
                                       unsigned long long* __restrict__ cnt) {
    int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    for (int64_t q = conn_ptr[e]; q < conn_ptr[e + 1]; ++q)
        atomicAdd(&cnt[conn[q]], 1ull);
}

__global__ void fill_incidence_kernel(const int64_t* __restrict__ conn_ptr,
                                      const int32_t* __restrict__ conn, int64_t n_elem,
                                      const int64_t* __restrict__ slot_ptr,
                                      unsigned long long* __restrict__ cursor,
                                      int64_t* __restrict__ keys) {
    int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    int64_t q0 = conn_ptr[e];
    for (int64_t q = q0; q < conn_ptr[e + 1]; ++q) {
        int32_t node = conn[q];
        unsigned long long pos = atomicAdd(&cursor[node], 1ull);
        keys[slot_ptr[node] + int64_t(pos)] = (e << 8) | int64_t(q - q0);
    }
}

// Per-node insertion sort of the (element, local) keys, then split.
__global__ void sort_slots_kernel(int64_t n_nodes, const int64_t* __restrict__ slot_ptr,
                                  int64_t* __restrict__ keys, int32_t* __restrict__ slot_elem,
                                  uint8_t* __restrict__ slot_local, int* max_slots) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t a = slot_ptr[i], b = slot_ptr[i + 1];
    for (int64_t x = a + 1; x < b; ++x) {
        int64_t key = keys[x];
        int64_t y = x;
        while (y > a && keys[y - 1] > key) {
            keys[y] = keys[y - 1];
            --y;
        }
        keys[y] = key;
    }
    for (int64_t x = a; x < b; ++x) {
        slot_elem[x] = int32_t(keys[x] >> 8);
        slot_local[x] = uint8_t(keys[x] & 0xff);
    }
    atomicMax(max_slots, int(b - a));
}

// ---- 2. adjacency ------------------------------------------------------------
// Smallest element node > last over the node's slots (INT_MAX if none).
__device__ __forceinline__ int32_t next_neighbour(int64_t s0, int64_t s1,
                                                  const int32_t* __restrict__ slot_elem,
                                                  const int64_t* __restrict__ conn_ptr,
                                                  const int32_t* __restrict__ conn, int32_t last) {
    int32_t best = INT_MAX;
    for (int64_t s = s0; s < s1; ++s) {
        int64_t e = slot_elem[s];
        for (int64_t q = conn_ptr[e]; q < conn_ptr[e + 1]; ++q) {
            int32_t v = conn[q];
            if (v > last && v < best) best = v;
        }
    }
    return best;
}

__global__ void adjacency_kernel(int64_t n_nodes, const int64_t* __restrict__ slot_ptr,
                                 const int32_t* __restrict__ slot_elem,
                                 const int64_t* __restrict__ conn_ptr,
                                 const int32_t* __restrict__ conn, int64_t* __restrict__ deg,
                                 const int64_t* __restrict__ adj_ptr, int32_t* __restrict__ adj,
                                 int* max_deg) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t s0 = slot_ptr[i], s1 = slot_ptr[i + 1];
    int32_t last = -1;
    int64_t d = 0;
    for (;;) {
        int32_t nx = next_neighbour(s0, s1, slot_elem, conn_ptr, conn, last);
        if (nx == INT_MAX) break;
        if (adj) adj[adj_ptr[i] + d] = nx;
        ++d;
        last = nx;
    }
    if (deg) {
        deg[i] = d;
        atomicMax(max_deg, int(d));
    }
}

// ---- 3. CSR rows --------------------------------------------------------------
__global__ void node_nnz_kernel(int64_t n_nodes, int ndof, const int64_t* __restrict__ adj_ptr,
                                int64_t* __restrict__ node_nnz) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t d = adj_ptr[i + 1] - adj_ptr[i];
    node_nnz[i] = d > 0 ? int64_t(ndof) * ndof * d : int64_t(ndof);
}

// One warp per node writes its ndof rows.
__global__ void csr_rows_kernel(int64_t n_nodes, int ndof, const int64_t* __restrict__ adj_ptr,
                                const int32_t* __restrict__ adj,
                                const int64_t* __restrict__ node_base,
                                int32_t* __restrict__ row_ptr, int32_t* __restrict__ col_idx,
                                int32_t* __restrict__ diag_pos, int64_t n_rows) {
    int64_t i = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= n_nodes) return;
    int64_t a0 = adj_ptr[i];
    int64_t d = adj_ptr[i + 1] - a0;
    int64_t base = node_base[i];
    if (d == 0) {
        if (lane < ndof) {
            int64_t row = i * ndof + lane;
            row_ptr[row] = int32_t(base + lane);
            col_idx[base + lane] = int32_t(row);
            diag_pos[row] = int32_t(base + lane);
        }
    } else {
        int64_t rowlen = int64_t(ndof) * d;
        if (lane < ndof) {
            int64_t row = i * ndof + lane;
            row_ptr[row] = int32_t(base + lane * rowlen);
            // position of i in its own adjacency (binary search)
            int64_t lo = 0, hi = d - 1;
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (adj[a0 + mid] < i) lo = mid + 1; else hi = mid;
            }
            diag_pos[row] = int32_t(base + lane * rowlen + lo * ndof + lane);
        }
        int64_t total = rowlen * ndof;
        for (int64_t q = lane; q < total; q += 32) {
            int64_t r = q % rowlen;
            int64_t k = r / ndof;
            int64_t b = r % ndof;
            col_idx[base + q] = int32_t(int64_t(adj[a0 + k]) * ndof + b);
        }
    }
    if (i == n_nodes - 1 && lane == 0) row_ptr[n_rows] = int32_t(node_base[n_nodes]);
}

// ---- 4. element -> nonzero map --------------------------------------------------
__global__ void slot_map_kernel(int64_t n_nodes, int max_nn, const int64_t* __restrict__ slot_ptr,
                                const int32_t* __restrict__ slot_elem,
                                const int64_t* __restrict__ conn_ptr,
                                const int32_t* __restrict__ conn,
                                const int64_t* __restrict__ adj_ptr,
                                const int32_t* __restrict__ adj, uint16_t* __restrict__ slot_map) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t a0 = adj_ptr[i];
    int64_t d = adj_ptr[i + 1] - a0;
    for (int64_t s = slot_ptr[i]; s < slot_ptr[i + 1]; ++s) {
        int64_t e = slot_elem[s];
        int64_t q0 = conn_ptr[e];
        int nn = int(conn_ptr[e + 1] - q0);
        for (int c = 0; c < nn; ++c) {
            int32_t v = conn[q0 + c];
            int64_t lo = 0, hi = d - 1;
            while (lo < hi) {
                int64_t mid = (lo + hi) >> 1;
                if (adj[a0 + mid] < v) lo = mid + 1; else hi = mid;
            }
            slot_map[s * max_nn + c] = uint16_t(lo);
        }
    }
}

inline unsigned blocks_for(int64_t n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace

void exclusive_scan_i64(svx_ctx* ctx, const int64_t* in, int64_t* out, int64_t n,
                        int64_t* total_host) {
    scan_rec(ctx, in, out, n);
    scan_total_kernel<<<1, 1, 0, ctx->stream>>>(in, out, n);
    SVX_LAUNCH_CHECK();
    if (total_host) {
        SVX_CUDA(cudaMemcpyAsync(total_host, out + n, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        SVX_CUDA(cudaStreamSynchronize(ctx->stream));
    }
}

void build_pattern(svx_ctx* ctx, svx_op* op) {
    Pattern& P = op->pat;
    cudaStream_t st = ctx->stream;
    const int64_t nn = op->n_nodes, ne = op->n_elem;
    P.n_nodes = nn;
    P.n_elem = ne;
    P.ndof = op->ndof;
    P.n = nn * op->ndof;

    DBuf<int> flags;  // [0] max_slots, [1] max_deg
    flags.alloc(ctx->pool, 2);
    SVX_CUDA(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), st));

    // 1. incidence
    DBuf<int64_t> cnt, cursor, keys;
    cnt.alloc(ctx->pool, nn + 1);
    cursor.alloc(ctx->pool, nn + 1);
    SVX_CUDA(cudaMemsetAsync(cnt.p, 0, (nn + 1) * sizeof(int64_t), st));
    SVX_CUDA(cudaMemsetAsync(cursor.p, 0, (nn + 1) * sizeof(int64_t), st));
    if (ne > 0) {
        count_incidence_kernel<<<blocks_for(ne, 256), 256, 0, st>>>(
            op->conn_ptr.p, op->conn.p, ne, reinterpret_cast<unsigned long long*>(cnt.p));
        SVX_LAUNCH_CHECK();
    }
    P.slot_ptr.alloc(ctx->pool, nn + 1);
    int64_t n_slots = 0;
    exclusive_scan_i64(ctx, cnt.p, P.slot_ptr.p, nn, &n_slots);
    P.n_slots = n_slots;
    keys.alloc(ctx->pool, n_slots + 1);
    P.slot_elem.alloc(ctx->pool, n_slots + 1);
    P.slot_local.alloc(ctx->pool, n_slots + 1);
    if (ne > 0) {
        fill_incidence_kernel<<<blocks_for(ne, 256), 256, 0, st>>>(
            op->conn_ptr.p, op->conn.p, ne, P.slot_ptr.p,
            reinterpret_cast<unsigned long long*>(cursor.p), keys.p);
        SVX_LAUNCH_CHECK();
    }
    if (nn > 0) {
        sort_slots_kernel<<<blocks_for(nn, 128), 128, 0, st>>>(nn, P.slot_ptr.p, keys.p,
                                                               P.slot_elem.p, P.slot_local.p,
                                                               flags.p);
        SVX_LAUNCH_CHECK();
    }
    keys.reset();
    cursor.reset();

    // 2. adjacency: count, scan, fill
    DBuf<int64_t> deg;
    deg.alloc(ctx->pool, nn + 1);
    if (nn > 0) {
        adjacency_kernel<<<blocks_for(nn, 128), 128, 0, st>>>(
            nn, P.slot_ptr.p, P.slot_elem.p, op->conn_ptr.p, op->conn.p, deg.p, nullptr,
            nullptr, flags.p + 1);
        SVX_LAUNCH_CHECK();
    }
    P.adj_ptr.alloc(ctx->pool, nn + 1);
    int64_t n_adj = 0;
    exclusive_scan_i64(ctx, deg.p, P.adj_ptr.p, nn, &n_adj);
    P.adj.alloc(ctx->pool, n_adj + 1);
    if (nn > 0) {
        adjacency_kernel<<<blocks_for(nn, 128), 128, 0, st>>>(
            nn, P.slot_ptr.p, P.slot_elem.p, op->conn_ptr.p, op->conn.p, nullptr, P.adj_ptr.p,
            P.adj.p, nullptr);
        SVX_LAUNCH_CHECK();
    }

    // 3. rows
    DBuf<int64_t> node_nnz;
    node_nnz.alloc(ctx->pool, nn + 1);
    if (nn > 0) {
        node_nnz_kernel<<<blocks_for(nn, 256), 256, 0, st>>>(nn, op->ndof, P.adj_ptr.p,
                                                             node_nnz.p);
        SVX_LAUNCH_CHECK();
    }
    P.node_base.alloc(ctx->pool, nn + 1);
    int64_t nnz = 0;
    exclusive_scan_i64(ctx, node_nnz.p, P.node_base.p, nn, &nnz);
    if (nnz >= int64_t(INT_MAX))
        throw ModelFail{SVX_OOM, 0, -1,
                        "stiffness has " + std::to_string(nnz) +
                            " nonzeros; the int32 CSR indices of the device path hold < 2^31"};
    P.nnz = nnz;
    P.row_ptr.alloc(ctx->pool, P.n + 1);
    P.col_idx.alloc(ctx->pool, nnz + 1);
    P.diag_pos.alloc(ctx->pool, P.n + 1);
    if (nn > 0) {
        csr_rows_kernel<<<blocks_for(nn * 32, 256), 256, 0, st>>>(
            nn, op->ndof, P.adj_ptr.p, P.adj.p, P.node_base.p, P.row_ptr.p, P.col_idx.p,
            P.diag_pos.p, P.n);
        SVX_LAUNCH_CHECK();
    }

    // 4. element -> nonzero map
    P.slot_map.alloc(ctx->pool, size_t(n_slots) * P.max_nn + 1);
    if (nn > 0) {
        slot_map_kernel<<<blocks_for(nn, 128), 128, 0, st>>>(
            nn, P.max_nn, P.slot_ptr.p, P.slot_elem.p, op->conn_ptr.p, op->conn.p, P.adj_ptr.p,
            P.adj.p, P.slot_map.p);
        SVX_LAUNCH_CHECK();
    }
    int h_flags[2] = {0, 0};
    SVX_CUDA(cudaMemcpyAsync(h_flags, flags.p, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaStreamSynchronize(st));
    P.max_slots = h_flags[0];
    P.max_deg = h_flags[1];
    if (P.max_deg > 65535)
        throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                        "a node shares elements with more than 65535 nodes"};
}

}  // namespace svx

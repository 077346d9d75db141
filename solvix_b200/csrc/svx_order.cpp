// svx_order.cpp - the equation ordering of the direct path.
//
// The direct path factorizes K in the reverse Cuthill-McKee order of the
// reference (rcm, ldl.rs:27-60), so that its pivots, its D-based condition
// estimate and the equation number of a failed pivot are those of the same
// ordering: every connected component starts at its first unvisited row of
// least degree, neighbours are enqueued in ascending column order, and the
// breadth-first order is reversed.  The reference picks each start by a scan
// over all rows; here rows are bucketed once by degree (a stable counting
// sort, so ties stay in index order) and a cursor skips the visited ones,
// which gives the same starts in O(n + nnz).

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "svx_internal.h"

namespace svx {

template <class P>
void rcm_order_impl(int64_t n, const P* row_ptr, const int32_t* col_idx,
                    std::vector<int32_t>& perm, int64_t& bandwidth) {
    perm.assign(size_t(n), 0);
    bandwidth = 0;
    if (n <= 0) return;
    int64_t max_deg = 0;
    for (int64_t i = 0; i < n; ++i)
        max_deg = std::max<int64_t>(max_deg, row_ptr[i + 1] - row_ptr[i]);
    std::vector<int64_t> start(size_t(max_deg) + 2, 0);
    for (int64_t i = 0; i < n; ++i) ++start[size_t(row_ptr[i + 1] - row_ptr[i]) + 1];
    for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
    std::vector<int32_t> by_degree(static_cast<size_t>(n));
    for (int64_t i = 0; i < n; ++i)
        by_degree[size_t(start[size_t(row_ptr[i + 1] - row_ptr[i])]++)] = int32_t(i);

    std::vector<uint8_t> seen(static_cast<size_t>(n), 0);
    std::vector<int32_t> order;
    order.reserve(size_t(n));
    size_t cursor = 0;
    while (int64_t(order.size()) < n) {
        while (seen[size_t(by_degree[cursor])]) ++cursor;
        const int32_t s = by_degree[cursor];
        seen[size_t(s)] = 1;
        size_t head = order.size();
        order.push_back(s);
        while (head < order.size()) {
            const int32_t u = order[head++];
            for (P p = row_ptr[u]; p < row_ptr[u + 1]; ++p) {
                const int32_t v = col_idx[p];
                if (!seen[size_t(v)]) {
                    seen[size_t(v)] = 1;
                    order.push_back(v);
                }
            }
        }
    }
    for (int64_t pos = 0; pos < n; ++pos) perm[size_t(order[size_t(n - 1 - pos)])] = int32_t(pos);
    for (int64_t r = 0; r < n; ++r)
        for (P p = row_ptr[r]; p < row_ptr[r + 1]; ++p)
            bandwidth = std::max<int64_t>(bandwidth, std::llabs(int64_t(perm[size_t(r)]) -
                                                                int64_t(perm[size_t(col_idx[p])])));
}

void rcm_order(int64_t n, const int32_t* row_ptr, const int32_t* col_idx,
               std::vector<int32_t>& perm, int64_t& bandwidth) {
    rcm_order_impl(n, row_ptr, col_idx, perm, bandwidth);
}

}  // namespace svx

extern "C" int svx_order_rcm(int64_t n, const int64_t* row_ptr, const int32_t* col_idx,
                             int32_t* perm, int64_t* bandwidth) {
    if (n < 0 || n > INT32_MAX || (n > 0 && (!row_ptr || !col_idx || !perm)))
        return SVX_BAD_ARGUMENT;
    for (int64_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return SVX_BAD_ARGUMENT;
    for (int64_t p = 0; n > 0 && p < row_ptr[n]; ++p)
        if (col_idx[p] < 0 || col_idx[p] >= n) return SVX_BAD_ARGUMENT;
    try {
        std::vector<int32_t> pv;
        int64_t bw = 0;
        svx::rcm_order_impl(n, row_ptr, col_idx, pv, bw);
        std::copy(pv.begin(), pv.end(), perm);
        if (bandwidth) *bandwidth = bw;
    } catch (const std::bad_alloc&) {
        return SVX_OOM;
    }
    return SVX_OK;
}

// svx_ldlt.cu - the direct path: LDL^T of the Dirichlet-modified K in the
// reverse Cuthill-McKee order, factorized and solved on the device.
//
// Replaces Ldlt::factorize / Ldlt::solve / cond_estimate (ldl.rs:144-265)
// and the residual of the direct closure of the static solve
// (lib.rs:645-663).  The reference runs an up-looking sparse LDL^T row by
// row on one core; an RCM-ordered stiffness matrix is banded, so here the
// lower band is stored as dense 32 x 32 tiles and factorized right-looking,
// one block column per step:
//
//   panel kernel   every block factors the diagonal tile (J, J) into L_JJ and
//                  D_J (the whole block, in shared memory, one column per
//                  step); block 0 stores them apart from the band (the
//                  other blocks are still reading tile (J, J)); block g
//                  solves the panel tile (J+1+g, J): W = A L_JJ^-T,
//                  L = W D_J^-1;
//   update kernel  one 64-thread block per tile pair J < K <= I <= J + w:
//                  A_IK -= W_IJ L_KJ^T (W keeps the product L D) with FP64
//                  tensor-core products (mma.sync m8n8k4 f64).
//
// Each step is two ordinary launches, so nothing on the device waits for
// another block.  The pivot test is the reference's: D_i not finite or
// D_i <= 1e-13 * max(max_j |K_ij|, DBL_MIN) fails with the reference's
// message and equation number (i in the RCM order); the first failing
// equation is kept with an atomic minimum.  The forward, diagonal and
// backward solves run in one block, block row by block row.
//
// The summation order differs from the reference's up-looking one, so D, u
// and the residual agree with it to rounding (D to a few ulps times the
// growth of the elimination), not bit for bit.
//
// Tile (I, d) holds block row I, block column I - d (0 <= d <= w, w the
// half-bandwidth in tiles); tile_off is the only address computation of the
// band, and the host sizes the band as tile_off(nb, 0, w).

#include <cfloat>
#include <cmath>

#include "svx_internal.h"
#include "svx_grid.h"

namespace svx {

void rcm_order(int64_t n, const int32_t* row_ptr, const int32_t* col_idx,
               std::vector<int32_t>& perm, int64_t& bandwidth);

namespace {

constexpr int LT = 32;           // tile edge
constexpr int LT2 = LT * LT;
constexpr int LBLOCK = 256;      // threads of the band kernels (8 warps)
constexpr int SBLOCK = 1024;     // threads of the solve and finish kernels
constexpr unsigned long long NO_FAIL = ~0ull;

__host__ __device__ __forceinline__ size_t tile_off(int64_t I, int d, int w) {
    return (size_t(I) * size_t(w + 1) + size_t(d)) * size_t(LT2);
}

// Reads the failure word once per block so that every thread of the block
// takes the same early exit.
__device__ __forceinline__ bool stopped(const unsigned long long* fail, int* s_flag) {
    if (threadIdx.x == 0) *s_flag = (*(volatile const unsigned long long*)fail != NO_FAIL);
    __syncthreads();
    return *s_flag != 0;
}

// One thread per row r of K: its lower-triangle entries in the RCM order go
// to the band, and max |K_rj| (the reference's row_max) to row_max[perm[r]].
__global__ void band_fill_kernel(int64_t n, int w, const int32_t* __restrict__ perm,
                                 const int32_t* __restrict__ row_ptr,
                                 const int32_t* __restrict__ col_idx,
                                 const double* __restrict__ vals, double* __restrict__ band,
                                 double* __restrict__ row_max, int* __restrict__ bad) {
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t i = perm[r];
    if (i < 0 || i >= n) {
        atomicExch(bad, 1);
        return;
    }
    const int64_t I = i / LT;
    const int ri = int(i % LT);
    double acc = 0.0;
    for (int32_t p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
        const int32_t c = col_idx[p];
        const double v = vals[p];
        acc = fmax(acc, fabs(v));
        if (c < 0 || c >= n) {
            atomicExch(bad, 1);
            continue;
        }
        const int64_t j = perm[c];
        if (j < 0 || j >= n) {
            atomicExch(bad, 1);
            continue;
        }
        if (j > i) continue;
        const int64_t d = I - j / LT;
        if (d > w) {
            atomicExch(bad, 1);
            continue;
        }
        band[tile_off(I, int(d), w) + size_t(ri) * LT + size_t(j % LT)] = v;
    }
    row_max[i] = acc;
}

// Rows n .. nb*LT-1 of the last block row: identity, so that the last
// diagonal tile factorizes whole.
__global__ void band_pad_kernel(int64_t n, int64_t rows, int w, double* __restrict__ band,
                                double* __restrict__ row_max) {
    const int64_t i = n + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    band[tile_off(i / LT, 0, w) + size_t(i % LT) * (LT + 1)] = 1.0;
    row_max[i] = 1.0;
}

// Step J, first half (grid: max(1, wj) blocks, wj = min(w, nb - 1 - J)).
__global__ void __launch_bounds__(LBLOCK)
ldlt_panel_kernel(int64_t J, int64_t n, int w, int wj, double* __restrict__ band,
                  double* __restrict__ panel, double* __restrict__ dfac,
                  double* __restrict__ dvec, const double* __restrict__ row_max,
                  unsigned long long* fail) {
    __shared__ double s_l[LT][LT + 1];
    __shared__ int s_flag;
    if (stopped(fail, &s_flag)) return;
    const double* dt = band + tile_off(J, 0, w);
    for (int k = threadIdx.x; k < LT2; k += LBLOCK) s_l[k / LT][k % LT] = dt[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // Right-looking LDL^T of the tile in shared memory, the whole block at
    // once: at column c every entry (r, k), c < k <= r, takes
    // A[r][k] -= (W[r][c] / D_c) W[k][c] with W column c still unscaled,
    // then column c becomes L = W / D_c; so each entry gets
    // A[r][k] - sum_c L[r][c] W[k][c] in column order.
    for (int c = 0; c < LT; ++c) {
        const double dc = s_l[c][c];
        const int64_t eq = J * LT + c;
        if (threadIdx.x == 0 && blockIdx.x == 0 && eq < n) {
            const double lim = 1e-13 * fmax(row_max[eq], DBL_MIN);
            if (!isfinite(dc) || dc <= lim)
                atomicMin(fail, (unsigned long long)(eq) << 1 | (dc < 0.0 ? 1ull : 0ull));
        }
        {
            // thread (r, g) takes row r, columns c + 1 + g, c + 9 + g, ... <= r
            const int r = threadIdx.x >> 3, g = threadIdx.x & 7;
            if (r > c) {
                const double l = s_l[r][c] / dc;
                for (int k = c + 1 + g; k <= r; k += 8) s_l[r][k] -= l * s_l[k][c];
            }
        }
        __syncthreads();
        if (threadIdx.x > c && threadIdx.x < LT) s_l[threadIdx.x][c] /= dc;
        __syncthreads();
    }
    if (blockIdx.x == 0) {
        double* out = dfac + size_t(J) * LT2;
        for (int k = threadIdx.x; k < LT2; k += LBLOCK) out[k] = s_l[k / LT][k % LT];
        if (threadIdx.x < LT) dvec[J * LT + threadIdx.x] = s_l[threadIdx.x][threadIdx.x];
    }
    const int d = 1 + int(blockIdx.x);
    if (d > wj) return;
    // Panel tile (J + d, J): warp w takes rows w, w + 8, w + 16, w + 24
    // together; lane c' keeps row c' of L_JJ in registers and ends with
    // W[row][c'] = A[row][c'] - sum_{c < c'} W[row][c] L_JJ[c'][c].
    static_assert(LT == 4 * (LBLOCK / 32), "four panel rows per warp");
    double lrow[LT];
#pragma unroll
    for (int k = 0; k < LT; ++k) lrow[k] = s_l[lane][k];
    const double dl = s_l[lane][lane];
    double* tile = band + tile_off(J + d, d, w);
    double* wt = panel + size_t(d - 1) * LT2;
    double x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = tile[(warp + 8 * q) * LT + lane];
#pragma unroll
    for (int c = 0; c < LT; ++c) {
        const double lc = lrow[c];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double v = __shfl_sync(0xffffffffu, x[q], c);
            if (lane > c) x[q] -= v * lc;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        wt[(warp + 8 * q) * LT + lane] = x[q];
        tile[(warp + 8 * q) * LT + lane] = x[q] / dl;
    }
}

// Step J, second half (grid: wj (wj + 1) / 2 blocks): block q takes the
// pair (di, dk), 1 <= dk <= di <= wj, q = di (di - 1) / 2 + dk - 1, and
// updates tile (J + di, di - dk) with W_(J+di) L_(J+dk)^T.
//
// 64 threads (two warps) a pair on the FP64 tensor cores: each warp takes
// 16 rows of the target as 2 x 4 blocks of 8 x 8 and accumulates
// W L^T over k in steps of 4 with mma.sync m8n8k4 f64 (tcgen05 has no FP64
// kind), both operand tiles staged row-major in shared memory and every
// global load of the block issued at once.  Each output is summed over k
// in column order, as in the FP64-FMA loop it replaced (the C2 residual is
// bitwise the same), 7.5% faster on the 160 x 16 x 16 cantilever
// (244 against 263 ms a solve).
constexpr int UBLOCK = 64;
// c += a b on an 8 x 8 x 4 FP64 tile (one element of A and B, two of C a lane)
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1) : "d"(a), "d"(b));
}
__global__ void __launch_bounds__(UBLOCK)
ldlt_update_kernel(int64_t J, int w, int wj, double* __restrict__ band,
                   const double* __restrict__ panel, const unsigned long long* fail) {
    __shared__ double s_w[LT][LT + 1];  // W[r][c]
    __shared__ double s_k[LT][LT + 1];  // L[s][c]: B = L^T, column-major
    __shared__ int s_flag;
    if (stopped(fail, &s_flag)) return;
    int q = int(blockIdx.x), di = 1;
    while (q >= di) {
        q -= di;
        ++di;
    }
    const int dk = q + 1;
    if (di > wj) return;
    const double2* wt = reinterpret_cast<const double2*>(panel + size_t(di - 1) * LT2);
    const double2* lk = reinterpret_cast<const double2*>(band + tile_off(J + dk, dk, w));
    double* tb = band + tile_off(J + di, di - dk, w);
    constexpr int Q = LT2 / 2 / UBLOCK;
    double2 wv[Q], lv[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        wv[q] = __ldg(wt + threadIdx.x + UBLOCK * q);
        lv[q] = __ldg(lk + threadIdx.x + UBLOCK * q);
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int fr = lane >> 2, fc = lane & 3;
    double tv[2][4][2];
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
        for (int sb = 0; sb < 4; ++sb)
#pragma unroll
            for (int i = 0; i < 2; ++i)
                tv[rb][sb][i] = tb[size_t((2 * wp + rb) * 8 + fr) * LT + sb * 8 + fc * 2 + i];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int e = 2 * (int(threadIdx.x) + UBLOCK * q), row = e / LT, col = e % LT;
        s_w[row][col] = wv[q].x;
        s_w[row][col + 1] = wv[q].y;
        s_k[row][col] = lv[q].x;
        s_k[row][col + 1] = lv[q].y;
    }
    __syncthreads();
    double acc[2][4][2];
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
        for (int sb = 0; sb < 4; ++sb) acc[rb][sb][0] = acc[rb][sb][1] = 0.0;
#pragma unroll
    for (int k4 = 0; k4 < LT / 4; ++k4) {
        double a[2], b[4];
#pragma unroll
        for (int rb = 0; rb < 2; ++rb) a[rb] = s_w[(2 * wp + rb) * 8 + fr][4 * k4 + fc];
#pragma unroll
        for (int sb = 0; sb < 4; ++sb) b[sb] = s_k[sb * 8 + fr][4 * k4 + fc];
#pragma unroll
        for (int rb = 0; rb < 2; ++rb)
#pragma unroll
            for (int sb = 0; sb < 4; ++sb) dmma(acc[rb][sb][0], acc[rb][sb][1], a[rb], b[sb]);
    }
#pragma unroll
    for (int rb = 0; rb < 2; ++rb)
#pragma unroll
        for (int sb = 0; sb < 4; ++sb)
#pragma unroll
            for (int i = 0; i < 2; ++i)
                tb[size_t((2 * wp + rb) * 8 + fr) * LT + sb * 8 + fc * 2 + i] =
                        tv[rb][sb][i] - acc[rb][sb][i];
}

// L y = P f, y /= D, L^T x = y, u = P^T x in one block (y: nb * LT
// scratch; the diagonal tiles' L in dfac).  Warp p sums the off-diagonal
// tiles d = p + 1, p + 33, ... of a block row; warp 0 adds the partials in
// a fixed order and solves the diagonal tile with shuffles.
__global__ void __launch_bounds__(SBLOCK)
ldlt_solve_kernel(int64_t n, int64_t nb, int w, const double* __restrict__ band,
                  const double* __restrict__ dfac, const double* __restrict__ dvec,
                  const int32_t* __restrict__ perm,
                  const double* __restrict__ f, double* y, double* __restrict__ u,
                  const unsigned long long* fail) {
    __shared__ double s_part[SBLOCK / 32][LT + 1];
    __shared__ int s_flag;
    if (stopped(fail, &s_flag)) return;
    const int lane = threadIdx.x & 31;
    const int part = threadIdx.x >> 5;
    constexpr int PARTS = SBLOCK / 32;
    const int64_t rows = nb * LT;
    for (int64_t i = threadIdx.x; i < rows; i += SBLOCK) y[i] = 0.0;
    __syncthreads();
    for (int64_t r = threadIdx.x; r < n; r += SBLOCK) y[perm[r]] = f[r];
    __syncthreads();
    for (int64_t I = 0; I < nb; ++I) {
        const int dmax = int(I < w ? I : w);
        double s = 0.0;
        for (int d = 1 + part; d <= dmax; d += PARTS) {
            const double* t = band + tile_off(I, d, w) + size_t(lane) * LT;
            const double* yy = y + (I - d) * LT;
            for (int c = 0; c < LT; ++c) s += t[c] * yy[c];
        }
        s_part[part][lane] = s;
        __syncthreads();
        if (part == 0) {
            double tot = 0.0;
            for (int k = 0; k < PARTS; ++k) tot += s_part[k][lane];
            double x = y[I * LT + lane] - tot;
            const double* t = dfac + size_t(I) * LT2 + size_t(lane) * LT;
            for (int c = 0; c < LT; ++c) {
                const double v = __shfl_sync(0xffffffffu, x, c);
                if (lane > c) x -= t[c] * v;
            }
            y[I * LT + lane] = x;
        }
        __syncthreads();
    }
    for (int64_t i = threadIdx.x; i < rows; i += SBLOCK) y[i] /= dvec[i];
    __syncthreads();
    for (int64_t J = nb - 1; J >= 0; --J) {
        const int dmax = int(nb - 1 - J < w ? nb - 1 - J : w);
        double s = 0.0;
        for (int d = 1 + part; d <= dmax; d += PARTS) {
            const double* t = band + tile_off(J + d, d, w) + lane;
            const double* xx = y + (J + d) * LT;
            for (int r = 0; r < LT; ++r) s += t[size_t(r) * LT] * xx[r];
        }
        s_part[part][lane] = s;
        __syncthreads();
        if (part == 0) {
            double tot = 0.0;
            for (int k = 0; k < PARTS; ++k) tot += s_part[k][lane];
            double z = y[J * LT + lane] - tot;
            const double* t = dfac + size_t(J) * LT2 + lane;
            for (int r = LT - 1; r >= 0; --r) {
                const double v = __shfl_sync(0xffffffffu, z, r);
                if (lane < r) z -= t[size_t(r) * LT] * v;
            }
            y[J * LT + lane] = z;
        }
        __syncthreads();
    }
    for (int64_t r = threadIdx.x; r < n; r += SBLOCK) u[r] = y[perm[r]];
}

// L y = P f, y /= D, L^T x = y, u = P^T x over the whole GPU (cooperative
// launch, one block per SM, a bounded grid barrier per block row).  In the
// forward sweep, iteration I: block 0 finishes y_I from the partial sums
// the other blocks left for row I (tiles d >= 2, part[I & 1]) plus its own
// T(I, 1) y_(I-1), then solves the diagonal tile; meanwhile block b >= 1
// forms T(I+1, d) y_(I+1-d) for its tiles d = 1 + b, 1 + b + (B - 1), ...
// (d >= 2: those y are final a barrier earlier) into part[(I+1) & 1].  The
// backward sweep mirrors it with transposed tiles, z = y / D taken when a
// block row is finished.  Every tile product has the same thread mapping
// wherever it runs and block 0 adds the partial sums in d order, so the
// result does not depend on the block count.
constexpr int TBLOCK = 256;
static_assert(TBLOCK == 8 * LT, "eight column (or row) groups of four per tile");

// the 32 results of one tile product (forward: rows of T times x over its
// columns; backward: columns of T times x over its rows), summed over the
// eight groups in order; valid in threads 0..31 of the block.  x was
// written by another block during the launch and is read from L2.
template <bool TRANS>
__device__ __forceinline__ double tile_product(const double* __restrict__ t,
                                               const double* x, double (*s_red)[LT]) {
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int k = 4 * g + j;
        const double xk = __ldcg(x + k);
        s += TRANS ? t[size_t(k) * LT + lane] * xk : t[size_t(lane) * LT + k] * xk;
    }
    s_red[g][lane] = s;
    __syncthreads();
    double tot = 0.0;
    if (threadIdx.x < LT)
#pragma unroll
        for (int q = 0; q < 8; ++q) tot += s_red[q][threadIdx.x];
    __syncthreads();
    return tot;
}

__global__ void __launch_bounds__(TBLOCK)
ldlt_solve_coop_kernel(int64_t n, int64_t nb, int w, const double* __restrict__ band,
                       const double* __restrict__ dfac, const double* __restrict__ dvec,
                       const int32_t* __restrict__ perm, const double* __restrict__ f,
                       double* y, double* __restrict__ u, double* part, GridBarrier* gb,
                       const unsigned long long* fail) {
    __shared__ double s_red[8][LT];
    __shared__ double s_acc[8][LT];
    __shared__ int s_flag;
    if (stopped(fail, &s_flag)) return;
    const unsigned int B = gridDim.x;
    unsigned int target = 0;
    const int64_t rows = nb * LT;
    const int64_t tid = int64_t(blockIdx.x) * TBLOCK + threadIdx.x, nthr = int64_t(B) * TBLOCK;
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    const size_t pstride = size_t(w + 1) * LT;  // one buffer of part
    for (int64_t i = tid; i < rows; i += nthr) y[i] = 0.0;
    if (!grid_sync(gb, B, target)) return;
    for (int64_t r = tid; r < n; r += nthr) y[perm[r]] = f[r];
    if (!grid_sync(gb, B, target)) return;
    // block 0's sum of the others' partials for block row R (d = 2..dmax):
    // thread (lane, g) adds d = 2 + g, 10 + g, ... in order, then the groups
    // are added in order
    auto partial_sum = [&](int64_t R, int dmax) -> double {
        const double* pb = part + size_t(R & 1) * pstride;
        double s = 0.0;
        for (int d = 2 + g; d <= dmax; d += 8) s += __ldcg(pb + size_t(d) * LT + lane);
        s_acc[g][lane] = s;
        __syncthreads();
        double tot = 0.0;
        if (threadIdx.x < LT)
#pragma unroll
            for (int q = 0; q < 8; ++q) tot += s_acc[q][threadIdx.x];
        __syncthreads();
        return tot;
    };
    for (int64_t I = 0; I < nb; ++I) {
        if (blockIdx.x == 0) {
            const int dmax = int(I < w ? I : w);
            double tot = partial_sum(I, dmax);
            if (dmax >= 1) {
                const double t1 = tile_product<false>(band + tile_off(I, 1, w),
                                                       y + (I - 1) * LT, s_red);
                tot = t1 + tot;
            }
            if (threadIdx.x < LT) {
                double x = __ldcg(y + I * LT + lane) - tot;
                const double* t = dfac + size_t(I) * LT2 + size_t(lane) * LT;
                for (int c = 0; c < LT; ++c) {
                    const double v = __shfl_sync(0xffffffffu, x, c);
                    if (lane > c) x -= t[c] * v;
                }
                y[I * LT + lane] = x;
            }
        } else if (I + 1 < nb) {
            const int64_t R = I + 1;
            const int dmax = int(R < w ? R : w);
            double* pb = part + size_t(R & 1) * pstride;
            for (int d = 1 + int(blockIdx.x); d <= dmax; d += int(B) - 1) {
                const double v = tile_product<false>(band + tile_off(R, d, w), y + (R - d) * LT,
                                                      s_red);
                if (threadIdx.x < LT) pb[size_t(d) * LT + lane] = v;
            }
        }
        if (!grid_sync(gb, B, target)) return;
    }
    for (int64_t J = nb - 1; J >= 0; --J) {
        if (blockIdx.x == 0) {
            const int dmax = int(nb - 1 - J < w ? nb - 1 - J : w);
            double tot = partial_sum(J, dmax);
            if (dmax >= 1) {
                const double t1 = tile_product<true>(band + tile_off(J + 1, 1, w),
                                                      y + (J + 1) * LT, s_red);
                tot = t1 + tot;
            }
            if (threadIdx.x < LT) {
                double z = __ldcg(y + J * LT + lane) / dvec[J * LT + lane] - tot;
                const double* t = dfac + size_t(J) * LT2 + lane;
                for (int r = LT - 1; r >= 0; --r) {
                    const double v = __shfl_sync(0xffffffffu, z, r);
                    if (lane < r) z -= t[size_t(r) * LT] * v;
                }
                y[J * LT + lane] = z;
            }
        } else if (J >= 1) {
            const int64_t R = J - 1;
            const int dmax = int(nb - 1 - R < w ? nb - 1 - R : w);
            double* pb = part + size_t(R & 1) * pstride;
            for (int d = 1 + int(blockIdx.x); d <= dmax; d += int(B) - 1) {
                const double v = tile_product<true>(band + tile_off(R + d, d, w),
                                                     y + (R + d) * LT, s_red);
                if (threadIdx.x < LT) pb[size_t(d) * LT + lane] = v;
            }
        }
        if (!grid_sync(gb, B, target)) return;
    }
    for (int64_t r = tid; r < n; r += nthr) u[r] = __ldcg(y + perm[r]);
}

// ||f||^2, ||f - K u||^2, max |D_i| and min |D_i| (one block, fixed order).
__global__ void __launch_bounds__(SBLOCK)
ldlt_finish_kernel(int64_t n, const double* __restrict__ f, const double* __restrict__ ku,
                   const double* __restrict__ dvec, double* __restrict__ out) {
    __shared__ double sh[4][SBLOCK / 32];
    double ff = 0.0, rr = 0.0, hi = 0.0, lo = INFINITY;
    for (int64_t i = threadIdx.x; i < n; i += SBLOCK) {
        const double fi = f[i];
        const double e = fi - ku[i];
        ff += fi * fi;
        rr += e * e;
        const double a = fabs(dvec[i]);
        hi = fmax(hi, a);
        lo = fmin(lo, a);
    }
    for (int o = 16; o > 0; o >>= 1) {
        ff += __shfl_xor_sync(0xffffffffu, ff, o);
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = ff;
        sh[1][warp] = rr;
        sh[2][warp] = hi;
        sh[3][warp] = lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, h = 0.0, l = INFINITY;
        for (int k = 0; k < SBLOCK / 32; ++k) {
            a += sh[0][k];
            b += sh[1][k];
            h = fmax(h, sh[2][k]);
            l = fmin(l, sh[3][k]);
        }
        out[0] = a;
        out[1] = b;
        out[2] = h;
        out[3] = l;
    }
}

}  // namespace

LdltOutcome ldlt_direct(svx_ctx* ctx, svx_op* op, double* u) {
    const cudaStream_t st = ctx->stream;
    const int64_t n = op->n;
    LdltOutcome res;
    if (n <= 0) return res;
    const int64_t nnz = op->pat.nnz;
    std::vector<int32_t> h_ptr(static_cast<size_t>(n) + 1);
    std::vector<int32_t> h_col(static_cast<size_t>(nnz));
    SVX_CUDA(cudaMemcpyAsync(h_ptr.data(), op->pat.row_ptr.p, h_ptr.size() * sizeof(int32_t),
                             cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaMemcpyAsync(h_col.data(), op->pat.col_idx.p, h_col.size() * sizeof(int32_t),
                             cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaStreamSynchronize(st));
    std::vector<int32_t> perm;
    int64_t bw = 0;
    rcm_order(n, h_ptr.data(), h_col.data(), perm, bw);
    res.bandwidth = bw;

    const int64_t nb = (n + LT - 1) / LT;
    const int w = int((bw + LT - 1) / LT);
    const size_t band_elems = tile_off(nb, 0, w);
    const size_t panel_elems = size_t(std::max(w, 1)) * LT2;
    const size_t rows = size_t(nb) * LT;
    const size_t need = (band_elems + panel_elems + size_t(nb) * LT2 + 3 * rows + size_t(n)) *
                            sizeof(double) +
                        size_t(n) * sizeof(int32_t) + 4096;
    size_t free_b = 0, total_b = 0;
    SVX_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (need > free_b / 10 * 9) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "the direct path needs %.2f GB of device memory for the band factor "
                      "(half-bandwidth %lld in the RCM order); %.2f GB are free",
                      double(need) / 1e9, (long long)bw, double(free_b) / 1e9);
        throw ModelFail{SVX_OOM, 0, -1, msg};
    }
    DBuf<double> band, panel, dfac, dvec, row_max, y, ku, out;
    DBuf<int32_t> d_perm;
    DBuf<unsigned long long> fail;
    DBuf<int> bad;
    band.alloc(ctx->pool, band_elems);
    panel.alloc(ctx->pool, panel_elems);
    dfac.alloc(ctx->pool, size_t(nb) * LT2);
    dvec.alloc(ctx->pool, rows);
    row_max.alloc(ctx->pool, rows);
    y.alloc(ctx->pool, rows);
    ku.alloc(ctx->pool, size_t(n));
    out.alloc(ctx->pool, 4);
    d_perm.alloc(ctx->pool, size_t(n));
    fail.alloc(ctx->pool, 1);
    bad.alloc(ctx->pool, 1);
    SVX_CUDA(cudaEventRecord(ctx->ev[6], st));
    SVX_CUDA(cudaMemsetAsync(band.p, 0, band_elems * sizeof(double), st));
    SVX_CUDA(cudaMemsetAsync(fail.p, 0xff, sizeof(unsigned long long), st));
    SVX_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    SVX_CUDA(cudaMemcpyAsync(d_perm.p, perm.data(), size_t(n) * sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
    band_fill_kernel<<<unsigned((n + 255) / 256), 256, 0, st>>>(
        n, w, d_perm.p, op->pat.row_ptr.p, op->pat.col_idx.p, op->vals.p, band.p, row_max.p,
        bad.p);
    SVX_LAUNCH_CHECK();
    if (int64_t(rows) > n) {
        band_pad_kernel<<<1, LT, 0, st>>>(n, int64_t(rows), w, band.p, row_max.p);
        SVX_LAUNCH_CHECK();
    }
    for (int64_t J = 0; J < nb; ++J) {
        const int wj = int(std::min<int64_t>(w, nb - 1 - J));
        ldlt_panel_kernel<<<unsigned(std::max(wj, 1)), LBLOCK, 0, st>>>(
            J, n, w, wj, band.p, panel.p, dfac.p, dvec.p, row_max.p, fail.p);
        SVX_LAUNCH_CHECK();
        if (wj > 0) {
            ldlt_update_kernel<<<unsigned(int64_t(wj) * (wj + 1) / 2), UBLOCK, 0, st>>>(
                J, w, wj, band.p, panel.p, fail.p);
            SVX_LAUNCH_CHECK();
        }
    }
    // the substitutions over the whole GPU when a cooperative launch of one
    // block per SM is possible, else in one block
    int coop = 0, bps = 0;
    SVX_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    SVX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, ldlt_solve_coop_kernel,
                                                           TBLOCK, 0));
    DBuf<double> part;
    DBuf<GridBarrier> gb;
    const bool coop_solve = coop && bps >= 1 && ctx->sm_count >= 2;
    if (coop_solve) {
        part.alloc(ctx->pool, 2 * (size_t(w) + 1) * LT);
        gb.alloc(ctx->pool, 1);
        SVX_CUDA(cudaMemsetAsync(gb.p, 0, sizeof(GridBarrier), st));
        const double* band_p = band.p;
        const double* dfac_p = dfac.p;
        const double* dvec_p = dvec.p;
        const int32_t* perm_p = d_perm.p;
        const double* f_p = op->f.p;
        double* y_p = y.p;
        double* part_p = part.p;
        GridBarrier* gb_p = gb.p;
        const unsigned long long* fail_p = fail.p;
        int64_t n_a = n, nb_a = nb;
        int w_a = w;
        void* args[] = {&n_a, &nb_a, &w_a, (void*)&band_p, (void*)&dfac_p, (void*)&dvec_p,
                        (void*)&perm_p, (void*)&f_p, (void*)&y_p, (void*)&u, (void*)&part_p,
                        (void*)&gb_p, (void*)&fail_p};
        SVX_CUDA(cudaLaunchCooperativeKernel((void*)ldlt_solve_coop_kernel,
                                             dim3(unsigned(ctx->sm_count)), dim3(TBLOCK), args,
                                             0, st));
        SVX_LAUNCH_CHECK();
    } else {
        ldlt_solve_kernel<<<1, SBLOCK, 0, st>>>(n, nb, w, band.p, dfac.p, dvec.p, d_perm.p,
                                                op->f.p, y.p, u, fail.p);
        SVX_LAUNCH_CHECK();
    }
    spmv_fp64(ctx, op, op->vals.p, u, ku.p);
    ldlt_finish_kernel<<<1, SBLOCK, 0, st>>>(n, op->f.p, ku.p, dvec.p, out.p);
    SVX_LAUNCH_CHECK();
    SVX_CUDA(cudaEventRecord(ctx->ev[7], st));
    unsigned long long h_fail = 0;
    int h_bad = 0;
    double h_out[4] = {0.0, 0.0, 0.0, 0.0};
    SVX_CUDA(cudaMemcpyAsync(&h_fail, fail.p, sizeof h_fail, cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaMemcpyAsync(&h_bad, bad.p, sizeof h_bad, cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaMemcpyAsync(h_out, out.p, sizeof h_out, cudaMemcpyDeviceToHost, st));
    GridBarrier h_gb{};
    if (coop_solve)
        SVX_CUDA(cudaMemcpyAsync(&h_gb, gb.p, sizeof h_gb, cudaMemcpyDeviceToHost, st));
    SVX_CUDA(cudaStreamSynchronize(st));
    if (h_gb.error)
        throw ModelFail{SVX_CUDA_ERROR, 0, -1,
                        "direct path: a grid barrier wait of the substitutions ran out"};
    float ms = 0.0f;
    SVX_CUDA(cudaEventElapsedTime(&ms, ctx->ev[6], ctx->ev[7]));
    res.ms = ms;
    if (h_bad) throw ModelFail{SVX_CUDA_ERROR, 0, -1, "direct path: band index out of range"};
    if (h_fail != NO_FAIL) {
        const long long eq = (long long)(h_fail >> 1);
        throw ModelFail{SVX_INVALID_MODEL, 0, -1,
                        std::string("stiffness matrix is not positive definite (pivot ") +
                            ((h_fail & 1ull) ? "negative" : "near-zero") + " at equation " +
                            std::to_string(eq) + ")"};
    }
    const double b_norm = std::sqrt(h_out[0]);
    res.residual = b_norm == 0.0 ? 0.0 : std::sqrt(h_out[1]) / b_norm;
    res.cond = h_out[2] / h_out[3];
    return res;
}

}  // namespace svx

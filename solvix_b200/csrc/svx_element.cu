// svx_element.cu - K1 element integration and K9/K10 stress + reaction
// recovery.  Compiled with -fmad=false: every product and sum rounds on its
// own, in the order of the reference's Rust code, so the element matrices,
// stresses and reactions are bit-identical to the oracle's for the same
// inputs (crates/solvix-core/src/element.rs, stress.rs).
//
// K1 layout: one warp per element.  Per Gauss point the warp builds J,
// det J, J^-1 and B in shared memory, forms DB = D*B (lanes over the S x N
// entries) and accumulates the upper triangle of w * B^T DB into per-lane
// registers (lanes own fixed (a, c) pairs, a <= c), exactly as btdb does
// (element.rs:830-851).  The finished Ke (mirrored) is staged in shared
// memory and written out with coalesced stores into a per-element slot of
// the Ke buffer, which the fixed-order assembly then gathers.

#include "svx_internal.h"

#include <cfloat>

namespace svx {

namespace {

constexpr int WARPS = 4;            // warps (elements) per block in K1
constexpr int MAX_PAIRS_PER_LANE = 10;  // ceil(300 / 32)

struct ElemSmem {
    double D[36];
    double B[6 * 24];
    double DB[6 * 24];
    double ke[576];
    double dn[3 * 8];
    double J[9];
    double xyz[24];
};

__device__ __forceinline__ double hexc(int i, int a) {
    // HEX_CORNERS (element.rs:427-437): bottom face CCW, then top face.
    const int sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const int sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const int sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    return double(a == 0 ? sx[i] : (a == 1 ? sy[i] : sz[i]));
}

__device__ __forceinline__ double quadc(int i, int a) {
    // QUAD_CORNERS (element.rs:131)
    const int sx[4] = {-1, 1, 1, -1};
    const int sy[4] = {-1, -1, 1, 1};
    return double(a == 0 ? sx[i] : sy[i]);
}

// element.rs:10-17
__device__ void d_matrix(double e, double nu, double d[3][3]) {
    double c = e / (1.0 - nu * nu);
    d[0][0] = c; d[0][1] = nu * c; d[0][2] = 0.0;
    d[1][0] = nu * c; d[1][1] = c; d[1][2] = 0.0;
    d[2][0] = 0.0; d[2][1] = 0.0; d[2][2] = c * (1.0 - nu) / 2.0;
}

// element.rs:33-47 (only the non-zero pattern is needed by callers; the
// full matrix is produced for the DB product, zeros included).
__device__ void d3_matrix(double e, double nu, double d[6][6]) {
    double lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = e / (2.0 * (1.0 + nu));
    double diag = lam + 2.0 * mu;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 6; ++c) d[r][c] = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) d[r][c] = (r == c) ? diag : lam;
    d[3][3] = mu; d[4][4] = mu; d[5][5] = mu;
}

// element.rs:441-445
__device__ __forceinline__ double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
           m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// element.rs:448-463: out[i][j] = cof(j, i) / det.
__device__ __forceinline__ double inv3_entry(const double* m, double id, int i, int j) {
    int r = j, c = i;
    int a = (r + 1) % 3, b = (r + 2) % 3;
    int d = (c + 1) % 3, e = (c + 2) % 3;
    double sign = ((r + c) % 2 == 0) ? 1.0 : -1.0;
    double cof = sign * (m[a * 3 + d] * m[b * 3 + e] - m[a * 3 + e] * m[b * 3 + d]);
    return cof * id;
}

// Linear upper-triangle pair index -> (a, c), a <= c, row-major.
__device__ __forceinline__ void pair_of(int p, int N, int* a, int* c) {
    int row = 0, start = 0;
    while (p >= start + (N - row)) {
        start += N - row;
        ++row;
    }
    *a = row;
    *c = row + (p - start);
}

// Fold one Gauss point into the lane's pair accumulators:
// DB = D * B (lanes over S*N), then acc(a, c) += w * sum_r B[r][a] DB[r][c].
template <int N, int S>
__device__ __forceinline__ void btdb_warp(ElemSmem& sm, double w, int lane,
                                          const int* pa, const int* pc, int npairs,
                                          double* acc) {
    for (int q = lane; q < S * N; q += 32) {
        int r = q / N, c = q % N;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < S; ++k) s += sm.D[r * 6 + k] * sm.B[k * N + c];
        sm.DB[r * N + c] = s;
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < MAX_PAIRS_PER_LANE; ++t) {
        if (t < npairs) {
            int a = pa[t], c = pc[t];
            double s = 0.0;
#pragma unroll
            for (int r = 0; r < S; ++r) s += sm.B[r * N + a] * sm.DB[r * N + c];
            double v = w * s;
            acc[t] += v;
        }
    }
    __syncwarp();
}

// C3D8 B at a natural point into sm.B; returns det J (element.rs:479-521).
__device__ double hex_b_warp(ElemSmem& sm, double xi, double eta, double zeta, int lane) {
    if (lane < 24) {
        int a = lane / 8, i = lane % 8;
        double ca = hexc(i, 0), cb = hexc(i, 1), cc = hexc(i, 2);
        double v;
        if (a == 0) v = 0.125 * ca * (1.0 + eta * cb) * (1.0 + zeta * cc);
        else if (a == 1) v = 0.125 * cb * (1.0 + xi * ca) * (1.0 + zeta * cc);
        else v = 0.125 * cc * (1.0 + xi * ca) * (1.0 + eta * cb);
        sm.dn[a * 8 + i] = v;
    }
    for (int q = lane; q < 144; q += 32) sm.B[q] = 0.0;
    __syncwarp();
    if (lane < 9) {
        int a = lane / 3, b = lane % 3;
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) s += sm.dn[a * 8 + i] * sm.xyz[i * 3 + b];
        sm.J[a * 3 + b] = s;
    }
    __syncwarp();
    double detj = det3(sm.J);
    if (!(detj <= 0.0) && lane < 24) {
        double id = 1.0 / detj;
        int i = lane / 3, b = lane % 3;
        double g = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) g += inv3_entry(sm.J, id, b, a) * sm.dn[a * 8 + i];
        int c = 3 * i;
        if (b == 0) {
            sm.B[0 * 24 + c] = g;
            sm.B[3 * 24 + c + 1] = g;
            sm.B[5 * 24 + c + 2] = g;
        } else if (b == 1) {
            sm.B[1 * 24 + c + 1] = g;
            sm.B[3 * 24 + c] = g;
            sm.B[4 * 24 + c + 2] = g;
        } else {
            sm.B[2 * 24 + c + 2] = g;
            sm.B[4 * 24 + c + 1] = g;
            sm.B[5 * 24 + c] = g;
        }
    }
    __syncwarp();
    return detj;
}

// CPS4 B at (xi, eta) into sm.B (3 x 8); returns det J (element.rs:147-171).
__device__ double quad_b_warp(ElemSmem& sm, double xi, double eta, int lane) {
    double dxi[4], deta[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double xi_i = quadc(i, 0), eta_i = quadc(i, 1);
        dxi[i] = 0.25 * xi_i * (1.0 + eta * eta_i);
        deta[i] = 0.25 * eta_i * (1.0 + xi * xi_i);
    }
    double j00 = 0.0, j01 = 0.0, j10 = 0.0, j11 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        j00 += dxi[i] * sm.xyz[i * 3];
        j01 += dxi[i] * sm.xyz[i * 3 + 1];
        j10 += deta[i] * sm.xyz[i * 3];
        j11 += deta[i] * sm.xyz[i * 3 + 1];
    }
    double detj = j00 * j11 - j01 * j10;
    for (int q = lane; q < 24; q += 32) sm.B[q] = 0.0;
    __syncwarp();
    if (!(detj <= 0.0) && lane < 4) {
        double inv = 1.0 / detj;
        int i = lane;
        double dnx = inv * (j11 * dxi[i] - j01 * deta[i]);
        double dny = inv * (j00 * deta[i] - j10 * dxi[i]);
        sm.B[0 * 8 + 2 * i] = dnx;
        sm.B[1 * 8 + 2 * i + 1] = dny;
        sm.B[2 * 8 + 2 * i] = dny;
        sm.B[2 * 8 + 2 * i + 1] = dnx;
    }
    __syncwarp();
    return detj;
}

// ---------------------------------------------------------------------- K1
__global__ void __launch_bounds__(WARPS * 32)
integrate_kernel(int64_t n_elem, const uint8_t* __restrict__ kind,
                 const int64_t* __restrict__ conn_ptr, const int32_t* __restrict__ conn,
                 const double* __restrict__ xyz, const double* __restrict__ youngs,
                 const double* __restrict__ poisson, double thickness_all,
                 const double* __restrict__ thick_elem,
                 double* __restrict__ ke_out, int ke_stride,
                 unsigned long long* __restrict__ first_fail) {
    __shared__ ElemSmem smem[WARPS];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    ElemSmem& sm = smem[w];
    const double g = 1.0 / sqrt(3.0);
    const int64_t warps_total = int64_t(gridDim.x) * WARPS;
    for (int64_t e = int64_t(blockIdx.x) * WARPS + w; e < n_elem; e += warps_total) {
        const int k = kind[e];
        const int64_t q0 = conn_ptr[e];
        const int nn = (k == SVX_C3D8) ? 8 : (k == SVX_CPS4 ? 4 : 3);
        if (lane < nn * 3) sm.xyz[lane] = xyz[int64_t(conn[q0 + lane / 3]) * 3 + lane % 3];
        __syncwarp();
        const double E = youngs[e], nu = poisson[e];
        const double thickness = thick_elem ? thick_elem[e] : thickness_all;
        const int N = (k == SVX_C3D8) ? 24 : nn * 2;
        const int n_pairs = N * (N + 1) / 2;
        int pa[MAX_PAIRS_PER_LANE], pc[MAX_PAIRS_PER_LANE];
        double acc[MAX_PAIRS_PER_LANE];
        int np = 0;
#pragma unroll
        for (int t = 0; t < MAX_PAIRS_PER_LANE; ++t) {
            acc[t] = 0.0;
            int p = lane + 32 * t;
            if (p < n_pairs) {
                pair_of(p, N, &pa[t], &pc[t]);
                np = t + 1;
            } else {
                pa[t] = 0;
                pc[t] = 0;
            }
        }
        bool ok = true;
        if (k == SVX_C3D8) {
            if (lane == 0) {
                double d[6][6];
                d3_matrix(E, nu, d);
                for (int q = 0; q < 36; ++q) sm.D[q] = d[q / 6][q % 6];
            }
            __syncwarp();
            for (int gp = 0; gp < 8 && ok; ++gp) {
                double xi = (gp & 4) ? g : -g, eta = (gp & 2) ? g : -g, zeta = (gp & 1) ? g : -g;
                double detj = hex_b_warp(sm, xi, eta, zeta, lane);
                if (detj <= 0.0) { ok = false; break; }
                btdb_warp<24, 6>(sm, detj, lane, pa, pc, np, acc);
            }
            if (ok) {
                double detc = hex_b_warp(sm, 0.0, 0.0, 0.0, lane);
                if (detc <= 0.0) ok = false;
            }
        } else if (k == SVX_CPS4) {
            if (lane == 0) {
                double d3[3][3];
                d_matrix(E, nu, d3);
                for (int q = 0; q < 9; ++q) sm.D[(q / 3) * 6 + q % 3] = d3[q / 3][q % 3];
            }
            __syncwarp();
            for (int gp = 0; gp < 4 && ok; ++gp) {
                double xi = (gp & 2) ? g : -g, eta = (gp & 1) ? g : -g;
                double detj = quad_b_warp(sm, xi, eta, lane);
                if (detj <= 0.0) { ok = false; break; }
                btdb_warp<8, 3>(sm, thickness * detj, lane, pa, pc, np, acc);
            }
            if (ok) {
                double detc = quad_b_warp(sm, 0.0, 0.0, lane);
                if (detc <= 0.0) ok = false;
            }
        } else {  // CPS3 (element.rs:91-129)
            if (lane == 0) {
                double d3[3][3];
                d_matrix(E, nu, d3);
                for (int q = 0; q < 9; ++q) sm.D[(q / 3) * 6 + q % 3] = d3[q / 3][q % 3];
            }
            __syncwarp();
            double x0 = sm.xyz[0], y0 = sm.xyz[1], x1 = sm.xyz[3], y1 = sm.xyz[4];
            double x2 = sm.xyz[6], y2 = sm.xyz[7];
            double b[3] = {y1 - y2, y2 - y0, y0 - y1};
            double c[3] = {x2 - x1, x0 - x2, x1 - x0};
            double two_a = b[0] * c[1] - b[1] * c[0];
            if (two_a == 0.0) {
                ok = false;
            } else {
                double inv = 1.0 / two_a;
                for (int q = lane; q < 18; q += 32) sm.B[q] = 0.0;
                __syncwarp();
                if (lane < 3) {
                    int i = lane;
                    sm.B[0 * 6 + 2 * i] = b[i] * inv;
                    sm.B[1 * 6 + 2 * i + 1] = c[i] * inv;
                    sm.B[2 * 6 + 2 * i] = c[i] * inv;
                    sm.B[2 * 6 + 2 * i + 1] = b[i] * inv;
                }
                __syncwarp();
                btdb_warp<6, 3>(sm, thickness * fabs(two_a) / 2.0, lane, pa, pc, np, acc);
            }
        }
        if (!ok) {
            if (lane == 0)
                atomicMin(first_fail, (unsigned long long)(e << 8) |
                                          (k == SVX_CPS3 ? SVX_REASON_DEGENERATE_TRI
                                                         : SVX_REASON_BAD_JACOBIAN));
            __syncwarp();
            continue;
        }
        // mirror into shared memory, then coalesced store of N*N values
#pragma unroll
        for (int t = 0; t < MAX_PAIRS_PER_LANE; ++t) {
            if (t < np) {
                sm.ke[pa[t] * N + pc[t]] = acc[t];
                sm.ke[pc[t] * N + pa[t]] = acc[t];
            }
        }
        __syncwarp();
        double* dst = ke_out + e * int64_t(ke_stride);
        for (int q = lane; q < N * N; q += 32) dst[q] = sm.ke[q];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------- K9
__device__ __forceinline__ double von_mises(const double* s) {
    // element.rs:917-923
    return sqrt(0.5 * ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) +
                       (s[2] - s[0]) * (s[2] - s[0])) +
                3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

__device__ __forceinline__ double hfun(double s) { return 0.5 * (1.0 + s * sqrt(3.0)); }

// Strain of a C3D8 at a natural point from u_e (B applied without forming
// it; skipped zero entries of B cannot change a non-zero sum).  Returns
// false when det J <= 0 (never for an element that assembled).
__device__ bool hex_strain(const double* x, const double* ue, double xi, double eta, double zeta,
                           double* eps) {
    double dn[3][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double a = hexc(i, 0), b = hexc(i, 1), c = hexc(i, 2);
        dn[0][i] = 0.125 * a * (1.0 + eta * b) * (1.0 + zeta * c);
        dn[1][i] = 0.125 * b * (1.0 + xi * a) * (1.0 + zeta * c);
        dn[2][i] = 0.125 * c * (1.0 + xi * a) * (1.0 + eta * b);
    }
    double J[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i) s += dn[a][i] * x[i * 3 + b];
            J[a * 3 + b] = s;
        }
    double detj = det3(J);
    if (detj <= 0.0) return false;
    double id = 1.0 / detj;
    double inv[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) inv[i * 3 + j] = inv3_entry(J, id, i, j);
#pragma unroll
    for (int r = 0; r < 6; ++r) eps[r] = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double g[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a) s += inv[b * 3 + a] * dn[a][i];
            g[b] = s;
        }
        const double u0 = ue[3 * i], u1 = ue[3 * i + 1], u2 = ue[3 * i + 2];
        // columns 3i, 3i+1, 3i+2 in ascending order per strain row
        eps[0] += g[0] * u0;
        eps[1] += g[1] * u1;
        eps[2] += g[2] * u2;
        eps[3] += g[1] * u0;
        eps[3] += g[0] * u1;
        eps[4] += g[2] * u1;
        eps[4] += g[1] * u2;
        eps[5] += g[2] * u0;
        eps[5] += g[0] * u2;
    }
    return true;
}

// solid_stress (element.rs:904-915) with the zero entries of D skipped.
__device__ __forceinline__ void solid_stress(double lam, double mu, double diag, const double* e,
                                             double* s) {
    s[0] = diag * e[0] + lam * e[1] + lam * e[2];
    s[1] = lam * e[0] + diag * e[1] + lam * e[2];
    s[2] = lam * e[0] + lam * e[1] + diag * e[2];
    s[3] = mu * e[3];
    s[4] = mu * e[4];
    s[5] = mu * e[5];
}

__device__ bool quad_strain(const double* x, const double* ue, double xi, double eta,
                            double* eps) {
    double dxi[4], deta[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double xi_i = quadc(i, 0), eta_i = quadc(i, 1);
        dxi[i] = 0.25 * xi_i * (1.0 + eta * eta_i);
        deta[i] = 0.25 * eta_i * (1.0 + xi * xi_i);
    }
    double j00 = 0.0, j01 = 0.0, j10 = 0.0, j11 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        j00 += dxi[i] * x[i * 3];
        j01 += dxi[i] * x[i * 3 + 1];
        j10 += deta[i] * x[i * 3];
        j11 += deta[i] * x[i * 3 + 1];
    }
    double detj = j00 * j11 - j01 * j10;
    if (detj <= 0.0) return false;
    double inv = 1.0 / detj;
    eps[0] = 0.0; eps[1] = 0.0; eps[2] = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double dnx = inv * (j11 * dxi[i] - j01 * deta[i]);
        double dny = inv * (j00 * deta[i] - j10 * dxi[i]);
        eps[0] += dnx * ue[2 * i];
        eps[1] += dny * ue[2 * i + 1];
        eps[2] += dny * ue[2 * i];
        eps[2] += dnx * ue[2 * i + 1];
    }
    return true;
}

// plane_stress (element.rs:867-881)
__device__ __forceinline__ void plane_stress(const double (*d)[3], const double* e, double* s) {
    s[0] = d[0][0] * e[0] + d[0][1] * e[1];
    s[1] = d[1][0] * e[0] + d[1][1] * e[1];
    s[2] = 0.0;
    s[3] = d[2][2] * e[2];
    s[4] = 0.0;
    s[5] = 0.0;
}

// One thread per element: centroid von Mises and the extrapolated nodal
// stress components (element.rs:926-1053), written to nodal[e][a][6].
__global__ void stress_elem_kernel(int64_t n_elem, int ndof, int max_nn,
                                   const uint8_t* __restrict__ kind,
                                   const int64_t* __restrict__ conn_ptr,
                                   const int32_t* __restrict__ conn,
                                   const double* __restrict__ xyz,
                                   const double* __restrict__ youngs,
                                   const double* __restrict__ poisson,
                                   const double* __restrict__ u, double* __restrict__ vm_elem,
                                   double* __restrict__ nodal) {
    int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    const int k = kind[e];
    const int64_t q0 = conn_ptr[e];
    const double g = 1.0 / sqrt(3.0);
    double* out = nodal + e * int64_t(max_nn) * 6;
    if (k == SVX_C3D8) {
        double x[24], ue[24];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int64_t nd = conn[q0 + i];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                x[i * 3 + b] = xyz[nd * 3 + b];
                ue[i * 3 + b] = u[nd * ndof + b];
            }
        }
        double E = youngs[e], nu = poisson[e];
        double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        double mu = E / (2.0 * (1.0 + nu));
        double diag = lam + 2.0 * mu;
        double eps[6], s[6];
        hex_strain(x, ue, 0.0, 0.0, 0.0, eps);
        solid_stress(lam, mu, diag, eps, s);
        vm_elem[e] = von_mises(s);
        double gp[8][6];
#pragma unroll 1
        for (int j = 0; j < 8; ++j) {
            double xi = (j & 4) ? g : -g, eta = (j & 2) ? g : -g, zeta = (j & 1) ? g : -g;
            hex_strain(x, ue, xi, eta, zeta, eps);
            solid_stress(lam, mu, diag, eps, gp[j]);
        }
#pragma unroll 1
        for (int i = 0; i < 8; ++i) {
            double o[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                double gx = (j & 4) ? 1.0 : -1.0, gy = (j & 2) ? 1.0 : -1.0,
                       gz = (j & 1) ? 1.0 : -1.0;
                double w = hfun(hexc(i, 0) * gx) * hfun(hexc(i, 1) * gy) * hfun(hexc(i, 2) * gz);
#pragma unroll
                for (int m = 0; m < 6; ++m) o[m] += w * gp[j][m];
            }
#pragma unroll
            for (int m = 0; m < 6; ++m) out[i * 6 + m] = o[m];
        }
    } else if (k == SVX_CPS4) {
        double x[12], ue[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int64_t nd = conn[q0 + i];
            x[i * 3] = xyz[nd * 3];
            x[i * 3 + 1] = xyz[nd * 3 + 1];
            x[i * 3 + 2] = xyz[nd * 3 + 2];
            ue[2 * i] = u[nd * ndof];
            ue[2 * i + 1] = u[nd * ndof + 1];
        }
        double d[3][3];
        d_matrix(youngs[e], poisson[e], d);
        double eps[3], s[6];
        quad_strain(x, ue, 0.0, 0.0, eps);
        plane_stress(d, eps, s);
        vm_elem[e] = von_mises(s);
        double gp[4][6];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double xi = (j & 2) ? g : -g, eta = (j & 1) ? g : -g;
            quad_strain(x, ue, xi, eta, eps);
            plane_stress(d, eps, gp[j]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            double o[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                double gx = (j & 2) ? 1.0 : -1.0, gy = (j & 1) ? 1.0 : -1.0;
                double w = hfun(quadc(i, 0) * gx) * hfun(quadc(i, 1) * gy);
#pragma unroll
                for (int m = 0; m < 6; ++m) o[m] += w * gp[j][m];
            }
#pragma unroll
            for (int m = 0; m < 6; ++m) out[i * 6 + m] = o[m];
        }
    } else {  // CPS3: constant strain, the same stress at the three nodes
        double x[9], ue[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            int64_t nd = conn[q0 + i];
            x[i * 3] = xyz[nd * 3];
            x[i * 3 + 1] = xyz[nd * 3 + 1];
            ue[2 * i] = u[nd * ndof];
            ue[2 * i + 1] = u[nd * ndof + 1];
        }
        double d[3][3];
        d_matrix(youngs[e], poisson[e], d);
        double b[3] = {x[4] - x[7], x[7] - x[1], x[1] - x[4]};
        double c[3] = {x[6] - x[3], x[0] - x[6], x[3] - x[0]};
        double two_a = b[0] * c[1] - b[1] * c[0];
        double inv = 1.0 / two_a;
        double eps[3] = {0.0, 0.0, 0.0}, s[6];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            eps[0] += (b[i] * inv) * ue[2 * i];
            eps[1] += (c[i] * inv) * ue[2 * i + 1];
            eps[2] += (c[i] * inv) * ue[2 * i];
            eps[2] += (b[i] * inv) * ue[2 * i + 1];
        }
        plane_stress(d, eps, s);
        vm_elem[e] = von_mises(s);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int m = 0; m < 6; ++m) out[i * 6 + m] = s[m];
    }
}

// Nodal average in slot order (element ascending, then local position),
// stress.rs:53-98; no atomics.
__global__ void nodal_average_kernel(int64_t n_nodes, int max_nn,
                                     const int64_t* __restrict__ slot_ptr,
                                     const int32_t* __restrict__ slot_elem,
                                     const uint8_t* __restrict__ slot_local,
                                     const double* __restrict__ nodal,
                                     double* __restrict__ vm_node) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    double sum[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int64_t s0 = slot_ptr[i], s1 = slot_ptr[i + 1];
    for (int64_t s = s0; s < s1; ++s) {
        const double* src = nodal + (int64_t(slot_elem[s]) * max_nn + slot_local[s]) * 6;
#pragma unroll
        for (int m = 0; m < 6; ++m) sum[m] += src[m];
    }
    if (s1 == s0) {
        vm_node[i] = 0.0;
        return;
    }
    double c = double(s1 - s0);
    double avg[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) avg[m] = sum[m] / c;
    vm_node[i] = von_mises(avg);
}

// K10: reactions K_orig u - f_orig at each constrained entry
// (stress.rs:103-118), serial row order like Csr::mat_vec.
__global__ void reactions_kernel(int64_t n_fixed, const int64_t* __restrict__ fixed_row,
                                 const int32_t* __restrict__ fixed_slot,
                                 const int32_t* __restrict__ kc_ptr,
                                 const int32_t* __restrict__ kc_col,
                                 const double* __restrict__ kc_val,
                                 const double* __restrict__ u,
                                 const double* __restrict__ f_orig, double* __restrict__ out) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_fixed) return;
    int r = fixed_slot[i];
    double o = 0.0;
    for (int j = kc_ptr[r]; j < kc_ptr[r + 1]; ++j) o += kc_val[j] * u[kc_col[j]];
    out[i] = o - f_orig[fixed_row[i]];
}

__global__ void displacements_kernel(int64_t n_nodes, int ndof, const double* __restrict__ u,
                                     double* __restrict__ disp3) {
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    disp3[3 * i] = u[i * ndof];
    disp3[3 * i + 1] = u[i * ndof + 1];
    disp3[3 * i + 2] = ndof == 3 ? u[i * ndof + 2] : 0.0;
}

// ---------------------------------------------------------------- conduction
// Steady heat conduction (heat.rs:149-296), one thread per element: the
// conduction matrix k * integral of grad N . grad N (N x N, N = nodes) into
// the element's Ke slot, and the consistent heat-source load into fe.  The
// gradients are built exactly as quad_b / hex_b build the first rows of B
// (element.rs:147-171, 479-521), in the reference's loop and sum order, so
// the values are bit-identical to the oracle's.  Kinds outside CPS3, CPS4 /
// CPE4 and C3D8 flag SVX_REASON_UNSUPPORTED_KIND.
__global__ void conduction_kernel(int64_t n_elem, const uint8_t* __restrict__ kind,
                                  const int64_t* __restrict__ conn_ptr,
                                  const int32_t* __restrict__ conn,
                                  const double* __restrict__ xyz, double k, double t, int has_q,
                                  double q, double* __restrict__ ke, int ke_stride,
                                  double* __restrict__ fe, int max_nn,
                                  unsigned long long* first_fail) {
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    const int kd = kind[e];
    const int64_t q0 = conn_ptr[e];
    double* ke_e = ke + e * int64_t(ke_stride);
    double* fe_e = fe + e * int64_t(max_nn);
    const double qq = has_q ? q : 0.0;
    auto fail = [&](int reason) {
        atomicMin(first_fail, (unsigned long long)(e << 8) | (unsigned long long)reason);
    };
    if (kd == SVX_CPS3) {
        double p[3][2];
        for (int i = 0; i < 3; ++i) {
            const int64_t nd = conn[q0 + i];
            p[i][0] = xyz[nd * 3];
            p[i][1] = xyz[nd * 3 + 1];
        }
        // heat.rs:140-145
        const double b[3] = {p[1][1] - p[2][1], p[2][1] - p[0][1], p[0][1] - p[1][1]};
        const double c[3] = {p[2][0] - p[1][0], p[0][0] - p[2][0], p[1][0] - p[0][0]};
        const double two_a = b[0] * c[1] - b[1] * c[0];
        if (two_a == 0.0) {
            fail(SVX_REASON_DEGENERATE_TRI);
            return;
        }
        const double w = k * t / (2.0 * fabs(two_a));
        for (int i = 0; i < 3; ++i) {
            fe_e[i] = has_q ? q * t * fabs(two_a) / 6.0 : 0.0;
            for (int j = 0; j < 3; ++j) ke_e[i * 3 + j] = w * (b[i] * b[j] + c[i] * c[j]);
        }
        return;
    }
    const double g = 1.0 / sqrt(3.0);
    if (kd == SVX_CPS4 || kd == SVX_CPE4) {
        double x[8];
        for (int i = 0; i < 4; ++i) {
            const int64_t nd = conn[q0 + i];
            x[2 * i] = xyz[nd * 3];
            x[2 * i + 1] = xyz[nd * 3 + 1];
        }
        double kl[16], fl[4];
        for (int i = 0; i < 16; ++i) kl[i] = 0.0;
        for (int i = 0; i < 4; ++i) fl[i] = 0.0;
        for (int a = 0; a < 2; ++a)
            for (int bq = 0; bq < 2; ++bq) {
                const double xi = a ? g : -g, eta = bq ? g : -g;
                double dxi[4], deta[4];
                for (int i = 0; i < 4; ++i) {
                    const double xi_i = quadc(i, 0), eta_i = quadc(i, 1);
                    dxi[i] = 0.25 * xi_i * (1.0 + eta * eta_i);
                    deta[i] = 0.25 * eta_i * (1.0 + xi * xi_i);
                }
                double j00 = 0.0, j01 = 0.0, j10 = 0.0, j11 = 0.0;
                for (int i = 0; i < 4; ++i) {
                    j00 += dxi[i] * x[2 * i];
                    j01 += dxi[i] * x[2 * i + 1];
                    j10 += deta[i] * x[2 * i];
                    j11 += deta[i] * x[2 * i + 1];
                }
                const double detj = j00 * j11 - j01 * j10;
                if (detj <= 0.0) {
                    fail(SVX_REASON_BAD_JACOBIAN);
                    return;
                }
                const double inv = 1.0 / detj;
                double dnx[4], dny[4], n[4];
                for (int i = 0; i < 4; ++i) {
                    dnx[i] = inv * (j11 * dxi[i] - j01 * deta[i]);
                    dny[i] = inv * (j00 * deta[i] - j10 * dxi[i]);
                    n[i] = 0.25 * (1.0 + xi * quadc(i, 0)) * (1.0 + eta * quadc(i, 1));
                }
                for (int i = 0; i < 4; ++i) {
                    fl[i] += qq * t * detj * n[i];
                    for (int j = 0; j < 4; ++j)
                        kl[i * 4 + j] += k * t * detj * (dnx[i] * dnx[j] + dny[i] * dny[j]);
                }
            }
        for (int i = 0; i < 16; ++i) ke_e[i] = kl[i];
        for (int i = 0; i < 4; ++i) fe_e[i] = fl[i];
        return;
    }
    if (kd == SVX_C3D8) {
        double x[24];
        for (int i = 0; i < 8; ++i) {
            const int64_t nd = conn[q0 + i];
            for (int b = 0; b < 3; ++b) x[i * 3 + b] = xyz[nd * 3 + b];
        }
        double kl[64], fl[8];
        for (int i = 0; i < 64; ++i) kl[i] = 0.0;
        for (int i = 0; i < 8; ++i) fl[i] = 0.0;
        for (int gp = 0; gp < 8; ++gp) {
            const double xi = (gp & 4) ? g : -g, eta = (gp & 2) ? g : -g,
                         zeta = (gp & 1) ? g : -g;
            double dn[3][8];
            for (int i = 0; i < 8; ++i) {
                const double a = hexc(i, 0), b = hexc(i, 1), c = hexc(i, 2);
                dn[0][i] = 0.125 * a * (1.0 + eta * b) * (1.0 + zeta * c);
                dn[1][i] = 0.125 * b * (1.0 + xi * a) * (1.0 + zeta * c);
                dn[2][i] = 0.125 * c * (1.0 + xi * a) * (1.0 + eta * b);
            }
            double J[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double sum = 0.0;
                    for (int i = 0; i < 8; ++i) sum += dn[a][i] * x[i * 3 + b];
                    J[a * 3 + b] = sum;
                }
            const double detj = det3(J);
            if (detj <= 0.0) {
                fail(SVX_REASON_BAD_JACOBIAN);
                return;
            }
            const double id = 1.0 / detj;
            double inv[9];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) inv[i * 3 + j] = inv3_entry(J, id, i, j);
            double gr[8][3], n[8];
            for (int i = 0; i < 8; ++i) {
                for (int b = 0; b < 3; ++b) {
                    double sum = 0.0;
                    for (int a = 0; a < 3; ++a) sum += inv[b * 3 + a] * dn[a][i];
                    gr[i][b] = sum;
                }
                n[i] = 0.125 * (1.0 + xi * hexc(i, 0)) * (1.0 + eta * hexc(i, 1)) *
                       (1.0 + zeta * hexc(i, 2));
            }
            for (int i = 0; i < 8; ++i) {
                fl[i] += qq * detj * n[i];
                for (int j = 0; j < 8; ++j) {
                    double v = 0.0;
                    for (int r = 0; r < 3; ++r) v += gr[i][r] * gr[j][r];
                    kl[i * 8 + j] += k * detj * v;
                }
            }
        }
        for (int i = 0; i < 64; ++i) ke_e[i] = kl[i];
        for (int i = 0; i < 8; ++i) fe_e[i] = fl[i];
        return;
    }
    fail(SVX_REASON_UNSUPPORTED_KIND);
}

// ---------------------------------------------------------------- consistent mass
// Consistent mass matrices (modal.rs:82-146), one thread per element, into
// the element's Ke slot (row-major (ND nn)^2) for the fixed-order assembly:
// CPS3 closed form rho t |2A| / 24 x (2 on the diagonal, 1 off it);
// CPS4 / CPE4 rho t detJ N_i N_j under 2x2 Gauss (xi outer); C3D8
// rho detJ N_i N_j under 2x2x2 Gauss (xi, eta, zeta nested), each value on
// every dof pair (d, d) of nodes i, j and zero elsewhere.  The Jacobians
// are built as quad_b / hex_b build them (the conduction kernel's code), the
// node-pair values summed over the Gauss points in the reference's order,
// so the values are bit-identical to the oracle's.  Failures: a zero-area
// triangle, det J <= 0 at a Gauss point, a kind outside CPS3 / CPS4 / CPE4
// / C3D8.
__global__ void mass_kernel(int64_t n_elem, int ndof, const uint8_t* __restrict__ kind,
                            const int64_t* __restrict__ conn_ptr,
                            const int32_t* __restrict__ conn, const double* __restrict__ xyz,
                            double rho, double t, double* __restrict__ ke, int ke_stride,
                            unsigned long long* first_fail) {
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n_elem) return;
    const int kd = kind[e];
    const int64_t q0 = conn_ptr[e];
    double* ke_e = ke + e * int64_t(ke_stride);
    auto fail = [&](int reason) {
        atomicMin(first_fail, (unsigned long long)(e << 8) | (unsigned long long)reason);
    };
    // writes the (nn ndof)^2 matrix whose dof pairs (d, d) of nodes i, j
    // hold v[i * nn + j]
    auto put = [&](const double* v, int nn) {
        const int N = nn * ndof;
        for (int a = 0; a < N; ++a)
            for (int c = 0; c < N; ++c)
                ke_e[a * N + c] = (a % ndof == c % ndof) ? v[(a / ndof) * nn + c / ndof] : 0.0;
    };
    if (kd == SVX_CPS3) {
        double p[3][2];
        for (int i = 0; i < 3; ++i) {
            const int64_t nd = conn[q0 + i];
            p[i][0] = xyz[nd * 3];
            p[i][1] = xyz[nd * 3 + 1];
        }
        const double two_a = (p[1][0] - p[0][0]) * (p[2][1] - p[0][1]) -
                             (p[2][0] - p[0][0]) * (p[1][1] - p[0][1]);
        if (two_a == 0.0) {
            fail(SVX_REASON_DEGENERATE_TRI);
            return;
        }
        const double w = rho * t * fabs(two_a) / 24.0;
        double v[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) v[i * 3 + j] = w * (i == j ? 2.0 : 1.0);
        put(v, 3);
        return;
    }
    const double g = 1.0 / sqrt(3.0);
    if (kd == SVX_CPS4 || kd == SVX_CPE4) {
        double x[8];
        for (int i = 0; i < 4; ++i) {
            const int64_t nd = conn[q0 + i];
            x[2 * i] = xyz[nd * 3];
            x[2 * i + 1] = xyz[nd * 3 + 1];
        }
        double v[16];
        for (int i = 0; i < 16; ++i) v[i] = 0.0;
        for (int a = 0; a < 2; ++a)
            for (int bq = 0; bq < 2; ++bq) {
                const double xi = a ? g : -g, eta = bq ? g : -g;
                double dxi[4], deta[4], n[4];
                for (int i = 0; i < 4; ++i) {
                    const double xi_i = quadc(i, 0), eta_i = quadc(i, 1);
                    dxi[i] = 0.25 * xi_i * (1.0 + eta * eta_i);
                    deta[i] = 0.25 * eta_i * (1.0 + xi * xi_i);
                    n[i] = 0.25 * (1.0 + xi * xi_i) * (1.0 + eta * eta_i);
                }
                double j00 = 0.0, j01 = 0.0, j10 = 0.0, j11 = 0.0;
                for (int i = 0; i < 4; ++i) {
                    j00 += dxi[i] * x[2 * i];
                    j01 += dxi[i] * x[2 * i + 1];
                    j10 += deta[i] * x[2 * i];
                    j11 += deta[i] * x[2 * i + 1];
                }
                const double detj = j00 * j11 - j01 * j10;
                if (detj <= 0.0) {
                    fail(SVX_REASON_BAD_JACOBIAN);
                    return;
                }
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j) v[i * 4 + j] += rho * t * detj * n[i] * n[j];
            }
        put(v, 4);
        return;
    }
    if (kd == SVX_C3D8) {
        double x[24];
        for (int i = 0; i < 8; ++i) {
            const int64_t nd = conn[q0 + i];
            for (int b = 0; b < 3; ++b) x[i * 3 + b] = xyz[nd * 3 + b];
        }
        double v[64];
        for (int i = 0; i < 64; ++i) v[i] = 0.0;
        for (int gp = 0; gp < 8; ++gp) {
            const double xi = (gp & 4) ? g : -g, eta = (gp & 2) ? g : -g,
                         zeta = (gp & 1) ? g : -g;
            double dn[3][8], n[8];
            for (int i = 0; i < 8; ++i) {
                const double a = hexc(i, 0), b = hexc(i, 1), c = hexc(i, 2);
                dn[0][i] = 0.125 * a * (1.0 + eta * b) * (1.0 + zeta * c);
                dn[1][i] = 0.125 * b * (1.0 + xi * a) * (1.0 + zeta * c);
                dn[2][i] = 0.125 * c * (1.0 + xi * a) * (1.0 + eta * b);
                n[i] = 0.125 * (1.0 + xi * a) * (1.0 + eta * b) * (1.0 + zeta * c);
            }
            double J[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double sum = 0.0;
                    for (int i = 0; i < 8; ++i) sum += dn[a][i] * x[i * 3 + b];
                    J[a * 3 + b] = sum;
                }
            const double detj = det3(J);
            if (detj <= 0.0) {
                fail(SVX_REASON_BAD_JACOBIAN);
                return;
            }
            for (int i = 0; i < 8; ++i)
                for (int j = 0; j < 8; ++j) v[i * 8 + j] += rho * detj * n[i] * n[j];
        }
        put(v, 8);
        return;
    }
    fail(SVX_REASON_UNSUPPORTED_KIND);
}


// Element source loads summed per node over its incident (element, local)
// slots in ascending element order: the reference's f[idx[i]] += fe[i] in
// element enumeration order (heat.rs:207-212, 283-288).
__global__ void node_source_kernel(int64_t n_nodes, const int64_t* __restrict__ slot_ptr,
                                   const int32_t* __restrict__ slot_elem,
                                   const uint8_t* __restrict__ slot_local,
                                   const double* __restrict__ fe, int max_nn,
                                   double* __restrict__ f) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    double s = 0.0;
    for (int64_t sl = slot_ptr[i]; sl < slot_ptr[i + 1]; ++sl)
        s += fe[int64_t(slot_elem[sl]) * max_nn + slot_local[sl]];
    f[i] = s;
}

// heat.rs:298-358 for linear plane edges, one thread in flux order (the
// host has checked kinds, faces and edge lengths).
__global__ void flux_load_kernel(int64_t n_flux, const int64_t* __restrict__ flux_elem,
                                 const int32_t* __restrict__ flux_face,
                                 const double* __restrict__ flux_value,
                                 const uint8_t* __restrict__ kind,
                                 const int64_t* __restrict__ conn_ptr,
                                 const int32_t* __restrict__ conn,
                                 const double* __restrict__ xyz, double t, double* f) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int64_t q = 0; q < n_flux; ++q) {
        const int64_t e = flux_elem[q];
        const int face = flux_face[q];
        const int corners = (kind[e] == SVX_CPS3) ? 3 : 4;
        const int64_t q0 = conn_ptr[e];
        const int64_t na = conn[q0 + face - 1], nb = conn[q0 + face % corners];
        const double dx = xyz[nb * 3] - xyz[na * 3], dy = xyz[nb * 3 + 1] - xyz[na * 3 + 1];
        const double len = sqrt(dx * dx + dy * dy);
        const double total = flux_value[q] * t * len;
        f[na] += total / 2.0;
        f[nb] += total / 2.0;
    }
}

// heat.rs:361-407, one thread per row: a free row moves K_rc T_c of every
// prescribed column to its right-hand side in column order and zeroes the
// entry; a prescribed row becomes an identity row with T on the right.
__global__ void temperature_rows_kernel(int64_t n, const int32_t* __restrict__ row_ptr,
                                        const int32_t* __restrict__ col_idx,
                                        const double* __restrict__ pres,
                                        double* __restrict__ vals, double* __restrict__ f) {
    const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const double tr = pres[r];
    if (isnan(tr)) {
        double fr = f[r];
        for (int32_t ii = row_ptr[r]; ii < row_ptr[r + 1]; ++ii) {
            const double tc = pres[col_idx[ii]];
            if (!isnan(tc)) {
                fr -= vals[ii] * tc;
                vals[ii] = 0.0;
            }
        }
        f[r] = fr;
    } else {
        for (int32_t ii = row_ptr[r]; ii < row_ptr[r + 1]; ++ii)
            vals[ii] = (col_idx[ii] == r) ? 1.0 : 0.0;
        f[r] = tr;
    }
}

inline unsigned blocks_for(int64_t n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace

uint64_t integrate_elements(svx_ctx* ctx, svx_op* op, double* ke, int ke_stride) {
    DBuf<unsigned long long> fail;
    fail.alloc(ctx->pool, 1);
    SVX_CUDA(cudaMemsetAsync(fail.p, 0xff, sizeof(unsigned long long), ctx->stream));
    if (op->n_elem > 0) {
        int64_t blocks = (op->n_elem + WARPS - 1) / WARPS;
        int64_t cap = int64_t(ctx->sm_count) * 64;
        if (blocks > cap) blocks = cap;
        integrate_kernel<<<unsigned(blocks), WARPS * 32, 0, ctx->stream>>>(
            op->n_elem, op->kind.p, op->conn_ptr.p, op->conn.p, op->xyz.p, op->youngs.p,
            op->poisson.p, op->thickness, op->thick_elem.p, ke, ke_stride, fail.p);
        SVX_LAUNCH_CHECK();
    }
    unsigned long long h = 0;
    SVX_CUDA(cudaMemcpyAsync(&h, fail.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    SVX_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
}

void recover_stress(svx_ctx* ctx, svx_op* op, const double* u, double* vm_elem, double* vm_node,
                    double* reactions, double* disp3) {
    cudaStream_t st = ctx->stream;
    const Pattern& P = op->pat;
    if (vm_elem || vm_node) {
        DBuf<double> nodal, vme;
        nodal.alloc(ctx->pool, size_t(op->n_elem) * P.max_nn * 6 + 1);
        double* vm_e = vm_elem;
        if (!vm_e) {
            vme.alloc(ctx->pool, op->n_elem + 1);
            vm_e = vme.p;
        }
        if (op->n_elem > 0) {
            stress_elem_kernel<<<blocks_for(op->n_elem, 128), 128, 0, st>>>(
                op->n_elem, op->ndof, P.max_nn, op->kind.p, op->conn_ptr.p, op->conn.p,
                op->xyz.p, op->youngs.p, op->poisson.p, u, vm_e, nodal.p);
            SVX_LAUNCH_CHECK();
        }
        if (vm_node && op->n_nodes > 0) {
            nodal_average_kernel<<<blocks_for(op->n_nodes, 256), 256, 0, st>>>(
                op->n_nodes, P.max_nn, P.slot_ptr.p, P.slot_elem.p, P.slot_local.p, nodal.p,
                vm_node);
            SVX_LAUNCH_CHECK();
        }
        SVX_CUDA(cudaStreamSynchronize(st));
    }
    if (reactions && op->n_fixed > 0) {
        reactions_kernel<<<blocks_for(op->n_fixed, 128), 128, 0, st>>>(
            op->n_fixed, op->fixed_row.p, op->fixed_slot.p, op->kc_ptr.p, op->kc_col.p,
            op->kc_val.p, u, op->f_orig.p, reactions);
        SVX_LAUNCH_CHECK();
    }
    if (disp3 && op->n_nodes > 0) {
        displacements_kernel<<<blocks_for(op->n_nodes, 256), 256, 0, st>>>(op->n_nodes,
                                                                           op->ndof, u, disp3);
        SVX_LAUNCH_CHECK();
    }
}

uint64_t integrate_mass(svx_ctx* ctx, svx_op* op, double rho, double* ke, int ke_stride) {
    DBuf<unsigned long long> fail;
    fail.alloc(ctx->pool, 1);
    SVX_CUDA(cudaMemsetAsync(fail.p, 0xff, sizeof(unsigned long long), ctx->stream));
    if (op->n_elem > 0) {
        mass_kernel<<<blocks_for(op->n_elem, 128), 128, 0, ctx->stream>>>(
            op->n_elem, op->ndof, op->kind.p, op->conn_ptr.p, op->conn.p, op->xyz.p, rho,
            op->thickness, ke, ke_stride, fail.p);
        SVX_LAUNCH_CHECK();
    }
    unsigned long long h = 0;
    SVX_CUDA(cudaMemcpyAsync(&h, fail.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    SVX_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
}

uint64_t integrate_conduction(svx_ctx* ctx, svx_op* op, double conductivity, int has_source,
                              double source, double* ke, int ke_stride, double* fe) {
    DBuf<unsigned long long> fail;
    fail.alloc(ctx->pool, 1);
    SVX_CUDA(cudaMemsetAsync(fail.p, 0xff, sizeof(unsigned long long), ctx->stream));
    if (op->n_elem > 0) {
        conduction_kernel<<<blocks_for(op->n_elem, 128), 128, 0, ctx->stream>>>(
            op->n_elem, op->kind.p, op->conn_ptr.p, op->conn.p, op->xyz.p, conductivity,
            op->thickness, has_source, source, ke, ke_stride, fe, op->pat.max_nn, fail.p);
        SVX_LAUNCH_CHECK();
    }
    unsigned long long h = 0;
    SVX_CUDA(cudaMemcpyAsync(&h, fail.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    SVX_CUDA(cudaStreamSynchronize(ctx->stream));
    return h;
}

void thermal_loads(svx_ctx* ctx, svx_op* op, const double* fe, int has_source, int64_t n_flux,
                   const int64_t* flux_elem, const int32_t* flux_face, const double* flux_value,
                   double* f) {
    cudaStream_t st = ctx->stream;
    const Pattern& P = op->pat;
    if (has_source && op->n_nodes > 0) {
        node_source_kernel<<<blocks_for(op->n_nodes, 256), 256, 0, st>>>(
            op->n_nodes, P.slot_ptr.p, P.slot_elem.p, P.slot_local.p, fe, P.max_nn, f);
        SVX_LAUNCH_CHECK();
    } else if (op->n_nodes > 0) {
        SVX_CUDA(cudaMemsetAsync(f, 0, sizeof(double) * size_t(op->n_nodes), st));
    }
    if (n_flux > 0) {
        flux_load_kernel<<<1, 32, 0, st>>>(n_flux, flux_elem, flux_face, flux_value, op->kind.p,
                                           op->conn_ptr.p, op->conn.p, op->xyz.p, op->thickness,
                                           f);
        SVX_LAUNCH_CHECK();
    }
}

void apply_temperatures(svx_ctx* ctx, svx_op* op, const double* pres) {
    const Pattern& P = op->pat;
    if (op->n > 0) {
        temperature_rows_kernel<<<blocks_for(op->n, 256), 256, 0, ctx->stream>>>(
            op->n, P.row_ptr.p, P.col_idx.p, pres, op->vals.p, op->f.p);
        SVX_LAUNCH_CHECK();
    }
}

}  // namespace svx

// svx_oracle.cpp - CPU oracle (test infrastructure) for the Solvix
// linear-static path.  A C++ restatement of the reference's Rust code; every
// function cites the file:line it follows.  Build with -O2 -ffp-contract=off
// (Rust never fuses a*b+c) and without -ffast-math, so that each expression
// rounds exactly like the reference's.
//
// csr_from_triplets (assembly.rs:87-116) sums duplicate (row, col) triplets
// in the order `sort_unstable_by_key` leaves them.  The oracle restates that
// sort (the row-sort section below), so its K, and with it the whole PCG
// trajectory, is bit-identical to the reference's: every published iteration
// count and residual of the reference's decks is reproduced.  A stable mode
// (triplet-stream order) is kept for bit-exact comparison with the CUDA
// assembly, which sums in ascending element order.
//
// Only the serial sums and the threaded row-chunked SpMV of the reference are
// restated; the threaded element loop writes each element's triplets at a
// fixed offset, which equals the reference's chunk-ordered merge
// (assembly.rs:306-363).

#include "svx_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

using std::size_t;

// ---------------------------------------------------------------- D matrices
// element.rs:10-17
void d_matrix(double e, double nu, double d[3][3]) {
    double c = e / (1.0 - nu * nu);
    d[0][0] = c;
    d[0][1] = nu * c;
    d[0][2] = 0.0;
    d[1][0] = nu * c;
    d[1][1] = c;
    d[1][2] = 0.0;
    d[2][0] = 0.0;
    d[2][1] = 0.0;
    d[2][2] = c * (1.0 - nu) / 2.0;
}

// element.rs:33-47
void d3_matrix(double e, double nu, double d[6][6]) {
    double lam = e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = e / (2.0 * (1.0 + nu));
    double diag = lam + 2.0 * mu;
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) d[r][c] = 0.0;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) d[r][c] = (r == c) ? diag : lam;
    d[3][3] = mu;
    d[4][4] = mu;
    d[5][5] = mu;
}

// ---------------------------------------------------------------- btdb
// element.rs:830-851: DB = D*B first, then for a <= c the w-scaled
// B^T*DB entry is added to ke[a][c] and mirrored to ke[c][a].
template <int N, int S>
void btdb(double* ke, const double b[S][N], const double d[S][S], double w) {
    double db[S][N];
    for (int r = 0; r < S; ++r)
        for (int c = 0; c < N; ++c) {
            double s = 0.0;
            for (int k = 0; k < S; ++k) s += d[r][k] * b[k][c];
            db[r][c] = s;
        }
    for (int a = 0; a < N; ++a)
        for (int c = a; c < N; ++c) {
            double s = 0.0;
            for (int r = 0; r < S; ++r) s += b[r][a] * db[r][c];
            double v = w * s;
            ke[a * N + c] += v;
            if (a != c) ke[c * N + a] += v;
        }
}

// ---------------------------------------------------------------- CPS3
// element.rs:91-116; returns false for a zero signed area.
bool cps3_b_matrix(const double xy[3][2], double bm[3][6], double* two_a_out) {
    double b[3] = {xy[1][1] - xy[2][1], xy[2][1] - xy[0][1], xy[0][1] - xy[1][1]};
    double c[3] = {xy[2][0] - xy[1][0], xy[0][0] - xy[2][0], xy[1][0] - xy[0][0]};
    double two_a = b[0] * c[1] - b[1] * c[0];
    if (two_a == 0.0) return false;
    double inv = 1.0 / two_a;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 6; ++k) bm[r][k] = 0.0;
    for (int i = 0; i < 3; ++i) {
        bm[0][2 * i] = b[i] * inv;
        bm[1][2 * i + 1] = c[i] * inv;
        bm[2][2 * i] = c[i] * inv;
        bm[2][2 * i + 1] = b[i] * inv;
    }
    *two_a_out = two_a;
    return true;
}

// ---------------------------------------------------------------- CPS4
const double QUAD_CORNERS[4][2] = {{-1.0, -1.0}, {1.0, -1.0}, {1.0, 1.0}, {-1.0, 1.0}};

// element.rs:134-144
void quad_shape_derivs(double xi, double eta, double dxi[4], double deta[4]) {
    for (int i = 0; i < 4; ++i) {
        double xi_i = QUAD_CORNERS[i][0], eta_i = QUAD_CORNERS[i][1];
        dxi[i] = 0.25 * xi_i * (1.0 + eta * eta_i);
        deta[i] = 0.25 * eta_i * (1.0 + xi * xi_i);
    }
}

// element.rs:147-171; false when det(J) <= 0 (a NaN determinant passes).
bool quad_b(const double xy[4][2], double xi, double eta, double bm[3][8], double* detj_out) {
    double dxi[4], deta[4];
    quad_shape_derivs(xi, eta, dxi, deta);
    double j00 = 0.0, j01 = 0.0, j10 = 0.0, j11 = 0.0;
    for (int i = 0; i < 4; ++i) {
        j00 += dxi[i] * xy[i][0];
        j01 += dxi[i] * xy[i][1];
        j10 += deta[i] * xy[i][0];
        j11 += deta[i] * xy[i][1];
    }
    double detj = j00 * j11 - j01 * j10;
    if (detj <= 0.0) return false;
    double inv = 1.0 / detj;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 8; ++k) bm[r][k] = 0.0;
    for (int i = 0; i < 4; ++i) {
        double dnx = inv * (j11 * dxi[i] - j01 * deta[i]);
        double dny = inv * (j00 * deta[i] - j10 * dxi[i]);
        bm[0][2 * i] = dnx;
        bm[1][2 * i + 1] = dny;
        bm[2][2 * i] = dny;
        bm[2][2 * i + 1] = dnx;
    }
    *detj_out = detj;
    return true;
}

// ---------------------------------------------------------------- C3D8
const double HEX_CORNERS[8][3] = {{-1.0, -1.0, -1.0}, {1.0, -1.0, -1.0}, {1.0, 1.0, -1.0},
                                  {-1.0, 1.0, -1.0},  {-1.0, -1.0, 1.0}, {1.0, -1.0, 1.0},
                                  {1.0, 1.0, 1.0},    {-1.0, 1.0, 1.0}};

// element.rs:441-445
double det3(const double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// element.rs:448-463: transposed cofactors times 1/det.
void inv3(const double m[3][3], double det, double out[3][3]) {
    double id = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            int r = j, c = i;  // cof(j, i)
            int a = (r + 1) % 3, b = (r + 2) % 3;
            int d = (c + 1) % 3, e = (c + 2) % 3;
            double sign = ((r + c) % 2 == 0) ? 1.0 : -1.0;
            double cof = sign * (m[a][d] * m[b][e] - m[a][e] * m[b][d]);
            out[i][j] = cof * id;
        }
}

// element.rs:467-475
void hex_shape_derivs(double xi, double eta, double zeta, double dn[3][8]) {
    for (int i = 0; i < 8; ++i) {
        double a = HEX_CORNERS[i][0], b = HEX_CORNERS[i][1], c = HEX_CORNERS[i][2];
        dn[0][i] = 0.125 * a * (1.0 + eta * b) * (1.0 + zeta * c);
        dn[1][i] = 0.125 * b * (1.0 + xi * a) * (1.0 + zeta * c);
        dn[2][i] = 0.125 * c * (1.0 + xi * a) * (1.0 + eta * b);
    }
}

// element.rs:479-521
bool hex_b(const double xyz[8][3], double xi, double eta, double zeta, double bm[6][24],
           double* detj_out) {
    double dn[3][8];
    hex_shape_derivs(xi, eta, zeta, dn);
    double j[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int i = 0; i < 8; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) j[a][b] += dn[a][i] * xyz[i][b];
    double detj = det3(j);
    if (detj <= 0.0) return false;
    double inv[3][3];
    inv3(j, detj, inv);
    for (int r = 0; r < 6; ++r)
        for (int k = 0; k < 24; ++k) bm[r][k] = 0.0;
    for (int i = 0; i < 8; ++i) {
        double dnv[3] = {dn[0][i], dn[1][i], dn[2][i]};
        double g[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < 3; ++b)
            for (int a = 0; a < 3; ++a) g[b] += inv[b][a] * dnv[a];
        int c = 3 * i;
        bm[0][c] = g[0];
        bm[1][c + 1] = g[1];
        bm[2][c + 2] = g[2];
        bm[3][c] = g[1];
        bm[3][c + 1] = g[0];
        bm[4][c + 1] = g[2];
        bm[4][c + 2] = g[1];
        bm[5][c] = g[2];
        bm[5][c + 2] = g[0];
    }
    *detj_out = detj;
    return true;
}

int node_count(int kind) {
    switch (kind) {
        case SVX_CPS3: return 3;
        case SVX_CPS4: return 4;
        case SVX_C3D8: return 8;
        default: return 0;
    }
}

// Element stiffness for the three kinds on the path.  Returns 0 or the
// svx_elem_reason.  Follows cps3_stiffness (element.rs:121-129),
// cps4_stiffness (:186-211; xi outer, eta inner, unit weights, w = t*detJ)
// and c3d8_stiffness (:535-561; xi, eta, zeta loops, w = detJ).
int element_ke(int kind, const double* coords, double e, double nu, double t, double* ke) {
    const double g = 1.0 / std::sqrt(3.0);
    if (kind == SVX_CPS3) {
        double d[3][3];
        d_matrix(e, nu, d);
        double xy[3][2];
        for (int i = 0; i < 3; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        double bm[3][6], two_a;
        if (!cps3_b_matrix(xy, bm, &two_a)) return SVX_REASON_DEGENERATE_TRI;
        std::memset(ke, 0, sizeof(double) * 36);
        btdb<6, 3>(ke, bm, d, t * std::fabs(two_a) / 2.0);
        return 0;
    }
    if (kind == SVX_CPS4) {
        double d[3][3];
        d_matrix(e, nu, d);
        double xy[4][2];
        for (int i = 0; i < 4; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        std::memset(ke, 0, sizeof(double) * 64);
        const double pts[2] = {-g, g};
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                double bm[3][8], detj;
                if (!quad_b(xy, pts[a], pts[b], bm, &detj)) return SVX_REASON_BAD_JACOBIAN;
                btdb<8, 3>(ke, bm, d, t * detj);
            }
        double bc[3][8], dj;
        if (!quad_b(xy, 0.0, 0.0, bc, &dj)) return SVX_REASON_BAD_JACOBIAN;
        return 0;
    }
    if (kind == SVX_C3D8) {
        double d[6][6];
        d3_matrix(e, nu, d);
        double xyz[8][3];
        for (int i = 0; i < 8; ++i)
            for (int k = 0; k < 3; ++k) xyz[i][k] = coords[3 * i + k];
        std::memset(ke, 0, sizeof(double) * 576);
        const double pts[2] = {-g, g};
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) {
                    double bm[6][24], detj;
                    if (!hex_b(xyz, pts[a], pts[b], pts[c], bm, &detj))
                        return SVX_REASON_BAD_JACOBIAN;
                    btdb<24, 6>(ke, bm, d, detj);
                }
        double bc[6][24], dj;
        if (!hex_b(xyz, 0.0, 0.0, 0.0, bc, &dj)) return SVX_REASON_BAD_JACOBIAN;
        return 0;
    }
    return SVX_REASON_UNSUPPORTED_KIND;
}

// ---------------------------------------------------------------- stress
// element.rs:854-863
template <int N, int S>
void strain(const double b[S][N], const double* ue, double* e) {
    for (int r = 0; r < S; ++r) {
        double s = 0.0;
        for (int c = 0; c < N; ++c) s += b[r][c] * ue[c];
        e[r] = s;
    }
}

// element.rs:867-881
template <int N>
void plane_stress(const double b[3][N], const double d[3][3], const double* ue, double s[6]) {
    double e[3];
    strain<N, 3>(b, ue, e);
    s[0] = d[0][0] * e[0] + d[0][1] * e[1];
    s[1] = d[1][0] * e[0] + d[1][1] * e[1];
    s[2] = 0.0;
    s[3] = d[2][2] * e[2];
    s[4] = 0.0;
    s[5] = 0.0;
}

// element.rs:904-915
template <int N>
void solid_stress(const double b[6][N], const double d[6][6], const double* ue, double s[6]) {
    double e[6];
    strain<N, 6>(b, ue, e);
    for (int r = 0; r < 6; ++r) {
        double acc = 0.0;
        for (int k = 0; k < 6; ++k) acc += d[r][k] * e[k];
        s[r] = acc;
    }
}

// element.rs:917-923
double von_mises(const double s[6]) {
    return std::sqrt(0.5 * ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) +
                            (s[2] - s[0]) * (s[2] - s[0])) +
                     3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

const double GP_SIGNS[4][2] = {{-1.0, -1.0}, {-1.0, 1.0}, {1.0, -1.0}, {1.0, 1.0}};
const double GP3_SIGNS[8][3] = {{-1.0, -1.0, -1.0}, {-1.0, -1.0, 1.0}, {-1.0, 1.0, -1.0},
                                {-1.0, 1.0, 1.0},   {1.0, -1.0, -1.0}, {1.0, -1.0, 1.0},
                                {1.0, 1.0, -1.0},   {1.0, 1.0, 1.0}};

double hfun(double s) { return 0.5 * (1.0 + s * std::sqrt(3.0)); }

// Centroid stress and the nodal (extrapolated) stresses of one element:
// centroid_stress (element.rs:926-943), nodal_stresses (:948-994),
// extrapolate_to_corners (:1005-1018) and extrapolate_to_corners3
// (:1040-1053).  nodal has room for 8 x 6 values.
void element_stresses(int kind, const double* coords, double e, double nu, double t,
                      const double* ue, double centroid[6], double nodal[8][6]) {
    (void)t;
    const double g = 1.0 / std::sqrt(3.0);
    if (kind == SVX_CPS3) {
        double d[3][3];
        d_matrix(e, nu, d);
        double xy[3][2];
        for (int i = 0; i < 3; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        double bm[3][6], two_a;
        cps3_b_matrix(xy, bm, &two_a);
        plane_stress<6>(bm, d, ue, centroid);
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 6; ++k) nodal[i][k] = centroid[k];
        return;
    }
    if (kind == SVX_CPS4) {
        double d[3][3];
        d_matrix(e, nu, d);
        double xy[4][2];
        for (int i = 0; i < 4; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        double bc[3][8], dj;
        quad_b(xy, 0.0, 0.0, bc, &dj);
        plane_stress<8>(bc, d, ue, centroid);
        double gp[4][6];
        const double pts[2] = {-g, g};
        int k = 0;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                double bm[3][8];
                quad_b(xy, pts[a], pts[b], bm, &dj);
                plane_stress<8>(bm, d, ue, gp[k]);
                ++k;
            }
        for (int i = 0; i < 4; ++i) {
            for (int m = 0; m < 6; ++m) nodal[i][m] = 0.0;
            for (int j = 0; j < 4; ++j) {
                double w = hfun(QUAD_CORNERS[i][0] * GP_SIGNS[j][0]) *
                           hfun(QUAD_CORNERS[i][1] * GP_SIGNS[j][1]);
                for (int m = 0; m < 6; ++m) nodal[i][m] += w * gp[j][m];
            }
        }
        return;
    }
    // C3D8
    double d[6][6];
    d3_matrix(e, nu, d);
    double xyz[8][3];
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) xyz[i][k] = coords[3 * i + k];
    double bc[6][24], dj;
    hex_b(xyz, 0.0, 0.0, 0.0, bc, &dj);
    solid_stress<24>(bc, d, ue, centroid);
    double gp[8][6];
    const double pts[2] = {-g, g};
    int k = 0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                double bm[6][24];
                hex_b(xyz, pts[a], pts[b], pts[c], bm, &dj);
                solid_stress<24>(bm, d, ue, gp[k]);
                ++k;
            }
    for (int i = 0; i < 8; ++i) {
        for (int m = 0; m < 6; ++m) nodal[i][m] = 0.0;
        for (int j = 0; j < 8; ++j) {
            double w = hfun(HEX_CORNERS[i][0] * GP3_SIGNS[j][0]) *
                       hfun(HEX_CORNERS[i][1] * GP3_SIGNS[j][1]) *
                       hfun(HEX_CORNERS[i][2] * GP3_SIGNS[j][2]);
            for (int m = 0; m < 6; ++m) nodal[i][m] += w * gp[j][m];
        }
    }
}

// ---------------------------------------------------------------- row sort
// csr_from_triplets sorts each row with `sort_unstable_by_key(|&(c, _)| c)`
// (assembly.rs:97), so the order in which duplicate (row, col) triplets are
// summed is whatever the Rust standard library's unstable sort leaves.  To
// reproduce the reference's K bit for bit, the oracle restates that
// published algorithm (Rust >= 1.81 `slice::sort_unstable`: insertion sort
// up to 20 elements, otherwise ipnsort = existing-run detection + quicksort
// with median-of-3 / recursive pseudo-median pivots, branchless cyclic
// Lomuto partitions, a stable small-sort below 33 elements and a heapsort
// fallback), specialised for 16-byte (usize, f64) items keyed by column.
struct Trip {
    int64_t c;
    double v;
};

inline bool trip_less(const Trip& a, const Trip& b) { return a.c < b.c; }

// Stable insertion of v[1..n) (insertion_sort_shift_left with offset 1).
void rs_insertion_sort(Trip* v, int64_t n) {
    for (int64_t i = 1; i < n; ++i) {
        if (!trip_less(v[i], v[i - 1])) continue;
        Trip tmp = v[i];
        int64_t j = i;
        do {
            v[j] = v[j - 1];
            --j;
        } while (j > 0 && trip_less(tmp, v[j - 1]));
        v[j] = tmp;
    }
}

// The general small-sort (sort8/sort4 presorting, insertion, bidirectional
// merge) is stable, so its result equals a stable sort of the slice.
void rs_small_sort(Trip* v, int64_t n) {
    std::stable_sort(v, v + n, trip_less);
}

const Trip* rs_median3(const Trip* a, const Trip* b, const Trip* c) {
    bool x = trip_less(*a, *b);
    bool y = trip_less(*a, *c);
    if (x == y) {
        bool z = trip_less(*b, *c);
        return (z ^ x) ? c : b;
    }
    return a;
}

const Trip* rs_median3_rec(const Trip* a, const Trip* b, const Trip* c, int64_t n) {
    if (n * 8 >= 64) {
        int64_t n8 = n / 8;
        a = rs_median3_rec(a, a + n8 * 4, a + n8 * 7, n8);
        b = rs_median3_rec(b, b + n8 * 4, b + n8 * 7, n8);
        c = rs_median3_rec(c, c + n8 * 4, c + n8 * 7, n8);
    }
    return rs_median3(a, b, c);
}

int64_t rs_choose_pivot(const Trip* v, int64_t len) {
    int64_t len_div_8 = len / 8;
    const Trip* a = v;
    const Trip* b = v + len_div_8 * 4;
    const Trip* c = v + len_div_8 * 7;
    const Trip* m = (len < 64) ? rs_median3(a, b, c) : rs_median3_rec(a, b, c, len_div_8);
    return int64_t(m - v);
}

// Branchless cyclic Lomuto partition of v[0..len) around `pivot`: elements
// are visited in order v[1], ..., v[len-1] and finally the saved v[0].
template <class Less>
int64_t rs_lomuto_cyclic(Trip* v, int64_t len, const Trip& pivot, Less less) {
    if (len == 0) return 0;
    Trip gap_value = v[0];
    int64_t gap = 0, num_lt = 0;
    for (int64_t r = 1; r < len; ++r) {
        Trip x = v[r];
        bool lt = less(x, pivot);
        v[gap] = v[num_lt];
        v[num_lt] = x;
        gap = r;
        num_lt += lt ? 1 : 0;
    }
    bool lt = less(gap_value, pivot);
    v[gap] = v[num_lt];
    v[num_lt] = gap_value;
    num_lt += lt ? 1 : 0;
    return num_lt;
}

template <class Less>
int64_t rs_partition(Trip* v, int64_t len, int64_t pivot, Less less) {
    std::swap(v[0], v[pivot]);
    Trip pv = v[0];
    int64_t num_lt = rs_lomuto_cyclic(v + 1, len - 1, pv, less);
    std::swap(v[0], v[num_lt]);
    return num_lt;
}

void rs_sift_down(Trip* v, int64_t len, int64_t node) {
    for (;;) {
        int64_t child = 2 * node + 1;
        if (child >= len) break;
        if (child + 1 < len) child += trip_less(v[child], v[child + 1]) ? 1 : 0;
        if (!trip_less(v[node], v[child])) break;
        std::swap(v[node], v[child]);
        node = child;
    }
}

void rs_heapsort(Trip* v, int64_t len) {
    for (int64_t i = len + len / 2 - 1; i >= 0; --i) {
        int64_t sift_idx;
        if (i >= len) {
            sift_idx = i - len;
        } else {
            std::swap(v[0], v[i]);
            sift_idx = 0;
        }
        rs_sift_down(v, std::min(i, len), sift_idx);
    }
}

void rs_quicksort(Trip* v, int64_t len, const Trip* ancestor, uint32_t limit) {
    for (;;) {
        if (len <= 32) {
            rs_small_sort(v, len);
            return;
        }
        if (limit == 0) {
            rs_heapsort(v, len);
            return;
        }
        --limit;
        int64_t pivot_pos = rs_choose_pivot(v, len);
        if (ancestor && !trip_less(*ancestor, v[pivot_pos])) {
            int64_t num_lt = rs_partition(
                v, len, pivot_pos, [](const Trip& a, const Trip& b) { return !trip_less(b, a); });
            v += num_lt + 1;
            len -= num_lt + 1;
            ancestor = nullptr;
            continue;
        }
        int64_t num_lt = rs_partition(v, len, pivot_pos, trip_less);
        rs_quicksort(v, num_lt, ancestor, limit);
        ancestor = v + num_lt;
        v += num_lt + 1;
        len -= num_lt + 1;
    }
}

void rust_sort_unstable(Trip* v, int64_t len) {
    if (len < 2) return;
    if (len <= 20) {
        rs_insertion_sort(v, len);
        return;
    }
    // ipnsort: an existing ascending / strictly descending run of the whole
    // slice is kept (descending reversed).
    int64_t run = 2;
    bool desc = trip_less(v[1], v[0]);
    if (desc)
        while (run < len && trip_less(v[run], v[run - 1])) ++run;
    else
        while (run < len && !trip_less(v[run], v[run - 1])) ++run;
    if (run == len) {
        if (desc) std::reverse(v, v + len);
        return;
    }
    uint32_t lg = 0;
    for (uint64_t x = uint64_t(len) | 1; x > 1; x >>= 1) ++lg;
    rs_quicksort(v, len, nullptr, 2 * lg);
}

// Row-sort mode: 0 = the reference's unstable sort (default), 1 = stable
// (triplet-stream order: seed first, then elements in enumeration order).
int g_sort_mode = 0;

// ---------------------------------------------------------------- helpers
template <class F>
void parallel_for(int64_t n, int threads, F&& fn) {
    if (threads <= 1 || n < 2) {
        fn(int64_t(0), n);
        return;
    }
    int64_t chunk = (n + threads - 1) / threads;
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        int64_t a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        pool.emplace_back([&fn, a, b] { fn(a, b); });
    }
    for (auto& th : pool) th.join();
}

uint32_t elem_id_of(const svx_flat_model_t* m, int64_t e) {
    return m->elem_id ? m->elem_id[e] : uint32_t(e + 1);
}

void set_error(svx_error_t* err, int code, int reason, int64_t elem, const char* msg) {
    if (!err) return;
    err->code = code;
    err->reason = reason;
    err->elem_index = elem;
    err->iterations = 0;
    err->residual = 0.0;
    std::snprintf(err->message, sizeof(err->message), "%s", msg);
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

// element_entry's checks before geometry (assembly.rs:143-160).
int material_check(const svx_flat_model_t* m, int64_t e) {
    if (m->no_material && m->no_material[e]) return SVX_REASON_NO_MATERIAL;
    double E = m->youngs[e], nu = m->poisson[e];
    if (E <= 0.0 || std::fabs(nu) >= 1.0) return SVX_REASON_BAD_MATERIAL;
    int kind = m->kind[e];
    bool solid = (kind == SVX_C3D8 || kind == SVX_C3D4);
    bool plane_strain = (kind == SVX_CPE4 || kind == SVX_CPE8);
    if ((solid || plane_strain) && nu >= 0.5) return SVX_REASON_SOLID_POISSON;
    if (node_count(kind) == 0) return SVX_REASON_UNSUPPORTED_KIND;
    return 0;
}

// ---------------------------------------------------------------- conduction
// heat.rs:140-145: CPS3 constant-gradient ingredients (b_i, c_i, signed 2A).
void tri_constants(const double p[3][2], double b[3], double c[3], double* two_a) {
    b[0] = p[1][1] - p[2][1];
    b[1] = p[2][1] - p[0][1];
    b[2] = p[0][1] - p[1][1];
    c[0] = p[2][0] - p[1][0];
    c[1] = p[0][0] - p[2][0];
    c[2] = p[1][0] - p[0][0];
    *two_a = b[0] * c[1] - b[1] * c[0];
}

// element.rs:175-182
void quad_shapes(double xi, double eta, double n[4]) {
    for (int i = 0; i < 4; ++i)
        n[i] = 0.25 * (1.0 + xi * QUAD_CORNERS[i][0]) * (1.0 + eta * QUAD_CORNERS[i][1]);
}

// element.rs:525-531
void hex_shapes(double xi, double eta, double zeta, double n[8]) {
    for (int i = 0; i < 8; ++i)
        n[i] = 0.125 * (1.0 + xi * HEX_CORNERS[i][0]) * (1.0 + eta * HEX_CORNERS[i][1]) *
               (1.0 + zeta * HEX_CORNERS[i][2]);
}

// heat.rs:149-296 (conduction_element) for CPS3, CPS4 / CPE4 and C3D8:
// C_e into ke (row-major N x N) and the consistent heat-source load into fe.
// fe_used is false when the reference adds nothing to f for this element
// (CPS3 without a source); otherwise it adds fe, zeros included.
int conduction_ke(int kind, const double* coords, double k, double t, bool has_q, double q,
                  double* ke, double* fe, bool* fe_used) {
    const double qq = has_q ? q : 0.0;
    if (kind == SVX_CPS3) {
        double p[3][2], b[3], c[3], two_a;
        for (int i = 0; i < 3; ++i) {
            p[i][0] = coords[3 * i];
            p[i][1] = coords[3 * i + 1];
        }
        tri_constants(p, b, c, &two_a);
        if (two_a == 0.0) return SVX_REASON_DEGENERATE_TRI;
        const double w = k * t / (2.0 * std::fabs(two_a));
        for (int i = 0; i < 3; ++i) {
            fe[i] = has_q ? q * t * std::fabs(two_a) / 6.0 : 0.0;
            for (int j = 0; j < 3; ++j) ke[i * 3 + j] = w * (b[i] * b[j] + c[i] * c[j]);
        }
        *fe_used = has_q;
        return 0;
    }
    if (kind == SVX_CPS4 || kind == SVX_CPE4) {
        double xy[4][2];
        for (int i = 0; i < 4; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        const double g = 1.0 / std::sqrt(3.0);
        const double pts[2] = {-g, g};
        for (int i = 0; i < 16; ++i) ke[i] = 0.0;
        for (int i = 0; i < 4; ++i) fe[i] = 0.0;
        for (double xi : pts)
            for (double eta : pts) {
                double bm[3][8], detj;
                if (!quad_b(xy, xi, eta, bm, &detj)) return SVX_REASON_BAD_JACOBIAN;
                double n[4];
                quad_shapes(xi, eta, n);
                for (int i = 0; i < 4; ++i) {
                    fe[i] += qq * t * detj * n[i];
                    for (int j = 0; j < 4; ++j)
                        ke[i * 4 + j] += k * t * detj *
                                         (bm[0][2 * i] * bm[0][2 * j] +
                                          bm[1][2 * i + 1] * bm[1][2 * j + 1]);
                }
            }
        *fe_used = true;
        return 0;
    }
    if (kind == SVX_C3D8) {
        double xyz[8][3];
        for (int i = 0; i < 8; ++i)
            for (int a = 0; a < 3; ++a) xyz[i][a] = coords[3 * i + a];
        const double g = 1.0 / std::sqrt(3.0);
        const double pts[2] = {-g, g};
        for (int i = 0; i < 64; ++i) ke[i] = 0.0;
        for (int i = 0; i < 8; ++i) fe[i] = 0.0;
        for (double xi : pts)
            for (double eta : pts)
                for (double zeta : pts) {
                    double bm[6][24], detj;
                    if (!hex_b(xyz, xi, eta, zeta, bm, &detj)) return SVX_REASON_BAD_JACOBIAN;
                    double n[8];
                    hex_shapes(xi, eta, zeta, n);
                    for (int i = 0; i < 8; ++i) {
                        fe[i] += qq * detj * n[i];
                        for (int j = 0; j < 8; ++j) {
                            double v = 0.0;
                            for (int r = 0; r < 3; ++r) v += bm[r][3 * i + r] * bm[r][3 * j + r];
                            ke[i * 8 + j] += k * detj * v;
                        }
                    }
                }
        *fe_used = true;
        return 0;
    }
    return SVX_REASON_UNSUPPORTED_KIND;
}

// The reference's Debug names of ElemKind (in its flux error texts).
const char* kind_debug(int kind) {
    static const char* names[] = {"Cps3", "Cps4", "Cps8", "Cpe4", "Cpe8", "C3d8", "C3d4", "B31"};
    return (kind >= 0 && kind < 8) ? names[kind] : "Unknown";
}

}  // namespace

extern "C" void svx_oracle_spmv(const svx_oracle_csr_t* k, const double* x, double* y, int threads);

namespace {

// assembly.rs:87-116 csr_from_triplets: bucket by row in stream order,
// sort each row by column (the reference's unstable sort restated, or a
// stable one), sum runs left to right starting from 0.0.  Allocates
// out->row_ptr, col_idx, vals and an n-long out->f the caller fills.
void csr_from_triplets(int64_t n, const std::vector<int64_t>& tr, const std::vector<int64_t>& tc,
                       const std::vector<double>& tv, svx_oracle_csr_t* out) {
    const int64_t nt = int64_t(tr.size());
    std::vector<int64_t> rcount(n + 1, 0);
    for (int64_t t = 0; t < nt; ++t) rcount[tr[t] + 1]++;
    for (int64_t i = 0; i < n; ++i) rcount[i + 1] += rcount[i];
    std::vector<int64_t> pos(rcount.begin(), rcount.end() - 1);
    std::vector<int64_t> perm(nt);
    for (int64_t t = 0; t < nt; ++t) perm[pos[tr[t]]++] = t;
    std::vector<int64_t> rp(n + 1, 0);
    std::vector<int64_t> ci;
    std::vector<double> cv;
    ci.reserve(nt / 2 + n);
    cv.reserve(nt / 2 + n);
    std::vector<Trip> row;
    for (int64_t i = 0; i < n; ++i) {
        row.clear();
        for (int64_t q = rcount[i]; q < rcount[i + 1]; ++q) {
            int64_t t = perm[q];
            row.push_back(Trip{tc[t], tv[t]});
        }
        if (g_sort_mode == 0)
            rust_sort_unstable(row.data(), int64_t(row.size()));
        else
            std::stable_sort(row.begin(), row.end(), trip_less);
        size_t k = 0;
        while (k < row.size()) {
            int64_t c = row[k].c;
            double v = 0.0;
            while (k < row.size() && row[k].c == c) {
                v += row[k].v;
                ++k;
            }
            ci.push_back(c);
            cv.push_back(v);
        }
        rp[i + 1] = int64_t(ci.size());
    }
    out->n = n;
    out->nnz = int64_t(ci.size());
    out->row_ptr = (int64_t*)std::malloc(sizeof(int64_t) * (n + 1));
    out->col_idx = (int64_t*)std::malloc(sizeof(int64_t) * (ci.size() + 1));
    out->vals = (double*)std::malloc(sizeof(double) * (cv.size() + 1));
    out->f = (double*)std::malloc(sizeof(double) * (n + 1));
    std::memcpy(out->row_ptr, rp.data(), sizeof(int64_t) * (n + 1));
    std::memcpy(out->col_idx, ci.data(), sizeof(int64_t) * ci.size());
    std::memcpy(out->vals, cv.data(), sizeof(double) * cv.size());
}

// stress.rs:22-118: centroid von Mises, nodal (extrapolated, averaged)
// von Mises and reactions K_orig u - f_orig at the constrained rows.
void recover(const svx_flat_model_t* m, const double* u, const svx_oracle_csr_t* k_orig,
             const double* f_orig, int threads, double* vm, double* vm_node, double* reactions) {
    const int ndof = m->ndof;
    const int64_t n = m->n_nodes * ndof;
    // stress.rs:22-98
    std::vector<double> sum(6 * m->n_nodes, 0.0);
    std::vector<uint32_t> count(m->n_nodes, 0);
    for (int64_t e = 0; e < m->n_elem; ++e) {
        int kind = m->kind[e];
        int nn = node_count(kind);
        const int32_t* cn = m->conn + m->conn_ptr[e];
        double coords[24], ue[24], cen[6], nod[8][6];
        for (int i = 0; i < nn; ++i) {
            for (int q = 0; q < 3; ++q) coords[3 * i + q] = m->xyz[3 * int64_t(cn[i]) + q];
            for (int q = 0; q < ndof; ++q) ue[i * ndof + q] = u[int64_t(cn[i]) * ndof + q];
        }
        element_stresses(kind, coords, m->youngs[e], m->poisson[e], m->thickness, ue, cen, nod);
        if (vm) vm[e] = von_mises(cen);
        for (int i = 0; i < nn; ++i) {
            int64_t node = cn[i];
            for (int q = 0; q < 6; ++q) sum[6 * node + q] += nod[i][q];
            count[node] += 1;
        }
    }
    if (vm_node)
        for (int64_t i = 0; i < m->n_nodes; ++i) {
            if (count[i] == 0) {
                vm_node[i] = 0.0;
                continue;
            }
            double c = double(count[i]);
            double avg[6];
            for (int q = 0; q < 6; ++q) avg[q] = sum[6 * i + q] / c;
            vm_node[i] = von_mises(avg);
        }
    // stress.rs:103-118
    if (reactions) {
        std::vector<double> ku(n);
        svx_oracle_spmv(k_orig, u, ku.data(), threads);
        for (int64_t i = 0; i < m->n_fixed; ++i) {
            int64_t row = m->fixed_row[i];
            reactions[i] = ku[row] - f_orig[row];
        }
    }
}

}  // namespace

extern "C" {

void svx_oracle_set_sort_mode(int mode) { g_sort_mode = mode; }

int svx_oracle_element_stiffness(int kind, const double* coords, double E, double nu,
                                 double thickness, double* ke) {
    return element_ke(kind, coords, E, nu, thickness, ke);
}

// assembly.rs:291-386 with csr_from_triplets (:87-116) and scatter (:120-133).
int svx_oracle_assemble(const svx_flat_model_t* m, int threads, svx_oracle_csr_t* out,
                        svx_error_t* err) {
    std::memset(out, 0, sizeof(*out));
    const int ndof = m->ndof;
    const int64_t n = m->n_nodes * ndof;
    const int64_t ne = m->n_elem;
    // Triplet stream: n diagonal seeds, then each element's N*N entries.
    std::vector<int64_t> toff(ne + 1, 0);
    for (int64_t e = 0; e < ne; ++e) {
        int64_t nn = m->conn_ptr[e + 1] - m->conn_ptr[e];
        int64_t N = nn * ndof;
        toff[e + 1] = toff[e] + N * N;
    }
    const int64_t nt = n + toff[ne];
    std::vector<int64_t> tr(nt), tc(nt);
    std::vector<double> tv(nt);
    for (int64_t i = 0; i < n; ++i) {
        tr[i] = i;
        tc[i] = i;
        tv[i] = 0.0;
    }
    std::vector<int> fail(ne, 0);
    auto run = [&](int64_t a, int64_t b) {
        double ke[576];
        double coords[24];
        for (int64_t e = a; e < b; ++e) {
            int r = material_check(m, e);
            if (r) {
                fail[e] = r;
                continue;
            }
            int kind = m->kind[e];
            int nn = node_count(kind);
            const int32_t* cn = m->conn + m->conn_ptr[e];
            for (int i = 0; i < nn; ++i)
                for (int k = 0; k < 3; ++k) coords[3 * i + k] = m->xyz[3 * int64_t(cn[i]) + k];
            r = element_ke(kind, coords, m->youngs[e], m->poisson[e], m->thickness, ke);
            if (r) {
                fail[e] = r;
                continue;
            }
            const int N = nn * ndof;
            int64_t o = n + toff[e];
            for (int aa = 0; aa < N; ++aa) {
                int64_t gr = int64_t(cn[aa / ndof]) * ndof + aa % ndof;
                for (int cc = 0; cc < N; ++cc) {
                    int64_t gc = int64_t(cn[cc / ndof]) * ndof + cc % ndof;
                    tr[o] = gr;
                    tc[o] = gc;
                    tv[o] = ke[aa * N + cc];
                    ++o;
                }
            }
        }
    };
    int n_chunks = (threads > 1 && ne >= 256) ? 2 * threads : 1;
    if (n_chunks == 1)
        run(0, ne);
    else
        parallel_for(ne, threads, run);
    for (int64_t e = 0; e < ne; ++e)
        if (fail[e]) {
            char msg[400];
            std::snprintf(msg, sizeof msg, "element %u: %s", elem_id_of(m, e),
                          reason_text(fail[e]));
            set_error(err, SVX_INVALID_MODEL, fail[e], e, msg);
            return SVX_INVALID_MODEL;
        }
    csr_from_triplets(n, tr, tc, tv, out);
    for (int64_t i = 0; i < n; ++i) out->f[i] = m->f ? m->f[i] : 0.0;
    if (err) set_error(err, SVX_OK, 0, -1, "");
    return SVX_OK;
}

void svx_oracle_csr_free(svx_oracle_csr_t* csr) {
    if (!csr) return;
    std::free(csr->row_ptr);
    std::free(csr->col_idx);
    std::free(csr->vals);
    std::free(csr->f);
    std::memset(csr, 0, sizeof(*csr));
}

// assembly.rs:46-72: row-chunked when threads > 1 and n > 20,000; each row
// keeps its serial order.
void svx_oracle_spmv(const svx_oracle_csr_t* k, const double* x, double* y, int threads) {
    const int64_t n = k->n;
    auto rows = [&](int64_t a, int64_t b) {
        for (int64_t r = a; r < b; ++r) {
            double o = 0.0;
            for (int64_t idx = k->row_ptr[r]; idx < k->row_ptr[r + 1]; ++idx)
                o += k->vals[idx] * x[k->col_idx[idx]];
            y[r] = o;
        }
    };
    if (threads > 1 && n > 20000)
        parallel_for(n, threads, rows);
    else
        rows(0, n);
}

// solver.rs:45-62
void svx_oracle_apply_dirichlet(svx_oracle_csr_t* k, double* f, const int64_t* rows,
                                int64_t n_rows) {
    const int64_t n = k->n;
    std::vector<char> is_c(n, 0);
    for (int64_t i = 0; i < n_rows; ++i) is_c[rows[i]] = 1;
    for (int64_t r = 0; r < n; ++r)
        for (int64_t idx = k->row_ptr[r]; idx < k->row_ptr[r + 1]; ++idx) {
            int64_t c = k->col_idx[idx];
            if (is_c[r] || is_c[c]) k->vals[idx] = (r == c) ? 1.0 : 0.0;
        }
    for (int64_t i = 0; i < n_rows; ++i) f[rows[i]] = 0.0;
}

// solver.rs:82-149 (serial dots, threaded SpMV).
int svx_oracle_pcg(const svx_oracle_csr_t* k, const double* f, double tol, int64_t max_iter,
                   int threads, double* u, int64_t* iterations, double* residual) {
    const int64_t n = k->n;
    std::vector<double> r(f, f + n), z(n), p(n), kp(n), inv_diag(n);
    for (int64_t i = 0; i < n; ++i) u[i] = 0.0;
    auto dot = [n](const double* a, const double* b) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    };
    double b_norm = std::sqrt(dot(f, f));
    if (b_norm == 0.0) {
        *iterations = 0;
        *residual = 0.0;
        return SVX_OK;
    }
    for (int64_t i = 0; i < n; ++i) {
        double d = 0.0;
        for (int64_t idx = k->row_ptr[i]; idx < k->row_ptr[i + 1]; ++idx)
            if (k->col_idx[idx] == i) {
                d = k->vals[idx];
                break;
            }
        inv_diag[i] = (d == 0.0) ? 0.0 : 1.0 / d;
    }
    auto rel_res = [&]() { return std::sqrt(dot(r.data(), r.data())) / b_norm; };
    for (int64_t i = 0; i < n; ++i) z[i] = r[i] * inv_diag[i];
    p = z;
    double rz = dot(r.data(), z.data());
    for (int64_t it = 1; it <= max_iter; ++it) {
        svx_oracle_spmv(k, p.data(), kp.data(), threads);
        double pap = dot(p.data(), kp.data());
        if (pap <= 0.0 || std::isnan(pap)) {
            *iterations = it;
            *residual = rel_res();
            return SVX_NOT_CONVERGED;
        }
        double alpha = rz / pap;
        for (int64_t i = 0; i < n; ++i) u[i] += alpha * p[i];
        for (int64_t i = 0; i < n; ++i) r[i] -= alpha * kp[i];
        double res = rel_res();
        if (res <= tol) {
            *iterations = it;
            *residual = res;
            return SVX_OK;
        }
        for (int64_t i = 0; i < n; ++i) z[i] = r[i] * inv_diag[i];
        double rz_new = dot(r.data(), z.data());
        double beta = rz_new / rz;
        rz = rz_new;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    *iterations = max_iter;
    *residual = rel_res();
    return SVX_NOT_CONVERGED;
}

// lib.rs:593-716 (Method::Pcg): assemble -> keep K, f -> Dirichlet -> PCG
// -> jacobi_cond -> displacements -> stresses -> reactions.
namespace {

// ------------------------------------------------------------------- LDL^T
// ldl.rs restated: reverse Cuthill-McKee ordering, permuted copy, elimination
// tree, up-looking LDL^T with L in CSR rows, and its solve.  Every loop keeps
// the reference's order, so L, D and the solution are bit-identical.
constexpr int64_t kNone = -1;  // usize::MAX of the reference (root / unset)

// ldl.rs:27-60.  Returns perm (old index -> new index).
std::vector<int64_t> rcm_perm(const svx_oracle_csr_t& k) {
    const int64_t n = k.n;
    std::vector<int64_t> perm(n, kNone), order;
    order.reserve(n);
    std::vector<char> visited(n, 0);
    std::vector<int64_t> queue;
    while (int64_t(order.size()) < n) {
        // min_by_key keeps the first of equal minima
        int64_t start = kNone, best = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (visited[i]) continue;
            int64_t deg = k.row_ptr[i + 1] - k.row_ptr[i];
            if (start == kNone || deg < best) {
                start = i;
                best = deg;
            }
        }
        visited[start] = 1;
        queue.assign(1, start);
        for (size_t head = 0; head < queue.size(); ++head) {
            int64_t u = queue[head];
            order.push_back(u);
            for (int64_t idx = k.row_ptr[u]; idx < k.row_ptr[u + 1]; ++idx) {
                int64_t v = k.col_idx[idx];
                if (!visited[v]) {
                    visited[v] = 1;
                    queue.push_back(v);
                }
            }
        }
    }
    for (int64_t pos = 0; pos < n; ++pos) perm[order[n - 1 - pos]] = pos;
    return perm;
}

struct HostCsr {
    std::vector<int64_t> row_ptr, col_idx;
    std::vector<double> vals;
};

// ldl.rs:63-85: out[r][c] = a[invp[r]][invp[c]], each row sorted by column
// (columns are unique within a row, so the sort order is fully determined).
HostCsr permuted(const svx_oracle_csr_t& k, const std::vector<int64_t>& perm,
                 const std::vector<int64_t>& invp) {
    HostCsr a;
    a.row_ptr.reserve(k.n + 1);
    a.row_ptr.push_back(0);
    a.col_idx.reserve(k.nnz);
    a.vals.reserve(k.nnz);
    std::vector<std::pair<int64_t, double>> row;
    for (int64_t old : invp) {
        row.clear();
        for (int64_t p = k.row_ptr[old]; p < k.row_ptr[old + 1]; ++p)
            row.emplace_back(perm[k.col_idx[p]], k.vals[p]);
        std::sort(row.begin(), row.end(),
                  [](const auto& x, const auto& y) { return x.first < y.first; });
        for (const auto& cv : row) {
            a.col_idx.push_back(cv.first);
            a.vals.push_back(cv.second);
        }
        a.row_ptr.push_back(int64_t(a.col_idx.size()));
    }
    return a;
}

// ldl.rs:89-110 (path compression through `ancestor`).
std::vector<int64_t> elimination_tree(const HostCsr& a) {
    const int64_t n = int64_t(a.row_ptr.size()) - 1;
    std::vector<int64_t> parent(n, kNone), ancestor(n, kNone);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t p = a.row_ptr[i]; p < a.row_ptr[i + 1]; ++p) {
            int64_t node = a.col_idx[p];
            while (node < i) {
                int64_t next = ancestor[node];
                ancestor[node] = i;
                if (next == kNone) {
                    parent[node] = i;
                    break;
                }
                node = next;
            }
        }
    return parent;
}

// ldl.rs:115-136 (cs_ereach): the pattern of row i of L, unsorted.
void ereach(const HostCsr& a, const std::vector<int64_t>& parent, std::vector<int64_t>& seen,
            int64_t i, std::vector<int64_t>& pattern) {
    pattern.clear();
    seen[i] = i;
    for (int64_t p = a.row_ptr[i]; p < a.row_ptr[i + 1]; ++p) {
        int64_t node = a.col_idx[p];
        while (node < i && seen[node] != i) {
            pattern.push_back(node);
            seen[node] = i;
            if (parent[node] == kNone) break;
            node = parent[node];
        }
    }
}

struct Ldlt {
    std::vector<int64_t> l_row_ptr, l_col_idx, invp;
    std::vector<double> l_vals, d;
};

// ldl.rs:144-221.  Returns SVX_OK, or SVX_INVALID_MODEL with the reference's
// pivot message in msg.
int ldlt_factorize(const svx_oracle_csr_t& k, Ldlt& out, std::string& msg) {
    const int64_t n = k.n;
    std::vector<int64_t> perm = rcm_perm(k);
    out.invp.assign(n, 0);
    for (int64_t old = 0; old < n; ++old) out.invp[perm[old]] = old;
    HostCsr a = permuted(k, perm, out.invp);
    std::vector<int64_t> parent = elimination_tree(a);
    out.l_row_ptr.assign(1, 0);
    out.l_col_idx.clear();
    out.l_vals.clear();
    out.d.assign(n, 0.0);
    std::vector<double> x(n, 0.0);
    std::vector<int64_t> seen(n, kNone), pattern;
    for (int64_t i = 0; i < n; ++i) {
        ereach(a, parent, seen, i, pattern);
        std::sort(pattern.begin(), pattern.end());
        double aii = 0.0, row_max = 0.0;
        for (int64_t p = a.row_ptr[i]; p < a.row_ptr[i + 1]; ++p) {
            int64_t c = a.col_idx[p];
            x[c] = a.vals[p];
            row_max = std::fmax(row_max, std::fabs(a.vals[p]));
            if (c == i) aii = a.vals[p];
        }
        for (int64_t kk : pattern) {
            double w = x[kk];
            for (int64_t p = out.l_row_ptr[kk]; p < out.l_row_ptr[kk + 1]; ++p)
                w -= out.l_vals[p] * x[out.l_col_idx[p]];
            x[kk] = w;
            double lik = w / out.d[kk];
            aii -= lik * w;
            out.l_col_idx.push_back(kk);
            out.l_vals.push_back(lik);
        }
        out.l_row_ptr.push_back(int64_t(out.l_col_idx.size()));
        for (int64_t kk : pattern) x[kk] = 0.0;
        for (int64_t p = a.row_ptr[i]; p < a.row_ptr[i + 1]; ++p) x[a.col_idx[p]] = 0.0;
        if (!std::isfinite(aii) || aii <= 1e-13 * std::fmax(row_max, DBL_MIN)) {
            msg = std::string("stiffness matrix is not positive definite (pivot ") +
                  (aii < 0.0 ? "negative" : "near-zero") + " at equation " +
                  std::to_string(i) + ")";
            return SVX_INVALID_MODEL;
        }
        out.d[i] = aii;
    }
    return SVX_OK;
}

// ldl.rs:224-251.
void ldlt_solve(const Ldlt& fa, const double* b, double* xout) {
    const int64_t n = int64_t(fa.d.size());
    std::vector<double> y(n);
    for (int64_t i = 0; i < n; ++i) y[i] = b[fa.invp[i]];
    for (int64_t i = 0; i < n; ++i) {
        double s = y[i];
        for (int64_t p = fa.l_row_ptr[i]; p < fa.l_row_ptr[i + 1]; ++p)
            s -= fa.l_vals[p] * y[fa.l_col_idx[p]];
        y[i] = s;
    }
    for (int64_t i = 0; i < n; ++i) y[i] /= fa.d[i];
    for (int64_t i = n - 1; i >= 0; --i) {
        double xi = y[i];
        for (int64_t p = fa.l_row_ptr[i]; p < fa.l_row_ptr[i + 1]; ++p)
            y[fa.l_col_idx[p]] -= fa.l_vals[p] * xi;
    }
    for (int64_t i = 0; i < n; ++i) xout[fa.invp[i]] = y[i];
}

// ldl.rs:256-265.
double ldlt_cond(const Ldlt& fa) {
    double lo = INFINITY, hi = 0.0;
    for (double dv : fa.d) {
        lo = std::fmin(lo, std::fabs(dv));
        hi = std::fmax(hi, std::fabs(dv));
    }
    return hi / lo;
}

}  // namespace

namespace {

// ------------------------------------------------------------ consistent mass
// modal.rs:82-99 (CPS3, closed form rho t A / 12 x [2 1 1; 1 2 1; 1 1 2]),
// :103-121 (CPS4 / CPE4, 2x2 Gauss, xi outer), :125-146 (C3D8, 2x2x2 Gauss):
// rho [t] detJ N_i N_j on every dof pair (d, d) of nodes i, j, into me
// (row-major N x N, zeros elsewhere).  Returns 0 or the svx_elem_reason:
// zero area, or det J <= 0 at a Gauss point (the stiffness's triggers, but
// no centroid check).
int element_me(int kind, const double* coords, double rho, double t, double* me) {
    const double g = 1.0 / std::sqrt(3.0);
    const double pts[2] = {-g, g};
    if (kind == SVX_CPS3) {
        const double two_a = (coords[3] - coords[0]) * (coords[7] - coords[1]) -
                             (coords[6] - coords[0]) * (coords[4] - coords[1]);
        if (two_a == 0.0) return SVX_REASON_DEGENERATE_TRI;
        const double w = rho * t * std::fabs(two_a) / 24.0;
        std::memset(me, 0, sizeof(double) * 36);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int d = 0; d < 2; ++d)
                    me[(2 * i + d) * 6 + 2 * j + d] = w * (i == j ? 2.0 : 1.0);
        return 0;
    }
    if (kind == SVX_CPS4 || kind == SVX_CPE4) {
        double xy[4][2];
        for (int i = 0; i < 4; ++i) {
            xy[i][0] = coords[3 * i];
            xy[i][1] = coords[3 * i + 1];
        }
        std::memset(me, 0, sizeof(double) * 64);
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                double bm[3][8], detj, nsh[4];
                if (!quad_b(xy, pts[a], pts[b], bm, &detj)) return SVX_REASON_BAD_JACOBIAN;
                quad_shapes(pts[a], pts[b], nsh);
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j) {
                        const double v = rho * t * detj * nsh[i] * nsh[j];
                        for (int d = 0; d < 2; ++d) me[(2 * i + d) * 8 + 2 * j + d] += v;
                    }
            }
        return 0;
    }
    if (kind == SVX_C3D8) {
        double xyz[8][3];
        for (int i = 0; i < 8; ++i)
            for (int k = 0; k < 3; ++k) xyz[i][k] = coords[3 * i + k];
        std::memset(me, 0, sizeof(double) * 576);
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) {
                    double bm[6][24], detj, nsh[8];
                    if (!hex_b(xyz, pts[a], pts[b], pts[c], bm, &detj))
                        return SVX_REASON_BAD_JACOBIAN;
                    hex_shapes(pts[a], pts[b], pts[c], nsh);
                    for (int i = 0; i < 8; ++i)
                        for (int j = 0; j < 8; ++j) {
                            const double v = rho * detj * nsh[i] * nsh[j];
                            for (int d = 0; d < 3; ++d) me[(3 * i + d) * 24 + 3 * j + d] += v;
                        }
                }
        return 0;
    }
    return SVX_REASON_UNSUPPORTED_KIND;
}

}  // namespace

int svx_oracle_element_mass(int kind, const double* coords, double rho, double t,
                            double* me) {
    return element_me(kind, coords, rho, t, me);
}

// assemble_mass (modal.rs:203-271): n zero diagonal seeds, then every
// element's N x N consistent mass in enumeration order, summed by
// csr_from_triplets; the first failing element raises "element {id}: ...".
int svx_oracle_assemble_mass(const svx_flat_model_t* m, double rho, svx_oracle_csr_t* out,
                             svx_error_t* err) {
    std::memset(out, 0, sizeof(*out));
    const int ndof = m->ndof;
    const int64_t n = m->n_nodes * ndof;
    std::vector<int64_t> tr, tc;
    std::vector<double> tv;
    for (int64_t i = 0; i < n; ++i) {
        tr.push_back(i);
        tc.push_back(i);
        tv.push_back(0.0);
    }
    double me[576], coords[24];
    for (int64_t e = 0; e < m->n_elem; ++e) {
        const int kind = m->kind[e];
        const int nn = int(m->conn_ptr[e + 1] - m->conn_ptr[e]);
        const int32_t* cn = m->conn + m->conn_ptr[e];
        for (int i = 0; i < nn && i < 8; ++i)
            for (int k = 0; k < 3; ++k) coords[3 * i + k] = m->xyz[3 * int64_t(cn[i]) + k];
        const int r = element_me(kind, coords, rho, m->thickness, me);
        if (r) {
            char msg[400];
            std::snprintf(msg, sizeof msg, "element %u: %s", elem_id_of(m, e), reason_text(r));
            set_error(err, SVX_INVALID_MODEL, r, e, msg);
            return SVX_INVALID_MODEL;
        }
        const int N = nn * ndof;
        for (int a = 0; a < N; ++a)
            for (int c = 0; c < N; ++c) {
                tr.push_back(int64_t(cn[a / ndof]) * ndof + a % ndof);
                tc.push_back(int64_t(cn[c / ndof]) * ndof + c % ndof);
                tv.push_back(me[a * N + c]);
            }
    }
    csr_from_triplets(n, tr, tc, tv, out);
    for (int64_t i = 0; i < n; ++i) out->f[i] = 0.0;
    if (err) set_error(err, SVX_OK, 0, -1, "");
    return SVX_OK;
}

void svx_oracle_rcm(const svx_oracle_csr_t* k, int64_t* perm) {
    std::vector<int64_t> p = rcm_perm(*k);
    std::copy(p.begin(), p.end(), perm);
}

// The `direct` closure of lib.rs:645-663: factorize, solve, the relative
// residual ||f - K u|| / ||f|| (0 when f is zero) and the D-based estimate.
int svx_oracle_ldlt(const svx_oracle_csr_t* k, const double* f, int threads, double* u,
                    double* residual, double* cond, double* d, int64_t* nnz_l,
                    svx_error_t* err) {
    Ldlt fa;
    std::string msg;
    int st = ldlt_factorize(*k, fa, msg);
    if (st != SVX_OK) {
        set_error(err, st, 0, -1, msg.c_str());
        return st;
    }
    const int64_t n = k->n;
    ldlt_solve(fa, f, u);
    double b2 = 0.0;
    for (int64_t i = 0; i < n; ++i) b2 += f[i] * f[i];
    double b_norm = std::sqrt(b2);
    double res = 0.0;
    if (b_norm != 0.0) {
        std::vector<double> r(n);
        svx_oracle_spmv(k, u, r.data(), threads);
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            double v = f[i] - r[i];
            s += v * v;
        }
        res = std::sqrt(s) / b_norm;
    }
    if (residual) *residual = res;
    if (cond) *cond = ldlt_cond(fa);
    if (d) std::copy(fa.d.begin(), fa.d.end(), d);
    if (nnz_l) *nnz_l = int64_t(fa.l_vals.size());
    if (err) set_error(err, SVX_OK, 0, -1, "");
    return SVX_OK;
}

int svx_oracle_solve(const svx_flat_model_t* m, int threads, double tol, int64_t max_iter,
                     svx_solution_t* sol, svx_error_t* err) {
    return svx_oracle_solve_method(m, threads, tol, max_iter, SVX_ORACLE_METHOD_PCG, sol,
                                   nullptr, err);
}

int svx_oracle_solve_method(const svx_flat_model_t* m, int threads, double tol,
                            int64_t max_iter, int method, svx_solution_t* sol,
                            int* method_used, svx_error_t* err) {
    svx_oracle_csr_t k;
    int st = svx_oracle_assemble(m, threads, &k, err);
    if (st != SVX_OK) return st;
    const int ndof = m->ndof;
    const int64_t n = k.n;
    std::vector<double> f_orig(k.f, k.f + n);
    svx_oracle_csr_t k_orig;
    k_orig.n = k.n;
    k_orig.nnz = k.nnz;
    k_orig.row_ptr = k.row_ptr;
    k_orig.col_idx = k.col_idx;
    std::vector<double> vals_orig(k.vals, k.vals + k.nnz);
    k_orig.vals = vals_orig.data();
    k_orig.f = nullptr;
    std::vector<double> f(k.f, k.f + n);
    svx_oracle_apply_dirichlet(&k, f.data(), m->fixed_row, m->n_fixed);
    if (max_iter <= 0) max_iter = std::max<int64_t>(1000, 10 * n);
    std::vector<double> u(n, 0.0);
    int64_t iters = 0;
    double res = 0.0, cond = 0.0;
    // lib.rs:664-686: Pcg, Ldlt, or Auto (PCG, then the direct path when
    // PCG returns NotConverged).
    bool direct = method == SVX_ORACLE_METHOD_LDLT;
    if (!direct) {
        st = svx_oracle_pcg(&k, f.data(), tol, max_iter, threads, u.data(), &iters, &res);
        if (st != SVX_OK && method == SVX_ORACLE_METHOD_AUTO) {
            direct = true;
        } else if (st != SVX_OK) {
            char msg[200];
            std::snprintf(msg, sizeof msg, "not converged after %lld iterations",
                          (long long)iters);
            set_error(err, SVX_NOT_CONVERGED, 0, -1, msg);
            if (err) {
                err->iterations = iters;
                err->residual = res;
            }
            svx_oracle_csr_free(&k);
            return st;
        }
    }
    if (direct) {
        iters = 0;
        st = svx_oracle_ldlt(&k, f.data(), threads, u.data(), &res, &cond, nullptr, nullptr,
                             err);
        if (st != SVX_OK) {
            svx_oracle_csr_free(&k);
            return st;
        }
    } else {
        // jacobi_cond (lib.rs:634-644): extreme |diag| of the modified K.
        double hi = 0.0, lo = INFINITY;
        for (int64_t i = 0; i < n; ++i)
            for (int64_t idx = k.row_ptr[i]; idx < k.row_ptr[i + 1]; ++idx)
                if (k.col_idx[idx] == i) {
                    double a = std::fabs(k.vals[idx]);
                    hi = std::fmax(hi, a);
                    lo = std::fmin(lo, a);
                    break;
                }
        cond = hi / lo;
    }
    if (method_used) *method_used = direct ? SVX_ORACLE_METHOD_LDLT : SVX_ORACLE_METHOD_PCG;
    sol->iterations = iters;
    sol->outer_iterations = 0;
    sol->final_residual = res;
    sol->cond_estimate = cond;
    if (sol->u) std::memcpy(sol->u, u.data(), sizeof(double) * n);
    if (sol->displacements)
        for (int64_t i = 0; i < m->n_nodes; ++i) {
            int64_t b = i * ndof;
            sol->displacements[3 * i] = u[b];
            sol->displacements[3 * i + 1] = u[b + 1];
            sol->displacements[3 * i + 2] = (ndof == 3) ? u[b + 2] : 0.0;
        }
    recover(m, u.data(), &k_orig, f_orig.data(), threads, sol->von_mises, sol->nodal_von_mises,
            sol->reactions);
    svx_oracle_csr_free(&k);
    if (err) set_error(err, SVX_OK, 0, -1, "");
    return SVX_OK;
}

int svx_oracle_stress(const svx_flat_model_t* m, const double* u, int threads, double* vm,
                      double* vm_node, double* reactions, svx_error_t* err) {
    svx_oracle_csr_t k;
    int st = svx_oracle_assemble(m, threads, &k, err);
    if (st != SVX_OK) return st;
    recover(m, u, &k, k.f, threads, vm, vm_node, reactions);
    svx_oracle_csr_free(&k);
    return SVX_OK;
}

int svx_oracle_conduction_element(int kind, const double* coords, double conductivity,
                                  double thickness, int has_source, double source, double* ke,
                                  double* fe) {
    bool used = false;
    return conduction_ke(kind, coords, conductivity, thickness, has_source != 0, source, ke, fe,
                         &used);
}

// heat.rs:52-98 solve_thermal, elements of the linear-static path (CPS3,
// CPS4 / CPE4, C3D8): seeds and conduction triplets in element order, flux
// loads, csr_from_triplets, apply_temperatures (heat.rs:361-407), PCG.
int svx_oracle_solve_thermal(const svx_oracle_thermal_t* m, int threads, double tol,
                             double* temperatures, int64_t* iterations, double* residual,
                             svx_error_t* err) {
    auto fail = [&](int code, int reason, int64_t elem, const std::string& msg) {
        set_error(err, code, reason, elem, msg.c_str());
        return code;
    };
    auto eid = [&](int64_t e) { return m->elem_id ? m->elem_id[e] : uint32_t(e + 1); };
    if (m->n_nodes == 0 || m->n_elem == 0) return fail(SVX_EMPTY_MESH, 0, -1, "empty mesh");
    for (int64_t e = 0; e < m->n_elem; ++e)
        if (m->kind[e] == SVX_B31)
            return fail(SVX_INVALID_MODEL, 0, -1,
                        "beam elements have no conduction formulation (v1: plane and solid "
                        "only)");
    if (m->n_temp == 0) return fail(SVX_NO_CONSTRAINTS, 0, -1, "no constraints");
    if (!(m->thickness > 0.0) || !(m->conductivity > 0.0))
        return fail(SVX_INVALID_MODEL, 0, -1, "thickness and conductivity must be positive");
    const int64_t n = m->n_nodes;
    std::vector<int64_t> tr, tc;
    std::vector<double> tv;
    tr.reserve(size_t(n) + size_t(m->n_elem) * 64);
    tc.reserve(tr.capacity());
    tv.reserve(tr.capacity());
    for (int64_t i = 0; i < n; ++i) {
        tr.push_back(i);
        tc.push_back(i);
        tv.push_back(0.0);
    }
    std::vector<double> f(size_t(n), 0.0);
    double ke[64], fe[8], coords[24];
    for (int64_t e = 0; e < m->n_elem; ++e) {
        const int kind = m->kind[e];
        const int nn = node_count(kind);
        const int32_t* cn = m->conn + m->conn_ptr[e];
        for (int i = 0; i < nn && i < 8; ++i)
            for (int a = 0; a < 3; ++a) coords[3 * i + a] = m->xyz[3 * int64_t(cn[i]) + a];
        bool used = false;
        const int r = conduction_ke(kind, coords, m->conductivity, m->thickness,
                                    m->has_source != 0, m->source, ke, fe, &used);
        if (r) {
            char msg[300];
            std::snprintf(msg, sizeof msg, "element %u: %s", eid(e), reason_text(r));
            return fail(SVX_INVALID_MODEL, r, e, msg);
        }
        for (int i = 0; i < nn; ++i) {
            if (used) f[cn[i]] += fe[i];
            for (int j = 0; j < nn; ++j) {
                tr.push_back(cn[i]);
                tc.push_back(cn[j]);
                tv.push_back(ke[i * nn + j]);
            }
        }
    }
    // heat.rs:298-358: linear plane edges only on this path
    for (int64_t q = 0; q < m->n_flux; ++q) {
        const int64_t e = m->flux_elem[q];
        const int kind = m->kind[e];
        int max_face = 0;
        if (kind == SVX_CPS3)
            max_face = 3;
        else if (kind == SVX_CPS4 || kind == SVX_CPE4)
            max_face = 4;
        char msg[300];
        if (!max_face) {
            std::snprintf(msg, sizeof msg,
                          "heat flux on element %u (%s) unsupported (plane edges only)", eid(e),
                          kind_debug(kind));
            return fail(SVX_INVALID_MODEL, 0, e, msg);
        }
        const int face = m->flux_face[q];
        if (face <= 0 || face > max_face) {
            std::snprintf(msg, sizeof msg, "element %u (%s) has no face %d", eid(e),
                          kind_debug(kind), face);
            return fail(SVX_INVALID_MODEL, 0, e, msg);
        }
        const int32_t* cn = m->conn + m->conn_ptr[e];
        const int corners = node_count(kind);
        const int32_t na = cn[face - 1], nb = cn[face % corners];
        const double* pa = m->xyz + 3 * int64_t(na);
        const double* pb = m->xyz + 3 * int64_t(nb);
        const double dx = pb[0] - pa[0], dy = pb[1] - pa[1];
        const double len = std::sqrt(dx * dx + dy * dy);
        if (len == 0.0) {
            std::snprintf(msg, sizeof msg, "zero-length flux edge on element %u", eid(e));
            return fail(SVX_INVALID_MODEL, 0, e, msg);
        }
        const double total = m->flux_value[q] * m->thickness * len;
        f[na] += total / 2.0;
        f[nb] += total / 2.0;
    }
    svx_oracle_csr_t c;
    csr_from_triplets(n, tr, tc, tv, &c);
    // heat.rs:361-407: later constraints win; free rows carry K[r,c] T_c to
    // the right-hand side, prescribed rows become identity rows
    std::vector<double> pres(size_t(n), NAN);
    for (int64_t q = 0; q < m->n_temp; ++q) pres[m->temp_node[q]] = m->temp_value[q];
    for (int64_t r = 0; r < n; ++r) {
        if (!std::isnan(pres[r])) continue;
        for (int64_t ii = c.row_ptr[r]; ii < c.row_ptr[r + 1]; ++ii) {
            const int64_t col = c.col_idx[ii];
            if (!std::isnan(pres[col])) {
                f[r] -= c.vals[ii] * pres[col];
                c.vals[ii] = 0.0;
            }
        }
    }
    for (int64_t r = 0; r < n; ++r) {
        if (std::isnan(pres[r])) continue;
        for (int64_t ii = c.row_ptr[r]; ii < c.row_ptr[r + 1]; ++ii)
            c.vals[ii] = (c.col_idx[ii] == r) ? 1.0 : 0.0;
        f[r] = pres[r];
    }
    const int64_t max_iter = std::max<int64_t>(1000, 10 * n);
    int64_t it = 0;
    double res = 0.0;
    const int st = svx_oracle_pcg(&c, f.data(), tol, max_iter, threads, temperatures, &it, &res);
    svx_oracle_csr_free(&c);
    *iterations = it;
    *residual = res;
    if (st != SVX_OK) {
        char msg[200];
        std::snprintf(msg, sizeof msg, "not converged after %lld iterations", (long long)it);
        set_error(err, SVX_NOT_CONVERGED, 0, -1, msg);
        if (err) {
            err->iterations = it;
            err->residual = res;
        }
        return st;
    }
    if (err) set_error(err, SVX_OK, 0, -1, "");
    return SVX_OK;
}

}  // extern "C"

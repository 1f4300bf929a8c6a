// pado_common.h -- scheme constants and right-hand-side row formulas shared by
// the host table builder and the device kernels.
//
// The constants restate the parameter blocks of the reference modules
// (cd06.F90:14-59, cd10.F90:16-104, cf90.F90:16-48) with the same expression
// trees, so they round to the same doubles.  The row formulas restate the
// explicit stencils ComputeX/Y/ZD1RHS, ComputeX/Y/ZD2RHS and ComputeX/Y/ZRHS
// (cd06.F90:515-742, cd10.F90:1098-2027, cf90.F90:610-1018) with the
// reference's term grouping; X, Y and Z variants share one formula per row.
#pragma once

#include <cmath>
#include <cstddef>

#ifdef __CUDACC__
#define PADO_HD __host__ __device__
#define PADO_INLINE __forceinline__
#else
#define PADO_HD
#define PADO_INLINE inline
#endif

namespace pado {

enum Scheme { CD06 = 0, CD10 = 1, CF90 = 2 };
enum Kind { FILTER = 0, D1 = 1, D2 = 2 };

// Which explicit stencil a kernel applies.
enum RhsKind { RHS_CD06_D1 = 0, RHS_CD10_D1 = 1, RHS_CD10_D2 = 2, RHS_CF90 = 3 };

PADO_HD PADO_INLINE int rhs_kind_of(int scheme, int kind)
{
    return scheme == CD06 ? RHS_CD06_D1 : (scheme == CF90 ? RHS_CF90 : (kind == D2 ? RHS_CD10_D2 : RHS_CD10_D1));
}

// Half width of the widest stencil (cf90: +-4; the one-sided d2 closure at
// node 1 also reaches 4 rows in).
constexpr int HALO = 4;

// Number of closure rows at each end of a bounded line (rows that do not use
// the interior stencil).  cd06.F90:567-585, cd10.F90:1164-1258 / 1656-1730,
// cf90.F90:676-798.
PADO_HD PADO_INLINE int closure_rows(int rk) { return rk == RHS_CD06_D1 ? 3 : (rk == RHS_CD10_D2 ? 3 : 4); }
// Rows of an edge piece (the rows outside the constant-coefficient block,
// cut into pieces the kernels run fully unrolled) for segments of m rows:
// m/4 for cd06 and the cd10 second derivative, m for the bounded cf90, m/2
// for the others.  Measured on 512^3: the shorter pieces give cd06 and cd10
// d2 more resident threads and run 2-6% faster; the cd10 first derivative
// and cf90 lose 1-40% with them (cf90's longer edge region then needs more
// segments than a 16-line tile of 384 threads holds); pieces of m rows make
// the bounded cf90 4-10% faster and the periodic one 7-10% slower.
PADO_HD constexpr int edge_piece_rows(int rk, bool periodic, int m)
{
    return (rk == RHS_CD06_D1 || rk == RHS_CD10_D2) && m / 4 >= 5 ? m / 4
                                                                   : (rk == RHS_CF90 && !periodic ? m : m / 2);
}

// Stencil coefficients, already scaled by 1/dx or 1/dx^2 as the reference
// scales them inside ComputeXD1RHS & co.
struct RhsCoef {
    int rk;        // RhsKind
    int periodic;  // 1 = cyclic line
    double c[16];
};

// ---------------------------------------------------------------------------
// Scheme constants (host).
// ---------------------------------------------------------------------------
struct Cd06Const {
    // cd06.F90:14-59
    double alpha06d1 = 1.0 / 3.0, a06d1 = (14.0 / 9.0) / 2.0, b06d1 = (1.0 / 9.0) / 4.0;
    double alpha06d2 = 2.0 / 11.0;
    double alpha = 3.0, p = 17.0 / 6.0, q = 3.0 / 2.0, r = 3.0 / 2.0, s = -1.0 / 6.0;
    double alpha_hat = 1.0 / 3.0, q_p = 3.0 / 4.0, alpha_p = 1.0 / 4.0;
    double alpha_pp, q_pp, r_pp, w1, w2, w3;
    Cd06Const()
    {
        const double ah = alpha_hat;
        alpha_pp = ((40 * ah - 1) * q + 7 * (4 * ah - 1) * s) / (16 * (ah + 2) * q + 8 * (1 - 4 * ah) * s);
        q_pp = (1.0 / 3.0) * (alpha_pp + 2);
        r_pp = (1.0 / 12.0) * (4 * alpha_pp - 1);
        w1 = (2 * ah + 1) / (2 * (q + s));
        w2 = ((8 * ah + 7) * q - 6 * (2 * ah + 1) * r + (8 * ah + 7) * s) / (9 * (q + s));
        w3 = (4 * (ah + 2) * q + 2 * (1 - 4 * ah) * s) / (9 * (q + s));
    }
};

struct Cd10Const {
    // cd10.F90:16-104
    double alpha10d1 = 1.0 / 2.0, beta10d1 = 1.0 / 20.0;
    double a10d1 = (17.0 / 12.0) / 2.0, b10d1 = (101.0 / 150.0) / 4.0, c10d1 = (1.0 / 100.0) / 6.0;
    double alpha10d2 = 334.0 / 899.0, beta10d2 = 43.0 / 1798.0;
    double a10d2 = (1065.0 / 1798.0) / 1.0, b10d2 = (1038.0 / 899.0) / 4.0, c10d2 = (79.0 / 1798.0) / 9.0;
    double alpha = 3.0, p = -17.0 / 6.0, q = 3.0 / 2.0, r = 3.0 / 2.0, s = -1.0 / 6.0;
    double q_hat, r_hat, s_hat, alpha_hat, beta_hat, q_p = 3.0 / 4.0, alpha_p = 1.0 / 4.0;
    double alpha_ppp, beta_ppp, q_ppp, r_ppp, s_ppp, alpha_pp, beta_pp, q_pp, r_pp, w1, w2, w3, w4;
    // second-derivative closures, cd10.F90:88-104
    double b1_alpha = 11.0, b1_a, b1_b, b1_c, b1_d, b1_e, b2_alpha = 1.0 / 10.0, b2_a;
    double b3_alpha = 344.0 / 1179.0, b3_beta, b3_a, b3_b;
    Cd10Const()
    {
        q_hat = a10d1;
        r_hat = b10d1;
        s_hat = c10d1;
        alpha_hat = alpha10d1;
        beta_hat = beta10d1;
        alpha_ppp = (8 * r_hat - 175 * s_hat) / (18 * r_hat - 550 * s_hat);
        beta_ppp = (1.0 / 20.0) * (-3 + 8 * alpha_ppp);
        q_ppp = (1.0 / 12.0) * (12 - 7 * alpha_ppp);
        r_ppp = (1.0 / 600.0) * (568 * alpha_ppp - 183);
        s_ppp = (1.0 / 300.0) * (9 * alpha_ppp - 4);
        const double t1 = s * (r_hat + 2 * s_hat) - q * (q_hat + r_hat + s_hat);
        const double t2 = q_hat + r_hat - s_hat * (q_ppp / s_ppp - 1);
        alpha_pp = ((17 * t1) / (72 * (q + s) * t2) - 8.0 / 9.0) / ((19 * t1) / (24 * (q + s) * t2) - 1.0 / 3);
        beta_pp = (1.0 / 12.0) * (-1 + 3 * alpha_pp);
        q_pp = (2.0 / 18.0) * (8 - 3 * alpha_pp);
        r_pp = (1.0 / 72.0) * (-17 + 57 * alpha_pp);
        w1 = (q_hat + 2 * r_hat + 3 * s_hat) / (q + s);
        w2 = (1 / q_p) * (r_hat + s_hat * (1 + q_ppp / s_ppp) - r * (q_hat + 2 * r_hat + 3 * s_hat) / (q + s));
        w3 = (q_hat + r_hat + s_hat * (1 - q_ppp / s_ppp)) / (r_pp);
        w4 = s_hat / s_ppp;
        b1_a = (11 * b1_alpha + 35) / 12;
        b1_b = -(5 * b1_alpha + 26) / 3;
        b1_c = (b1_alpha + 19) / 2;
        b1_d = (b1_alpha - 14) / 3;
        b1_e = (11 - b1_alpha) / 12;
        b2_a = (4 * (1 - b2_alpha) / 3) / 1.0;
        b3_beta = (38.0 * b3_alpha - 9.0) / 214.0;
        b3_a = ((696 - 1191 * b3_alpha) / 428) / 1.0;
        b3_b = ((2454 * b3_alpha - 294) / 535) / 4.0;
    }
};

struct Cf90Const {
    // cf90.F90:16-48 (b..e already halved in the reference)
    double alpha = 6.6624e-1, beta = 1.6688e-1;
    double a = 9.9965e-1, b = 6.6652e-1, c = 1.6674e-1, d = 4.0e-5, e = -5.0e-6;
    double b2_alpha = 4.997e-1, b2_a = 9.997e-1, b2_b = 4.9985e-1;
    double b3_alpha = 6.6624e-1, b3_beta = 1.6688e-1, b3_a = 9.9952e-1, b3_b = 6.6656e-1, b3_c = 1.668e-1;
    double b4_alpha = 6.6624e-1, b4_beta = 1.6688e-1, b4_a = 9.9968e-1, b4_b = 6.6652e-1, b4_c = 1.6672e-1;
    double b4_d = 4.0e-5;
};

// ---------------------------------------------------------------------------
// A double whose products and sums round one at a time (no fused
// multiply-add).  The stencils below evaluate with it so that their
// cancelling sums round exactly like the reference's expressions: one-sided
// closures add terms of size f/dx whose sum is orders of magnitude smaller,
// and a contracted product there moves the result by more than the parity
// bar.  The recurrences of the solve are well conditioned and keep FMA.
// ---------------------------------------------------------------------------
struct NC {
    double v;
    PADO_HD PADO_INLINE explicit NC(double x) : v(x) {}
};
#ifdef __CUDA_ARCH__
PADO_HD PADO_INLINE NC operator*(NC a, NC b) { return NC(__dmul_rn(a.v, b.v)); }
PADO_HD PADO_INLINE NC operator+(NC a, NC b) { return NC(__dadd_rn(a.v, b.v)); }
PADO_HD PADO_INLINE NC operator-(NC a, NC b) { return NC(__dsub_rn(a.v, b.v)); }
#else
PADO_HD PADO_INLINE NC operator*(NC a, NC b) { return NC(a.v * b.v); }
PADO_HD PADO_INLINE NC operator+(NC a, NC b) { return NC(a.v + b.v); }
PADO_HD PADO_INLINE NC operator-(NC a, NC b) { return NC(a.v - b.v); }
#endif
PADO_HD PADO_INLINE NC operator-(NC a) { return NC(-a.v); }
PADO_HD PADO_INLINE NC operator*(double a, NC b) { return NC(a) * b; }

// ---------------------------------------------------------------------------
// Interior stencils on a 9-point window v[0..8] = f(i-4..i+4).
// ---------------------------------------------------------------------------
PADO_HD PADO_INLINE double rhs_interior(int rk, int periodic, const double *cc, const double *vv)
{
#define c(k) NC(cc[k])
#define v(k) NC(vv[k])
    switch (rk) {
    case RHS_CD06_D1:
        // periodic: cd06.F90:541-542; bounded rows 4..n-3: cd06.F90:575-576 (b term first)
        if (periodic) return (c(0) * (v(5) - v(3)) + c(1) * (v(6) - v(2))).v;
        return (c(1) * (v(6) - v(2)) + c(0) * (v(5) - v(3))).v;
    case RHS_CD10_D1:  // cd10.F90:1129-1131, 1209-1211
        return (c(0) * (v(5) - v(3)) + c(1) * (v(6) - v(2)) + c(2) * (v(7) - v(1))).v;
    case RHS_CD10_D2:  // cd10.F90:1619-1621, 1692-1694
        return (c(0) * (v(5) - 2.0 * v(4) + v(3)) + c(1) * (v(6) - 2.0 * v(4) + v(2)) +
                c(2) * (v(7) - 2.0 * v(4) + v(1))).v;
    default:  // cf90.F90:643-647, 735-739
        return (c(0) * (v(4)) + c(1) * (v(5) + v(3)) + c(2) * (v(6) + v(2)) + c(3) * (v(7) + v(1)) +
                c(4) * (v(8) + v(0))).v;
    }
#undef c
#undef v
}

// The same interior stencils with fused multiply-adds: for the interior
// (differences of neighbouring values, no one-sided cancellation) the result
// moves by a few ulps of the terms, far inside the parity bar, for two to
// four fewer FP64 operations per row.
PADO_HD PADO_INLINE double rhs_interior_fma(int rk, int periodic, const double *c, const double *v)
{
    switch (rk) {
    case RHS_CD06_D1:
        if (periodic) return fma(c[1], v[6] - v[2], c[0] * (v[5] - v[3]));
        return fma(c[0], v[5] - v[3], c[1] * (v[6] - v[2]));
    case RHS_CD10_D1:
        return fma(c[2], v[7] - v[1], fma(c[1], v[6] - v[2], c[0] * (v[5] - v[3])));
    case RHS_CD10_D2: {
        const double m2 = -2.0 * v[4];
        return fma(c[2], v[7] + m2 + v[1], fma(c[1], v[6] + m2 + v[2], c[0] * (v[5] + m2 + v[3])));
    }
    default:
        return fma(c[4], v[8] + v[0],
                   fma(c[3], v[7] + v[1], fma(c[2], v[6] + v[2], fma(c[1], v[5] + v[3], c[0] * v[4]))));
    }
}

// ---------------------------------------------------------------------------
// One closure row of a bounded line.  `line` is the whole line (element
// stride `stride`),
// `row` is 0-based and lies in the first or last closure_rows(rk) rows.
// F(j) below is the reference's 1-based f(j).
// ---------------------------------------------------------------------------
PADO_HD PADO_INLINE double rhs_closure_row(int rk, const double *c, const double *line, long long stride, int n, int row,
                                      int bc1, int bcn)
{
#define F(j) NC(line[(long long)((j)-1) * stride])
    const int i = row + 1;  // 1-based
    const bool left = i <= closure_rows(rk);
    switch (rk) {
    case RHS_CD06_D1: {
        // cd06.F90:565-585 (bc is fixed at init; only bc=0 closures exist)
        const NC a_np_1(c[2]), b_np_1(c[3]), c_np_1(c[4]), d_np_1(c[5]), a_np_2(c[6]), a_np_3(c[7]), b_np_3(c[8]);
        if (i == 1) return (a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4)).v;
        if (i == 2) return (a_np_2 * (F(3) - F(1))).v;
        if (i == 3) return (a_np_3 * (F(4) - F(2)) + b_np_3 * (F(5) - F(1))).v;
        if (i == n - 2) return (a_np_3 * (F(n - 1) - F(n - 3)) + b_np_3 * (F(n) - F(n - 4))).v;
        if (i == n - 1) return (a_np_2 * (F(n) - F(n - 2))).v;
        return (-(a_np_1 * F(n)) - b_np_1 * F(n - 1) - c_np_1 * F(n - 2) - d_np_1 * F(n - 3)).v;
    }
    case RHS_CD10_D1: {
        // cd10.F90:1164-1258
        const NC a10(c[0]), b10(c[1]), c10(c[2]), a_np_4(c[3]), b_np_4(c[4]), c_np_4(c[5]), a_np_3(c[6]),
                         b_np_3(c[7]), a_np_2(c[8]), a_np_1(c[9]), b_np_1(c[10]), c_np_1(c[11]), d_np_1(c[12]);
        if (left) {
            if (bc1 == 0) {
                if (i == 1) return (a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4)).v;
                if (i == 2) return (a_np_2 * (F(3) - F(1))).v;
                if (i == 3) return (a_np_3 * (F(4) - F(2)) + b_np_3 * (F(5) - F(1))).v;
                return (a_np_4 * (F(5) - F(3)) + b_np_4 * (F(6) - F(2)) + c_np_4 * (F(7) - F(1))).v;
            }
            if (bc1 == 1) {
                if (i == 1) return 0.0;
                if (i == 2) return (a10 * (F(3) - F(1)) + b10 * (F(4) - F(2)) + c10 * (F(5) - F(3))).v;
                if (i == 3) return (a10 * (F(4) - F(2)) + b10 * (F(5) - F(1)) + c10 * (F(6) - F(2))).v;
                return (a10 * (F(5) - F(3)) + b10 * (F(6) - F(2)) + c10 * (F(7) - F(1))).v;
            }
            if (i == 1) return (a10 * (F(2) + F(2)) + b10 * (F(3) + F(3)) + c10 * (F(4) + F(4))).v;
            if (i == 2) return (a10 * (F(3) - F(1)) + b10 * (F(4) + F(2)) + c10 * (F(5) + F(3))).v;
            if (i == 3) return (a10 * (F(4) - F(2)) + b10 * (F(5) - F(1)) + c10 * (F(6) + F(2))).v;
            return (a10 * (F(5) - F(3)) + b10 * (F(6) - F(2)) + c10 * (F(7) - F(1))).v;
        }
        if (bcn == 0) {
            if (i == n - 3) return (a_np_4 * (F(n - 2) - F(n - 4)) + b_np_4 * (F(n - 1) - F(n - 5)) + c_np_4 * (F(n) - F(n - 6))).v;
            if (i == n - 2) return (a_np_3 * (F(n - 1) - F(n - 3)) + b_np_3 * (F(n) - F(n - 4))).v;
            if (i == n - 1) return (a_np_2 * (F(n) - F(n - 2))).v;
            return (-(a_np_1 * F(n)) - b_np_1 * F(n - 1) - c_np_1 * F(n - 2) - d_np_1 * F(n - 3)).v;
        }
        if (bcn == 1) {
            if (i == n - 3) return (a10 * (F(n - 2) - F(n - 4)) + b10 * (F(n - 1) - F(n - 5)) + c10 * (F(n) - F(n - 6))).v;
            if (i == n - 2) return (a10 * (F(n - 1) - F(n - 3)) + b10 * (F(n) - F(n - 4)) + c10 * (F(n - 1) - F(n - 5))).v;
            if (i == n - 1) return (a10 * (F(n) - F(n - 2)) + b10 * (F(n - 1) - F(n - 3)) + c10 * (F(n - 2) - F(n - 4))).v;
            return 0.0;
        }
        if (i == n - 3) return (a10 * (F(n - 2) - F(n - 4)) + b10 * (F(n - 1) - F(n - 5)) + c10 * (F(n) - F(n - 6))).v;
        if (i == n - 2) return (a10 * (F(n - 1) - F(n - 3)) + b10 * (F(n) - F(n - 4)) + c10 * (-F(n - 1) - F(n - 5))).v;
        if (i == n - 1) return (a10 * (F(n) - F(n - 2)) + b10 * (-F(n - 1) - F(n - 3)) + c10 * (-F(n - 2) - F(n - 4))).v;
        return (a10 * (-F(n - 1) - F(n - 1)) + b10 * (-F(n - 2) - F(n - 2)) + c10 * (-F(n - 3) - F(n - 3))).v;
    }
    case RHS_CD10_D2: {
        // cd10.F90:1654-1730
        const NC a10(c[0]), b10(c[1]), c10(c[2]), a_np_3(c[3]), b_np_3(c[4]), a_np_2(c[5]), a_np_1(c[6]),
                         b_np_1(c[7]), c_np_1(c[8]), d_np_1(c[9]), e_np_1(c[10]);
        if (left) {
            if (bc1 == 0) {
                if (i == 1) return (a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4) + e_np_1 * F(5)).v;
                if (i == 2) return (a_np_2 * (F(3) - 2.0 * F(2) + F(1))).v;
                return (a_np_3 * (F(4) - 2.0 * F(3) + F(2)) + b_np_3 * (F(5) - 2.0 * F(3) + F(1))).v;
            }
            if (bc1 == 1) {
                if (i == 1) return (a10 * (F(2) - 2.0 * F(1) + F(2)) + b10 * (F(3) - 2.0 * F(1) + F(3)) + c10 * (F(4) - 2.0 * F(1) + F(4))).v;
                if (i == 2) return (a10 * (F(3) - 2.0 * F(2) + F(1)) + b10 * (F(4) - 2.0 * F(2) + F(2)) + c10 * (F(5) - 2.0 * F(2) + F(3))).v;
                return (a10 * (F(4) - 2.0 * F(3) + F(2)) + b10 * (F(5) - 2.0 * F(3) + F(1)) + c10 * (F(6) - 2.0 * F(3) + F(2))).v;
            }
            if (i == 1) return (a10 * (F(2) - 2.0 * F(1) - F(2)) + b10 * (F(3) - 2.0 * F(1) - F(3)) + c10 * (F(4) - 2.0 * F(1) - F(4))).v;
            if (i == 2) return (a10 * (F(3) - 2.0 * F(2) + F(1)) + b10 * (F(4) - 2.0 * F(2) - F(2)) + c10 * (F(5) - 2.0 * F(2) - F(3))).v;
            return (a10 * (F(4) - 2.0 * F(3) + F(2)) + b10 * (F(5) - 2.0 * F(3) + F(1)) + c10 * (F(6) - 2.0 * F(3) - F(2))).v;
        }
        if (bcn == 0) {
            if (i == n - 2) return (a_np_3 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b_np_3 * (F(n) - 2.0 * F(n - 2) + F(n - 4))).v;
            if (i == n - 1) return (a_np_2 * (F(n) - 2.0 * F(n - 1) + F(n - 2))).v;
            return (a_np_1 * F(n) + b_np_1 * F(n - 1) + c_np_1 * F(n - 2) + d_np_1 * F(n - 3) + e_np_1 * F(n - 4)).v;
        }
        if (bcn == 1) {
            if (i == n - 2) return (a10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b10 * (F(n) - 2.0 * F(n - 2) + F(n - 4)) + c10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 5))).v;
            if (i == n - 1) return (a10 * (F(n) - 2.0 * F(n - 1) + F(n - 2)) + b10 * (F(n - 1) - 2.0 * F(n - 1) + F(n - 3)) + c10 * (F(n - 2) - 2.0 * F(n - 1) + F(n - 4))).v;
            return (a10 * (F(n - 1) - 2.0 * F(n) + F(n - 1)) + b10 * (F(n - 2) - 2.0 * F(n) + F(n - 2)) + c10 * (F(n - 3) - 2.0 * F(n) + F(n - 3))).v;
        }
        if (i == n - 2) return (a10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b10 * (F(n) - 2.0 * F(n - 2) + F(n - 4)) + c10 * (-F(n - 1) - 2.0 * F(n - 2) + F(n - 5))).v;
        if (i == n - 1) return (a10 * (F(n) - 2.0 * F(n - 1) + F(n - 2)) + b10 * (-F(n - 1) - 2.0 * F(n - 1) + F(n - 3)) + c10 * (-F(n - 2) - 2.0 * F(n - 1) + F(n - 4))).v;
        return (a10 * (-F(n - 1) - 2.0 * F(n) + F(n - 1)) + b10 * (-F(n - 2) - 2.0 * F(n) + F(n - 2)) + c10 * (-F(n - 3) - 2.0 * F(n) + F(n - 3))).v;
    }
    default: {
        // cf90.F90:673-798
        const NC a90(c[0]), b90(c[1]), c90(c[2]), d90(c[3]), e90(c[4]);
        const NC b2_a(c[5]), b2_b(c[6]), b3_a(c[7]), b3_b(c[8]), b3_c(c[9]), b4_a(c[10]), b4_b(c[11]), b4_c(c[12]),
                         b4_d(c[13]);
        if (left) {
            if (bc1 == 0) {
                if (i == 1) return (1.0 * (F(1))).v;
                if (i == 2) return (b2_a * (F(2)) + b2_b * (F(3) + F(1))).v;
                if (i == 3) return (b3_a * (F(3)) + b3_b * (F(4) + F(2)) + b3_c * (F(5) + F(1))).v;
                return (b4_a * (F(4)) + b4_b * (F(5) + F(3)) + b4_c * (F(6) + F(2)) + b4_d * (F(7) + F(1))).v;
            }
            if (bc1 == 1) {
                if (i == 1) return (a90 * (F(1)) + b90 * (F(2) + F(2)) + c90 * (F(3) + F(3)) + d90 * (F(4) + F(4)) + e90 * (F(5) + F(5))).v;
                if (i == 2) return (a90 * (F(2)) + b90 * (F(3) + F(1)) + c90 * (F(4) + F(2)) + d90 * (F(5) + F(3)) + e90 * (F(6) + F(4))).v;
                if (i == 3) return (a90 * (F(3)) + b90 * (F(4) + F(2)) + c90 * (F(5) + F(1)) + d90 * (F(6) + F(2)) + e90 * (F(7) + F(3))).v;
                return (a90 * (F(4)) + b90 * (F(5) + F(3)) + c90 * (F(6) + F(2)) + d90 * (F(7) + F(1)) + e90 * (F(8) + F(2))).v;
            }
            if (i == 1) return (a90 * (F(1)) + b90 * (F(2) - F(2)) + c90 * (F(3) - F(3)) + d90 * (F(4) - F(4)) + e90 * (F(5) - F(5))).v;
            if (i == 2) return (a90 * (F(2)) + b90 * (F(3) + F(1)) + c90 * (F(4) - F(2)) + d90 * (F(5) - F(3)) + e90 * (F(6) - F(4))).v;
            if (i == 3) return (a90 * (F(3)) + b90 * (F(4) + F(2)) + c90 * (F(5) + F(1)) + d90 * (F(6) - F(2)) + e90 * (F(7) - F(3))).v;
            return (a90 * (F(4)) + b90 * (F(5) + F(3)) + c90 * (F(6) + F(2)) + d90 * (F(7) + F(1)) + e90 * (F(8) - F(2))).v;
        }
        if (bcn == 0) {
            if (i == n - 3) return (b4_a * (F(n - 3)) + b4_b * (F(n - 2) + F(n - 4)) + b4_c * (F(n - 1) + F(n - 5)) + b4_d * (F(n) + F(n - 6))).v;
            if (i == n - 2) return (b3_a * (F(n - 2)) + b3_b * (F(n - 1) + F(n - 3)) + b3_c * (F(n) + F(n - 4))).v;
            if (i == n - 1) return (b2_a * (F(n - 1)) + b2_b * (F(n) + F(n - 2))).v;
            return (1.0 * (F(n))).v;
        }
        if (bcn == 1) {
            if (i == n - 3) return (a90 * (F(n - 3)) + b90 * (F(n - 2) + F(n - 4)) + c90 * (F(n - 1) + F(n - 5)) + d90 * (F(n) + F(n - 6)) + e90 * (F(n - 1) + F(n - 7))).v;
            if (i == n - 2) return (a90 * (F(n - 2)) + b90 * (F(n - 1) + F(n - 3)) + c90 * (F(n) + F(n - 4)) + d90 * (F(n - 1) + F(n - 5)) + e90 * (F(n - 2) + F(n - 6))).v;
            if (i == n - 1) return (a90 * (F(n - 1)) + b90 * (F(n) + F(n - 2)) + c90 * (F(n - 1) + F(n - 3)) + d90 * (F(n - 2) + F(n - 4)) + e90 * (F(n - 3) + F(n - 5))).v;
            return (a90 * (F(n)) + b90 * (F(n - 1) + F(n - 1)) + c90 * (F(n - 2) + F(n - 2)) + d90 * (F(n - 3) + F(n - 3)) + e90 * (F(n - 4) + F(n - 4))).v;
        }
        if (i == n - 3) return (a90 * (F(n - 3)) + b90 * (F(n - 2) + F(n - 4)) + c90 * (F(n - 1) + F(n - 5)) + d90 * (F(n) + F(n - 6)) + e90 * (-F(n - 1) + F(n - 7))).v;
        if (i == n - 2) return (a90 * (F(n - 2)) + b90 * (F(n - 1) + F(n - 3)) + c90 * (F(n) + F(n - 4)) + d90 * (-F(n - 1) + F(n - 5)) + e90 * (-F(n - 2) + F(n - 6))).v;
        if (i == n - 1) return (a90 * (F(n - 1)) + b90 * (F(n) + F(n - 2)) + c90 * (-F(n - 1) + F(n - 3)) + d90 * (-F(n - 2) + F(n - 4)) + e90 * (-F(n - 3) + F(n - 5))).v;
        return (a90 * (F(n)) + b90 * (-F(n - 1) + F(n - 1)) + c90 * (-F(n - 2) + F(n - 2)) + d90 * (-F(n - 3) + F(n - 3)) + e90 * (-F(n - 4) + F(n - 4))).v;
    }
    }
#undef F
}

// Interior stencil as 9 taps (offset -4..4) -- the same operator as
// rhs_interior, used where a plain weighted sum is enough (the adjoint).
inline void interior_taps(const RhsCoef &rc, double taps[9])
{
    for (int k = 0; k < 9; ++k) taps[k] = 0.0;
    const double *c = rc.c;
    switch (rc.rk) {
    case RHS_CD06_D1:
        taps[5] += c[0]; taps[3] -= c[0]; taps[6] += c[1]; taps[2] -= c[1];
        break;
    case RHS_CD10_D1:
        taps[5] += c[0]; taps[3] -= c[0]; taps[6] += c[1]; taps[2] -= c[1]; taps[7] += c[2]; taps[1] -= c[2];
        break;
    case RHS_CD10_D2:
        for (int d = 1; d <= 3; ++d) {
            taps[4 + d] += c[d - 1];
            taps[4] -= 2.0 * c[d - 1];
            taps[4 - d] += c[d - 1];
        }
        break;
    default:
        taps[4] += c[0];
        for (int d = 1; d <= 4; ++d) {
            taps[4 + d] += c[d];
            taps[4 - d] += c[d];
        }
    }
}

// Scaled stencil coefficients for a (scheme, kind, dx, periodic) operator,
// as ComputeXD1RHS / ComputeXD2RHS / ComputeXRHS scale them.
inline RhsCoef make_rhs_coef(int scheme, int kind, double dx, int periodic)
{
    RhsCoef rc{};
    rc.rk = rhs_kind_of(scheme, kind);
    rc.periodic = periodic;
    const double ob = 1.0 / dx, ob2 = ob / dx;  // cd06.F90:140-141, cd10.F90:206-207
    if (rc.rk == RHS_CD06_D1) {
        const Cd06Const k;
        rc.c[0] = k.a06d1 * ob;  // cd06.F90:552-563
        rc.c[1] = k.b06d1 * ob;
        rc.c[2] = k.w1 * (-(k.p * ob));
        rc.c[3] = k.w1 * (k.q * ob);
        rc.c[4] = k.w1 * (k.r * ob);
        rc.c[5] = k.w1 * (k.s * ob);
        rc.c[6] = k.w2 * k.q_p * ob;
        rc.c[7] = k.w3 * k.q_pp * ob;
        rc.c[8] = k.w3 * k.r_pp * ob;
    } else if (rc.rk == RHS_CD10_D1) {
        const Cd10Const k;
        rc.c[0] = k.q_hat * ob;  // cd10.F90:1144-1160 (q_hat == a10d1 etc.)
        rc.c[1] = k.r_hat * ob;
        rc.c[2] = k.s_hat * ob;
        rc.c[3] = k.w4 * k.q_ppp * ob;
        rc.c[4] = k.w4 * k.r_ppp * ob;
        rc.c[5] = k.w4 * k.s_ppp * ob;
        rc.c[6] = k.w3 * k.q_pp * ob;
        rc.c[7] = k.w3 * k.r_pp * ob;
        rc.c[8] = k.w2 * k.q_p * ob;
        rc.c[9] = k.w1 * (k.p * ob);
        rc.c[10] = k.w1 * (k.q * ob);
        rc.c[11] = k.w1 * (k.r * ob);
        rc.c[12] = k.w1 * (k.s * ob);
    } else if (rc.rk == RHS_CD10_D2) {
        const Cd10Const k;
        rc.c[0] = k.a10d2 * ob2;  // cd10.F90:1638-1651
        rc.c[1] = k.b10d2 * ob2;
        rc.c[2] = k.c10d2 * ob2;
        rc.c[3] = k.b3_a * ob2;
        rc.c[4] = k.b3_b * ob2;
        rc.c[5] = k.b2_a * ob2;
        rc.c[6] = k.b1_a * ob2;
        rc.c[7] = k.b1_b * ob2;
        rc.c[8] = k.b1_c * ob2;
        rc.c[9] = k.b1_d * ob2;
        rc.c[10] = k.b1_e * ob2;
    } else {
        const Cf90Const k;
        rc.c[0] = k.a;
        rc.c[1] = k.b;
        rc.c[2] = k.c;
        rc.c[3] = k.d;
        rc.c[4] = k.e;
        rc.c[5] = k.b2_a;
        rc.c[6] = k.b2_b;
        rc.c[7] = k.b3_a;
        rc.c[8] = k.b3_b;
        rc.c[9] = k.b3_c;
        rc.c[10] = k.b4_a;
        rc.c[11] = k.b4_b;
        rc.c[12] = k.b4_c;
        rc.c[13] = k.b4_d;
    }
    return rc;
}

// ---------------------------------------------------------------------------
// Solver tables.  Every left-hand side the reference factorises (cyclic
// tridiagonal LU, Thomas, cyclic pentadiagonal LU, bounded penta LU) is run
// by the device as the same three-part sweep over the banded rows
// [0, nb) plus nbord = n - nb cyclic border rows:
//
//   forward   z_i = alpha_i r_i - c1_i z_{i-1} - c2_i z_{i-2}
//             sig_k = sum_i k_{k,i} z_i                      (cyclic only)
//   border    E = Mb (r_border - sig);  x_border = E        (cyclic only)
//   backward  x_i = gamma_i z_i - d1_i x_{i+1} - d2_i x_{i+2} - e1_i E_1 - e2_i E_2
//   output    out_i = delta_i x_i
//
// The adjoint solve (A^{-T}) has the same shape with transformed tables.
// A line is cut into S segments; the partition tables hold the responses of
// the forward (U, V) and backward (S, T) recurrences of each segment to a
// unit incoming state, so segments run concurrently and a short chain over
// segments stitches them together.
//
// Per banded row the device table holds 16 doubles (128 bytes):
// ---------------------------------------------------------------------------
// Staged per-row table of the streaming kernel: the fields its sweeps read,
// pairs that are loaded together kept adjacent.  The output scale delta of a
// transposed sweep is not 1 only for tridiagonal sweeps, which have no
// second lag: it shares the c2 slot (E_DELTA).
enum EtabField {
    E_C1 = 0, E_C2 = 1, E_ALPHA = 2, E_K1 = 3, E_K2 = 4, E_D2 = 5, E_U = 6, E_V = 7, E_GAMMA = 8, E_D1 = 9,
    E_S = 10, E_T = 11, E_NF = 12, E_DELTA = E_C2
};

enum TabField {
    T_C1 = 0, T_C2 = 1, T_ALPHA = 2, T_K1 = 3, T_K2 = 4, T_PAD = 5, T_U = 6, T_V = 7,
    T_GAMMA = 8, T_D1 = 9, T_D2 = 10, T_E1 = 11, T_E2 = 12, T_DELTA = 13, T_S = 14, T_T = 15,
    T_NF = 16
};

}  // namespace pado

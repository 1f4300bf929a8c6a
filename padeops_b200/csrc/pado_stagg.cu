// pado_stagg.cu -- the staggered sixth-order compact scheme (cd06stagg) along z:
// first derivatives edge->cell (E2C), cell->edge (C2E), cell->cell (C2C) and
// edge->edge (E2E), second derivatives C2C and E2E, and interpolation E2C and
// C2E, on periodic (cyclic LU) or non-periodic (Thomas; even / odd symmetric
// or one-sided closures) lines.  The cell grid has n points, the edge grid
// n + 1.
//
// Host side: every operator becomes a right-hand-side "row program" per output
// row -- up to four groups coef * (m0 f[i0] + m1 f[i1] + ...), summed in order
// -- that evaluates each row as the reference's array statement for it does
// (same differences, same grouping), plus the factor table of its solve.
// Device side: one thread per z line (lanes are consecutive x, so every row
// access of a warp is one coalesced segment): forward sweep with the
// right-hand side formed row by row, results through df, backward sweep.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "pado_internal.h"

namespace {

constexpr int SG_GROUPS = 4, SG_TERMS = 4;

struct SRow {
    double coef[SG_GROUPS];
    double mul[SG_GROUPS][SG_TERMS];
    int idx[SG_GROUPS][SG_TERMS];
    int nt[SG_GROUPS];
    int ng;
    int pad;
};

// One operator of a handle: its rows, its solve, its shapes.
struct StaggOp {
    int nin = 0, nout = 0, nsolve = 0;
    bool periodic = false, copy_first = false, valid = false;
    std::vector<SRow> rows;
    std::vector<double> fac;  // periodic: [nsolve][5] (bc, h, 1/c, a/c, v/c); else [nout][3] (ddn*den, den, cp)
    SRow *d_rows = nullptr;
    double *d_fac = nullptr;
};

struct Builder {
    std::vector<SRow> rows;
    explicit Builder(int nout) : rows((size_t)nout)
    {
        for (auto &r : rows) std::memset(&r, 0, sizeof(r));
    }
    // group g of row i (0-based): coef * (sum of mul * f[idx], in order); idx 1-based like the reference
    void add(int i, double coef, std::initializer_list<std::pair<double, int>> terms)
    {
        SRow &r = rows[(size_t)i - 1];
        const int g = r.ng++;
        r.coef[g] = coef;
        int t = 0;
        for (const auto &tm : terms) {
            r.mul[g][t] = tm.first;
            r.idx[g][t] = tm.second - 1;
            ++t;
        }
        r.nt[g] = t;
    }
    void clear(int i) { std::memset(&rows[(size_t)i - 1], 0, sizeof(SRow)); }
};

// cd06stagg.F90:18-57: the C2C first derivative's edge closures (Lele).
struct C2CClosure {
    double p = 17.0 / 6.0, q = 3.0 / 2.0, r = 3.0 / 2.0, s = -1.0 / 6.0;
    double alpha_hat = 1.0 / 3.0, q_p = 3.0 / 4.0, alpha_p = 1.0 / 4.0;
    double alpha_pp, q_pp, r_pp, w1, w2, w3;
    C2CClosure()
    {
        alpha_pp = ((40 * alpha_hat - 1) * q + 7 * (4 * alpha_hat - 1) * s) /
                   (16 * (alpha_hat + 2) * q + 8 * (1 - 4 * alpha_hat) * s);
        q_pp = (1.0 / 3.0) * (alpha_pp + 2);
        r_pp = (1.0 / 12.0) * (4 * alpha_pp - 1);
        w1 = (2 * alpha_hat + 1) / (2 * (q + s));
        w2 = ((8 * alpha_hat + 7) * q - 6 * (2 * alpha_hat + 1) * r + (8 * alpha_hat + 7) * s) / (9 * (q + s));
        w3 = (4 * (alpha_hat + 2) * q + 2 * (1 - 4 * alpha_hat) * s) / (9 * (q + s));
    }
};
constexpr double W0S = 223.0 / 186.0, W1S = 61.0 / 62.0;

// Cyclic tridiagonal LU of the periodic operators (the reference's ComputeLU,
// cd06stagg.F90:631-672): per row bc, h, 1/c, a/c, v/c.
std::vector<double> cyclic_lu(int n, double b, double d, double a)
{
    std::vector<double> bc(n, 0.0), h(n, 0.0), c(n, 0.0), aa(n, 0.0), v(n, 0.0);
    c[0] = d;
    v[0] = b;
    h[0] = a / c[0];
    for (int i = 1; i < n - 1; ++i) c[i] = d - (b / c[i - 1]) * a;
    for (int i = 1; i < n - 2; ++i) {
        v[i] = -(b / c[i - 1]) * v[i - 1];
        h[i] = -(a / c[i]) * h[i - 1];
    }
    v[n - 2] = a - (b / c[n - 3]) * v[n - 3];
    h[n - 2] = (b - h[n - 3] * a) / c[n - 2];
    double acc = 0.0;
    for (int i = 0; i < n - 1; ++i) acc += h[i] * v[i];
    c[n - 1] = d - acc;
    for (int i = 1; i < n - 1; ++i) bc[i] = b / c[i - 1];
    for (int i = 0; i < n - 2; ++i) aa[i] = a;
    std::vector<double> out((size_t)n * 5);
    for (int i = 0; i < n; ++i) {
        const double ci = 1.0 / c[i];
        out[(size_t)i * 5 + 0] = bc[i];
        out[(size_t)i * 5 + 1] = h[i];
        out[(size_t)i * 5 + 2] = ci;
        out[(size_t)i * 5 + 3] = aa[i] * ci;
        out[(size_t)i * 5 + 4] = v[i] * ci;
    }
    return out;
}

// Thomas factors of a tridiagonal system (STAGG_CD06_files/ComputeTri_common.F90):
// per row ddn*den, den, cp.
std::vector<double> thomas(const std::vector<double> &ddn, const std::vector<double> &dg, const std::vector<double> &dup)
{
    const int n = (int)dg.size();
    std::vector<double> cp(n, 0.0), den(n, 0.0), out((size_t)n * 3);
    cp[0] = dup[0] / dg[0];
    for (int i = 1; i < n - 1; ++i) cp[i] = dup[i] / (dg[i] - ddn[i] * cp[i - 1]);
    den[0] = 1.0 / dg[0];
    for (int i = 1; i < n; ++i) den[i] = 1.0 / (dg[i] - ddn[i] * cp[i - 1]);
    for (int i = 0; i < n; ++i) {
        out[(size_t)i * 3 + 0] = ddn[i] * den[i];
        out[(size_t)i * 3 + 1] = den[i];
        out[(size_t)i * 3 + 2] = cp[i];
    }
    return out;
}

}  // namespace

struct pado_stagg_s {
    int n = 0, periodic = 1, top_even = 1, bot_even = 1, top_sided = 0, bot_sided = 0, device = 0;
    double dx = 1.0;
    StaggOp ops[PADO_STAGG_NOPS];
};

namespace {

// ---- right-hand sides and solves of one handle ------------------------------------------------
void build_periodic(pado_stagg_s *h)
{
    const int n = h->n, nE = n + 1;
    const double odx = 1.0 / h->dx;
    auto wrap = [&](int j) { return j; };  // indices below are written out as the reference does
    (void)wrap;
    const std::vector<double> lu_d1 = cyclic_lu(n, 9.0 / 62.0, 1.0, 9.0 / 62.0);
    const std::vector<double> lu_d2 = cyclic_lu(n, 2.0 / 11.0, 1.0, 2.0 / 11.0);
    const std::vector<double> lu_in = cyclic_lu(n, 3.0 / 10.0, 1.0, 3.0 / 10.0);
    // E2C, first derivative (differences) and interpolation (sums): n rows from nE edges
    // (ComputeZD1RHS_E2C_REAL_periodic :301-322, ComputeZInterpRHS_E2C_REAL_periodic :526-547)
    for (int which = 0; which < 2; ++which) {
        const bool d1 = which == 0;
        const double a06 = d1 ? (63.0 / 62.0) * odx : (3.0 / 2.0) * 0.5;
        const double b06 = d1 ? ((17.0 / 62.0) / 3.0) * odx : (1.0 / 10.0) * 0.5;
        const double sg = d1 ? -1.0 : 1.0;
        Builder B(n);
        B.add(1, a06, {{1.0, 2}, {sg, 1}});
        B.add(1, b06, {{1.0, 3}, {sg, n}});
        for (int i = 2; i <= n - 1; ++i) {
            B.add(i, a06, {{1.0, i + 1}, {sg, i}});
            B.add(i, b06, {{1.0, i + 2}, {sg, i - 1}});
        }
        B.add(n, a06, {{1.0, n + 1}, {sg, n}});
        B.add(n, b06, {{1.0, 2}, {sg, n - 1}});
        StaggOp &o = h->ops[d1 ? PADO_STAGG_DDZ_E2C : PADO_STAGG_INTERPZ_E2C];
        o.nin = nE;
        o.nout = n;
        o.rows = B.rows;
        o.fac = d1 ? lu_d1 : lu_in;
    }
    // C2E, first derivative and interpolation: rows 1..n solved, row n+1 = row 1
    // (ComputeZD1RHS_C2E_REAL_periodic :349-375, ComputeZInterpRHS_C2E_REAL_periodic :573-600)
    for (int which = 0; which < 2; ++which) {
        const bool d1 = which == 0;
        const double a06 = d1 ? (63.0 / 62.0) * odx : (3.0 / 2.0) * 0.5;
        const double b06 = d1 ? ((17.0 / 62.0) / 3.0) * odx : (1.0 / 10.0) * 0.5;
        const double sg = d1 ? -1.0 : 1.0;
        Builder B(nE);
        B.add(1, a06, {{1.0, 1}, {sg, n}});
        B.add(1, b06, {{1.0, 2}, {sg, n - 1}});
        B.add(2, a06, {{1.0, 2}, {sg, 1}});
        B.add(2, b06, {{1.0, 3}, {sg, n}});
        for (int i = 3; i <= n - 1; ++i) {
            B.add(i, a06, {{1.0, i}, {sg, i - 1}});
            B.add(i, b06, {{1.0, i + 1}, {sg, i - 2}});
        }
        B.add(n, a06, {{1.0, n}, {sg, n - 1}});
        B.add(n, b06, {{1.0, 1}, {sg, n - 2}});
        StaggOp &o = h->ops[d1 ? PADO_STAGG_DDZ_C2E : PADO_STAGG_INTERPZ_C2E];
        o.nin = n;
        o.nout = nE;
        o.copy_first = true;
        o.rows = B.rows;
        o.fac = d1 ? lu_d1 : lu_in;
    }
    // second derivatives C2C (n rows) and E2E (n solved rows, row n+1 = row 1)
    // (ComputeZD2RHS_C2C_REAL_periodic :405-432, ComputeZD2RHS_E2E_REAL_periodic :465-495)
    const double a2 = (12.0 / 11.0) * (odx * odx), b2 = ((3.0 / 11.0) / 4.0) * (odx * odx);
    for (int which = 0; which < 2; ++which) {
        const bool e2e = which == 1;
        Builder B(e2e ? nE : n);
        auto d2 = [&](int i, int p1, int m1, int p2, int m2) {
            B.add(i, a2, {{1.0, p1}, {-2.0, i}, {1.0, m1}});
            B.add(i, b2, {{1.0, p2}, {-2.0, i}, {1.0, m2}});
        };
        d2(1, 2, n, 3, n - 1);
        d2(2, 3, 1, 4, n);
        for (int i = 3; i <= n - 2; ++i) d2(i, i + 1, i - 1, i + 2, i - 2);
        d2(n - 1, n, n - 2, 1, n - 3);
        d2(n, 1, n - 1, 2, n - 2);
        StaggOp &o = h->ops[e2e ? PADO_STAGG_D2DZ2_E2E : PADO_STAGG_D2DZ2_C2C];
        o.nin = e2e ? nE : n;
        o.nout = e2e ? nE : n;
        o.copy_first = e2e;
        o.rows = B.rows;
        o.fac = lu_d2;
    }
    for (int k : {PADO_STAGG_DDZ_E2C, PADO_STAGG_DDZ_C2E, PADO_STAGG_INTERPZ_E2C, PADO_STAGG_INTERPZ_C2E,
                  PADO_STAGG_D2DZ2_C2C, PADO_STAGG_D2DZ2_E2E}) {
        h->ops[k].periodic = true;
        h->ops[k].nsolve = n;
        h->ops[k].valid = true;
    }
    // C2C and E2E first derivatives exist only for non-periodic objects (the
    // reference solves them with tables a periodic init does not allocate)
}

void build_nonperiodic(pado_stagg_s *h)
{
    const int n = h->n, nE = n + 1;
    const bool te = h->top_even, be = h->bot_even, ts = h->top_sided, bs = h->bot_sided;
    const double odx = 1.0 / h->dx, odx2 = odx / h->dx;
    const C2CClosure C;
    auto setop = [&](int k, int nin, int nout, const Builder &B, std::vector<double> fac) {
        StaggOp &o = h->ops[k];
        o.nin = nin;
        o.nout = nout;
        o.nsolve = nout;
        o.rows = B.rows;
        o.fac = std::move(fac);
        o.valid = true;
    };
    // ---- ddz_E2C (D1RHS_E2C_common.F90, ComputeTriD1_E2C) ----
    {
        const double a = (63.0 / 62.0) / 1.0, b = (17.0 / 62.0) / 3.0;
        const double alpha1 = 37.0 / 183.0, alpha0 = -1.0;
        const double a0 = (1.0 / 24.0) * (alpha0 - 23.0), b0 = (1.0 / 8.0) * (-9.0 * alpha0 + 7.0);
        const double c0 = (1.0 / 8.0) * (9.0 * alpha0 + 1.0), d0 = -(1.0 / 24.0) * (alpha0 + 1.0);
        const double a1 = (3.0 / 8.0) * (3.0 - 2.0 * alpha1), b1 = (1.0 / 8.0) * (-1.0 + 22.0 * alpha1);
        const double a06 = a * odx, b06 = b * odx;
        Builder B(n);
        for (int i = 2; i <= n - 1; ++i) {
            B.add(i, b06, {{1.0, i + 2}, {-1.0, i - 1}});
            B.add(i, a06, {{1.0, i + 1}, {-1.0, i}});
        }
        if (bs) {
            B.clear(1);
            B.clear(2);
            B.add(1, W0S * odx, {{a0, 1}, {b0, 2}, {c0, 3}, {d0, 4}});
            B.add(2, W1S * odx, {{-b1 / 3.0, 1}, {-a1, 2}, {a1, 3}, {b1 / 3.0, 4}});
        } else {
            B.add(1, b06, {{1.0, 3}, {be ? -1.0 : 1.0, 2}});
            B.add(1, a06, {{1.0, 2}, {-1.0, 1}});
        }
        if (ts) {
            B.clear(n);
            B.clear(n - 1);
            B.add(n, -(W0S * odx), {{a0, nE}, {b0, nE - 1}, {c0, nE - 2}, {d0, nE - 3}});
            B.add(n - 1, W1S * odx, {{-b1 / 3.0, nE - 3}, {-a1, nE - 2}, {a1, nE - 1}, {b1 / 3.0, nE}});
        } else if (te) {
            B.add(n, b06, {{1.0, nE - 1}, {-1.0, nE - 2}});
            B.add(n, a06, {{1.0, nE}, {-1.0, nE - 1}});
        } else {
            B.add(n, -b06, {{1.0, nE - 1}, {1.0, nE - 2}});
            B.add(n, a06, {{1.0, nE}, {-1.0, nE - 1}});
        }
        const double al = 9.0 / 62.0;
        std::vector<double> ddn(n, al), dg(n, 1.0), dup(n, al);
        if (ts) {
            ddn[n - 1] = W0S * alpha0; dg[n - 1] = W0S;
            ddn[n - 2] = W1S * alpha1; dup[n - 2] = W1S * alpha1; dg[n - 2] = W1S;
        } else if (te) {
            dup[n - 1] = 0.0; dg[n - 1] = 1.0 - al;
        } else {
            dg[n - 1] = 1.0 + al; dup[n - 1] = 0.0;
        }
        if (bs) {
            dup[0] = W0S * alpha0; dg[0] = W0S;
            ddn[1] = W1S * alpha1; dup[1] = W1S * alpha1; dg[1] = W1S;
        } else {
            ddn[0] = 0.0; dg[0] = be ? 1.0 - al : 1.0 + al;
        }
        setop(PADO_STAGG_DDZ_E2C, nE, n, B, thomas(ddn, dg, dup));
    }
    // ---- ddz_C2E (D1RHS_C2E_common.F90, ComputeTriD1_C2E) ----
    {
        const double a = (63.0 / 62.0) / 1.0, b = (17.0 / 62.0) / 3.0;
        const double a0 = -71.0 / 24.0, b0 = 47.0 / 8.0, c0 = -31.0 / 8.0, d0 = 23.0 / 24.0, a1 = 12.0 / 11.0;
        const double a06 = a * odx, b06 = b * odx;
        Builder B(nE);
        for (int i = 2; i <= nE - 1; ++i) B.add(i, a06, {{1.0, i}, {-1.0, i - 1}});
        for (int i = 3; i <= nE - 2; ++i) B.add(i, b06, {{1.0, i + 1}, {-1.0, i - 2}});
        if (bs) {
            B.clear(1);
            B.clear(2);
            B.add(1, odx, {{a0, 1}, {b0, 2}, {c0, 3}, {d0, 4}});
            B.add(2, a1 * odx, {{1.0, 2}, {-1.0, 1}});
        } else if (be) {
            B.clear(1);
            B.add(2, b06, {{1.0, 3}, {-1.0, 1}});
        } else {
            B.clear(1);
            B.add(1, 2.0 * b06, {{1.0, 2}});
            B.add(1, 2.0 * a06, {{1.0, 1}});
            B.add(2, b06, {{1.0, 3}, {1.0, 1}});
        }
        if (ts) {
            B.clear(nE - 1);
            B.clear(nE);
            B.add(nE - 1, a1 * odx, {{1.0, n}, {-1.0, n - 1}});
            B.add(nE, -odx, {{a0, n}, {b0, n - 1}, {c0, n - 2}, {d0, n - 3}});
        } else if (te) {
            B.add(nE - 1, b06, {{1.0, n}, {-1.0, n - 2}});
            B.clear(nE);
        } else {
            B.add(nE - 1, -b06, {{1.0, n}, {1.0, n - 2}});
            B.clear(nE);
            B.add(nE, -2.0 * b06, {{1.0, n - 1}});
            B.add(nE, 2.0 * a06, {{-1.0, n}});
        }
        const double al = 9.0 / 62.0;
        std::vector<double> ddn(nE, al), dg(nE, 1.0), dup(nE, al);
        const int m = nE;
        if (ts) {
            ddn[m - 1] = 0.0; dup[m - 1] = 0.0;
            ddn[m - 2] = 1.0 / 22.0; dup[m - 2] = 1.0 / 22.0;
        } else if (te) {
            dup[m - 1] = 0.0; ddn[m - 1] = 0.0;
        } else {
            ddn[m - 1] = 2.0 * al; dup[m - 1] = 0.0;
        }
        if (bs) {
            dup[0] = 0.0; ddn[0] = 0.0;
            dup[1] = 1.0 / 22.0; ddn[1] = 1.0 / 22.0;
        } else if (be) {
            ddn[0] = 0.0; dup[0] = 0.0;
        } else {
            ddn[0] = 0.0; dup[0] = 2.0 * al;
        }
        setop(PADO_STAGG_DDZ_C2E, n, nE, B, thomas(ddn, dg, dup));
    }
    // ---- ddz_C2C (D1RHS_C2C_common.F90, ComputeTriD1_C2C) ----
    {
        const double a = (14.0 / 9.0) / 2.0, b = (1.0 / 9.0) / 4.0;
        const double a06 = a * odx, b06 = b * odx;
        const double a_np_3 = C.w3 * C.q_pp * odx, b_np_3 = C.w3 * C.r_pp * odx, a_np_2 = C.w2 * C.q_p * odx;
        const double a_np_1 = C.w1 * (-C.p * odx), b_np_1 = C.w1 * (C.q * odx);
        const double c_np_1 = C.w1 * (C.r * odx), d_np_1 = C.w1 * (C.s * odx);
        Builder B(n);
        if (bs) {
            B.add(1, a_np_1, {{1.0, 1}});
            B.add(1, b_np_1, {{1.0, 2}});
            B.add(1, c_np_1, {{1.0, 3}});
            B.add(1, d_np_1, {{1.0, 4}});
            B.add(2, a_np_2, {{1.0, 3}, {-1.0, 1}});
            B.add(3, a_np_3, {{1.0, 4}, {-1.0, 2}});
            B.add(3, b_np_3, {{1.0, 5}, {-1.0, 1}});
        } else if (be) {
            B.add(1, b06, {{1.0, 3}, {-1.0, 2}});
            B.add(1, a06, {{1.0, 2}, {-1.0, 1}});
            B.add(2, b06, {{1.0, 4}, {-1.0, 1}});
            B.add(2, a06, {{1.0, 3}, {-1.0, 1}});
            B.add(3, b06, {{1.0, 5}, {-1.0, 1}});
            B.add(3, a06, {{1.0, 4}, {-1.0, 2}});
        } else {
            B.add(1, b06, {{1.0, 3}, {1.0, 2}});
            B.add(1, a06, {{1.0, 2}, {1.0, 1}});
            B.add(2, b06, {{1.0, 4}, {1.0, 1}});
            B.add(2, a06, {{1.0, 3}, {-1.0, 1}});
            B.add(3, b06, {{1.0, 5}, {-1.0, 1}});
            B.add(3, a06, {{1.0, 4}, {-1.0, 2}});
        }
        for (int i = 4; i <= n - 3; ++i) {
            B.add(i, b06, {{1.0, i + 2}, {-1.0, i - 2}});
            B.add(i, a06, {{1.0, i + 1}, {-1.0, i - 1}});
        }
        if (ts) {
            B.add(n - 2, a_np_3, {{1.0, n - 1}, {-1.0, n - 3}});
            B.add(n - 2, b_np_3, {{1.0, n}, {-1.0, n - 4}});
            B.add(n - 1, a_np_2, {{1.0, n}, {-1.0, n - 2}});
            B.add(n, -a_np_1, {{1.0, n}});
            B.add(n, -b_np_1, {{1.0, n - 1}});
            B.add(n, -c_np_1, {{1.0, n - 2}});
            B.add(n, -d_np_1, {{1.0, n - 3}});
        } else if (te) {
            B.add(n - 2, b06, {{1.0, n}, {-1.0, n - 4}});
            B.add(n - 2, a06, {{1.0, n - 1}, {-1.0, n - 3}});
            B.add(n - 1, b06, {{1.0, n}, {-1.0, n - 3}});
            B.add(n - 1, a06, {{1.0, n}, {-1.0, n - 2}});
            B.add(n, b06, {{1.0, n - 1}, {-1.0, n - 2}});
            B.add(n, a06, {{1.0, n}, {-1.0, n - 1}});
        } else {
            B.add(n - 2, b06, {{1.0, n}, {-1.0, n - 4}});
            B.add(n - 2, a06, {{1.0, n - 1}, {-1.0, n - 3}});
            B.add(n - 1, -b06, {{1.0, n}, {1.0, n - 3}});
            B.add(n - 1, a06, {{1.0, n}, {-1.0, n - 2}});
            B.add(n, -b06, {{1.0, n - 1}, {1.0, n - 2}});
            B.add(n, -a06, {{1.0, n}, {1.0, n - 1}});
        }
        const double al = 1.0 / 3.0, alpha_low = 3.0;
        std::vector<double> ddn(n, al), dg(n, 1.0), dup(n, al);
        if (ts) {
            dup[n - 1] = C.w1 * 0.0; dup[n - 2] = C.w2 * C.alpha_p; dup[n - 3] = C.w3 * C.alpha_pp;
            dg[n - 1] = C.w1 * 1.0; dg[n - 2] = C.w2 * 1.0; dg[n - 3] = C.w3 * 1.0;
            ddn[n - 1] = C.w1 * alpha_low; ddn[n - 2] = C.w2 * C.alpha_p; ddn[n - 3] = C.w3 * C.alpha_pp;
        } else {
            dg[n - 1] = te ? 1.0 - al : 1.0 + al;
        }
        if (bs) {
            ddn[0] = C.w1 * 0.0; ddn[1] = C.w2 * C.alpha_p; ddn[2] = C.w3 * C.alpha_pp;
            dg[0] = C.w1 * 1.0; dg[1] = C.w2 * 1.0; dg[2] = C.w3 * 1.0;
            dup[0] = C.w1 * alpha_low; dup[1] = C.w2 * C.alpha_p; dup[2] = C.w3 * C.alpha_pp;
        } else {
            dg[0] = be ? 1.0 - al : 1.0 + al;
        }
        setop(PADO_STAGG_DDZ_C2C, n, n, B, thomas(ddn, dg, dup));
    }
    // ---- ddz_E2E (D1RHS_E2E_common.F90, ComputeTriD1_E2E) ----
    {
        const double a = (14.0 / 9.0) / 2.0, b = (1.0 / 9.0) / 4.0;
        const double a06 = a * odx, b06 = b * odx;
        Builder B(nE);
        for (int i = 2; i <= nE - 1; ++i) B.add(i, a06, {{1.0, i + 1}, {-1.0, i - 1}});
        for (int i = 3; i <= nE - 2; ++i) B.add(i, b06, {{1.0, i + 2}, {-1.0, i - 2}});
        if (be) {
            B.clear(1);
            B.add(2, b06, {{1.0, 4}, {-1.0, 2}});
        } else {
            B.clear(1);
            B.add(1, b06, {{1.0, 3}, {1.0, 3}});
            B.add(1, a06, {{1.0, 2}, {1.0, 2}});
            B.add(2, b06, {{1.0, 4}, {1.0, 2}});
        }
        if (te) {
            B.clear(nE);
            B.add(nE - 1, b06, {{1.0, nE - 1}, {-1.0, nE - 3}});
        } else {
            B.clear(nE);
            B.add(nE, -b06, {{1.0, nE - 2}, {1.0, nE - 2}});
            B.add(nE, a06, {{-1.0, nE - 1}, {-1.0, nE - 1}});
            B.add(nE - 1, -b06, {{1.0, nE - 1}, {1.0, nE - 3}});
        }
        const double al = 1.0 / 3.0;
        std::vector<double> ddn(nE, al), dg(nE, 1.0), dup(nE, al);
        dg[nE - 1] = 1.0; ddn[nE - 1] = te ? 0.0 : 2.0 * al;
        dg[0] = 1.0; dup[0] = be ? 0.0 : 2.0 * al;
        setop(PADO_STAGG_DDZ_E2E, nE, nE, B, thomas(ddn, dg, dup));
    }
    // ---- d2dz2_C2C and d2dz2_E2E (D2RHS_*_common.F90, ComputeTriD2_*) ----
    for (int which = 0; which < 2; ++which) {
        const bool e2e = which == 1;
        const int m = e2e ? nE : n;
        const double a = 12.0 / 11.0, b = (3.0 / 11.0) / 4.0;
        const double a06 = a * odx2, b06 = b * odx2;
        Builder B(m);
        for (int i = 2; i <= m - 1; ++i) B.add(i, a06, {{1.0, i + 1}, {1.0, i - 1}});
        for (int i = 3; i <= m - 2; ++i) B.add(i, b06, {{1.0, i + 2}, {1.0, i - 2}});
        if (!e2e) {
            if (be) {
                B.add(1, b06, {{1.0, 3}, {1.0, 2}});
                B.add(1, a06, {{1.0, 2}, {1.0, 1}});
                B.add(2, b06, {{1.0, 4}, {1.0, 1}});
            } else {
                B.add(1, b06, {{1.0, 3}, {-1.0, 2}});
                B.add(1, a06, {{1.0, 2}, {-1.0, 1}});
                B.add(2, b06, {{1.0, 4}, {-1.0, 1}});
            }
            if (te) {
                B.add(n, b06, {{1.0, n - 1}, {1.0, n - 2}});
                B.add(n, a06, {{1.0, n}, {1.0, n - 1}});
                B.add(n - 1, b06, {{1.0, n}, {1.0, n - 3}});
            } else {
                B.add(n, b06, {{-1.0, n - 1}, {1.0, n - 2}});
                B.add(n, a06, {{-1.0, n}, {1.0, n - 1}});
                B.add(n - 1, b06, {{-1.0, n}, {1.0, n - 3}});
            }
        } else {
            if (be) {
                B.add(1, b06, {{1.0, 3}, {1.0, 3}});
                B.add(1, a06, {{1.0, 2}, {1.0, 2}});
                B.add(2, b06, {{1.0, 4}, {1.0, 2}});
            } else {
                B.add(2, b06, {{1.0, 4}, {-1.0, 2}});
            }
            if (te) {
                B.add(nE, 2.0 * b06, {{1.0, nE - 2}});
                B.add(nE, 2.0 * a06, {{1.0, nE - 1}});
                B.add(nE - 1, b06, {{1.0, nE - 1}, {1.0, nE - 3}});
            } else {
                B.add(nE - 1, b06, {{-1.0, nE - 1}, {1.0, nE - 3}});
            }
        }
        // rhs = rhs - two*(b06 + a06)*f, row by row
        const double cdiag = 2.0 * (b06 + a06);
        for (int i = 1; i <= m; ++i) B.add(i, -cdiag, {{1.0, i}});
        const double al = 2.0 / 11.0;
        std::vector<double> ddn(m, al), dg(m, 1.0), dup(m, al);
        if (e2e) {
            dg[m - 1] = 1.0; ddn[m - 1] = te ? 2.0 * al : 0.0;
            dg[0] = 1.0; dup[0] = be ? 2.0 * al : 0.0;
        } else {
            dg[m - 1] = te ? 1.0 + al : 1.0 - al;
            dg[0] = be ? 1.0 + al : 1.0 - al;
        }
        setop(e2e ? PADO_STAGG_D2DZ2_E2E : PADO_STAGG_D2DZ2_C2C, m, m, B, thomas(ddn, dg, dup));
    }
    // ---- InterpZ_C2E (InterpRHS_C2E_common.F90, ComputeTriInterp_C2E) ----
    {
        const double b = (1.0 / 10.0) / 2.0, a = (3.0 / 2.0) / 2.0;
        const double a0 = 15.0 / 8.0, b0 = -5.0 / 4.0, c0 = 3.0 / 8.0;
        const double alpha1 = 1.0 / 6.0, a1 = (1.0 / 8.0) * (9.0 + 10.0 * alpha1);
        Builder B(nE);
        for (int i = 2; i <= nE - 1; ++i) B.add(i, a, {{1.0, i}, {1.0, i - 1}});
        for (int i = 3; i <= nE - 2; ++i) B.add(i, b, {{1.0, i + 1}, {1.0, i - 2}});
        if (bs) {
            B.clear(1);
            B.clear(2);
            B.add(1, a0, {{1.0, 1}});
            B.add(1, b0, {{1.0, 2}});
            B.add(1, c0, {{1.0, 3}});
            B.add(2, a1 / 2.0, {{1.0, 2}, {1.0, 1}});
        } else if (be) {
            B.clear(1);
            B.add(1, 2.0 * b, {{1.0, 2}});
            B.add(1, 2.0 * a, {{1.0, 1}});
            B.add(2, b, {{1.0, 3}, {1.0, 1}});
        } else {
            B.clear(1);
            B.add(2, b, {{1.0, 3}, {-1.0, 1}});
        }
        if (ts) {
            B.clear(nE);
            B.clear(nE - 1);
            B.add(nE, a0, {{1.0, n}});
            B.add(nE, b0, {{1.0, n - 1}});
            B.add(nE, c0, {{1.0, n - 2}});
            B.add(nE - 1, a1 / 2.0, {{1.0, n}, {1.0, n - 1}});
        } else if (te) {
            B.clear(nE);
            B.add(nE, 2.0 * b, {{1.0, n - 1}});
            B.add(nE, 2.0 * a, {{1.0, n}});
            B.add(nE - 1, b, {{1.0, n}, {1.0, n - 2}});
        } else {
            B.clear(nE);
            B.add(nE - 1, b, {{-1.0, n}, {1.0, n - 2}});
        }
        const double al = 3.0 / 10.0;
        std::vector<double> ddn(nE, al), dg(nE, 1.0), dup(nE, al);
        const int m = nE;
        if (ts) {
            dup[m - 1] = 0.0; ddn[m - 1] = 0.0;
            dup[m - 2] = alpha1; ddn[m - 2] = alpha1;
        } else if (te) {
            ddn[m - 1] = 2.0 * al; dg[m - 1] = 1.0;
        } else {
            ddn[m - 1] = 0.0; dg[m - 1] = 1.0;
        }
        if (bs) {
            dup[0] = 0.0; ddn[0] = 0.0; dg[0] = 1.0;
            dup[1] = alpha1; ddn[1] = alpha1; dg[1] = 1.0;
        } else if (be) {
            dup[0] = 2.0 * al; dg[0] = 1.0;
        } else {
            dup[0] = 0.0; dg[0] = 1.0;
        }
        setop(PADO_STAGG_INTERPZ_C2E, n, nE, B, thomas(ddn, dg, dup));
    }
    // ---- InterpZ_E2C (InterpRHS_E2C_common.F90, ComputeTriInterp_E2C) ----
    {
        const double b = (1.0 / 10.0) / 2.0, a = (3.0 / 2.0) / 2.0;
        const double alpha0 = 1.0;
        const double a0 = (1.0 / 16.0) * (5.0 - alpha0), b0 = (1.0 / 16.0) * (9.0 * alpha0 + 15.0);
        const double c0 = (1.0 / 16.0) * (9.0 * alpha0 - 5.0), d0 = (1.0 / 16.0) * (1.0 - alpha0);
        Builder B(n);
        if (bs) {
            B.add(1, a0, {{1.0, 1}});
            B.add(1, b0, {{1.0, 2}});
            B.add(1, c0, {{1.0, 3}});
            B.add(1, d0, {{1.0, 4}});
        } else {
            B.add(1, b, {{1.0, 3}, {be ? 1.0 : -1.0, 2}});
            B.add(1, a, {{1.0, 2}, {1.0, 1}});
        }
        for (int i = 2; i <= n - 1; ++i) {
            B.add(i, b, {{1.0, i + 2}, {1.0, i - 1}});
            B.add(i, a, {{1.0, i + 1}, {1.0, i}});
        }
        if (ts) {
            B.add(n, a0, {{1.0, nE}});
            B.add(n, b0, {{1.0, nE - 1}});
            B.add(n, c0, {{1.0, nE - 2}});
            B.add(n, d0, {{1.0, nE - 3}});
        } else if (te) {
            B.add(n, b, {{1.0, nE - 1}, {1.0, nE - 2}});
            B.add(n, a, {{1.0, nE}, {1.0, nE - 1}});
        } else {
            B.add(n, b, {{-1.0, nE - 1}, {1.0, nE - 2}});
            B.add(n, a, {{1.0, nE}, {1.0, nE - 1}});
        }
        const double al = 3.0 / 10.0;
        std::vector<double> ddn(n, al), dg(n, 1.0), dup(n, al);
        if (ts) {
            ddn[n - 1] = alpha0; dup[n - 1] = 0.0;
        } else {
            dg[n - 1] = te ? 1.0 + al : 1.0 - al;
        }
        if (bs) {
            dup[0] = alpha0; ddn[0] = 0.0;
        } else {
            dg[0] = be ? 1.0 + al : 1.0 - al;
        }
        setop(PADO_STAGG_INTERPZ_E2C, nE, n, B, thomas(ddn, dg, dup));
    }
}

// ---- device ------------------------------------------------------------------------------
struct StaggLaunch {
    const double *in;
    double *out;
    long long nlines, zs;  // lines (n1 * n2, x fastest) and the element stride between z planes
    int nout, nsolve, periodic, copy_first;
    const SRow *rows;
    const double *fac;
};

__device__ __forceinline__ double stagg_rhs(const SRow *__restrict__ rows, int k, const double *__restrict__ f,
                                            long long zs)
{
    const SRow *r = rows + k;
    const int ng = __ldg(&r->ng);
    double acc = 0.0;
    for (int g = 0; g < ng; ++g) {
        const int nt = __ldg(&r->nt[g]);
        double s = __ldg(&r->mul[g][0]) * f[(long long)__ldg(&r->idx[g][0]) * zs];
        for (int t = 1; t < nt; ++t) s += __ldg(&r->mul[g][t]) * f[(long long)__ldg(&r->idx[g][t]) * zs];
        const double v = __ldg(&r->coef[g]) * s;
        acc = g == 0 ? v : acc + v;
    }
    return acc;
}

__global__ void __launch_bounds__(256) stagg_kernel(const StaggLaunch p)
{
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= p.nlines) return;
    const double *f = p.in + q;
    double *y = p.out + q;
    const long long zs = p.zs;
    const double *__restrict__ F = p.fac;
    if (!p.periodic) {
        // Thomas (SolveZTriREAL): y1 = r1 den1; yk = rk denk - y(k-1) (ddn den)k; yk -= cp_k y(k+1)
        const int m = p.nout;
        double prev = stagg_rhs(p.rows, 0, f, zs) * __ldg(F + 1);
        y[0] = prev;
        for (int k = 1; k < m; ++k) {
            prev = stagg_rhs(p.rows, k, f, zs) * __ldg(F + 3 * k + 1) - prev * __ldg(F + 3 * k);
            y[(long long)k * zs] = prev;
        }
        for (int k = m - 2; k >= 0; --k) {
            prev = y[(long long)k * zs] - __ldg(F + 3 * k + 2) * prev;
            y[(long long)k * zs] = prev;
        }
        return;
    }
    // cyclic LU (SolveZLU_REAL): forward with the last row's spike sum, then backward
    const int n = p.nsolve;
    double ym = stagg_rhs(p.rows, 0, f, zs);
    y[0] = ym;
    double s1 = __ldg(F + 1) * ym;
    for (int k = 1; k < n - 1; ++k) {
        const double yk = stagg_rhs(p.rows, k, f, zs) - __ldg(F + 5 * k) * ym;
        s1 = s1 + __ldg(F + 5 * k + 1) * yk;
        y[(long long)k * zs] = yk;
        ym = yk;
    }
    double yn = stagg_rhs(p.rows, n - 1, f, zs) - s1;
    yn = yn * __ldg(F + 5 * (n - 1) + 2);
    y[(long long)(n - 1) * zs] = yn;
    double nxt = ym * __ldg(F + 5 * (n - 2) + 2) - yn * __ldg(F + 5 * (n - 2) + 4);
    y[(long long)(n - 2) * zs] = nxt;
    for (int k = n - 3; k >= 0; --k) {
        nxt = y[(long long)k * zs] * __ldg(F + 5 * k + 2) - nxt * __ldg(F + 5 * k + 3) - yn * __ldg(F + 5 * k + 4);
        y[(long long)k * zs] = nxt;
    }
    if (p.copy_first) y[(long long)(p.nout - 1) * zs] = nxt;
}

void free_ops(pado_stagg_s *h)
{
    for (auto &o : h->ops) {
        if (o.d_rows) cudaFree(o.d_rows);
        if (o.d_fac) cudaFree(o.d_fac);
        o.d_rows = nullptr;
        o.d_fac = nullptr;
    }
}

int upload(pado_stagg_s *h)
{
    for (auto &o : h->ops) {
        if (!o.valid) continue;
        cudaError_t e = cudaMalloc(&o.d_rows, o.rows.size() * sizeof(SRow));
        if (e == cudaSuccess) e = cudaMalloc(&o.d_fac, o.fac.size() * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMemcpy(o.d_rows, o.rows.data(), o.rows.size() * sizeof(SRow), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(o.d_fac, o.fac.data(), o.fac.size() * sizeof(double), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            free_ops(h);
            return pado::cuda_fail(e);
        }
    }
    return PADO_OK;
}

int create(pado_stagg_t *out, int nx, double dx, int periodic, int top_even, int bot_even, int top_sided,
           int bot_sided)
{
    if (!out) return PADO_E_NULL;
    *out = nullptr;
    if (nx <= 4) return PADO_STAGG_E_SHORT;  // cd06stagg.F90:183-185, 216-218
    if (!(dx > 0.0) && !(dx < 0.0)) return PADO_E_ARG;
    pado_stagg_s *h = new (std::nothrow) pado_stagg_s;
    if (!h) return PADO_E_NOMEM;
    h->n = nx;
    h->dx = dx;
    h->periodic = periodic != 0;
    h->top_even = top_even != 0;
    h->bot_even = bot_even != 0;
    h->top_sided = top_sided != 0;
    h->bot_sided = bot_sided != 0;
    cudaGetDevice(&h->device);
    if (h->periodic) build_periodic(h);
    else build_nonperiodic(h);
    const int rc = upload(h);
    if (rc != PADO_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return PADO_OK;
}

}  // namespace

extern "C" {

int pado_cd06stagg_init_periodic(pado_stagg_t *stagg, int nx, double dx)
{
    return create(stagg, nx, dx, 1, 1, 1, 0, 0);
}

int pado_cd06stagg_init_nonperiodic(pado_stagg_t *stagg, int nx, double dx, int is_top_even, int is_bot_even,
                                    int is_top_sided, int is_bot_sided)
{
    return create(stagg, nx, dx, 0, is_top_even, is_bot_even, is_top_sided, is_bot_sided);
}

void pado_cd06stagg_destroy(pado_stagg_t stagg)
{
    if (!stagg) return;
    free_ops(stagg);
    delete stagg;
}

int pado_cd06stagg_sizes(pado_stagg_t stagg, int op, int *nin, int *nout)
{
    if (!stagg || !nin || !nout) return PADO_E_NULL;
    if (op < 0 || op >= PADO_STAGG_NOPS) return PADO_E_ARG;
    const StaggOp &o = stagg->ops[op];
    if (!o.valid) return PADO_E_UNSUPPORTED;
    *nin = o.nin;
    *nout = o.nout;
    return PADO_OK;
}

int pado_cd06stagg_apply(pado_stagg_t stagg, int op, const double *f, double *df, long n1, long n2, void *stream)
{
    if (!stagg) return PADO_E_NULL;
    if (op < 0 || op >= PADO_STAGG_NOPS || n1 < 0 || n2 < 0) return PADO_E_ARG;
    const StaggOp &o = stagg->ops[op];
    if (!o.valid) return PADO_E_UNSUPPORTED;
    const long long lines = (long long)n1 * n2;
    if (lines == 0) return PADO_OK;
    if (!f || !df) return PADO_E_NULL;
    const long long in_total = lines * o.nin, out_total = lines * o.nout;
    if (f < df + out_total && df < f + in_total) return PADO_E_ALIAS;
    StaggLaunch p;
    p.in = f;
    p.out = df;
    p.nlines = lines;
    p.zs = lines;
    p.nout = o.nout;
    p.nsolve = o.nsolve;
    p.periodic = o.periodic;
    p.copy_first = o.copy_first;
    p.rows = o.d_rows;
    p.fac = o.d_fac;
    const long long blocks = (lines + 255) / 256;
    if (blocks > 0x7fffffffLL) return PADO_E_SIZE;
    stagg_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p);
    pado::g_launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : pado::cuda_fail(e);
}

}  // extern "C"

// pado_tables.cpp -- host-side solver tables (see pado_tables.h).
#include "pado_tables.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

namespace pado {

namespace {

// Column-major (n, ncol) table with the reference's 1-based (row, col) access.
struct Tab {
    int n, ncol;
    std::vector<double> v;
    Tab(int n_, int ncol_) : n(n_), ncol(ncol_), v((size_t)n_ * ncol_, 0.0) {}
    double &operator()(int i, int c) { return v[(size_t)(i - 1) + (size_t)n * (c - 1)]; }
};

}  // namespace

// Bordered cyclic-tridiagonal LU with fixed bands (b, d, a) -- cd06.F90:221-262.
// Columns: 1 sub-diagonal of L, 2 last-row spike of L, 3 inverse pivots,
// 4 super-diagonal times inverse pivot, 5 last-column spike times inverse pivot.
std::vector<double> cd06_cyclic_lu(int n, double b, double d, double a)
{
    Tab L(n, 5);
    std::vector<double> c(n + 1), v(n + 1, 0.0), h(n + 1, 0.0);
    c[1] = d;
    v[1] = b;
    h[1] = a / c[1];
    for (int i = 2; i <= n - 1; ++i) c[i] = d - (b / c[i - 1]) * a;
    for (int i = 2; i <= n - 2; ++i) {
        v[i] = -(b / c[i - 1]) * v[i - 1];
        h[i] = -(a / c[i]) * h[i - 1];
    }
    v[n - 1] = a - (b / c[n - 2]) * v[n - 2];
    h[n - 1] = (b - h[n - 2] * a) / c[n - 1];
    double acc = 0.0;
    for (int i = 1; i <= n - 1; ++i) acc += h[i] * v[i];
    c[n] = d - acc;
    for (int i = 2; i <= n - 1; ++i) L(i, 1) = b / c[i - 1];
    for (int i = 1; i <= n; ++i) {
        const double inv = 1.0 / c[i];
        L(i, 2) = h[i];
        L(i, 3) = inv;
        L(i, 4) = (i <= n - 2 ? a : 0.0) * inv;
        L(i, 5) = v[i] * inv;
    }
    return L.v;
}

// Thomas factors of the bounded cd06 system with the one-sided closures of
// Lele (1992) -- cd06.F90:264-327.  Columns: a*den, den, cp.
std::vector<double> cd06_tri1(int n, int bc1, int bcn)
{
    const Cd06Const k;
    std::vector<double> a(n + 1, k.alpha_hat), b(n + 1, 1.0), c(n + 1, k.alpha_hat), cp(n + 1, 0.0),
        den(n + 1, 0.0);
    if (bc1 == 0) {
        a[1] = k.w1 * 0.0; a[2] = k.w2 * k.alpha_p; a[3] = k.w3 * k.alpha_pp;
        b[1] = k.w1 * 1.0; b[2] = k.w2 * 1.0; b[3] = k.w3 * 1.0;
        c[1] = k.w1 * k.alpha; c[2] = k.w2 * k.alpha_p; c[3] = k.w3 * k.alpha_pp;
    }  // other bc1 values keep the interior bands, as the reference does ("Incomplete")
    if (bcn == 0) {
        c[n] = k.w1 * 0.0; c[n - 1] = k.w2 * k.alpha_p; c[n - 2] = k.w3 * k.alpha_pp;
        b[n] = k.w1 * 1.0; b[n - 1] = k.w2 * 1.0; b[n - 2] = k.w3 * 1.0;
        a[n] = k.w1 * k.alpha; a[n - 1] = k.w2 * k.alpha_p; a[n - 2] = k.w3 * k.alpha_pp;
    }
    cp[1] = c[1] / b[1];
    for (int i = 2; i <= n - 1; ++i) cp[i] = c[i] / (b[i] - a[i] * cp[i - 1]);
    den[1] = 1.0 / b[1];
    for (int i = 2; i <= n; ++i) den[i] = 1.0 / (b[i] - a[i] * cp[i - 1]);
    Tab T(n, 3);
    for (int i = 1; i <= n; ++i) {
        T(i, 1) = a[i] * den[i];
        T(i, 2) = den[i];
        T(i, 3) = cp[i];  // cp(n) is never read by the solve
    }
    return T.v;
}

// Bordered cyclic-pentadiagonal LU (Neossi Nguetchue & Abelman 2008) with
// bands (e, a, d, c, f) -- cd10.F90:351-427 / cf90.F90:198-274.
// Columns: 1 b, 2 e/g(i-2), 3 k, 4 l, 5 1/g, 6 h, 7 f, 8 v, 9 w.
std::vector<double> penta_cyclic_lu(int n, double e, double a, double d, double c, double f)
{
    std::vector<double> b(n + 1, 0.0), k(n + 1, 0.0), l(n + 1, 0.0), g(n + 1, 0.0), h(n + 1, 0.0),
        v(n + 1, 0.0), w(n + 1, 0.0);
    g[1] = d;
    b[2] = a / g[1];
    h[1] = c;
    k[1] = f / g[1];
    w[1] = a;
    v[1] = e;
    l[1] = c / g[1];
    g[2] = d - b[2] * h[1];
    k[2] = -k[1] * h[1] / g[2];
    w[2] = e - b[2] * w[1];
    v[2] = -b[2] * v[1];
    l[2] = (f - l[1] * h[1]) / g[2];
    h[2] = c - b[2] * f;
    for (int i = 3; i <= n - 3; ++i) {
        const double eg = e / g[i - 2];
        b[i] = (a - eg * h[i - 2]) / g[i - 1];
        h[i] = c - b[i] * f;
        g[i] = d - eg * f - b[i] * h[i - 1];
    }
    b[n - 2] = (a - (e / g[n - 4]) * h[n - 4]) / g[n - 3];
    g[n - 2] = d - (e / g[n - 4]) * f - b[n - 2] * h[n - 3];
    for (int i = 3; i <= n - 4; ++i) {
        k[i] = -(k[i - 2] * f + k[i - 1] * h[i - 1]) / g[i];
        v[i] = -(e / g[i - 2]) * v[i - 2] - b[i] * v[i - 1];
    }
    k[n - 3] = (e - k[n - 5] * f - k[n - 4] * h[n - 4]) / g[n - 3];
    k[n - 2] = (a - k[n - 4] * f - k[n - 3] * h[n - 3]) / g[n - 2];
    v[n - 3] = f - (e / g[n - 5]) * v[n - 5] - b[n - 3] * v[n - 4];
    v[n - 2] = c - (e / g[n - 4]) * v[n - 4] - b[n - 2] * v[n - 3];
    double acc = 0.0;
    for (int i = 1; i <= n - 2; ++i) acc += k[i] * v[i];
    g[n - 1] = d - acc;
    for (int i = 3; i <= n - 3; ++i) {
        w[i] = -(e / g[i - 2]) * w[i - 2] - b[i] * w[i - 1];
        l[i] = -(l[i - 2] * f + l[i - 1] * h[i - 1]) / g[i];
    }
    w[n - 2] = f - (e / g[n - 4]) * w[n - 4] - b[n - 2] * w[n - 3];
    acc = 0.0;
    for (int i = 1; i <= n - 2; ++i) acc += k[i] * w[i];
    w[n - 1] = c - acc;
    l[n - 2] = (e - l[n - 4] * f - l[n - 3] * h[n - 3]) / g[n - 2];
    acc = 0.0;
    for (int i = 1; i <= n - 2; ++i) acc += l[i] * v[i];
    l[n - 1] = (a - acc) / g[n - 1];
    acc = 0.0;
    for (int i = 1; i <= n - 1; ++i) acc += l[i] * w[i];
    g[n] = d - acc;
    Tab T(n, 9);
    for (int i = 1; i <= n; ++i) {
        T(i, 1) = b[i];
        T(i, 2) = (i >= 3 && i <= n - 2) ? e / g[i - 2] : 0.0;
        T(i, 3) = k[i];
        T(i, 4) = l[i];
        T(i, 6) = h[i];
        T(i, 7) = (i <= n - 4) ? f : 0.0;
        T(i, 8) = v[i];
        T(i, 9) = w[i];
    }
    for (int i = 1; i <= n; ++i) T(i, 5) = 1.0 / g[i];
    return T.v;
}

// Bands (bt, b, d, a, at) of a bounded pentadiagonal system with the
// reference's closures, factorised without pivoting.
// cd10.F90:429-578 (ComputePenta1), :580-709 (ComputePenta2), cf90.F90:276-418.
// Columns: 1 bt, 2 b, 3 d, 4 a, 5 at, 6 e, 7 1/pivot, 8 f, 9 g, 10 e/pivot.
std::vector<double> penta_bounded(int scheme, int kind, int n, int bc1, int bcn)
{
    Tab P(n, 11);
    auto set = [&](int i, double bt, double b, double d, double a, double at) {
        P(i, 1) = bt; P(i, 2) = b; P(i, 3) = d; P(i, 4) = a; P(i, 5) = at;
    };
    if (scheme == CD10 && kind == D1) {
        const Cd10Const k;
        const double ah = k.alpha_hat, bh = k.beta_hat;
        for (int i = 1; i <= n; ++i) set(i, bh, ah, 1.0, ah, bh);
        // one-sided closure rows 1..4 (weights w1..w4), mirrored at the far end
        const double W[4] = {k.w1, k.w2, k.w3, k.w4};
        const double R[4][5] = {{0.0, 0.0, 1.0, k.alpha, 0.0},
                                {0.0, k.alpha_p, 1.0, k.alpha_p, 0.0},
                                {k.beta_pp, k.alpha_pp, 1.0, k.alpha_pp, k.beta_pp},
                                {k.beta_ppp, k.alpha_ppp, 1.0, k.alpha_ppp, k.beta_ppp}};
        if (bc1 == 0) {
            for (int r = 0; r < 4; ++r)
                set(r + 1, W[r] * R[r][0], W[r] * R[r][1], W[r] * R[r][2], W[r] * R[r][3], W[r] * R[r][4]);
        } else if (bc1 == 1) {
            set(1, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(2, 0.0, ah, 1.0 - bh, ah, bh);
        } else if (bc1 == -1) {
            set(1, 0.0, 0.0, 1.0, 2.0 * ah, 2.0 * bh);
            set(2, 0.0, ah, 1.0 + bh, ah, bh);
        }
        if (bcn == 0) {
            for (int r = 0; r < 4; ++r)
                set(n - r, W[r] * R[r][4], W[r] * R[r][3], W[r] * R[r][2], W[r] * R[r][1], W[r] * R[r][0]);
        } else if (bcn == 1) {
            set(n, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(n - 1, bh, ah, 1.0 - bh, ah, 0.0);
        } else if (bcn == -1) {
            set(n, 2.0 * bh, 2.0 * ah, 1.0, 0.0, 0.0);
            set(n - 1, bh, ah, 1.0 + bh, ah, 0.0);
        }
    } else if (scheme == CD10) {
        const Cd10Const k;
        const double al = k.alpha10d2, be = k.beta10d2;
        for (int i = 1; i <= n; ++i) set(i, be, al, 1.0, al, be);
        if (bc1 == 0) {
            set(1, 0.0, 0.0, 1.0, k.b1_alpha, 0.0);
            set(2, 0.0, k.b2_alpha, 1.0, k.b2_alpha, 0.0);
            set(3, k.b3_beta, k.b3_alpha, 1.0, k.b3_alpha, k.b3_beta);
        } else if (bc1 == 1) {
            set(1, 0.0, 0.0, 1.0, 2.0 * al, 2.0 * be);
            set(2, 0.0, al, 1.0 + be, al, be);
        } else if (bc1 == -1) {
            set(1, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(2, 0.0, al, 1.0 - be, al, be);
        }
        if (bcn == 0) {
            set(n - 2, k.b3_beta, k.b3_alpha, 1.0, k.b3_alpha, k.b3_beta);
            set(n - 1, 0.0, k.b2_alpha, 1.0, k.b2_alpha, 0.0);
            set(n, 0.0, k.b1_alpha, 1.0, 0.0, 0.0);
        } else if (bcn == 1) {
            set(n - 1, be, al, 1.0 + be, al, 0.0);
            set(n, 2.0 * be, 2.0 * al, 1.0, 0.0, 0.0);
        } else if (bcn == -1) {
            set(n - 1, be, al, 1.0 - be, al, 0.0);
            set(n, 0.0, 0.0, 1.0, 0.0, 0.0);
        }
    } else {
        const Cf90Const k;
        const double al = k.alpha, be = k.beta;
        for (int i = 1; i <= n; ++i) set(i, be, al, 1.0, al, be);
        if (bc1 == 0) {
            set(1, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(2, 0.0, k.b2_alpha, 1.0, k.b2_alpha, 0.0);
            set(3, k.b3_beta, k.b3_alpha, 1.0, k.b3_alpha, k.b3_beta);
            set(4, k.b4_beta, k.b4_alpha, 1.0, k.b4_alpha, k.b4_beta);
        } else if (bc1 == 1) {
            set(1, 0.0, 0.0, 1.0, 2.0 * al, 2.0 * be);
            set(2, 0.0, al, 1.0 + be, al, be);
        } else if (bc1 == -1) {
            set(1, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(2, 0.0, al, 1.0 - be, al, be);
        }
        if (bcn == 0) {
            set(n, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(n - 1, 0.0, k.b2_alpha, 1.0, k.b2_alpha, 0.0);
            set(n - 2, k.b3_beta, k.b3_alpha, 1.0, k.b3_alpha, k.b3_beta);
            set(n - 3, k.b4_beta, k.b4_alpha, 1.0, k.b4_alpha, k.b4_beta);
        } else if (bcn == 1) {
            set(n, 2.0 * be, 2.0 * al, 1.0, 0.0, 0.0);
            set(n - 1, be, al, 1.0 + be, al, 0.0);
        } else if (bcn == -1) {
            set(n, 0.0, 0.0, 1.0, 0.0, 0.0);
            set(n - 1, be, al, 1.0 - be, al, 0.0);
        }
    }
    // Factorisation (cd10.F90:558-575).
    P(1, 7) = 1.0 / P(1, 3);
    P(2, 7) = 1.0 / (P(2, 3) - P(2, 2) * P(1, 4) * P(1, 7));
    P(1, 6) = P(1, 4);
    P(2, 8) = P(2, 2) * P(1, 7);
    for (int i = 3; i <= n; ++i) {
        P(i, 9) = P(i, 1) * P(i - 2, 7);
        P(i - 1, 6) = P(i - 1, 4) - P(i - 1, 8) * P(i - 2, 5);
        P(i, 8) = (P(i, 2) - P(i, 9) * P(i - 2, 6)) * P(i - 1, 7);
        P(i, 7) = 1.0 / (P(i, 3) - P(i, 8) * P(i - 1, 6) - P(i, 9) * P(i - 2, 5));
    }
    for (int i = 1; i <= n; ++i) P(i, 10) = P(i, 6) * P(i, 7);
    return P.v;
}

static Sweep make_sweep(int n, int nb)
{
    Sweep s;
    s.n = n;
    s.nb = nb;
    s.nbord = n - nb;
    for (auto *v : {&s.alpha, &s.c1, &s.c2, &s.k1, &s.k2, &s.gamma, &s.d1, &s.d2, &s.e1, &s.e2, &s.delta})
        v->assign(nb, 0.0);
    std::fill(s.alpha.begin(), s.alpha.end(), 1.0);
    std::fill(s.delta.begin(), s.delta.end(), 1.0);
    return s;
}

Sweep primal_sweep(int scheme, int kind, int n, int periodic, int bc1, int bcn)
{
    if (scheme == CD06 && periodic) {
        // cd06.F90:345-373: forward over rows 1..n-1 with one running sum,
        // border row n, backward with the last-column spike.
        const Cd06Const k;
        Tab L(n, 5);
        L.v = cd06_cyclic_lu(n, k.alpha06d1, 1.0, k.alpha06d1);
        Sweep s = make_sweep(n, n - 1);
        for (int i = 0; i < n - 1; ++i) {
            s.c1[i] = L(i + 1, 1);
            s.k1[i] = L(i + 1, 2);
            s.gamma[i] = L(i + 1, 3);
            s.d1[i] = L(i + 1, 4);
            s.e1[i] = L(i + 1, 5);
        }
        s.mb[0] = L(n, 3);
        return s;
    }
    if (scheme == CD06) {
        // cd06.F90:432-452: scaled forward sweep, unit backward sweep.
        Tab T(n, 3);
        T.v = cd06_tri1(n, bc1, bcn);
        Sweep s = make_sweep(n, n);
        for (int i = 0; i < n; ++i) {
            s.alpha[i] = T(i + 1, 2);
            s.c1[i] = i > 0 ? T(i + 1, 1) : 0.0;
            s.gamma[i] = 1.0;
            s.d1[i] = i < n - 1 ? T(i + 1, 3) : 0.0;
        }
        return s;
    }
    if (periodic) {
        // cd10.F90:712-749 / cf90.F90:421-458: forward over rows 1..n-2 with two
        // running sums, border rows n-1 and n, backward with two spike columns.
        Tab L(n, 9);
        if (scheme == CD10) {
            const Cd10Const k;
            if (kind == D1) L.v = penta_cyclic_lu(n, k.beta10d1, k.alpha10d1, 1.0, k.alpha10d1, k.beta10d1);
            else L.v = penta_cyclic_lu(n, k.beta10d2, k.alpha10d2, 1.0, k.alpha10d2, k.beta10d2);
        } else {
            const Cf90Const k;
            L.v = penta_cyclic_lu(n, k.beta, k.alpha, 1.0, k.alpha, k.beta);
        }
        Sweep s = make_sweep(n, n - 2);
        for (int i = 0; i < n - 2; ++i) {
            const double g = L(i + 1, 5);
            s.c1[i] = L(i + 1, 1);
            s.c2[i] = L(i + 1, 2);
            s.k1[i] = L(i + 1, 3);
            s.k2[i] = L(i + 1, 4);
            s.gamma[i] = g;
            s.d1[i] = L(i + 1, 6) * g;
            s.d2[i] = L(i + 1, 7) * g;
            s.e1[i] = L(i + 1, 8) * g;
            s.e2[i] = L(i + 1, 9) * g;
        }
        // Border (rows n-1, n): u = r_border - sums;
        //   y1 = u0;  x2 = (u1 - l(n-1) y1) / g(n);  x1 = (y1 - w(n-1) x2) / g(n-1).
        const double g1 = L(n - 1, 5), gn = L(n, 5), wv = L(n - 1, 9), lv = L(n - 1, 4);
        s.mb[0] = g1 + g1 * wv * gn * lv;
        s.mb[1] = -g1 * wv * gn;
        s.mb[2] = -gn * lv;
        s.mb[3] = gn;
        return s;
    }
    // Bounded penta: cd10.F90:823-851 / cf90.F90:532-558.
    Tab P(n, 11);
    P.v = penta_bounded(scheme, kind, n, bc1, bcn);
    Sweep s = make_sweep(n, n);
    for (int i = 0; i < n; ++i) {
        const int r = i + 1;
        s.c1[i] = i >= 1 ? P(r, 8) : 0.0;
        s.c2[i] = i >= 2 ? P(r, 9) : 0.0;
        s.gamma[i] = P(r, 7);
        s.d1[i] = i <= n - 2 ? P(r, 10) : 0.0;
        s.d2[i] = i <= n - 3 ? P(r, 5) * P(r, 7) : 0.0;
    }
    return s;
}

// Transposed sweep.  The forward recurrence of A^{-T} runs the primal
// backward coefficients shifted by their lag, and vice versa; sums and
// broadcast border terms swap roles; the border map is transposed.
Sweep adjoint_sweep(const Sweep &p)
{
    Sweep a = make_sweep(p.n, p.nb);
    const int nb = p.nb;
    for (int i = 0; i < nb; ++i) {
        a.alpha[i] = 1.0;
        a.c1[i] = i >= 1 ? p.d1[i - 1] : 0.0;
        a.c2[i] = i >= 2 ? p.d2[i - 2] : 0.0;
        a.k1[i] = p.e1[i];
        a.k2[i] = p.e2[i];
        a.gamma[i] = p.gamma[i];
        a.d1[i] = i + 1 < nb ? p.c1[i + 1] : 0.0;
        a.d2[i] = i + 2 < nb ? p.c2[i + 2] : 0.0;
        a.e1[i] = p.k1[i];
        a.e2[i] = p.k2[i];
        a.delta[i] = p.alpha[i];
    }
    if (p.nbord == 1) {
        a.mb[0] = p.mb[0];
    } else if (p.nbord == 2) {
        a.mb[0] = p.mb[0];
        a.mb[1] = p.mb[2];
        a.mb[2] = p.mb[1];
        a.mb[3] = p.mb[3];
    }
    return a;
}

Layout make_layout(int n, int m, int i0, int i1, int e_rows)
{
    Layout L;
    L.n = n;
    auto uniform = [&](int S) {
        L.S = std::max(1, std::min(S, n));
        L.st.assign(L.S + 1, 0);
        for (int s = 0; s <= L.S; ++s) L.st[s] = (int)((long long)n * s / L.S);
    };
    const int A0 = std::max(i0, HALO), B = std::min(i1, n - HALO);
    const int kmax = (i0 < i1 && B > A0) ? (B - A0) / m : 0;
    if (kmax < 1 || m < 8) {
        uniform((n + m - 1) / m);
        return L;
    }
    // Lines whose length is a multiple of E (e_rows, else m/2): pieces of
    // exactly E rows before and after the interior block, which the kernels
    // run on a fully unrolled per-row-table path (about as fast per row as
    // the interior); the block of k interior segments starts at a whole
    // number of pieces (one interior segment fewer where the rounding needs it).
    const int E = e_rows > 0 ? e_rows : m / 2;
    if (n % E == 0) {
        const int A = (A0 + E - 1) / E * E;
        for (int k = kmax; k >= std::max(1, kmax - 1); --k) {
            if (A + k * m > B) continue;
            std::vector<int> st;
            for (int r = 0; r < A; r += E) st.push_back(r);
            for (int j = 0; j < k; ++j) st.push_back(A + j * m);
            for (int r = A + k * m; r < n; r += E) st.push_back(r);
            st.push_back(n);
            if ((int)st.size() - 1 > MAX_SEGMENTS) break;
            L.st = st;
            L.S = (int)st.size() - 1;
            return L;
        }
    }
    // otherwise pieces of about m/3 rows (near-equal), on the generic per-row
    // loop, several times slower per row than the interior: short pieces keep
    // every thread of a tile near an interior segment's time
    int k = kmax;
    int e = std::max(4, (m + 2) / 3);
    auto pieces = [](int rows, int e_) { return rows <= 0 ? 0 : (rows + e_ - 1) / e_; };
    for (;;) {
        const int right = n - (A0 + k * m);
        const int S = k + pieces(A0, e) + pieces(right, e);
        if (S <= MAX_SEGMENTS) break;
        if (e < m) ++e;
        else if (k > 1) --k;
        else {
            uniform((n + m - 1) / m);
            return L;
        }
    }
    L.st.clear();
    auto cut = [&](int lo, int hi) {  // near-equal pieces of [lo, hi)
        const int np = pieces(hi - lo, e);
        for (int j = 0; j < np; ++j) L.st.push_back(lo + (int)((long long)(hi - lo) * j / np));
    };
    cut(0, A0);
    for (int j = 0; j < k; ++j) L.st.push_back(A0 + j * m);
    cut(A0 + k * m, n);
    L.st.push_back(n);
    L.S = (int)L.st.size() - 1;
    return L;
}

void interior_range(const Sweep &sw, int *i0, int *i1)
{
    *i0 = *i1 = 0;
    const int nb = sw.nb;
    if (nb < 16) return;
    const int mid = nb / 2;
    const double ref[7] = {sw.alpha[mid], sw.c1[mid], sw.c2[mid], sw.gamma[mid], sw.d1[mid], sw.d2[mid], sw.delta[mid]};
    // a row is interior when its coefficients equal the line-centre values to
    // 1e-14 relative (they settle to a few ulps); its cyclic spike terms are
    // handled per row (row_spiky)
    auto ok = [&](int i) {
        const double v[7] = {sw.alpha[i], sw.c1[i], sw.c2[i], sw.gamma[i], sw.d1[i], sw.d2[i], sw.delta[i]};
        for (int k = 0; k < 7; ++k)
            if (std::fabs(v[k] - ref[k]) > 1e-14 * std::fabs(ref[k])) return false;
        return true;
    };
    if (!ok(mid)) return;
    int a = mid, b = mid + 1;
    while (a > 0 && ok(a - 1)) --a;
    while (b < nb && ok(b)) ++b;
    *i0 = a;
    *i1 = b;
}

void build_device_table(const Sweep &sw, const Layout &lay, std::vector<double> &tab, std::vector<double> &segsum)
{
    const int nb = sw.nb;
    tab.assign((size_t)nb * T_NF, 0.0);
    segsum.assign((size_t)lay.S * 4, 0.0);
    auto T = [&](int i, int f) -> double & { return tab[(size_t)i * T_NF + f]; };
    for (int i = 0; i < nb; ++i) {
        T(i, T_C1) = sw.c1[i];
        T(i, T_C2) = sw.c2[i];
        T(i, T_ALPHA) = sw.alpha[i];
        T(i, T_K1) = sw.k1[i];
        T(i, T_K2) = sw.k2[i];
        T(i, T_GAMMA) = sw.gamma[i];
        T(i, T_D1) = sw.d1[i];
        T(i, T_D2) = sw.d2[i];
        T(i, T_E1) = sw.e1[i];
        T(i, T_E2) = sw.e2[i];
        T(i, T_DELTA) = sw.delta[i];
    }
    for (int s = 0; s < lay.S; ++s) {
        const int a = lay.start(s);
        const int b = std::min(lay.start(s) + lay.len(s), nb);  // banded end
        if (s > 0) {
            // forward responses to a unit incoming state (z_{a-1}, z_{a-2})
            for (int which = 0; which < 2; ++which) {
                double zm1 = which == 0 ? 1.0 : 0.0, zm2 = which == 0 ? 0.0 : 1.0;
                double ks1 = 0.0, ks2 = 0.0;
                for (int i = a; i < b; ++i) {
                    const double z = -sw.c1[i] * zm1 - sw.c2[i] * zm2;
                    T(i, which == 0 ? T_U : T_V) = z;
                    ks1 += sw.k1[i] * z;
                    ks2 += sw.k2[i] * z;
                    zm2 = zm1;
                    zm1 = z;
                }
                segsum[(size_t)s * 4 + (which == 0 ? 0 : 1)] = ks1;
                segsum[(size_t)s * 4 + (which == 0 ? 2 : 3)] = ks2;
            }
        }
        if (s < lay.S - 1) {
            // backward responses to a unit incoming state (x_b, x_{b+1})
            for (int which = 0; which < 2; ++which) {
                double xp1 = which == 0 ? 1.0 : 0.0, xp2 = which == 0 ? 0.0 : 1.0;
                for (int i = b - 1; i >= a; --i) {
                    const double x = -sw.d1[i] * xp1 - sw.d2[i] * xp2;
                    T(i, which == 0 ? T_S : T_T) = x;
                    xp2 = xp1;
                    xp1 = x;
                }
            }
        }
    }
}

Interior interior_info(const Sweep &sw, const Layout &lay, int m)
{
    Interior in;
    int i0, i1;
    interior_range(sw, &i0, &i1);
    if (i0 >= i1) return in;
    const int mid = sw.nb / 2;
    const double ref[7] = {sw.alpha[mid], sw.c1[mid], sw.c2[mid], sw.gamma[mid], sw.d1[mid], sw.d2[mid], sw.delta[mid]};
    in.i0 = i0;
    in.i1 = i1;
    for (int k = 0; k < 7; ++k) in.kc[k] = ref[k];
    const double c1 = ref[1], c2 = ref[2], d1 = ref[4], d2 = ref[5];
    if (m > MAXM) return in;
    // unit responses of a length-m segment under the constant recurrences
    double z1 = 1.0, z2 = 0.0, y1 = 0.0, y2 = 1.0;
    for (int t = 0; t < m; ++t) {
        const double z = -c1 * z1 - c2 * z2, y = -c1 * y1 - c2 * y2;
        in.pu[t] = z;
        in.pv[t] = y;
        z2 = z1; z1 = z; y2 = y1; y1 = y;
    }
    double x1 = 1.0, x2 = 0.0, w1 = 0.0, w2 = 1.0;
    for (int t = m - 1; t >= 0; --t) {
        const double x = -d1 * x1 - d2 * x2, w = -d1 * w1 - d2 * w2;
        in.ps[t] = x;
        in.pt[t] = w;
        x2 = x1; x1 = x; w2 = w1; w1 = w;
    }
    // cyclic spike terms below 1e-17 of their largest magnitude contribute far
    // below one rounding of the sums they enter; rows above that keep them
    double kmax = 0.0, emax = 0.0;
    for (int i = 0; i < sw.nb; ++i) {
        kmax = std::max({kmax, std::fabs(sw.k1[i]), std::fabs(sw.k2[i])});
        emax = std::max({emax, std::fabs(sw.e1[i]), std::fabs(sw.e2[i])});
    }
    auto spiky = [&](int i) {
        return std::fabs(sw.k1[i]) > 1e-17 * kmax || std::fabs(sw.k2[i]) > 1e-17 * kmax ||
               std::fabs(sw.e1[i]) > 1e-17 * emax || std::fabs(sw.e2[i]) > 1e-17 * emax;
    };
    for (int s = 1; s + 1 < lay.S && s < 32; ++s) {
        const int a = lay.start(s), len = lay.len(s);
        if (len == m && a >= i0 && a + len <= i1 && a >= HALO && a + len + HALO <= sw.n) {
            in.mask |= 1u << s;
            for (int i = a; i < a + len; ++i)
                if (spiky(i)) in.spk_mask |= 1u << s;
        }
    }
    return in;
}

ChainTables chain_tables(const std::vector<double> &tab, const std::vector<double> &segsum, const Layout &lay, int nb,
                         const Interior &in, int m)
{
    const int S = lay.S;
    auto T = [&](int i, int f) { return tab[(size_t)i * T_NF + f]; };
    // per-segment transfers
    std::vector<std::array<double, 4>> A(S, {0, 0, 0, 0}), B(S, {0, 0, 0, 0});
    for (int s = 0; s < S; ++s) {
        const bool fast = (in.mask >> s) & 1u;
        const int a = lay.start(s);
        if (s + 1 < S) {
            const int b = lay.start(s + 1);  // segments before the last are fully banded
            A[s] = {fast ? in.pu[m - 1] : T(b - 1, T_U), fast ? in.pv[m - 1] : T(b - 1, T_V),
                    fast ? in.pu[m - 2] : T(b - 2, T_U), fast ? in.pv[m - 2] : T(b - 2, T_V)};
        }
        if (s > 0) {
            B[s] = {fast ? in.ps[0] : T(a, T_S), fast ? in.pt[0] : T(a, T_T),
                    fast ? in.ps[1] : (a + 1 < nb ? T(a + 1, T_S) : 0.0),
                    fast ? in.pt[1] : (a + 1 < nb ? T(a + 1, T_T) : 0.0)};
        }
    }
    auto mul = [](const std::array<double, 4> &x, const std::array<double, 4> &y) {
        return std::array<double, 4>{x[0] * y[0] + x[1] * y[2], x[0] * y[1] + x[1] * y[3],
                                     x[2] * y[0] + x[3] * y[2], x[2] * y[1] + x[3] * y[3]};
    };
    auto norm = [](const std::array<double, 4> &x) {
        return std::max({std::fabs(x[0]), std::fabs(x[1]), std::fabs(x[2]), std::fabs(x[3])});
    };
    const std::array<double, 4> I = {1, 0, 0, 1};
    // phi[s][j], psi[s][j] for all pairs (S <= 32)
    std::vector<std::array<double, 4>> phi((size_t)S * S, {0, 0, 0, 0}), psi((size_t)S * S, {0, 0, 0, 0});
    for (int s = 0; s < S; ++s) {
        std::array<double, 4> M_ = I;
        for (int j = s - 1; j >= 0; --j) {  // Phi(s, j) = Phi(s, j+1) A_{j+1}
            if (j < s - 1) M_ = mul(M_, A[j + 1]);
            phi[(size_t)s * S + j] = M_;
        }
        M_ = I;
        for (int j = s + 1; j < S; ++j) {  // Psi(s, j) = Psi(s, j-1) B_{j-1}
            if (j > s + 1) M_ = mul(M_, B[j - 1]);
            psi[(size_t)s * S + j] = M_;
        }
    }
    ChainTables ct;
    int W = 0;
    for (int s = 0; s < S; ++s) {
        int wf = 0, wb = 0;
        for (int j = 0; j < S; ++j) {
            if (j < s && norm(phi[(size_t)s * S + j]) >= XFER_DROP) wf = std::max(wf, s - j);
            if (j > s && norm(psi[(size_t)s * S + j]) >= XFER_DROP) wb = std::max(wb, j - s);
        }
        ct.wf[s] = (unsigned char)wf;
        ct.wb[s] = (unsigned char)wb;
        W = std::max({W, wf, wb});
    }
    ct.W = W;
    ct.xtab.clear();
    for (int s = 0; s < S; ++s) {
        ct.xof[s] = (unsigned short)(ct.xtab.size() / 4);
        for (int d = 1; d <= ct.wf[s]; ++d) {
            const auto &p = phi[(size_t)s * S + (s - d)];
            for (int k = 0; k < 4; ++k) ct.xtab.push_back(norm(p) >= XFER_DROP ? p[k] : 0.0);
        }
    }
    for (int s = 0; s < S; ++s) {
        ct.xob[s] = (unsigned short)(ct.xtab.size() / 4);
        for (int d = 1; d <= ct.wb[s]; ++d) {
            const auto &p = psi[(size_t)s * S + (s + d)];
            for (int k = 0; k < 4; ++k) ct.xtab.push_back(norm(p) >= XFER_DROP ? p[k] : 0.0);
        }
    }
    // border-sum weights (every term kept)
    ct.ctab.assign((size_t)S * CT_NF, 0.0);
    for (int j = 0; j < S; ++j) {
        double g[4] = {0, 0, 0, 0};
        for (int t = j + 1; t < S; ++t) {
            const auto &p = phi[(size_t)t * S + j];
            const double k1u = segsum[(size_t)t * 4 + 0], k1v = segsum[(size_t)t * 4 + 1];
            const double k2u = segsum[(size_t)t * 4 + 2], k2v = segsum[(size_t)t * 4 + 3];
            g[0] += k1u * p[0] + k1v * p[2];
            g[1] += k1u * p[1] + k1v * p[3];
            g[2] += k2u * p[0] + k2v * p[2];
            g[3] += k2u * p[1] + k2v * p[3];
        }
        std::copy(g, g + 4, &ct.ctab[(size_t)j * CT_NF]);
    }
    return ct;
}

void edge_table(const std::vector<double> &tab, const Layout &lay, int nb, unsigned mask, unsigned spk, bool tri,
                std::vector<double> &etab, std::vector<double> &ktab, std::vector<int> &toff)
{
    etab.clear();
    ktab.clear();
    toff.assign(lay.S, 0);
    int rows = 0, krows = 0;
    for (int s = 0; s < lay.S; ++s) {
        const int a = lay.start(s), b = std::min(a + lay.len(s), nb);
        if (!((mask >> s) & 1u)) {
            toff[s] = rows;
            for (int i = a; i < b; ++i, ++rows) {
                const double *r = &tab[(size_t)i * T_NF];
                double e[E_NF];
                e[E_C1] = r[T_C1];
                e[E_C2] = tri ? r[T_DELTA] : r[T_C2];  // E_DELTA for tridiagonal sweeps
                e[E_ALPHA] = r[T_ALPHA];
                e[E_K1] = r[T_K1];
                e[E_K2] = r[T_K2];
                e[E_D2] = r[T_D2];
                e[E_U] = r[T_U];
                e[E_V] = r[T_V];
                e[E_GAMMA] = r[T_GAMMA];
                e[E_D1] = r[T_D1];
                e[E_S] = r[T_S];
                e[E_T] = r[T_T];
                etab.insert(etab.end(), e, e + E_NF);
            }
        } else if ((spk >> s) & 1u) {
            toff[s] = krows;
            for (int i = a; i < b; ++i, ++krows) {
                const double *r = &tab[(size_t)i * T_NF];
                ktab.insert(ktab.end(), {r[T_K1], r[T_K2]});
            }
        }
    }
}

OpTables make_op_tables(int scheme, int kind, int n, double dx, int periodic, int bc1, int bcn, int m, bool adjoint)
{
    OpTables ot;
    const Sweep prim = primal_sweep(scheme, kind, n, periodic, bc1, bcn);
    const Sweep sw = adjoint ? adjoint_sweep(prim) : prim;
    ot.nb = sw.nb;
    ot.nbord = sw.nbord;
    ot.m = m;
    std::memcpy(ot.mb, sw.mb, sizeof(ot.mb));
    ot.rc = make_rhs_coef(scheme, kind, dx, periodic);
    int i0, i1;
    interior_range(sw, &i0, &i1);
    ot.lay = make_layout(n, m, i0, i1, edge_piece_rows(ot.rc.rk, ot.rc.periodic != 0, m));
    std::vector<double> segsum;
    build_device_table(sw, ot.lay, ot.tab, segsum);
    ot.interior = interior_info(sw, ot.lay, m);
    ot.chain = chain_tables(ot.tab, segsum, ot.lay, sw.nb, ot.interior, m);
    ot.chain_exact = chain_tables(ot.tab, segsum, ot.lay, sw.nb, Interior{}, m);
    edge_table(ot.tab, ot.lay, sw.nb, ot.interior.mask, ot.interior.spk_mask, ot.rc.rk == RHS_CD06_D1, ot.etab,
               ot.ktab, ot.toff);
    if (sw.nbord > 0) {
        // backward sweep of the unit spike sources: x_i = -e_i - d1_i x_{i+1} - d2_i x_{i+2}
        const int nb = sw.nb;
        std::vector<double> r1(nb + 2, 0.0), r2(nb + 2, 0.0);
        double rmax = 0.0;
        for (int i = nb - 1; i >= 0; --i) {
            r1[i] = -sw.e1[i] - sw.d1[i] * r1[i + 1] - sw.d2[i] * r1[i + 2];
            r2[i] = -sw.e2[i] - sw.d1[i] * r2[i + 1] - sw.d2[i] * r2[i + 2];
            rmax = std::max({rmax, std::fabs(r1[i]), std::fabs(r2[i])});
        }
        auto big = [&](int i) { return std::fabs(r1[i]) > 1e-17 * rmax || std::fabs(r2[i]) > 1e-17 * rmax; };
        // the longest run of negligible rows splits the line into the two regions
        int best_a = nb, best_b = nb, run_a = -1;
        for (int i = 0; i <= nb; ++i) {
            const bool small = i < nb && !big(i);
            if (small && run_a < 0) run_a = i;
            if (!small && run_a >= 0) {
                if (i - run_a > best_b - best_a) {
                    best_a = run_a;
                    best_b = i;
                }
                run_a = -1;
            }
        }
        ot.ie = best_a;
        ot.je = best_b;
        ot.rtab.clear();
        for (int i = 0; i < nb; ++i)
            if (i < ot.ie || i >= ot.je) ot.rtab.insert(ot.rtab.end(), {r1[i], r2[i]});
    }
    // thread slots: segments on the per-row table first, so that a warp's
    // segments take one path
    int k = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (int s = 0; s < ot.lay.S && s < 32; ++s)
            if ((((ot.interior.mask >> s) & 1u) != 0) == (pass == 1)) ot.sperm[k++] = (unsigned char)s;
    if (adjoint) {
        double taps[9];
        interior_taps(ot.rc, taps);
        for (int k = 0; k < 9; ++k) ot.taps[k] = taps[8 - k];
        if (!periodic) ot.bt = transposed_stencil_blocks(ot.rc, n, bc1, bcn);
    }
    return ot;
}

int warp_slots(const OpTables &ot, int L, unsigned char *sperm, int max_slots, bool border_warp)
{
    const int S = ot.lay.S;
    // code-path classes: per-row table unrolled (pieces of m/2 rows), per-row
    // table loop (other lengths), then the interior with or without spike sums
    // and border responses
    auto cls = [&](int s) {
        const int a = ot.lay.start(s), len = ot.lay.len(s);
        if (!((ot.interior.mask >> s) & 1u)) return len == edge_piece_rows(ot.rc.rk, ot.rc.periodic != 0, ot.m) ? 0 : 1;
        const bool spk = (ot.interior.spk_mask >> s) & 1u;
        const bool resp = ot.nbord > 0 && (a < ot.ie || a + len > ot.je);
        return spk ? (resp ? 2 : 3) : (resp ? 4 : 5);
    };
    const int spw = L >= 32 ? 1 : 32 / L;
    int k = 0;
    if (border_warp && ot.nbord > 0) {
        // a warp of idle slots first: its first slot is the first idle one
        for (int j = 0; j < spw && k < max_slots; ++j) sperm[k++] = 0xff;
    }
    for (int c = 0; c <= 5; ++c) {
        int cnt = 0;
        for (int s = 0; s < S; ++s)
            if (cls(s) == c) {
                if (k >= max_slots) break;
                sperm[k++] = (unsigned char)s;
                ++cnt;
            }
        while (cnt % spw != 0 && k < max_slots) {
            sperm[k++] = 0xff;
            ++cnt;
        }
    }
    int used = 0;
    for (int i = 0; i < k; ++i) used += sperm[i] != 0xff;
    if (used != S) {
        // does not fit: the unpadded order
        std::memcpy(sperm, ot.sperm, (size_t)S);
        return S;
    }
    return k;
}

std::vector<double> stencil_matrix(const RhsCoef &rc, int n, int bc1, int bcn)
{
    std::vector<double> B((size_t)n * n, 0.0);
    std::vector<double> e(n, 0.0);
    double taps[9];
    interior_taps(rc, taps);
    const int cr = closure_rows(rc.rk);
    for (int i = 0; i < n; ++i) {
        const bool closure = !rc.periodic && (i < cr || i >= n - cr);
        if (!closure) {
            for (int k = 0; k < 9; ++k) {
                int j = i + k - 4;
                if (rc.periodic) j = ((j % n) + n) % n;
                if (j >= 0 && j < n) B[(size_t)i * n + j] += taps[k];
            }
            continue;
        }
        for (int j = 0; j < n; ++j) {
            e[j] = 1.0;
            B[(size_t)i * n + j] = rhs_closure_row(rc.rk, rc.c, e.data(), 1, n, i, bc1, bcn);
            e[j] = 0.0;
        }
    }
    return B;
}

std::vector<double> transposed_stencil_blocks(const RhsCoef &rc, int n, int bc1, int bcn)
{
    const std::vector<double> B = stencil_matrix(rc, n, bc1, bcn);
    if (n <= DENSE_BT_MAX) {
        std::vector<double> BT((size_t)n * n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) BT[(size_t)j * n + i] = B[(size_t)i * n + j];
        return BT;
    }
    // [0][j][i]: column j (0..7), rows 0..11;  [1][j'][i']: column n-8+j', rows n-12+i'.
    std::vector<double> blk((size_t)2 * BT_ZONE * BT_WIN, 0.0);
    for (int j = 0; j < BT_ZONE; ++j)
        for (int i = 0; i < BT_WIN; ++i) blk[(size_t)j * BT_WIN + i] = B[(size_t)i * n + j];
    for (int j = 0; j < BT_ZONE; ++j)
        for (int i = 0; i < BT_WIN; ++i)
            blk[(size_t)(BT_ZONE + j) * BT_WIN + i] = B[(size_t)(n - BT_WIN + i) * n + (n - BT_ZONE + j)];
    return blk;
}

}  // namespace pado

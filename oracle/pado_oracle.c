/*
 * pado_oracle.c -- CPU restatement of PadeOps' compact-difference hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker (and the timed
 * CPU baseline, "kind": "port") for the CUDA implementation in
 * padeops_b200/csrc.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load it.  The product never links
 * or calls it.
 *
 * It restates, in the reference's loop and operation order, the Fortran
 * modules
 *     src/derivatives/cd06.F90   (module cd06stuff)
 *     src/derivatives/cd10.F90   (module cd10stuff)
 *     src/filters/cf90.F90       (module cf90stuff, + CF90_files/*.F90)
 * Every function cites the routine and line range it follows.  Array
 * expressions of the reference are evaluated element by element with the same
 * term grouping; Fortran left-to-right evaluation is kept; the file is built
 * with -ffp-contract=off so no FMA contraction changes the rounding.
 *
 * Layout: Fortran column-major f(n1,n2,n3), f[i + n1*(j + n2*k)] (0-based).
 * Coefficient tables are column-major (n, ncol): T[(i-1) + n*(c-1)] for the
 * 1-based (i,c) of the reference.  Internally the code uses 1-based row
 * indices to keep the transcription checkable against the Fortran.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* Coefficients.  cd06.F90:14-59                                              */
/* ------------------------------------------------------------------------- */
static const double alpha06d1 = 1.0 / 3.0;
static const double a06d1 = (14.0 / 9.0) / 2.0;
static const double b06d1 = (1.0 / 9.0) / 4.0;
static const double alpha06d2 = 2.0 / 11.0;

#define C6_alpha 3.0
#define C6_p (17.0 / 6.0)
#define C6_q (3.0 / 2.0)
#define C6_r (3.0 / 2.0)
#define C6_s (-1.0 / 6.0)
#define C6_alpha_hat (1.0 / 3.0)
#define C6_q_p (3.0 / 4.0)
#define C6_alpha_p (1.0 / 4.0)
#define C6_alpha_pp                                                             \
    (((40 * C6_alpha_hat - 1) * C6_q + 7 * (4 * C6_alpha_hat - 1) * C6_s) /    \
     (16 * (C6_alpha_hat + 2) * C6_q + 8 * (1 - 4 * C6_alpha_hat) * C6_s))
#define C6_q_pp ((1.0 / 3.0) * (C6_alpha_pp + 2))
#define C6_r_pp ((1.0 / 12.0) * (4 * C6_alpha_pp - 1))
#define C6_w1 ((2 * C6_alpha_hat + 1) / (2 * (C6_q + C6_s)))
#define C6_w2                                                                   \
    (((8 * C6_alpha_hat + 7) * C6_q - 6 * (2 * C6_alpha_hat + 1) * C6_r +      \
      (8 * C6_alpha_hat + 7) * C6_s) /                                          \
     (9 * (C6_q + C6_s)))
#define C6_w3                                                                   \
    ((4 * (C6_alpha_hat + 2) * C6_q + 2 * (1 - 4 * C6_alpha_hat) * C6_s) /     \
     (9 * (C6_q + C6_s)))

/* ------------------------------------------------------------------------- */
/* Coefficients.  cd10.F90:16-104                                             */
/* ------------------------------------------------------------------------- */
static const double alpha10d1 = 1.0 / 2.0;
static const double beta10d1 = 1.0 / 20.0;
static const double a10d1 = (17.0 / 12.0) / 2.0;
static const double b10d1 = (101.0 / 150.0) / 4.0;
static const double c10d1 = (1.0 / 100.0) / 6.0;
static const double alpha10d2 = 334.0 / 899.0;
static const double beta10d2 = 43.0 / 1798.0;
static const double a10d2 = (1065.0 / 1798.0) / 1.0;
static const double b10d2 = (1038.0 / 899.0) / 4.0;
static const double c10d2 = (79.0 / 1798.0) / 9.0;

#define C10_alpha 3.0
#define C10_p (-17.0 / 6.0)
#define C10_q (3.0 / 2.0)
#define C10_r (3.0 / 2.0)
#define C10_s (-1.0 / 6.0)
#define C10_q_hat ((17.0 / 12.0) / 2.0)
#define C10_r_hat ((101.0 / 150.0) / 4.0)
#define C10_s_hat ((1.0 / 100.0) / 6.0)
#define C10_alpha_hat (1.0 / 2.0)
#define C10_beta_hat (1.0 / 20.0)
#define C10_q_p (3.0 / 4.0)
#define C10_alpha_p (1.0 / 4.0)
#define C10_alpha_ppp ((8 * C10_r_hat - 175 * C10_s_hat) / (18 * C10_r_hat - 550 * C10_s_hat))
#define C10_beta_ppp ((1.0 / 20.0) * (-3 + 8 * C10_alpha_ppp))
#define C10_q_ppp ((1.0 / 12.0) * (12 - 7 * C10_alpha_ppp))
#define C10_r_ppp ((1.0 / 600.0) * (568 * C10_alpha_ppp - 183))
#define C10_s_ppp ((1.0 / 300.0) * (9 * C10_alpha_ppp - 4))
#define C10_APP_T1 (C10_s * (C10_r_hat + 2 * C10_s_hat) - C10_q * (C10_q_hat + C10_r_hat + C10_s_hat))
#define C10_APP_T2 (C10_q_hat + C10_r_hat - C10_s_hat * (C10_q_ppp / C10_s_ppp - 1))
#define C10_alpha_pp                                                            \
    (((17 * C10_APP_T1) / (72 * (C10_q + C10_s) * C10_APP_T2) - 8.0 / 9.0) /   \
     ((19 * C10_APP_T1) / (24 * (C10_q + C10_s) * C10_APP_T2) - 1.0 / 3))
#define C10_beta_pp ((1.0 / 12.0) * (-1 + 3 * C10_alpha_pp))
#define C10_q_pp ((2.0 / 18.0) * (8 - 3 * C10_alpha_pp))
#define C10_r_pp ((1.0 / 72.0) * (-17 + 57 * C10_alpha_pp))
#define C10_w1 ((C10_q_hat + 2 * C10_r_hat + 3 * C10_s_hat) / (C10_q + C10_s))
#define C10_w2                                                                  \
    ((1 / C10_q_p) * (C10_r_hat + C10_s_hat * (1 + C10_q_ppp / C10_s_ppp) -    \
                      C10_r * (C10_q_hat + 2 * C10_r_hat + 3 * C10_s_hat) / (C10_q + C10_s)))
#define C10_w3 ((C10_q_hat + C10_r_hat + C10_s_hat * (1 - C10_q_ppp / C10_s_ppp)) / (C10_r_pp))
#define C10_w4 (C10_s_hat / C10_s_ppp)

#define B1_alpha10d2 11.0
#define B1_a10d2 ((11 * B1_alpha10d2 + 35) / 12)
#define B1_b10d2 (-(5 * B1_alpha10d2 + 26) / 3)
#define B1_c10d2 ((B1_alpha10d2 + 19) / 2)
#define B1_d10d2 ((B1_alpha10d2 - 14) / 3)
#define B1_e10d2 ((11 - B1_alpha10d2) / 12)
#define B2_alpha10d2 (1.0 / 10.0)
#define B2_a10d2 ((4 * (1 - B2_alpha10d2) / 3) / 1.0)
#define B3_alpha10d2 (344.0 / 1179.0)
#define B3_beta10d2 ((38.0 * B3_alpha10d2 - 9.0) / 214.0)
#define B3_a10d2 (((696 - 1191 * B3_alpha10d2) / 428) / 1.0)
#define B3_b10d2 (((2454 * B3_alpha10d2 - 294) / 535) / 4.0)

/* ------------------------------------------------------------------------- */
/* Coefficients.  cf90.F90:16-48                                              */
/* ------------------------------------------------------------------------- */
#define alpha90 6.6624e-1
#define beta90 1.6688e-1
#define a90 9.9965e-1
#define b90 6.6652e-1
#define c90 1.6674e-1
#define d90 4.0e-5
#define e90 (-5.0e-6)
#define b2_alpha90 4.997e-1
#define b2_a90 9.997e-1
#define b2_b90 4.9985e-1
#define b3_alpha90 6.6624e-1
#define b3_beta90 1.6688e-1
#define b3_a90 9.9952e-1
#define b3_b90 6.6656e-1
#define b3_c90 1.668e-1
#define b4_alpha90 6.6624e-1
#define b4_beta90 1.6688e-1
#define b4_a90 9.9968e-1
#define b4_b90 6.6652e-1
#define b4_c90 1.6672e-1
#define b4_d90 4.0e-5

enum { SCHEME_CD06 = 0, SCHEME_CD10 = 1, SCHEME_CF90 = 2 };

/* Handle: the coefficient tables each reference object owns. */
typedef struct {
    int scheme, n, periodic, bc1, bcn;
    double dx, onebydx, onebydx2;
    double *LU1, *LU2; /* cd06: (n,5); cd10: (n,9); cf90: LU1 only (n,9) */
    double *Tri1;      /* cd06 bounded: (n,3)                            */
    double *penta1[9]; /* cd10 d1 / cf90 bounded: (n,11) per bc pair      */
    double *penta2[9]; /* cd10 d2 bounded                                 */
} oracle_op;

#define T(M, i, c) (M)[((i)-1) + (size_t)n * ((c)-1)]

static int bcidx(int bc) { return bc == 0 ? 0 : (bc == 1 ? 1 : 2); }
static int pidx(int bc1, int bcn) { return 3 * bcidx(bc1) + bcidx(bcn); }

/* cd06.F90:221-262  ComputeLU(LU,n,b,d,a): bordered cyclic-tridiagonal LU. */
static void cd06_compute_lu(double *LU, int n, double b, double d, double a)
{
    memset(LU, 0, sizeof(double) * (size_t)n * 5);
#define BC(i) T(LU, i, 1)
#define H(i) T(LU, i, 2)
#define CC(i) T(LU, i, 3)
#define AA(i) T(LU, i, 4)
#define V(i) T(LU, i, 5)
    CC(1) = d;
    V(1) = b;
    H(1) = a / CC(1);
    for (int i = 2; i <= n - 1; ++i) CC(i) = d - (b / CC(i - 1)) * a;
    for (int i = 2; i <= n - 2; ++i) {
        V(i) = -(b / CC(i - 1)) * V(i - 1);
        H(i) = -(a / CC(i)) * H(i - 1);
    }
    V(n - 1) = a - (b / CC(n - 2)) * V(n - 2);
    H(n - 1) = (b - H(n - 2) * a) / CC(n - 1);
    {
        double sum = 0.0;
        for (int i = 1; i <= n - 1; ++i) sum += H(i) * V(i);
        CC(n) = d - sum;
    }
    for (int i = 2; i <= n - 1; ++i) BC(i) = b / CC(i - 1);
    for (int i = 1; i <= n - 2; ++i) AA(i) = a;
    for (int i = 1; i <= n; ++i) CC(i) = 1.0 / CC(i);
    for (int i = 1; i <= n; ++i) AA(i) = AA(i) * CC(i);
    for (int i = 1; i <= n; ++i) V(i) = V(i) * CC(i);
#undef BC
#undef H
#undef CC
#undef AA
#undef V
}

/* cd06.F90:264-327  ComputeTri1(bc1,bcn): Thomas factors with one-sided closures. */
static void cd06_compute_tri1(double *Tri, int n, int bc1, int bcn)
{
    double *a = calloc((size_t)n + 1, sizeof(double));
    double *b = calloc((size_t)n + 1, sizeof(double));
    double *c = calloc((size_t)n + 1, sizeof(double));
    double *cp = calloc((size_t)n + 1, sizeof(double));
    double *den = calloc((size_t)n + 1, sizeof(double));
    for (int i = 1; i <= n; ++i) {
        a[i] = C6_alpha_hat;
        b[i] = 1.0;
        c[i] = C6_alpha_hat;
    }
    if (bc1 == 0) {
        a[1] = C6_w1 * 0.0;
        a[2] = C6_w2 * C6_alpha_p;
        a[3] = C6_w3 * C6_alpha_pp;
        b[1] = C6_w1 * 1.0;
        b[2] = C6_w2 * 1.0;
        b[3] = C6_w3 * 1.0;
        c[1] = C6_w1 * C6_alpha;
        c[2] = C6_w2 * C6_alpha_p;
        c[3] = C6_w3 * C6_alpha_pp;
    } /* bc1 == 1: "Incomplete" in the reference (cd06.F90:288-291): interior bands kept. */
    if (bcn == 0) {
        c[n] = C6_w1 * 0.0;
        c[n - 1] = C6_w2 * C6_alpha_p;
        c[n - 2] = C6_w3 * C6_alpha_pp;
        b[n] = C6_w1 * 1.0;
        b[n - 1] = C6_w2 * 1.0;
        b[n - 2] = C6_w3 * 1.0;
        a[n] = C6_w1 * C6_alpha;
        a[n - 1] = C6_w2 * C6_alpha_p;
        a[n - 2] = C6_w3 * C6_alpha_pp;
    }
    cp[1] = c[1] / b[1];
    for (int i = 2; i <= n - 1; ++i) cp[i] = c[i] / (b[i] - a[i] * cp[i - 1]);
    den[1] = 1.0 / b[1];
    for (int i = 2; i <= n; ++i) den[i] = 1.0 / (b[i] - a[i] * cp[i - 1]);
    /* cp(n) is never assigned in the reference and never read by the solve. */
    for (int i = 1; i <= n; ++i) {
        T(Tri, i, 1) = a[i] * den[i];
        T(Tri, i, 2) = den[i];
        T(Tri, i, 3) = cp[i];
    }
    free(a); free(b); free(c); free(cp); free(den);
}

/* cd10.F90:351-427 and cf90.F90:198-274  ComputeLU(LU,n,e,a,d,c,f):
 * bordered cyclic-pentadiagonal LU (Neossi Nguetchue & Abelman 2008). */
static void penta_compute_lu(double *LU, int n, double e, double a, double d, double c, double f)
{
    memset(LU, 0, sizeof(double) * (size_t)n * 9);
#define B(i) T(LU, i, 1)
#define EG(i) T(LU, i, 2)
#define K(i) T(LU, i, 3)
#define L(i) T(LU, i, 4)
#define G(i) T(LU, i, 5)
#define H(i) T(LU, i, 6)
#define FF(i) T(LU, i, 7)
#define V(i) T(LU, i, 8)
#define W(i) T(LU, i, 9)
    /* Step 1 */
    G(1) = d;
    B(2) = a / G(1);
    H(1) = c;
    K(1) = f / G(1);
    W(1) = a;
    V(1) = e;
    L(1) = c / G(1);
    G(2) = d - B(2) * H(1);
    K(2) = -K(1) * H(1) / G(2);
    W(2) = e - B(2) * W(1);
    V(2) = -B(2) * V(1);
    L(2) = (f - L(1) * H(1)) / G(2);
    H(2) = c - B(2) * f;
    /* Step 2 */
    for (int i = 3; i <= n - 3; ++i) {
        B(i) = (a - (e / G(i - 2)) * H(i - 2)) / G(i - 1);
        H(i) = c - B(i) * f;
        G(i) = d - (e / G(i - 2)) * f - B(i) * H(i - 1);
    }
    /* Step 3 */
    B(n - 2) = (a - (e / G(n - 4)) * H(n - 4)) / G(n - 3);
    G(n - 2) = d - (e / G(n - 4)) * f - B(n - 2) * H(n - 3);
    /* Step 4 */
    for (int i = 3; i <= n - 4; ++i) {
        K(i) = -(K(i - 2) * f + K(i - 1) * H(i - 1)) / G(i);
        V(i) = -(e / G(i - 2)) * V(i - 2) - B(i) * V(i - 1);
    }
    /* Step 5 */
    K(n - 3) = (e - K(n - 5) * f - K(n - 4) * H(n - 4)) / G(n - 3);
    K(n - 2) = (a - K(n - 4) * f - K(n - 3) * H(n - 3)) / G(n - 2);
    V(n - 3) = f - (e / G(n - 5)) * V(n - 5) - B(n - 3) * V(n - 4);
    V(n - 2) = c - (e / G(n - 4)) * V(n - 4) - B(n - 2) * V(n - 3);
    {
        double sum = 0.0;
        for (int i = 1; i <= n - 2; ++i) sum += K(i) * V(i);
        G(n - 1) = d - sum;
    }
    /* Step 6 */
    for (int i = 3; i <= n - 3; ++i) {
        W(i) = -(e / G(i - 2)) * W(i - 2) - B(i) * W(i - 1);
        L(i) = -(L(i - 2) * f + L(i - 1) * H(i - 1)) / G(i);
    }
    /* Step 7 */
    W(n - 2) = f - (e / G(n - 4)) * W(n - 4) - B(n - 2) * W(n - 3);
    {
        double sum = 0.0;
        for (int i = 1; i <= n - 2; ++i) sum += K(i) * W(i);
        W(n - 1) = c - sum;
    }
    L(n - 2) = (e - L(n - 4) * f - L(n - 3) * H(n - 3)) / G(n - 2);
    {
        double sum = 0.0;
        for (int i = 1; i <= n - 2; ++i) sum += L(i) * V(i);
        L(n - 1) = (a - sum) / G(n - 1);
    }
    {
        double sum = 0.0;
        for (int i = 1; i <= n - 1; ++i) sum += L(i) * W(i);
        G(n) = d - sum;
    }
    for (int i = 3; i <= n - 2; ++i) EG(i) = e / G(i - 2);
    for (int i = 1; i <= n - 4; ++i) FF(i) = f;
    for (int i = 1; i <= n; ++i) G(i) = 1.0 / G(i);
#undef B
#undef EG
#undef K
#undef L
#undef G
#undef H
#undef FF
#undef V
#undef W
}

/* Bands (bt,b,d,a,at) -> penta LU factors.  Shared tail of
 * cd10.F90:558-575 (ComputePenta1), :689-706 (ComputePenta2) and
 * cf90.F90:398-415 (ComputePenta).  The reference's unassigned entries
 * (f(1), g(1:2), e(n), column 11) are zero here; the solve never reads them. */
static void penta_factor(double *P, int n)
{
#define BT(i) T(P, i, 1)
#define BB(i) T(P, i, 2)
#define DD(i) T(P, i, 3)
#define AA(i) T(P, i, 4)
#define AT(i) T(P, i, 5)
#define EE(i) T(P, i, 6)
#define OBC(i) T(P, i, 7)
#define FF(i) T(P, i, 8)
#define GG(i) T(P, i, 9)
#define EOBC(i) T(P, i, 10)
    OBC(1) = 1.0 / DD(1);
    OBC(2) = 1.0 / (DD(2) - BB(2) * AA(1) * OBC(1));
    EE(1) = AA(1);
    FF(2) = BB(2) * OBC(1);
    for (int i = 3; i <= n; ++i) {
        GG(i) = BT(i) * OBC(i - 2);
        EE(i - 1) = AA(i - 1) - FF(i - 1) * AT(i - 2);
        FF(i) = (BB(i) - GG(i) * EE(i - 2)) * OBC(i - 1);
        OBC(i) = 1.0 / (DD(i) - FF(i) * EE(i - 1) - GG(i) * AT(i - 2));
    }
    for (int i = 1; i <= n; ++i) EOBC(i) = EE(i) * OBC(i);
}

static void set5(double *P, int n, int i, double bt, double b, double d, double a, double at)
{
    BT(i) = bt;
    BB(i) = b;
    DD(i) = d;
    AA(i) = a;
    AT(i) = at;
}

/* cd10.F90:429-578  ComputePenta1(penta1,bc1,bcn). */
static void cd10_compute_penta1(double *P, int n, int bc1, int bcn)
{
    memset(P, 0, sizeof(double) * (size_t)n * 11);
    for (int i = 1; i <= n; ++i) set5(P, n, i, C10_beta_hat, C10_alpha_hat, 1.0, C10_alpha_hat, C10_beta_hat);
    const double w1 = C10_w1, w2 = C10_w2, w3 = C10_w3, w4 = C10_w4;
    if (bc1 == 0) {
        set5(P, n, 1, w1 * 0.0, w1 * 0.0, w1 * 1.0, w1 * C10_alpha, w1 * 0.0);
        set5(P, n, 2, w2 * 0.0, w2 * C10_alpha_p, w2 * 1.0, w2 * C10_alpha_p, w2 * 0.0);
        set5(P, n, 3, w3 * C10_beta_pp, w3 * C10_alpha_pp, w3 * 1.0, w3 * C10_alpha_pp, w3 * C10_beta_pp);
        set5(P, n, 4, w4 * C10_beta_ppp, w4 * C10_alpha_ppp, w4 * 1.0, w4 * C10_alpha_ppp, w4 * C10_beta_ppp);
    } else if (bc1 == 1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, 2, 0.0, C10_alpha_hat, 1.0 - C10_beta_hat, C10_alpha_hat, C10_beta_hat);
    } else if (bc1 == -1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 2.0 * C10_alpha_hat, 2.0 * C10_beta_hat);
        set5(P, n, 2, 0.0, C10_alpha_hat, 1.0 + C10_beta_hat, C10_alpha_hat, C10_beta_hat);
    }
    if (bcn == 0) {
        set5(P, n, n, w1 * 0.0, w1 * C10_alpha, w1 * 1.0, w1 * 0.0, w1 * 0.0);
        set5(P, n, n - 1, w2 * 0.0, w2 * C10_alpha_p, w2 * 1.0, w2 * C10_alpha_p, w2 * 0.0);
        set5(P, n, n - 2, w3 * C10_beta_pp, w3 * C10_alpha_pp, w3 * 1.0, w3 * C10_alpha_pp, w3 * C10_beta_pp);
        set5(P, n, n - 3, w4 * C10_beta_ppp, w4 * C10_alpha_ppp, w4 * 1.0, w4 * C10_alpha_ppp, w4 * C10_beta_ppp);
    } else if (bcn == 1) {
        set5(P, n, n, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, n - 1, C10_beta_hat, C10_alpha_hat, 1.0 - C10_beta_hat, C10_alpha_hat, 0.0);
    } else if (bcn == -1) {
        set5(P, n, n, 2.0 * C10_beta_hat, 2.0 * C10_alpha_hat, 1.0, 0.0, 0.0);
        set5(P, n, n - 1, C10_beta_hat, C10_alpha_hat, 1.0 + C10_beta_hat, C10_alpha_hat, 0.0);
    }
    penta_factor(P, n);
}

/* cd10.F90:580-709  ComputePenta2(penta2,bc1,bcn). */
static void cd10_compute_penta2(double *P, int n, int bc1, int bcn)
{
    memset(P, 0, sizeof(double) * (size_t)n * 11);
    for (int i = 1; i <= n; ++i) set5(P, n, i, beta10d2, alpha10d2, 1.0, alpha10d2, beta10d2);
    if (bc1 == 0) {
        set5(P, n, 1, 0.0, 0.0, 1.0, B1_alpha10d2, 0.0);
        set5(P, n, 2, 0.0, B2_alpha10d2, 1.0, B2_alpha10d2, 0.0);
        set5(P, n, 3, B3_beta10d2, B3_alpha10d2, 1.0, B3_alpha10d2, B3_beta10d2);
    } else if (bc1 == 1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 2.0 * alpha10d2, 2.0 * beta10d2);
        set5(P, n, 2, 0.0, alpha10d2, 1.0 + beta10d2, alpha10d2, beta10d2);
    } else if (bc1 == -1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, 2, 0.0, alpha10d2, 1.0 - beta10d2, alpha10d2, beta10d2);
    }
    if (bcn == 0) {
        set5(P, n, n - 2, B3_beta10d2, B3_alpha10d2, 1.0, B3_alpha10d2, B3_beta10d2);
        set5(P, n, n - 1, 0.0, B2_alpha10d2, 1.0, B2_alpha10d2, 0.0);
        set5(P, n, n, 0.0, B1_alpha10d2, 1.0, 0.0, 0.0);
    } else if (bcn == 1) {
        set5(P, n, n - 1, beta10d2, alpha10d2, 1.0 + beta10d2, alpha10d2, 0.0);
        set5(P, n, n, 2.0 * beta10d2, 2.0 * alpha10d2, 1.0, 0.0, 0.0);
    } else if (bcn == -1) {
        set5(P, n, n - 1, beta10d2, alpha10d2, 1.0 - beta10d2, alpha10d2, 0.0);
        set5(P, n, n, 0.0, 0.0, 1.0, 0.0, 0.0);
    }
    penta_factor(P, n);
}

/* cf90.F90:276-418  ComputePenta(penta,bc1,bcn). */
static void cf90_compute_penta(double *P, int n, int bc1, int bcn)
{
    memset(P, 0, sizeof(double) * (size_t)n * 11);
    for (int i = 1; i <= n; ++i) set5(P, n, i, beta90, alpha90, 1.0, alpha90, beta90);
    if (bc1 == 0) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, 2, 0.0, b2_alpha90, 1.0, b2_alpha90, 0.0);
        set5(P, n, 3, b3_beta90, b3_alpha90, 1.0, b3_alpha90, b3_beta90);
        set5(P, n, 4, b4_beta90, b4_alpha90, 1.0, b4_alpha90, b4_beta90);
    } else if (bc1 == 1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 2.0 * alpha90, 2.0 * beta90);
        set5(P, n, 2, 0.0, alpha90, 1.0 + beta90, alpha90, beta90);
    } else if (bc1 == -1) {
        set5(P, n, 1, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, 2, 0.0, alpha90, 1.0 - beta90, alpha90, beta90);
    }
    if (bcn == 0) {
        set5(P, n, n, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, n - 1, 0.0, b2_alpha90, 1.0, b2_alpha90, 0.0);
        set5(P, n, n - 2, b3_beta90, b3_alpha90, 1.0, b3_alpha90, b3_beta90);
        set5(P, n, n - 3, b4_beta90, b4_alpha90, 1.0, b4_alpha90, b4_beta90);
    } else if (bcn == 1) {
        set5(P, n, n, 2.0 * beta90, 2.0 * alpha90, 1.0, 0.0, 0.0);
        set5(P, n, n - 1, beta90, alpha90, 1.0 + beta90, alpha90, 0.0);
    } else if (bcn == -1) {
        set5(P, n, n, 0.0, 0.0, 1.0, 0.0, 0.0);
        set5(P, n, n - 1, beta90, alpha90, 1.0 - beta90, alpha90, 0.0);
    }
    penta_factor(P, n);
}
#undef BT
#undef BB
#undef DD
#undef AA
#undef AT
#undef EE
#undef OBC
#undef FF
#undef GG
#undef EOBC

/* ------------------------------------------------------------------------- */
/* Handle life cycle: cd06.F90:129-201, cd10.F90:195-315, cf90.F90:107-175.  */
/* Returns the reference's ierr (0 ok; cd06 3 periodic / 2 bounded; cd10 2;  */
/* cf90 7).                                                                  */
/* ------------------------------------------------------------------------- */
void oracle_destroy(oracle_op *op);

int oracle_create(oracle_op **out, int scheme, int n, double dx, int periodic, int bc1, int bcn)
{
    oracle_op *op = calloc(1, sizeof(oracle_op));
    *out = op;
    op->scheme = scheme;
    op->n = n;
    op->dx = dx;
    op->onebydx = 1.0 / dx;
    op->onebydx2 = op->onebydx / dx;
    op->periodic = periodic;
    op->bc1 = bc1;
    op->bcn = bcn;
    if (scheme == SCHEME_CD06) {
        if (periodic) {
            op->LU1 = calloc((size_t)n * 5, sizeof(double));
            if (n >= 6) {
                cd06_compute_lu(op->LU1, n, alpha06d1, 1.0, alpha06d1);
                op->LU2 = calloc((size_t)n * 5, sizeof(double));
                cd06_compute_lu(op->LU2, n, alpha06d2, 1.0, alpha06d2);
            } else if (n == 1) {
                op->LU1[0] = 1.0;
            } else {
                return 3;
            }
        } else {
            op->Tri1 = calloc((size_t)n * 3, sizeof(double));
            if (n >= 8) cd06_compute_tri1(op->Tri1, n, bc1, bcn);
            else if (n != 1) return 2;
        }
        return 0;
    }
    if (scheme == SCHEME_CD10) {
        if (periodic) {
            op->LU1 = calloc((size_t)n * 9, sizeof(double));
            op->LU2 = calloc((size_t)n * 9, sizeof(double));
            if (n >= 8) {
                penta_compute_lu(op->LU1, n, beta10d1, alpha10d1, 1.0, alpha10d1, beta10d1);
                penta_compute_lu(op->LU2, n, beta10d2, alpha10d2, 1.0, alpha10d2, beta10d2);
            } else if (n != 1) {
                return 2;
            }
        } else {
            for (int q = 0; q < 9; ++q) {
                op->penta1[q] = calloc((size_t)n * 11, sizeof(double));
                op->penta2[q] = calloc((size_t)n * 11, sizeof(double));
            }
            if (n >= 8) {
                static const int bcs[3] = {0, 1, -1};
                for (int p = 0; p < 3; ++p)
                    for (int q = 0; q < 3; ++q) {
                        cd10_compute_penta1(op->penta1[pidx(bcs[p], bcs[q])], n, bcs[p], bcs[q]);
                        cd10_compute_penta2(op->penta2[pidx(bcs[p], bcs[q])], n, bcs[p], bcs[q]);
                    }
            } else if (n != 1) {
                return 2;
            }
        }
        return 0;
    }
    if (scheme == SCHEME_CF90) {
        if (periodic) {
            op->LU1 = calloc((size_t)n * 9, sizeof(double));
            if (n >= 10) penta_compute_lu(op->LU1, n, beta90, alpha90, 1.0, alpha90, beta90);
            else if (n != 1) return 7;
        } else {
            for (int q = 0; q < 9; ++q) op->penta1[q] = calloc((size_t)n * 11, sizeof(double));
            if (n >= 10) {
                static const int bcs[3] = {0, 1, -1};
                for (int p = 0; p < 3; ++p)
                    for (int q = 0; q < 3; ++q)
                        cf90_compute_penta(op->penta1[pidx(bcs[p], bcs[q])], n, bcs[p], bcs[q]);
            } else if (n != 1) {
                return 7;
            }
        }
        return 0;
    }
    return -1;
}

void oracle_destroy(oracle_op *op)
{
    if (!op) return;
    free(op->LU1);
    free(op->LU2);
    free(op->Tri1);
    for (int q = 0; q < 9; ++q) {
        free(op->penta1[q]);
        free(op->penta2[q]);
    }
    free(op);
}

/* Copies a coefficient table out (tests compare the device tables to these).
 * which: 0 LU1, 1 LU2, 2 Tri1, 10+q penta1[q], 20+q penta2[q]. */
int oracle_table(const oracle_op *op, int which, double *dst)
{
    const double *src = NULL;
    size_t cols = 0;
    int n = op->n;
    if (which == 0) { src = op->LU1; cols = op->scheme == SCHEME_CD06 ? 5 : 9; }
    else if (which == 1) { src = op->LU2; cols = op->scheme == SCHEME_CD06 ? 5 : 9; }
    else if (which == 2) { src = op->Tri1; cols = 3; }
    else if (which >= 10 && which < 19) { src = op->penta1[which - 10]; cols = 11; }
    else if (which >= 20 && which < 29) { src = op->penta2[which - 20]; cols = 11; }
    if (!src) return -1;
    memcpy(dst, src, sizeof(double) * (size_t)n * cols);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* RHS rows.  A "line" is p[(i-1)*s], i = 1..n.  Each function returns the    */
/* reference's value for one row, with the reference's term grouping.        */
/* ------------------------------------------------------------------------- */
#define F(i) p[(ptrdiff_t)((i)-1) * s]

/* cd06.F90:515-592 (X), 596-671 (Y), 674-742 (Z): identical row formulas. */
static inline double cd06_d1_row(const double *p, ptrdiff_t s, int n, int i, int periodic, double ob)
{
    const double a06 = a06d1 * ob, b06 = b06d1 * ob;
    if (periodic) {
        int ip1 = i + 1 > n ? i + 1 - n : i + 1, ip2 = i + 2 > n ? i + 2 - n : i + 2;
        int im1 = i - 1 < 1 ? i - 1 + n : i - 1, im2 = i - 2 < 1 ? i - 2 + n : i - 2;
        return a06 * (F(ip1) - F(im1)) + b06 * (F(ip2) - F(im2));
    }
    const double a_np_3 = C6_w3 * C6_q_pp * ob, b_np_3 = C6_w3 * C6_r_pp * ob;
    const double a_np_2 = C6_w2 * C6_q_p * ob;
    const double a_np_1 = C6_w1 * (-(C6_p * ob)), b_np_1 = C6_w1 * (C6_q * ob);
    const double c_np_1 = C6_w1 * (C6_r * ob), d_np_1 = C6_w1 * (C6_s * ob);
    if (i == 1) return a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4);
    if (i == 2) return a_np_2 * (F(3) - F(1));
    if (i == 3) return a_np_3 * (F(4) - F(2)) + b_np_3 * (F(5) - F(1));
    if (i == n - 2) return a_np_3 * (F(n - 1) - F(n - 3)) + b_np_3 * (F(n) - F(n - 4));
    if (i == n - 1) return a_np_2 * (F(n) - F(n - 2));
    if (i == n) return -(a_np_1 * F(n)) - b_np_1 * F(n - 1) - c_np_1 * F(n - 2) - d_np_1 * F(n - 3);
    return b06 * (F(i + 2) - F(i - 2)) + a06 * (F(i + 1) - F(i - 1));
}

static inline int wrap(int i, int n) { return i > n ? i - n : (i < 1 ? i + n : i); }

/* cd10.F90:1098-1585  ComputeX/Y/ZD1RHS. */
static inline double cd10_d1_row(const double *p, ptrdiff_t s, int n, int i, int periodic, int bc1, int bcn,
                                 double ob)
{
    if (periodic) {
        const double a10 = a10d1 * ob, b10 = b10d1 * ob, c10 = c10d1 * ob;
        return a10 * (F(wrap(i + 1, n)) - F(wrap(i - 1, n))) + b10 * (F(wrap(i + 2, n)) - F(wrap(i - 2, n))) +
               c10 * (F(wrap(i + 3, n)) - F(wrap(i - 3, n)));
    }
    const double a10 = C10_q_hat * ob, b10 = C10_r_hat * ob, c10 = C10_s_hat * ob;
    const double a_np_4 = C10_w4 * C10_q_ppp * ob, b_np_4 = C10_w4 * C10_r_ppp * ob, c_np_4 = C10_w4 * C10_s_ppp * ob;
    const double a_np_3 = C10_w3 * C10_q_pp * ob, b_np_3 = C10_w3 * C10_r_pp * ob;
    const double a_np_2 = C10_w2 * C10_q_p * ob;
    const double a_np_1 = C10_w1 * (C10_p * ob), b_np_1 = C10_w1 * (C10_q * ob);
    const double c_np_1 = C10_w1 * (C10_r * ob), d_np_1 = C10_w1 * (C10_s * ob);
    if (i <= 4) {
        if (bc1 == 0) {
            if (i == 1) return a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4);
            if (i == 2) return a_np_2 * (F(3) - F(1));
            if (i == 3) return a_np_3 * (F(4) - F(2)) + b_np_3 * (F(5) - F(1));
            return a_np_4 * (F(5) - F(3)) + b_np_4 * (F(6) - F(2)) + c_np_4 * (F(7) - F(1));
        } else if (bc1 == 1) {
            if (i == 1) return 0.0;
            if (i == 2) return a10 * (F(3) - F(1)) + b10 * (F(4) - F(2)) + c10 * (F(5) - F(3));
            if (i == 3) return a10 * (F(4) - F(2)) + b10 * (F(5) - F(1)) + c10 * (F(6) - F(2));
            return a10 * (F(5) - F(3)) + b10 * (F(6) - F(2)) + c10 * (F(7) - F(1));
        } else {
            if (i == 1) return a10 * (F(2) + F(2)) + b10 * (F(3) + F(3)) + c10 * (F(4) + F(4));
            if (i == 2) return a10 * (F(3) - F(1)) + b10 * (F(4) + F(2)) + c10 * (F(5) + F(3));
            if (i == 3) return a10 * (F(4) - F(2)) + b10 * (F(5) - F(1)) + c10 * (F(6) + F(2));
            return a10 * (F(5) - F(3)) + b10 * (F(6) - F(2)) + c10 * (F(7) - F(1));
        }
    }
    if (i >= n - 3) {
        if (bcn == 0) {
            if (i == n - 3) return a_np_4 * (F(n - 2) - F(n - 4)) + b_np_4 * (F(n - 1) - F(n - 5)) + c_np_4 * (F(n) - F(n - 6));
            if (i == n - 2) return a_np_3 * (F(n - 1) - F(n - 3)) + b_np_3 * (F(n) - F(n - 4));
            if (i == n - 1) return a_np_2 * (F(n) - F(n - 2));
            return -(a_np_1 * F(n)) - b_np_1 * F(n - 1) - c_np_1 * F(n - 2) - d_np_1 * F(n - 3);
        } else if (bcn == 1) {
            if (i == n - 3) return a10 * (F(n - 2) - F(n - 4)) + b10 * (F(n - 1) - F(n - 5)) + c10 * (F(n) - F(n - 6));
            if (i == n - 2) return a10 * (F(n - 1) - F(n - 3)) + b10 * (F(n) - F(n - 4)) + c10 * (F(n - 1) - F(n - 5));
            if (i == n - 1) return a10 * (F(n) - F(n - 2)) + b10 * (F(n - 1) - F(n - 3)) + c10 * (F(n - 2) - F(n - 4));
            return 0.0;
        } else {
            if (i == n - 3) return a10 * (F(n - 2) - F(n - 4)) + b10 * (F(n - 1) - F(n - 5)) + c10 * (F(n) - F(n - 6));
            if (i == n - 2) return a10 * (F(n - 1) - F(n - 3)) + b10 * (F(n) - F(n - 4)) + c10 * (-F(n - 1) - F(n - 5));
            if (i == n - 1) return a10 * (F(n) - F(n - 2)) + b10 * (-F(n - 1) - F(n - 3)) + c10 * (-F(n - 2) - F(n - 4));
            return a10 * (-F(n - 1) - F(n - 1)) + b10 * (-F(n - 2) - F(n - 2)) + c10 * (-F(n - 3) - F(n - 3));
        }
    }
    return a10 * (F(i + 1) - F(i - 1)) + b10 * (F(i + 2) - F(i - 2)) + c10 * (F(i + 3) - F(i - 3));
}

/* cd10.F90:1587-2027  ComputeX/Y/ZD2RHS. */
static inline double cd10_d2_row(const double *p, ptrdiff_t s, int n, int i, int periodic, int bc1, int bcn,
                                 double ob2)
{
    const double a10 = a10d2 * ob2, b10 = b10d2 * ob2, c10 = c10d2 * ob2;
    if (periodic) {
        return a10 * (F(wrap(i + 1, n)) - 2.0 * F(i) + F(wrap(i - 1, n))) +
               b10 * (F(wrap(i + 2, n)) - 2.0 * F(i) + F(wrap(i - 2, n))) +
               c10 * (F(wrap(i + 3, n)) - 2.0 * F(i) + F(wrap(i - 3, n)));
    }
    const double a_np_3 = B3_a10d2 * ob2, b_np_3 = B3_b10d2 * ob2, a_np_2 = B2_a10d2 * ob2;
    const double a_np_1 = B1_a10d2 * ob2, b_np_1 = B1_b10d2 * ob2, c_np_1 = B1_c10d2 * ob2;
    const double d_np_1 = B1_d10d2 * ob2, e_np_1 = B1_e10d2 * ob2;
    if (i <= 3) {
        if (bc1 == 0) {
            if (i == 1) return a_np_1 * F(1) + b_np_1 * F(2) + c_np_1 * F(3) + d_np_1 * F(4) + e_np_1 * F(5);
            if (i == 2) return a_np_2 * (F(3) - 2.0 * F(2) + F(1));
            return a_np_3 * (F(4) - 2.0 * F(3) + F(2)) + b_np_3 * (F(5) - 2.0 * F(3) + F(1));
        } else if (bc1 == 1) {
            if (i == 1) return a10 * (F(2) - 2.0 * F(1) + F(2)) + b10 * (F(3) - 2.0 * F(1) + F(3)) + c10 * (F(4) - 2.0 * F(1) + F(4));
            if (i == 2) return a10 * (F(3) - 2.0 * F(2) + F(1)) + b10 * (F(4) - 2.0 * F(2) + F(2)) + c10 * (F(5) - 2.0 * F(2) + F(3));
            return a10 * (F(4) - 2.0 * F(3) + F(2)) + b10 * (F(5) - 2.0 * F(3) + F(1)) + c10 * (F(6) - 2.0 * F(3) + F(2));
        } else {
            if (i == 1) return a10 * (F(2) - 2.0 * F(1) - F(2)) + b10 * (F(3) - 2.0 * F(1) - F(3)) + c10 * (F(4) - 2.0 * F(1) - F(4));
            if (i == 2) return a10 * (F(3) - 2.0 * F(2) + F(1)) + b10 * (F(4) - 2.0 * F(2) - F(2)) + c10 * (F(5) - 2.0 * F(2) - F(3));
            return a10 * (F(4) - 2.0 * F(3) + F(2)) + b10 * (F(5) - 2.0 * F(3) + F(1)) + c10 * (F(6) - 2.0 * F(3) - F(2));
        }
    }
    if (i >= n - 2) {
        if (bcn == 0) {
            if (i == n - 2) return a_np_3 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b_np_3 * (F(n) - 2.0 * F(n - 2) + F(n - 4));
            if (i == n - 1) return a_np_2 * (F(n) - 2.0 * F(n - 1) + F(n - 2));
            return a_np_1 * F(n) + b_np_1 * F(n - 1) + c_np_1 * F(n - 2) + d_np_1 * F(n - 3) + e_np_1 * F(n - 4);
        } else if (bcn == 1) {
            if (i == n - 2) return a10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b10 * (F(n) - 2.0 * F(n - 2) + F(n - 4)) + c10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 5));
            if (i == n - 1) return a10 * (F(n) - 2.0 * F(n - 1) + F(n - 2)) + b10 * (F(n - 1) - 2.0 * F(n - 1) + F(n - 3)) + c10 * (F(n - 2) - 2.0 * F(n - 1) + F(n - 4));
            return a10 * (F(n - 1) - 2.0 * F(n) + F(n - 1)) + b10 * (F(n - 2) - 2.0 * F(n) + F(n - 2)) + c10 * (F(n - 3) - 2.0 * F(n) + F(n - 3));
        } else {
            if (i == n - 2) return a10 * (F(n - 1) - 2.0 * F(n - 2) + F(n - 3)) + b10 * (F(n) - 2.0 * F(n - 2) + F(n - 4)) + c10 * (-F(n - 1) - 2.0 * F(n - 2) + F(n - 5));
            if (i == n - 1) return a10 * (F(n) - 2.0 * F(n - 1) + F(n - 2)) + b10 * (-F(n - 1) - 2.0 * F(n - 1) + F(n - 3)) + c10 * (-F(n - 2) - 2.0 * F(n - 1) + F(n - 4));
            return a10 * (-F(n - 1) - 2.0 * F(n) + F(n - 1)) + b10 * (-F(n - 2) - 2.0 * F(n) + F(n - 2)) + c10 * (-F(n - 3) - 2.0 * F(n) + F(n - 3));
        }
    }
    return a10 * (F(i + 1) - 2.0 * F(i) + F(i - 1)) + b10 * (F(i + 2) - 2.0 * F(i) + F(i - 2)) +
           c10 * (F(i + 3) - 2.0 * F(i) + F(i - 3));
}

/* cf90.F90:610-994, CF90_files/ComputeZRHS_common.F90:1-174. */
static inline double cf90_row(const double *p, ptrdiff_t s, int n, int i, int periodic, int bc1, int bcn)
{
    if (periodic) {
        return a90 * (F(i)) + b90 * (F(wrap(i + 1, n)) + F(wrap(i - 1, n))) +
               c90 * (F(wrap(i + 2, n)) + F(wrap(i - 2, n))) + d90 * (F(wrap(i + 3, n)) + F(wrap(i - 3, n))) +
               e90 * (F(wrap(i + 4, n)) + F(wrap(i - 4, n)));
    }
    if (i <= 4) {
        if (bc1 == 0) {
            if (i == 1) return 1.0 * (F(1));
            if (i == 2) return b2_a90 * (F(2)) + b2_b90 * (F(3) + F(1));
            if (i == 3) return b3_a90 * (F(3)) + b3_b90 * (F(4) + F(2)) + b3_c90 * (F(5) + F(1));
            return b4_a90 * (F(4)) + b4_b90 * (F(5) + F(3)) + b4_c90 * (F(6) + F(2)) + b4_d90 * (F(7) + F(1));
        } else if (bc1 == 1) {
            if (i == 1) return a90 * (F(1)) + b90 * (F(2) + F(2)) + c90 * (F(3) + F(3)) + d90 * (F(4) + F(4)) + e90 * (F(5) + F(5));
            if (i == 2) return a90 * (F(2)) + b90 * (F(3) + F(1)) + c90 * (F(4) + F(2)) + d90 * (F(5) + F(3)) + e90 * (F(6) + F(4));
            if (i == 3) return a90 * (F(3)) + b90 * (F(4) + F(2)) + c90 * (F(5) + F(1)) + d90 * (F(6) + F(2)) + e90 * (F(7) + F(3));
            return a90 * (F(4)) + b90 * (F(5) + F(3)) + c90 * (F(6) + F(2)) + d90 * (F(7) + F(1)) + e90 * (F(8) + F(2));
        } else {
            if (i == 1) return a90 * (F(1)) + b90 * (F(2) - F(2)) + c90 * (F(3) - F(3)) + d90 * (F(4) - F(4)) + e90 * (F(5) - F(5));
            if (i == 2) return a90 * (F(2)) + b90 * (F(3) + F(1)) + c90 * (F(4) - F(2)) + d90 * (F(5) - F(3)) + e90 * (F(6) - F(4));
            if (i == 3) return a90 * (F(3)) + b90 * (F(4) + F(2)) + c90 * (F(5) + F(1)) + d90 * (F(6) - F(2)) + e90 * (F(7) - F(3));
            return a90 * (F(4)) + b90 * (F(5) + F(3)) + c90 * (F(6) + F(2)) + d90 * (F(7) + F(1)) + e90 * (F(8) - F(2));
        }
    }
    if (i >= n - 3) {
        if (bcn == 0) {
            if (i == n - 3) return b4_a90 * (F(n - 3)) + b4_b90 * (F(n - 2) + F(n - 4)) + b4_c90 * (F(n - 1) + F(n - 5)) + b4_d90 * (F(n) + F(n - 6));
            if (i == n - 2) return b3_a90 * (F(n - 2)) + b3_b90 * (F(n - 1) + F(n - 3)) + b3_c90 * (F(n) + F(n - 4));
            if (i == n - 1) return b2_a90 * (F(n - 1)) + b2_b90 * (F(n) + F(n - 2));
            return 1.0 * (F(n));
        } else if (bcn == 1) {
            if (i == n - 3) return a90 * (F(n - 3)) + b90 * (F(n - 2) + F(n - 4)) + c90 * (F(n - 1) + F(n - 5)) + d90 * (F(n) + F(n - 6)) + e90 * (F(n - 1) + F(n - 7));
            if (i == n - 2) return a90 * (F(n - 2)) + b90 * (F(n - 1) + F(n - 3)) + c90 * (F(n) + F(n - 4)) + d90 * (F(n - 1) + F(n - 5)) + e90 * (F(n - 2) + F(n - 6));
            if (i == n - 1) return a90 * (F(n - 1)) + b90 * (F(n) + F(n - 2)) + c90 * (F(n - 1) + F(n - 3)) + d90 * (F(n - 2) + F(n - 4)) + e90 * (F(n - 3) + F(n - 5));
            return a90 * (F(n)) + b90 * (F(n - 1) + F(n - 1)) + c90 * (F(n - 2) + F(n - 2)) + d90 * (F(n - 3) + F(n - 3)) + e90 * (F(n - 4) + F(n - 4));
        } else {
            if (i == n - 3) return a90 * (F(n - 3)) + b90 * (F(n - 2) + F(n - 4)) + c90 * (F(n - 1) + F(n - 5)) + d90 * (F(n) + F(n - 6)) + e90 * (-F(n - 1) + F(n - 7));
            if (i == n - 2) return a90 * (F(n - 2)) + b90 * (F(n - 1) + F(n - 3)) + c90 * (F(n) + F(n - 4)) + d90 * (-F(n - 1) + F(n - 5)) + e90 * (-F(n - 2) + F(n - 6));
            if (i == n - 1) return a90 * (F(n - 1)) + b90 * (F(n) + F(n - 2)) + c90 * (-F(n - 1) + F(n - 3)) + d90 * (-F(n - 2) + F(n - 4)) + e90 * (-F(n - 3) + F(n - 5));
            return a90 * (F(n)) + b90 * (-F(n - 1) + F(n - 1)) + c90 * (-F(n - 2) + F(n - 2)) + d90 * (-F(n - 3) + F(n - 3)) + e90 * (-F(n - 4) + F(n - 4));
        }
    }
    return a90 * (F(i)) + b90 * (F(i + 1) + F(i - 1)) + c90 * (F(i + 2) + F(i - 2)) + d90 * (F(i + 3) + F(i - 3)) +
           e90 * (F(i + 4) + F(i - 4));
}
#undef F

/* ------------------------------------------------------------------------- */
/* Block kernels: nl lines, lines contiguous in memory (stride 1 between      */
/* lines), element stride s along a line.  For X the block is one line       */
/* (nl = 1, s = 1); for Y one k-plane slice; for Z a slice of the (i,j)      */
/* plane -- the loop nests of the reference's X, Y and Z routines.           */
/* ------------------------------------------------------------------------- */
enum { KIND_D1 = 1, KIND_D2 = 2, KIND_FILTER = 0 };

static inline __attribute__((always_inline)) void rhs_block(const oracle_op *op, int kind, const double *f,
                                                            double *r, int nl, ptrdiff_t s, int bc1, int bcn)
{
    const int n = op->n;
    /* Interior rows [lo, hi] use the plain stencil (no wrap, no closure):
     * these are the reference's array-section statements, e.g.
     * cd10.F90:1129-1131 / 1209-1211, cd06.F90:541-542 / 575-576,
     * cf90.F90:643-647 / 735-739, cd10.F90:1619-1621 / 1692-1694. */
    int lo, hi;
    if (op->scheme == SCHEME_CD06) { lo = op->periodic ? 3 : 4; hi = op->periodic ? n - 2 : n - 3; }
    else if (op->scheme == SCHEME_CD10 && kind == KIND_D1) { lo = op->periodic ? 4 : 5; hi = op->periodic ? n - 3 : n - 4; }
    else if (op->scheme == SCHEME_CD10) { lo = 4; hi = n - 3; }
    else { lo = 5; hi = n - 4; }
    for (int i = 1; i <= n; ++i) {
        double *ri = r + (ptrdiff_t)(i - 1) * s;
        if (i >= lo && i <= hi) {
            const double *c0 = f + (ptrdiff_t)(i - 1) * s;
            if (op->scheme == SCHEME_CD06) {
                const double a06 = a06d1 * op->onebydx, b06 = b06d1 * op->onebydx;
                if (op->periodic)
                    for (int l = 0; l < nl; ++l) ri[l] = a06 * (c0[l + s] - c0[l - s]) + b06 * (c0[l + 2 * s] - c0[l - 2 * s]);
                else
                    for (int l = 0; l < nl; ++l) ri[l] = b06 * (c0[l + 2 * s] - c0[l - 2 * s]) + a06 * (c0[l + s] - c0[l - s]);
            } else if (op->scheme == SCHEME_CD10 && kind == KIND_D1) {
                const double a10 = a10d1 * op->onebydx, b10 = b10d1 * op->onebydx, c10 = c10d1 * op->onebydx;
                for (int l = 0; l < nl; ++l)
                    ri[l] = a10 * (c0[l + s] - c0[l - s]) + b10 * (c0[l + 2 * s] - c0[l - 2 * s]) +
                            c10 * (c0[l + 3 * s] - c0[l - 3 * s]);
            } else if (op->scheme == SCHEME_CD10) {
                const double a10 = a10d2 * op->onebydx2, b10 = b10d2 * op->onebydx2, c10 = c10d2 * op->onebydx2;
                for (int l = 0; l < nl; ++l)
                    ri[l] = a10 * (c0[l + s] - 2.0 * c0[l] + c0[l - s]) + b10 * (c0[l + 2 * s] - 2.0 * c0[l] + c0[l - 2 * s]) +
                            c10 * (c0[l + 3 * s] - 2.0 * c0[l] + c0[l - 3 * s]);
            } else {
                for (int l = 0; l < nl; ++l)
                    ri[l] = a90 * (c0[l]) + b90 * (c0[l + s] + c0[l - s]) + c90 * (c0[l + 2 * s] + c0[l - 2 * s]) +
                            d90 * (c0[l + 3 * s] + c0[l - 3 * s]) + e90 * (c0[l + 4 * s] + c0[l - 4 * s]);
            }
            continue;
        }
        if (op->scheme == SCHEME_CD06) {
            for (int l = 0; l < nl; ++l) ri[l] = cd06_d1_row(f + l, s, n, i, op->periodic, op->onebydx);
        } else if (op->scheme == SCHEME_CD10 && kind == KIND_D1) {
            for (int l = 0; l < nl; ++l) ri[l] = cd10_d1_row(f + l, s, n, i, op->periodic, bc1, bcn, op->onebydx);
        } else if (op->scheme == SCHEME_CD10) {
            for (int l = 0; l < nl; ++l) ri[l] = cd10_d2_row(f + l, s, n, i, op->periodic, bc1, bcn, op->onebydx2);
        } else {
            for (int l = 0; l < nl; ++l) ri[l] = cf90_row(f + l, s, n, i, op->periodic, bc1, bcn);
        }
    }
}

#define Y(i) y[(ptrdiff_t)((i)-1) * s + l]

/* cd06.F90:345-429  SolveX/Y/ZLU1. */
static inline __attribute__((always_inline)) void solve_cd06_lu(const double *LU, int n, double *y, int nl,
                                                                ptrdiff_t s, double *sum1)
{
    for (int l = 0; l < nl; ++l) sum1[l] = T(LU, 1, 2) * Y(1);
    for (int i = 2; i <= n - 1; ++i)
        for (int l = 0; l < nl; ++l) {
            Y(i) = Y(i) - T(LU, i, 1) * Y(i - 1);
            sum1[l] = sum1[l] + T(LU, i, 2) * Y(i);
        }
    for (int l = 0; l < nl; ++l) {
        Y(n) = Y(n) - sum1[l];
        Y(n) = Y(n) * T(LU, n, 3);
        Y(n - 1) = Y(n - 1) * T(LU, n - 1, 3) - Y(n) * T(LU, n - 1, 5);
    }
    for (int i = n - 2; i >= 1; --i)
        for (int l = 0; l < nl; ++l) Y(i) = Y(i) * T(LU, i, 3) - Y(i + 1) * T(LU, i, 4) - Y(n) * T(LU, i, 5);
}

/* cd06.F90:432-490  SolveX/Y/ZTri1. */
static inline __attribute__((always_inline)) void solve_cd06_tri(const double *Tri, int n, double *y, int nl,
                                                                 ptrdiff_t s)
{
    for (int l = 0; l < nl; ++l) Y(1) = Y(1) * T(Tri, 1, 2);
    for (int i = 2; i <= n; ++i)
        for (int l = 0; l < nl; ++l) Y(i) = Y(i) * T(Tri, i, 2) - Y(i - 1) * T(Tri, i, 1);
    for (int i = n - 1; i >= 1; --i)
        for (int l = 0; l < nl; ++l) Y(i) = Y(i) - T(Tri, i, 3) * Y(i + 1);
}

/* cd10.F90:712-821 / 904-1013, cf90.F90:421-530  SolveX/Y/ZLU{,1,2}. */
static inline __attribute__((always_inline)) void solve_penta_lu(const double *LU, int n, double *y, int nl,
                                                                 ptrdiff_t s, double *sum1, double *sum2)
{
    for (int l = 0; l < nl; ++l) {
        Y(2) = Y(2) - T(LU, 2, 1) * Y(1);
        sum1[l] = T(LU, 1, 3) * Y(1) + T(LU, 2, 3) * Y(2);
        sum2[l] = T(LU, 1, 4) * Y(1) + T(LU, 2, 4) * Y(2);
    }
    for (int i = 3; i <= n - 2; ++i)
        for (int l = 0; l < nl; ++l) {
            Y(i) = Y(i) - T(LU, i, 1) * Y(i - 1) - T(LU, i, 2) * Y(i - 2);
            sum1[l] = sum1[l] + T(LU, i, 3) * Y(i);
            sum2[l] = sum2[l] + T(LU, i, 4) * Y(i);
        }
    for (int l = 0; l < nl; ++l) {
        Y(n - 1) = Y(n - 1) - sum1[l];
        Y(n) = (Y(n) - sum2[l] - T(LU, n - 1, 4) * Y(n - 1)) * T(LU, n, 5);
        Y(n - 1) = (Y(n - 1) - T(LU, n - 1, 9) * Y(n)) * T(LU, n - 1, 5);
        Y(n - 2) = (Y(n - 2) - T(LU, n - 2, 8) * Y(n - 1) - T(LU, n - 2, 9) * Y(n)) * T(LU, n - 2, 5);
        Y(n - 3) = (Y(n - 3) - T(LU, n - 3, 6) * Y(n - 2) - T(LU, n - 3, 8) * Y(n - 1) - T(LU, n - 3, 9) * Y(n)) *
                   T(LU, n - 3, 5);
    }
    for (int i = n - 4; i >= 1; --i)
        for (int l = 0; l < nl; ++l)
            Y(i) = (Y(i) - T(LU, i, 6) * Y(i + 1) - T(LU, i, 7) * Y(i + 2) - T(LU, i, 8) * Y(n - 1) -
                    T(LU, i, 9) * Y(n)) *
                   T(LU, i, 5);
}

/* cd10.F90:823-901 / 1016-1095, cf90.F90:532-608  SolveX/Y/ZPenta{,1,2}. */
static inline __attribute__((always_inline)) void solve_penta(const double *P, int n, double *y, int nl,
                                                              ptrdiff_t s)
{
    for (int l = 0; l < nl; ++l) Y(2) = Y(2) - T(P, 2, 8) * Y(1);
    for (int i = 3; i <= n; ++i)
        for (int l = 0; l < nl; ++l) Y(i) = Y(i) - T(P, i, 9) * Y(i - 2) - T(P, i, 8) * Y(i - 1);
    for (int l = 0; l < nl; ++l) {
        Y(n) = Y(n) * T(P, n, 7);
        Y(n - 1) = Y(n - 1) * T(P, n - 1, 7) - T(P, n - 1, 10) * Y(n);
    }
    for (int i = n - 2; i >= 1; --i)
        for (int l = 0; l < nl; ++l)
            Y(i) = Y(i) * T(P, i, 7) - Y(i + 2) * T(P, i, 5) * T(P, i, 7) - Y(i + 1) * T(P, i, 10);
}
#undef Y

/* One block: RHS then the solve that the reference's dd, d2d and filter dispatch
 * selects (cd06.F90:775-839, cd10.F90:2029-2447, cf90.F90:1020-1228). */
static inline __attribute__((always_inline)) void apply_block(const oracle_op *op, int kind, const double *f,
                                                              double *df, int nl, ptrdiff_t s, int bc1, int bcn,
                                                              double *tmp1, double *tmp2)
{
    const int n = op->n;
    rhs_block(op, kind, f, df, nl, s, bc1, bcn);
    if (op->scheme == SCHEME_CD06) {
        if (op->periodic) solve_cd06_lu(op->LU1, n, df, nl, s, tmp1);
        else solve_cd06_tri(op->Tri1, n, df, nl, s);
    } else if (op->periodic) {
        const double *LU = (op->scheme == SCHEME_CD10 && kind == KIND_D2) ? op->LU2 : op->LU1;
        solve_penta_lu(LU, n, df, nl, s, tmp1, tmp2);
    } else {
        const double *P = (op->scheme == SCHEME_CD10 && kind == KIND_D2) ? op->penta2[pidx(bc1, bcn)]
                                                                          : op->penta1[pidx(bc1, bcn)];
        solve_penta(P, n, df, nl, s);
    }
}

/* Line-block worker for axis 1 (x): lines are the (j,k) pairs. */
static void apply_x(const oracle_op *op, int kind, const double *f, double *df, long nlines, int bc1, int bcn,
                    int nthreads)
{
    const int n = op->n;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
    for (long line = 0; line < nlines; ++line) {
        double t1, t2;
        apply_block(op, kind, f + line * n, df + line * n, 1, 1, bc1, bcn, &t1, &t2);
    }
}

/* Plane-slice worker for axes 2 and 3: `nplanes` planes of `nl` contiguous
 * lines, element stride s, plane stride ps.  Work is split over planes and,
 * when there are few planes, over chunks of lines within a plane. */
static void apply_planes(const oracle_op *op, int kind, const double *f, double *df, long nplanes, long nl,
                         ptrdiff_t s, ptrdiff_t ps, int bc1, int bcn, int nthreads)
{
    long chunks = 1;
    if (nthreads > 1 && nplanes < 4L * nthreads) {
        chunks = (4L * nthreads + nplanes - 1) / nplanes;
        if (chunks > nl) chunks = nl;
    }
    const long items = nplanes * chunks;
    const long cl = (nl + chunks - 1) / chunks;
#pragma omp parallel num_threads(nthreads) if (nthreads > 1)
    {
        double *t1 = malloc(sizeof(double) * (size_t)cl);
        double *t2 = malloc(sizeof(double) * (size_t)cl);
#pragma omp for schedule(static)
        for (long it = 0; it < items; ++it) {
            long pl = it / chunks, c = it % chunks;
            long l0 = c * cl, l1 = l0 + cl < nl ? l0 + cl : nl;
            if (l1 <= l0) continue;
            apply_block(op, kind, f + pl * ps + l0, df + pl * ps + l0, (int)(l1 - l0), s, bc1, bcn, t1, t2);
        }
        free(t1);
        free(t2);
    }
}

/* ------------------------------------------------------------------------- */
/* Public entry: the reference's dd1/dd2/dd3, d2d1/2/3 and filter1/2/3.      */
/*   kind: 1 = first derivative, 2 = second derivative, 0 = filter.          */
/*   axis: 1, 2, 3.  Shapes (n,na,nb) / (na,n,nb) / (na,nb,n).               */
/*   bc1/bcn are the optional arguments (ignored by cd06, whose closures come */
/*   from init; ignored when periodic).                                       */
/* Returns 0, or 324 (the reference's GracefulExit code) for a bad bc, or    */
/* -2 for an operator the reference does not implement (cd06 d2, cf90 d1).   */
/* ------------------------------------------------------------------------- */
int oracle_apply(const oracle_op *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                 int bcn, int nthreads)
{
    const int n = op->n;
    if (op->scheme == SCHEME_CD06 && kind != KIND_D1) return -2;
    if (op->scheme == SCHEME_CF90 && kind != KIND_FILTER) return -2;
    if (op->scheme == SCHEME_CD10 && kind == KIND_FILTER) return -2;
    const long total = (long)n * na * nb;
    if (n == 1) {
        /* cd06.F90:781-784, cd10.F90:2037-2040 (zero); cf90.F90:1028-1031 (copy) */
        for (long q = 0; q < total; ++q) df[q] = (kind == KIND_FILTER) ? f[q] : 0.0;
        return 0;
    }
    if (op->scheme != SCHEME_CD06) {
        if ((bc1 != 0 && bc1 != 1 && bc1 != -1) || (bcn != 0 && bcn != 1 && bcn != -1)) return 324;
    } else {
        bc1 = op->bc1;
        bcn = op->bcn;
    }
    if (nthreads < 1) nthreads = 1;
    if (axis == 1) apply_x(op, kind, f, df, na * nb, bc1, bcn, nthreads);
    else if (axis == 2) apply_planes(op, kind, f, df, nb, na, na, na * (long)n, bc1, bcn, nthreads);
    else apply_planes(op, kind, f, df, 1, na * nb, na * nb, 0, bc1, bcn, nthreads);
    return 0;
}

/* cf90.F90:1230-1251  filter3_CMPLX.  A complex (na,nb,n) field stores (re, im)
 * pairs, so to the stencil and the solve -- which act on each part alone -- it
 * is the real (2*na,nb,n) field.  The right-hand side takes the closures
 * (bc1, bcn) (ComputeZRHS_CMPLX, CF90_files/ComputeZRHS_common.F90); the solve
 * always uses penta_nn (SolveZPenta_CMPLX, CF90_files/SolveZPenta_common.F90).
 * Returns 0; -3 for a periodic object (it has no penta_nn: the reference reads
 * an unallocated array); 324 for a bc outside {0, 1, -1} (the reference does
 * not check and leaves those rows unset). */
int oracle_filter3_complex(const oracle_op *op, const double *f, double *df, long na, long nb, int bc1, int bcn,
                           int nthreads)
{
    const int n = op->n;
    const long nl = 2 * na * nb;
    if (op->scheme != SCHEME_CF90) return -2;
    if (n == 1) {
        for (long q = 0; q < nl; ++q) df[q] = f[q];
        return 0;
    }
    if (op->periodic) return -3;
    if ((bc1 != 0 && bc1 != 1 && bc1 != -1) || (bcn != 0 && bcn != 1 && bcn != -1)) return 324;
    if (nthreads < 1) nthreads = 1;
    const long chunks = nthreads > 1 ? 4L * nthreads : 1;
    const long cl = (nl + chunks - 1) / chunks;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
    for (long c = 0; c < chunks; ++c) {
        const long l0 = c * cl, l1 = l0 + cl < nl ? l0 + cl : nl;
        if (l1 <= l0) continue;
        rhs_block(op, KIND_FILTER, f + l0, df + l0, (int)(l1 - l0), nl, bc1, bcn);
        solve_penta(op->penta1[pidx(0, 0)], n, df + l0, (int)(l1 - l0), nl);
    }
    return 0;
}

int oracle_n(const oracle_op *op) { return op->n; }

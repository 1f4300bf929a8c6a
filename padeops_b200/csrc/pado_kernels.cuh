// pado_kernels.cuh -- the line kernel: explicit stencil fused with the banded
// solve, for one line family (all lines of a field along one axis).
//
// A CTA owns a tile of L lines and cuts every line into S segments; thread
// (l, s) = line lane l (fastest), segment s.  Lanes are lines, so for lines
// along a strided axis (y, z) a warp's accesses to one row are contiguous in
// memory.  The input of a tile comes from one of three places (IN):
//   IN_GLOBAL  straight from global memory into registers (strided lines)
//   IN_ROWS    a shared-memory tile [n][L] (strided lines), filled by cp.async
//   IN_LINES   a shared-memory tile [L][P], P odd (contiguous x lines)
// and results go straight from registers to global memory.  The persistent
// kernel prefetches the next tile with cp.async while the current one runs
// its chains and backward sweep.  Per tile:
//
//   fwd      stencil rows of the segment (reference grouping), then the local
//            forward recurrence with zero incoming state, in registers
//   chainF   every thread: its incoming state from the W segments before it
//            (precomputed transfer products); per line, the cyclic border
//            unknowns
//   bwd      local backward recurrence (forward values corrected on the fly)
//   chainB   every thread: its incoming state from the W segments after it
//   fin      x = local + incoming-state corrections -> df
//
// The adjoint kernel runs the transposed sweep first and the transposed
// stencil last (through the tile).  Each phase is a __host__ __device__
// function so the tests run the same code on the CPU.
#pragma once

#include "pado_common.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace pado {

constexpr int KMAXM = 64;  // longest segment (MAXM of pado_tables.h)
constexpr int KMAXSLOT = 48;  // thread slots per line (segments plus warp padding)
constexpr unsigned char SLOT_IDLE = 0xff;
constexpr int KCT_NF = 4;  // border-sum weights per segment (CT_NF of pado_tables.h)

// Parameters of one launch (passed by value).
struct KParams {
    const double *in;
    double *out;
    long long nlines;      // lines in the family
    long long line_ia;     // base(q) = (q % line_ia) + (q / line_ia) * line_oc
    long long line_oc;
    long long stride;      // element stride along a line
    int n, nb, nbord, P;   // line length, banded rows, border rows, tile pitch
    int S;                 // segments per line
    int L;                 // lines per CTA
    int bc1, bcn;
    const double *tab;     // [nb][T_NF]
    const double *ctab;    // [S][KCT_NF] border-sum weights G1, G2
    const double *xtab;    // packed transfer products Phi(s, s-d), Psi(s, s+d) (4 doubles each)
    int W;                 // largest coupling window
    int xd;                // doubles in xtab
    const double *bt;      // adjoint: transposed stencil blocks (bounded)
    double mb[4];
    double taps[9];        // adjoint: interior transposed taps
    RhsCoef rc;
    // constant-coefficient interior (see Interior in pado_tables.h)
    unsigned int_mask;     // bit s: segment s takes the constant-coefficient path
    unsigned spk_mask;     // bit s: ... and adds its rows' cyclic spike terms (per-row table)
    double kc[8];          // alpha, c1, c2, gamma, d1, d2, delta
    double pu[KMAXM], pv[KMAXM], ps[KMAXM], pt[KMAXM];  // unit responses, rows 0..m-1
    unsigned char sperm[KMAXSLOT];  // thread slot -> segment, SLOT_IDLE for an idle slot
    int nslots;                     // slots per line (S, or more when warps are padded)
    int border_slot;                // idle slot whose threads solve a cyclic line's border
                                    // unknowns (-1: segment 0's threads do)
    unsigned short sstart[33];  // segment s = rows [sstart[s], sstart[s+1])
    unsigned char wf[32], wb[32];    // coupling window of each segment (forward, backward)
    unsigned short xof[32], xob[32]; // first xtab block of each segment's forward / backward list
    const double *rtab;    // cyclic: (R1, R2) per row for rows [0, ie) then [je, nb) (streaming kernel)
    int ie, je;
    // how results reach df (OutMode): stored, scaled by out_alpha, or
    // out_alpha * result added to df
    int out_mode;
    double out_alpha;
};

enum OutMode { OUT_STORE = 0, OUT_SCALE = 1, OUT_ACC = 2 };

// One result x to its place p in df, through the launch's output mode.
PADO_HD PADO_INLINE void out_put(const KParams &kp, double *p, double x)
{
    if (kp.out_mode == OUT_ACC) *p = fma(kp.out_alpha, x, *p);
    else if (kp.out_mode == OUT_SCALE) *p = kp.out_alpha * x;
    else *p = x;
}

// Staged response row of banded row i (i < ie or i >= je).
PADO_HD PADO_INLINE const double *resp_row(const KParams &kp, const double *rtab, int i)
{
    return rtab + (size_t)(i < kp.ie ? i : kp.ie + (i - kp.je)) * 2;
}
PADO_HD PADO_INLINE int resp_rows(const KParams &kp) { return kp.ie + (kp.nb - kp.je); }

// Segment of thread slot `slot` (= tid / L), or -1 for an idle slot.
PADO_HD PADO_INLINE int slot_segment(const KParams &kp, int slot)
{
    return (slot < kp.nslots && kp.sperm[slot] != SLOT_IDLE) ? (int)kp.sperm[slot] : -1;
}

PADO_HD PADO_INLINE int seg_start(const KParams &kp, int s) { return kp.sstart[s]; }
PADO_HD PADO_INLINE int seg_len(const KParams &kp, int s) { return kp.sstart[s + 1] - kp.sstart[s]; }
PADO_HD PADO_INLINE long long line_base(const KParams &kp, long long q)
{
    return (q % kp.line_ia) + (q / kp.line_ia) * kp.line_oc;
}

// Shared-memory carve-up (doubles).  The tile is only allocated by kernels
// that use it.  etab/toff: the per-row table of the segments that read it,
// staged in shared memory by the persistent kernel (null: read kp.tab).
struct Smem {
    double *buf4;        // [S][4][L]  forward summaries, later backward summaries
    double *buf2;        // [S][2][L]  forward incoming states, later backward ones
    double *eb;          // [L][4]     border unknowns E (0..1) and border rhs (2..3)
    double *ctab;        // [S][KCT_NF] border-sum weights
    double *xtab;        // packed transfer products (xd doubles)
    double *tile;        // [L][P] or [n][L]
    const double *etab;  // packed table rows of the segments that read the table
    const int *toff;     // [S] first packed row of each segment
    const double *ktab;  // packed spike values (k1, k2) of the spiky segments' rows
    const double *rtab;  // staged (R1, R2) rows (streaming kernel)
};

// tile_doubles: 0 (no tile), L*P ([L][P] tile) or n*L ([n][L] tile)
PADO_HD PADO_INLINE size_t smem_doubles(int L, int S, int xd, size_t tile_doubles)
{
    return (size_t)S * L * 6 + (size_t)L * 4 + (size_t)S * KCT_NF + (size_t)xd + tile_doubles;
}

PADO_HD PADO_INLINE Smem carve(double *base, int L, int P, int S, int xd)
{
    Smem sm;
    sm.buf4 = base;
    sm.buf2 = sm.buf4 + (size_t)S * L * 4;
    sm.eb = sm.buf2 + (size_t)S * L * 2;
    sm.ctab = sm.eb + (size_t)L * 4;
    sm.xtab = sm.ctab + (size_t)S * KCT_NF;
    sm.tile = sm.xtab + (size_t)xd;
    sm.etab = nullptr;
    sm.toff = nullptr;
    sm.ktab = nullptr;
    sm.rtab = nullptr;
    (void)P;
    return sm;
}

// Per-segment summaries, segment-major so that the lanes (lines) of a warp
// touch consecutive doubles: value k of segment s, line l at p[k * L].
PADO_HD PADO_INLINE double *sum4(const Smem &sm, int L, int s, int l) { return sm.buf4 + (size_t)s * 4 * L + l; }
PADO_HD PADO_INLINE double *sum2(const Smem &sm, int L, int s, int l) { return sm.buf2 + (size_t)s * 2 * L + l; }

// Where one line's input comes from and its output goes (set per thread by
// the kernel driver): row r of the input is src[r * ss], of the output
// dst[r * ds].  live: the line exists (the last tile may be partial).
struct LineIO {
    const double *src;
    long long ss;
    double *dst;
    long long ds;
    bool live;
    bool tile = false;  // dst is the shared-memory tile (results reach df later)
};

// Per-thread segment values: M rows plus the 8-row stencil window margin.
template <int M>
struct Regs {
    double r[M + 8];
};

struct Dbl2 {
    double x, y;
};

#ifdef __CUDA_ARCH__
#define PADO_LDG(p) __ldg(p)
__device__ __forceinline__ Dbl2 ldg2(const double *p)
{
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return Dbl2{v.x, v.y};
}
#else
#define PADO_LDG(p) (*(p))
inline Dbl2 ldg2(const double *p) { return Dbl2{p[0], p[1]}; }
#endif

// ---------------------------------------------------------------------------
// Tile load / store for contiguous lines (x): the L lines of a tile are one
// contiguous run of L*n doubles; all threads stream it with independent loads.
// ---------------------------------------------------------------------------
PADO_HD PADO_INLINE void tile_load(const KParams &kp, const Smem &sm, long long q0, int tid, int nthreads)
{
    const int n = kp.n, L = kp.L, P = kp.P;
    const int nl = (int)(kp.nlines - q0 < L ? kp.nlines - q0 : L);
    const int total = nl * n;
    const double *src = kp.in + line_base(kp, q0);
    // element e = tid + k*nthreads sits at (line l, row r); advance (l, r) without divisions
    int l = tid / n, r = tid - (tid / n) * n;
    const int dl = nthreads / n, dr = nthreads - dl * n;
    for (int e = tid; e < total; e += 4 * nthreads) {
        double v[4];
        int ls[4], rs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int ee = e + u * nthreads;
            v[u] = ee < total ? src[ee] : 0.0;
            ls[u] = l;
            rs[u] = r;
            l += dl;
            r += dr;
            if (r >= n) {
                r -= n;
                ++l;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (e + u * nthreads < total) sm.tile[(size_t)ls[u] * P + rs[u]] = v[u];
    }
}

PADO_HD PADO_INLINE void tile_store(const KParams &kp, const Smem &sm, long long q0, int tid, int nthreads)
{
    const int n = kp.n, L = kp.L, P = kp.P;
    const int nl = (int)(kp.nlines - q0 < L ? kp.nlines - q0 : L);
    const int total = nl * n;
    double *dst = kp.out + line_base(kp, q0);
    int l = tid / n, r = tid - (tid / n) * n;
    const int dl = nthreads / n, dr = nthreads - dl * n;
    for (int e = tid; e < total; e += nthreads) {
        out_put(kp, dst + e, sm.tile[(size_t)l * P + r]);
        l += dl;
        r += dr;
        if (r >= n) {
            r -= n;
            ++l;
        }
    }
}

// Closure rows are rare (first/last few rows of a bounded line): evaluate
// them out of line from memory (the tile, or global memory with a stride),
// one function per stencil so that each holds only its own closures.
template <int RK>
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
    double
    closure_row_noinline(const RhsCoef *rc, const double *line, long long stride, int n, int row, int bc1, int bcn)
{
    return rhs_closure_row(RK, rc->c, line, stride, n, row, bc1, bcn);
}

// Transposed stencil at one column j of a bounded line from explicit blocks.
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
    double
    bt_column_noinline(const double *bt, const double *line, int n, int j)
{
    double acc = 0.0;
    if (n <= 32) {
        const double *w = bt + (size_t)j * n;
        for (int i = 0; i < n; ++i) acc += PADO_LDG(w + i) * line[i];
        return acc;
    }
    if (j < 8) {
        const double *w = bt + (size_t)j * 12;
        for (int i = 0; i < 12; ++i) acc += PADO_LDG(w + i) * line[i];
    } else {
        const double *w = bt + (size_t)(8 + j - (n - 8)) * 12;
        for (int i = 0; i < 12; ++i) acc += PADO_LDG(w + i) * line[n - 12 + i];
    }
    return acc;
}

enum InputSource { IN_GLOBAL = 0, IN_ROWS = 1, IN_LINES = 2 };

// Table rows of segment s (first row a) in global memory (T_NF fields per row).
PADO_HD PADO_INLINE const double *seg_table(const KParams &kp, const Smem &sm, int s, int a)
{
    (void)sm;
    (void)s;
    return kp.tab + (size_t)a * T_NF;
}
// ... and in the streaming kernel's staged copy (E_NF fields per row).
PADO_HD PADO_INLINE const double *seg_etab(const Smem &sm, int s) { return sm.etab + (size_t)sm.toff[s] * E_NF; }

// Table loads: read-only cache for global memory, plain loads for shared memory.
template <bool STAGED>
PADO_HD PADO_INLINE double tld(const double *p)
{
    if (STAGED) return *p;
    return PADO_LDG(p);
}
template <bool STAGED>
PADO_HD PADO_INLINE Dbl2 tld2(const double *p)
{
    if (STAGED) return Dbl2{p[0], p[1]};
    return ldg2(p);
}

// Cyclic spike values of the rows of segment s (first row a): the compact
// staged copy (k1, k2, e1, e2 per row) or the full global table.
template <bool STAGED>
struct SpikeRows {
    static constexpr int STRIDE = STAGED ? 2 : T_NF;
    static constexpr int K1 = STAGED ? 0 : T_K1, K2 = STAGED ? 1 : T_K2, E1 = T_E1, E2 = T_E2;  // E: global only
    static PADO_HD PADO_INLINE const double *rows(const KParams &kp, const Smem &sm, int s, int a)
    {
        return STAGED ? sm.ktab + (size_t)sm.toff[s] * 2 : kp.tab + (size_t)a * T_NF;
    }
};

template <int RK, bool PER, bool ADJ, int M, int IN>
struct LineKernel {
    static constexpr bool CYC = PER;
    static constexpr bool ORDER2 = RK != RHS_CD06_D1;  // tridiagonal (cd06) sweeps have no second lag
    // only the bounded cd06 (Thomas) sweep scales its input (alpha != 1), and
    // only its adjoint scales the output (delta != 1)
    static constexpr bool HAS_ALPHA = RK == RHS_CD06_D1 && !PER && !ADJ;
    static constexpr bool HAS_DELTA = RK == RHS_CD06_D1 && !PER && ADJ;
    static_assert(M <= KMAXM, "segment longer than the response tables");

    static PADO_HD PADO_INLINE bool fast(const KParams &kp, int s) { return (kp.int_mask >> s) & 1u; }

    // ---- constant-coefficient interior segment: stencil + forward sweep ----
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fwd_fast(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s,
                                             const LineIO &io)
    {
        const int a = seg_start(kp, s);
        const long long gs = io.ss;
        if (!ADJ) {
            const double *p = io.src + (long long)(a - 4) * gs;
#pragma unroll
            for (int j = 0; j < M + 8; ++j) R.r[j] = p[(long long)j * gs];
#pragma unroll
            for (int t = 0; t < M; ++t) R.r[t] = rhs_interior(RK, PER, kp.rc.c, &R.r[t]);
        } else {
            const double *p = io.src + (long long)a * gs;
#pragma unroll
            for (int t = 0; t < M; ++t) R.r[t] = p[(long long)t * gs];
        }
        const double al = kp.kc[0], c1 = kp.kc[1], c2 = kp.kc[2];
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0;
        const bool spk = CYC && ((kp.spk_mask >> s) & 1u);
        using SR = SpikeRows<STAGED>;
        const double *tb = SR::rows(kp, sm, s, a);
#pragma unroll
        for (int t = 0; t < M; ++t) {
            double z = HAS_ALPHA ? al * R.r[t] : R.r[t];
            if (ORDER2) z -= c2 * z2;
            z -= c1 * z1;
            R.r[t] = z;
            if (CYC && spk) {
                const double *tr = tb + (size_t)t * SR::STRIDE;
                s1 += tld<STAGED>(tr + SR::K1) * z;
                if (ORDER2) s2 += tld<STAGED>(tr + SR::K2) * z;
            }
            z2 = z1;
            z1 = z;
        }
        summarize_fwd<STAGED>(kp, sm, l, s, z1, z2, s1, s2);
    }

    // forward summary of segment s: end values y = (z1, z2) and, for a cyclic
    // line, its share of the border sums (local sums + G_s . y)
    template <bool STAGED>
    static PADO_HD PADO_INLINE void summarize_fwd(const KParams &kp, const Smem &sm, int l, int s, double z1,
                                                  double z2, double s1, double s2)
    {
        const int L = kp.L;
        double *o = sum4(sm, L, s, l);
        o[0] = z1;
        o[L] = z2;
        if (CYC) {
            const double *g = (STAGED ? sm.ctab : kp.ctab) + (size_t)s * KCT_NF;
            const Dbl2 g1 = tld2<STAGED>(g), g2 = tld2<STAGED>(g + 2);
            o[2 * L] = s1 + g1.x * z1 + g1.y * z2;
            o[3 * L] = s2 + g2.x * z1 + g2.y * z2;
        }
    }

    // ---- constant-coefficient interior segment: backward sweep -------------
    // forward values = local + P1*U + P2*V (the incoming state's response)
    template <bool STAGED>
    static PADO_HD PADO_INLINE void bwd_fast(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const double *st = sum2(sm, kp.L, s, l);
        const double ga = kp.kc[3], d1 = kp.kc[4], d2 = kp.kc[5];
        const double P1 = st[0], P2 = st[kp.L];
        const bool spk = CYC && ((kp.spk_mask >> s) & 1u);
        const double E1 = CYC ? sm.eb[(size_t)l * 4 + 0] : 0.0, E2 = CYC ? sm.eb[(size_t)l * 4 + 1] : 0.0;
        using SR = SpikeRows<STAGED>;
        const double *tb = SR::rows(kp, sm, s, seg_start(kp, s));
        double x1 = 0.0, x2 = 0.0;
#pragma unroll
        for (int t = M - 1; t >= 0; --t) {
            double z = R.r[t] + P1 * kp.pu[t];
            if (ORDER2) z += P2 * kp.pv[t];
            double x = ga * z;
            if (CYC && spk) {
                const double *tr = tb + (size_t)t * SR::STRIDE;
                x -= tld<STAGED>(tr + SR::E1) * E1;
                if (ORDER2) x -= tld<STAGED>(tr + SR::E2) * E2;
            }
            if (ORDER2) x -= d2 * x2;
            x -= d1 * x1;
            R.r[t] = x;
            x2 = x1;
            x1 = x;
        }
        double *o = sum4(sm, kp.L, s, l);
        o[0] = x1;
        o[kp.L] = x2;
    }

    // ---- constant-coefficient interior segment: corrections + output ------
    static PADO_HD PADO_INLINE void fin_fast(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s,
                                             const LineIO &io)
    {
        const int a = seg_start(kp, s);
        const double *st = sum2(sm, kp.L, s, l);
        const double de = kp.kc[6];
        const double Q1 = st[0], Q2 = st[kp.L];
        double *p = io.dst + (long long)a * io.ds;
        if (!io.tile && kp.out_mode != OUT_STORE) {
#pragma unroll
            for (int t = 0; t < M; ++t) {
                double x = R.r[t] + Q1 * kp.ps[t];
                if (ORDER2) x += Q2 * kp.pt[t];
                if (HAS_DELTA) x *= de;
                out_put(kp, p + (long long)t * io.ds, x);
            }
            return;
        }
#pragma unroll
        for (int t = 0; t < M; ++t) {
            double x = R.r[t] + Q1 * kp.ps[t];
            if (ORDER2) x += Q2 * kp.pt[t];
            if (HAS_DELTA) x *= de;
            p[(long long)t * io.ds] = x;
        }
    }

    static PADO_HD PADO_INLINE int wrap(int row, int n) { return row < 0 ? row + n : (row >= n ? row - n : row); }

    // ---- phase fwd: right-hand side (primal) + local forward sweep ---------
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fwd(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s, const LineIO &io)
    {
        const int n = kp.n, nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;  // banded rows of this segment
        const bool live = io.live;
        const double *gline = io.src;
        const long long gs = io.ss;
        if (fast(kp, s)) {
            fwd_fast<STAGED>(kp, sm, R, l, s, io);
            return;
        }
        if (!ADJ) {
            // Closure rows of a bounded line (first/last segment only) are
            // evaluated first, out of line, while few registers are live.
            const int cr = closure_rows(RK);
            double cv[4] = {0.0, 0.0, 0.0, 0.0};
            const bool first = !PER && s == 0, last = !PER && s == kp.S - 1;
            if (first || last) {
                for (int k = 0; k < cr; ++k) {
                    if (live && first) cv[k] = closure_row_noinline<RK>(&kp.rc, gline, gs, n, k, kp.bc1, kp.bcn);
                }
            }
            double cl[4] = {0.0, 0.0, 0.0, 0.0};
            if (last) {
                for (int k = 0; k < cr; ++k)
                    if (live) cl[k] = closure_row_noinline<RK>(&kp.rc, gline, gs, n, n - cr + k, kp.bc1, kp.bcn);
            }
            // window rows a-4 .. a+len+3, all loads issued up front; the
            // stencil result of row t overwrites R.r[t], the oldest window entry
#pragma unroll
            for (int j = 0; j < M + 8; ++j) {
                const int row = a - 4 + j;
                const bool ok = live && j < len + 8 && (PER || (row >= 0 && row < n));
                R.r[j] = ok ? gline[(long long)(PER ? wrap(row, n) : row) * gs] : 0.0;
            }
#pragma unroll
            for (int t = 0; t < M; ++t)
                if (t < len) R.r[t] = rhs_interior(RK, PER, kp.rc.c, &R.r[t]);
            if (first) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (k < cr && k < len) R.r[k] = cv[k];
            }
            if (last) {
#pragma unroll
                for (int t = 0; t < M; ++t) {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k < cr && t == len - cr + k) R.r[t] = cl[k];
                }
            }
        } else {
#pragma unroll
            for (int t = 0; t < M; ++t)
                if (t < len) R.r[t] = live ? gline[(long long)(a + t) * gs] : 0.0;
        }
        // local forward sweep with zero incoming state; the coefficients of
        // eight rows are read before their recurrence steps
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0;
        const double *tb = seg_table(kp, sm, s, a);
        if (lenb > 0) {
#pragma unroll
            for (int c0 = 0; c0 < M; c0 += 8) {
                Dbl2 cc[8], ak[8];
                double k2[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int tt = c0 + u < lenb ? c0 + u : lenb - 1;
                    const double *tr = tb + (size_t)tt * T_NF;
                    cc[u] = tld2<STAGED>(tr + T_C1);
                    ak[u] = (HAS_ALPHA || CYC) ? tld2<STAGED>(tr + T_ALPHA) : Dbl2{1.0, 0.0};
                    k2[u] = (CYC && ORDER2) ? tld<STAGED>(tr + T_K2) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int t = c0 + u;
                    if (t < lenb) {
                        double z = HAS_ALPHA ? ak[u].x * R.r[t] : R.r[t];
                        if (ORDER2) z -= cc[u].y * z2;
                        z -= cc[u].x * z1;
                        R.r[t] = z;
                        if (CYC) {
                            s1 += ak[u].y * z;
                            if (ORDER2) s2 += k2[u] * z;
                        }
                        z2 = z1;
                        z1 = z;
                    }
                }
            }
        }
        summarize_fwd<STAGED>(kp, sm, l, s, z1, z2, s1, s2);
        if (CYC && s == kp.S - 1) {
            // border rows' right-hand sides (the last nbord rows of the line)
            double rb0 = 0.0, rb1 = 0.0;
#pragma unroll
            for (int t = 0; t < M; ++t) {
                if (t == lenb) rb0 = R.r[t];
                if (t == lenb + 1) rb1 = R.r[t];
            }
            sm.eb[(size_t)l * 4 + 2] = rb0;
            sm.eb[(size_t)l * 4 + 3] = rb1;
        }
    }

    // ---- phase chainF: forward incoming states + border ------------------
    // Every thread sums the transfers of the wf[s] segments before its own
    // (no serial walk over the segments); the thread of segment 0, whose
    // incoming state is zero, adds up the border sums of its line.
    static PADO_HD PADO_INLINE void chain_fwd(const KParams &kp, const Smem &sm, int l, int s)
    {
        const int L = kp.L, wf = kp.wf[s];
        // four independent partial sums so that the loads of four segments
        // are in flight together
        double P1[4] = {0.0, 0.0, 0.0, 0.0}, P2[4] = {0.0, 0.0, 0.0, 0.0};
        const double *xt = sm.xtab + (size_t)kp.xof[s] * 4;
        for (int d0 = 1; d0 <= wf; d0 += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int d = d0 + u;
                if (d <= wf) {
                    const double *y = sum4(sm, L, s - d, l);
                    const double *ph = xt + (size_t)(d - 1) * 4;
                    const double y0 = y[0], y1 = y[L];
                    P1[u] += ph[0] * y0 + ph[1] * y1;
                    P2[u] += ph[2] * y0 + ph[3] * y1;
                }
            }
        }
        double *st = sum2(sm, L, s, l);
        st[0] = (P1[0] + P1[1]) + (P1[2] + P1[3]);
        st[L] = (P2[0] + P2[1]) + (P2[2] + P2[3]);
        if (CYC && s == 0) {
            double g1[4] = {0.0, 0.0, 0.0, 0.0}, g2[4] = {0.0, 0.0, 0.0, 0.0};
            for (int j0 = 0; j0 < kp.S; j0 += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (j0 + u < kp.S) {
                        const double *c = sum4(sm, L, j0 + u, l);
                        g1[u] += c[2 * L];
                        g2[u] += c[3 * L];
                    }
                }
            }
            const double sg1 = (g1[0] + g1[1]) + (g1[2] + g1[3]), sg2 = (g2[0] + g2[1]) + (g2[2] + g2[3]);
            double *eb = sm.eb + (size_t)l * 4;
            const double u0 = eb[2] - sg1, u1 = eb[3] - sg2;
            if (kp.nbord == 1) {
                eb[0] = kp.mb[0] * u0;
                eb[1] = 0.0;
            } else {
                eb[0] = kp.mb[0] * u0 + kp.mb[1] * u1;
                eb[1] = kp.mb[2] * u0 + kp.mb[3] * u1;
            }
        }
    }

    // ---- phase bwd: local backward sweep ---------------------------------
    template <bool STAGED>
    static PADO_HD PADO_INLINE void bwd(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        if (fast(kp, s)) {
            bwd_fast<STAGED>(kp, sm, R, l, s);
            return;
        }
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        const double *st = sum2(sm, kp.L, s, l);
        const double P1 = st[0], P2 = st[kp.L];
        double E1 = 0.0, E2 = 0.0;
        if (CYC) {
            E1 = sm.eb[(size_t)l * 4 + 0];
            E2 = sm.eb[(size_t)l * 4 + 1];
        }
        const double *tb = seg_table(kp, sm, s, a);
        double x1 = 0.0, x2 = 0.0;
        if (lenb > 0) {
#pragma unroll
            for (int c0 = M - 4; c0 >= 0; c0 -= 4) {
                Dbl2 uv[4], gd[4], de[4];
                double e2[4];
#pragma unroll
                for (int u = 3; u >= 0; --u) {
                    const int tt = c0 + u < lenb ? c0 + u : lenb - 1;
                    const double *tr = tb + (size_t)tt * T_NF;
                    uv[u] = tld2<STAGED>(tr + T_U);
                    gd[u] = tld2<STAGED>(tr + T_GAMMA);
                    de[u] = tld2<STAGED>(tr + T_D2);
                    e2[u] = (CYC && ORDER2) ? tld<STAGED>(tr + T_E2) : 0.0;
                }
#pragma unroll
                for (int u = 3; u >= 0; --u) {
                    const int t = c0 + u;
                    if (t < lenb) {
                        double z = R.r[t] + P1 * uv[u].x;
                        if (ORDER2) z += P2 * uv[u].y;
                        double x = gd[u].x * z;
                        if (CYC) {
                            x -= de[u].y * E1;
                            if (ORDER2) x -= e2[u] * E2;
                        }
                        if (ORDER2) x -= de[u].x * x2;
                        x -= gd[u].y * x1;
                        R.r[t] = x;
                        x2 = x1;
                        x1 = x;
                    }
                }
            }
        }
        double *o = sum4(sm, kp.L, s, l);
        o[0] = x1;     // x at the segment's first row
        o[kp.L] = x2;  // and the second
    }

    // ---- phase chainB: backward incoming states ---------------------------
    static PADO_HD PADO_INLINE void chain_bwd(const KParams &kp, const Smem &sm, int l, int s)
    {
        const int L = kp.L, wb = kp.wb[s];
        double Q1[4] = {0.0, 0.0, 0.0, 0.0}, Q2[4] = {0.0, 0.0, 0.0, 0.0};
        const double *xt = sm.xtab + (size_t)kp.xob[s] * 4;
        for (int d0 = 1; d0 <= wb; d0 += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int d = d0 + u;
                if (d <= wb) {
                    const double *w = sum4(sm, L, s + d, l);
                    const double *ps_ = xt + (size_t)(d - 1) * 4;
                    const double w0 = w[0], w1 = w[L];
                    Q1[u] += ps_[0] * w0 + ps_[1] * w1;
                    Q2[u] += ps_[2] * w0 + ps_[3] * w1;
                }
            }
        }
        double *st = sum2(sm, L, s, l);
        st[0] = (Q1[0] + Q1[1]) + (Q1[2] + Q1[3]);
        st[L] = (Q2[0] + Q2[1]) + (Q2[2] + Q2[3]);
    }

    // ---- phase fin: corrected values -> the line's output -----------------
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fin(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s, const LineIO &io)
    {
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        const double *st = sum2(sm, kp.L, s, l);
        const double Q1 = st[0], Q2 = st[kp.L];
        if (!io.live) return;
        double *line = io.dst;
        const long long gs = io.ds;
        const bool xf = !io.tile && kp.out_mode != OUT_STORE;
        if (fast(kp, s)) {
            fin_fast(kp, sm, R, l, s, io);
            return;
        }
        const double *tb = seg_table(kp, sm, s, a);
#pragma unroll
        for (int t = 0; t < M; ++t) {
            if (t < lenb) {
                const double *tr = tb + (size_t)t * T_NF;
                const Dbl2 stt = tld2<STAGED>(tr + T_S);
                double x = R.r[t] + Q1 * stt.x;
                if (ORDER2) x += Q2 * stt.y;
                if (HAS_DELTA) x = tld<STAGED>(tr + T_DELTA) * x;
                if (xf) out_put(kp, line + (long long)(a + t) * gs, x);
                else line[(long long)(a + t) * gs] = x;
            }
        }
        if (CYC && s == kp.S - 1) {
            if (xf) {
                out_put(kp, line + (long long)nb * gs, sm.eb[(size_t)l * 4 + 0]);
                if (kp.nbord == 2) out_put(kp, line + (long long)(nb + 1) * gs, sm.eb[(size_t)l * 4 + 1]);
            } else {
                line[(long long)nb * gs] = sm.eb[(size_t)l * 4 + 0];
                if (kp.nbord == 2) line[(long long)(nb + 1) * gs] = sm.eb[(size_t)l * 4 + 1];
            }
        }
    }

    // ---- phase adjoint stencil: tile (A^{-T} g) -> registers (B^T ...) ----
    static PADO_HD PADO_INLINE void adj_stencil(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int n = kp.n;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const double *line = sm.tile + (size_t)l * kp.P;
        const int zone = n <= 32 ? n : 8;
#pragma unroll
        for (int j = 0; j < M + 8; ++j) {
            const int row = a - 4 + j;
            const bool ok = j < len + 8 && (PER || (row >= 0 && row < n));
            R.r[j] = ok ? line[PER ? wrap(row, n) : row] : 0.0;
        }
#pragma unroll
        for (int t = 0; t < M; ++t) {
            if (t < len) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < 9; ++k) acc += kp.taps[k] * R.r[t + k];
                R.r[t] = acc;
            }
        }
        if (!PER && (a < zone || a + len > n - zone)) {
            // boundary columns of B^T (explicit blocks), rare: first/last segments
#pragma unroll
            for (int t = 0; t < M; ++t) {
                const int j = a + t;
                if (t < len && (j < zone || j >= n - zone)) R.r[t] = bt_column_noinline(kp.bt, line, n, j);
            }
        }
    }

    // ---- phase adjoint output ----------------------------------------------
    static PADO_HD PADO_INLINE void adj_out(const KParams &kp, Regs<M> &R, int s, const LineIO &io)
    {
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        if (!io.live) return;
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < len) io.dst[(long long)(a + t) * io.ds] = R.r[t];
    }
};

// Phase schedule of one tile.  Phases are separated by a CTA barrier.
enum Phase {
    PH_LOAD = 0, PH_FWD, PH_CHAINF, PH_BWD, PH_CHAINB, PH_FIN, PH_ADJ_STENCIL, PH_ADJ_OUT, PH_STORE, NPHASES
};

// x lines (IN_LINES) load and store their tile cooperatively; the adjoint
// runs its transposed stencil after the solve
template <bool ADJ, int IN>
PADO_HD PADO_INLINE constexpr bool phase_used(int ph)
{
    return (ph == PH_LOAD || ph == PH_STORE) ? IN == IN_LINES && !(ph == PH_STORE && ADJ)
         : (ph == PH_ADJ_STENCIL || ph == PH_ADJ_OUT) ? ADJ
         : true;
}

// Line l of the tile starting at line q0, for the one-CTA-per-tile kernels:
// input from global memory (IN_GLOBAL) or the tile; the sweep's output goes
// to the [L][P] tile (adjoint, x lines) or to global memory.
template <bool ADJ, int IN>
PADO_HD PADO_INLINE LineIO tile_line_io(const KParams &kp, const Smem &sm, int l, long long q0)
{
    const long long q = q0 + l;
    LineIO io;
    io.live = q < kp.nlines;
    const long long base = line_base(kp, io.live ? q : 0);
    io.src = IN == IN_GLOBAL ? kp.in + base : IN == IN_ROWS ? sm.tile + l : sm.tile + (size_t)l * kp.P;
    io.ss = IN == IN_GLOBAL ? kp.stride : IN == IN_ROWS ? kp.L : 1;
    const bool out_tile = ADJ || IN == IN_LINES;
    io.dst = out_tile ? sm.tile + (size_t)l * kp.P : kp.out + base;
    io.ds = out_tile ? 1 : kp.stride;
    io.tile = out_tile;
    return io;
}

PADO_HD PADO_INLINE void stage_chain_table(const KParams &kp, const Smem &sm, int tid, int nthreads)
{
    for (int i = tid; i < kp.S * KCT_NF; i += nthreads) sm.ctab[i] = kp.ctab[i];
    for (int i = tid; i < kp.xd; i += nthreads) sm.xtab[i] = kp.xtab[i];
}

// One tile of kp.L lines on a CTA of nthreads threads (nthreads >= L*S;
// extra threads only help with the tile load).
template <int RK, bool PER, bool ADJ, int M, int IN>
PADO_HD PADO_INLINE void tile_phase(int phase, const KParams &kp, const Smem &sm, Regs<M> &R, long long q0, int tid,
                                    int nthreads)
{
    using K = LineKernel<RK, PER, ADJ, M, IN>;
    const int l = tid % kp.L, slot = tid / kp.L, s = slot_segment(kp, slot);
    const bool active = s >= 0;
    switch (phase) {
    case PH_LOAD: tile_load(kp, sm, q0, tid, nthreads); break;
    case PH_FWD:
        stage_chain_table(kp, sm, tid, nthreads);
        if (active) K::template fwd<false>(kp, sm, R, l, s, tile_line_io<ADJ, IN>(kp, sm, l, q0));
        break;
    case PH_CHAINF: if (active) K::chain_fwd(kp, sm, l, s); break;
    case PH_BWD: if (active) K::template bwd<false>(kp, sm, R, l, s); break;
    case PH_CHAINB: if (active) K::chain_bwd(kp, sm, l, s); break;
    case PH_FIN: if (active) K::template fin<false>(kp, sm, R, l, s, tile_line_io<ADJ, IN>(kp, sm, l, q0)); break;
    case PH_ADJ_STENCIL: if (active) K::adj_stencil(kp, sm, R, l, s); break;
    case PH_ADJ_OUT:
        if (active) {
            const long long q = q0 + l;
            const LineIO io{nullptr, 0, kp.out + line_base(kp, q < kp.nlines ? q : 0), kp.stride, q < kp.nlines};
            K::adj_out(kp, R, s, io);
        }
        break;
    default: tile_store(kp, sm, q0, tid, nthreads); break;
    }
}

// ---------------------------------------------------------------------------
// Asynchronous tile prefetch (persistent kernel).  Each thread copies its
// share of the tile with 8-byte cp.async; on the host it is a plain copy.
// ---------------------------------------------------------------------------
PADO_HD PADO_INLINE void copy8_async(double *dst_smem, const double *src)
{
#ifdef __CUDA_ARCH__
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
#else
    *dst_smem = *src;
#endif
}
PADO_HD PADO_INLINE void copy_async_commit()
{
#ifdef __CUDA_ARCH__
    asm volatile("cp.async.commit_group;\n" ::: "memory");
#endif
}
PADO_HD PADO_INLINE void copy_async_wait_all()
{
#ifdef __CUDA_ARCH__
    asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
}

PADO_HD PADO_INLINE void prefetch_l2(const void *p)
{
#ifdef __CUDA_ARCH__
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
#else
    (void)p;
#endif
}

template <int IN>
PADO_HD PADO_INLINE void tile_prefetch(const KParams &kp, const Smem &sm, long long q0, int tid, int nthreads)
{
    const int n = kp.n, L = kp.L;
    if (IN == IN_GLOBAL) {
        // strided lines read straight into registers: warm L2 with the tile's
        // rows (each row of L lines is contiguous when the lines are)
        const long long nl = kp.nlines - q0 < L ? kp.nlines - q0 : L;
        if (nl <= 0) return;
        const double *first = kp.in + line_base(kp, q0), *last = kp.in + line_base(kp, q0 + nl - 1);
        const long long span = (long long)(last - first) + 1;  // doubles from the first to the last line of a row
        const int per_row = (int)((span * 8 + 127) / 128);
        if (per_row > 8) {
            // lines not adjacent: one prefetch per line and row
            for (long long e = tid; e < nl * n; e += nthreads) {
                const long long l = e % nl, r = e / nl;
                prefetch_l2(kp.in + line_base(kp, q0 + l) + r * kp.stride);
            }
            return;
        }
        for (int e = tid; e < n * per_row; e += nthreads) {
            const int r = e / per_row, c = e - r * per_row;
            prefetch_l2(reinterpret_cast<const char *>(first + (long long)r * kp.stride) + c * 128);
        }
        return;
    }
    if (IN == IN_ROWS) {
        // thread (l, s) copies rows s, s+Sn, ... of line l; lanes read consecutive lines
        const int l = tid % L, s0 = tid / L, Sn = nthreads / L;
        const long long q = q0 + l;
        if (s0 >= Sn || q >= kp.nlines) return;
        const double *src = kp.in + line_base(kp, q);
        for (int r = s0; r < n; r += Sn) copy8_async(sm.tile + (size_t)r * L + l, src + (long long)r * kp.stride);
    } else {
        // the tile's lines are one contiguous run of nl*n doubles
        const int P = kp.P;
        const int nl = (int)(kp.nlines - q0 < L ? kp.nlines - q0 : L);
        const int total = nl * n;
        const double *src = kp.in + line_base(kp, q0);
        int l = tid / n, r = tid - (tid / n) * n;
        const int dl = nthreads / n, dr = nthreads - dl * n;
        for (int e = tid; e < total; e += nthreads) {
            copy8_async(sm.tile + (size_t)l * P + r, src + e);
            l += dl;
            r += dr;
            if (r >= n) {
                r -= n;
                ++l;
            }
        }
    }
}

#ifdef __CUDACC__
template <int RK, bool PER, bool ADJ, int M, int IN>
__device__ __forceinline__ void run_tile(const KParams &kp, const Smem &sm, long long q0)
{
    Regs<M> R;
    const int tid = threadIdx.x, nthreads = blockDim.x;
#pragma unroll
    for (int ph = 0; ph < NPHASES; ++ph) {
        if (!phase_used<ADJ, IN>(ph)) continue;
        tile_phase<RK, PER, ADJ, M, IN>(ph, kp, sm, R, q0, tid, nthreads);
        if (ph + 1 < NPHASES) __syncthreads();
    }
}

// One CTA = one tile of kp.L lines; blockDim.x >= kp.L * kp.S.
template <int RK, bool PER, bool ADJ, int M, int IN>
__global__ void __launch_bounds__(M <= 8 ? 1024 : (M <= 32 ? 512 : 256), 1) line_kernel(const KParams kp)
{
    extern __shared__ double smem_raw[];
    const Smem sm = carve(smem_raw, kp.L, kp.P, kp.S, kp.xd);
    run_tile<RK, PER, ADJ, M, IN>(kp, sm, (long long)blockIdx.x * kp.L);
}

// Persistent CTAs walk the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// The next tile is copied into the shared tile (cp.async) as soon as the
// current tile's stencil has read it -- or, for IN_GLOBAL, prefetched into L2
// -- so the copy overlaps the chains, the backward sweep and the stores.
template <int RK, bool PER, int M, int IN>
__global__ void __launch_bounds__(M <= 8 ? 1024 : (M <= 32 ? 512 : 256), 1) line_kernel_persist(const KParams kp)
{
    extern __shared__ double smem_raw[];
    using K = LineKernel<RK, PER, false, M, IN>;
    const Smem sm = carve(smem_raw, kp.L, kp.P, kp.S, kp.xd);
    const int tid = threadIdx.x, nthreads = blockDim.x;
    const int l = tid % kp.L, slot = tid / kp.L, s = slot_segment(kp, slot);
    const bool active = s >= 0;
    const long long ntiles = (kp.nlines + kp.L - 1) / kp.L;
    Regs<M> R;
    long long t = blockIdx.x;
    stage_chain_table(kp, sm, tid, nthreads);
    if (IN != IN_GLOBAL && t < ntiles) tile_prefetch<IN>(kp, sm, t * kp.L, tid, nthreads);
    copy_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        const long long q0 = t * kp.L;
        if (IN != IN_GLOBAL) copy_async_wait_all();
        __syncthreads();
        const LineIO io = tile_line_io<false, IN>(kp, sm, l, q0);
        if (active) K::template fwd<false>(kp, sm, R, l, s, io);
        __syncthreads();
        if (t + gridDim.x < ntiles) tile_prefetch<IN>(kp, sm, (t + gridDim.x) * kp.L, tid, nthreads);
        copy_async_commit();
        if (active) K::chain_fwd(kp, sm, l, s);
        __syncthreads();
        if (active) K::template bwd<false>(kp, sm, R, l, s);
        __syncthreads();
        if (active) K::chain_bwd(kp, sm, l, s);
        __syncthreads();
        // results go straight to global memory (the tile already holds the next input)
        LineIO out = io;
        out.dst = kp.out + line_base(kp, io.live ? q0 + l : 0);
        out.ds = kp.stride;
        out.tile = false;
        if (active) K::template fin<false>(kp, sm, R, l, s, out);
    }
}
#endif

// Host emulation (tests): the phases in kernel order over all threads of the CTA.
template <int RK, bool PER, bool ADJ, int M, int IN>
inline void emulate_tile(const KParams &kp, double *smem, long long q0, int nthreads)
{
    const Smem sm = carve(smem, kp.L, kp.P, kp.S, kp.xd);
    Regs<M> *R = new Regs<M>[nthreads];
    if (IN == IN_ROWS)
        for (int tid = 0; tid < nthreads; ++tid) tile_prefetch<IN_ROWS>(kp, sm, q0, tid, nthreads);
    for (int ph = 0; ph < NPHASES; ++ph) {
        if (!phase_used<ADJ, IN>(ph)) continue;
        for (int tid = 0; tid < nthreads; ++tid) tile_phase<RK, PER, ADJ, M, IN>(ph, kp, sm, R[tid], q0, tid, nthreads);
    }
    delete[] R;
}

}  // namespace pado

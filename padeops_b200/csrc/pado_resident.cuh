// pado_resident.cuh -- per-thread phases of the tile-resident sweep used by
// the streaming kernel: the tile of lines stays in shared memory and every
// pass works on it in place, so a thread keeps only a 9-row stencil window
// and a few states in registers (instead of its whole segment), and several
// CTAs of many threads fit on one SM to hide the latency of the serial
// recurrences.
//
// Thread (l, s) owns rows [a, a + len) of line l; row r of the line is
// line[r * rs].  Per tile:
//   prep    the 4 rows before and after the segment (the neighbours' rows,
//           read before anyone overwrites them) and the closure rows of a
//           bounded line
//   fwd     stencil + local forward sweep; z overwrites f row by row; the
//           segment's end values (and border-sum share) go to buf4
//   bwd     incoming forward state from the wf[s] segments before (and, for
//           the segments that need them, the cyclic border unknowns), then
//           the local backward sweep; x overwrites z; first values -> buf2
//   fin     incoming backward state from the wb[s] segments after, corrected
//           x -> the output line (global memory, or the tile)
// Three barriers separate prep, fwd, bwd and fin: the chains run inside the
// phases that use them.
//
// The adjoint (ADJ) solves A^T z = g with the transposed sweep tables: fwd
// reads g from the tile (no stencil, no prep), fin writes z back into the
// tile (scaled by the transposed sweep's delta), and adj_out applies B^T
// (reversed interior taps; explicit columns at a bounded line's ends) from
// the tile to the output after one more barrier.
#pragma once

#include "pado_kernels.cuh"

namespace pado {

// fin with the launch's output mode (scaled / accumulated results), defined
// after ResidentLine.  The shared-memory carve-up comes by value: by
// reference, the caller keeps it in local memory for the call, and every
// kernel then reads the tile through generic loads.
template <int RK, bool PER, int M, bool ADJ, bool STAGED>
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
    void
    fin_out_mode(const KParams &kp, const Smem sm, const double *line, long long rs, int l, int s, double *out,
                 long long os);

template <int RK, bool PER, int M, bool ADJ = false>
struct ResidentLine {
    static constexpr bool CYC = PER;
    static constexpr bool ORDER2 = RK != RHS_CD06_D1;
    // only the bounded cd06 (Thomas) sweep scales its input (alpha != 1), and
    // only its adjoint scales the output (delta != 1)
    static constexpr bool HAS_ALPHA = RK == RHS_CD06_D1 && !PER && !ADJ;
    static constexpr bool HAS_DELTA = RK == RHS_CD06_D1 && !PER && ADJ;
    static constexpr int CR = (RK == RHS_CD06_D1 || RK == RHS_CD10_D2) ? 3 : 4;  // closure_rows(RK)
    using LK = LineKernel<RK, PER, false, M, IN_ROWS>;

    // Rows a thread needs from outside its segment, and its closure rows.
    struct Halo {
        double hp[4];  // rows a-4 .. a-1
        double hn[4];  // rows a+len .. a+len+3
        double cv[4];  // closure rows 0 .. CR-1 (first segment of a bounded line)
        double cl[4];  // closure rows n-CR .. n-1 (last segment of a bounded line)
    };

    static PADO_HD PADO_INLINE bool fast(const KParams &kp, int s) { return (kp.int_mask >> s) & 1u; }
    static PADO_HD PADO_INLINE int wrap(int row, int n) { return row < 0 ? row + n : (row >= n ? row - n : row); }
    // h[j] for a runtime j in [0, 4) without indexing a register array at run
    // time (which would move the array to local memory)
    static PADO_HD PADO_INLINE double pick4(const double (&h)[4], int j)
    {
        double v = h[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (j == k) v = h[k];
        return v;
    }
    static PADO_HD PADO_INLINE double row_or_zero(const double *line, long long rs, int row, int n)
    {
        if (PER) return line[(long long)wrap(row, n) * rs];
        return (row >= 0 && row < n) ? line[(long long)row * rs] : 0.0;
    }

    // ---- prep: halo rows and closure rows, before any in-place write ------
    static PADO_HD PADO_INLINE void prep(const KParams &kp, const double *line, long long rs, int s, Halo &h)
    {
        const int n = kp.n, a = seg_start(kp, s), len = seg_len(kp, s);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            h.hp[k] = row_or_zero(line, rs, a - 4 + k, n);
            h.hn[k] = row_or_zero(line, rs, a + len + k, n);
            h.cv[k] = 0.0;
            h.cl[k] = 0.0;
        }
        if (!PER) {
            if (s == 0) {
#pragma unroll
                for (int k = 0; k < CR; ++k) h.cv[k] = closure_row_noinline<RK>(&kp.rc, line, rs, n, k, kp.bc1, kp.bcn);
            }
            if (s == kp.S - 1) {
#pragma unroll
                for (int k = 0; k < CR; ++k)
                    h.cl[k] = closure_row_noinline<RK>(&kp.rc, line, rs, n, n - CR + k, kp.bc1, kp.bcn);
            }
        }
    }

    // constant-coefficient segment: stencil + forward sweep (w[0..3] preset)
    template <bool STAGED, bool SPK>
    static PADO_HD PADO_INLINE void fwd_fast(const KParams &kp, const Smem &sm, double *p, long long rs, int l, int s,
                                             int a, double (&w)[9], const Halo &h)
    {
        if (!ADJ) {
#pragma unroll
            for (int k = 0; k < 5; ++k) w[4 + k] = p[(long long)k * rs];
        }
        const double al = kp.kc[0], c1 = kp.kc[1], c2 = kp.kc[2];
        double cst[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) cst[k] = kp.rc.c[k];
        using SR = SpikeRows<STAGED>;
        const double *tbs = SPK ? SR::rows(kp, sm, s, a) : nullptr;
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int t = 0; t < M; ++t) {
            double z = ADJ ? p[(long long)t * rs] : rhs_interior_fma(RK, PER, cst, w);
            if (HAS_ALPHA) z *= al;
            if (ORDER2) z -= c2 * z2;
            z -= c1 * z1;
            p[(long long)t * rs] = z;
            if (SPK) {
                const double *tr = tbs + (size_t)t * SR::STRIDE;
                s1 += tld<STAGED>(tr + SR::K1) * z;
                if (ORDER2) s2 += tld<STAGED>(tr + SR::K2) * z;
            }
            z2 = z1;
            z1 = z;
            if (!ADJ) {
#pragma unroll
                for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
                if (t + 5 < M) w[8] = p[(long long)(t + 5) * rs];
                else if (t + 5 - M < 4) w[8] = h.hn[t + 5 - M];
            }
        }
        LK::template summarize_fwd<STAGED>(kp, sm, l, s, z1, z2, s1, s2);
    }

    // constant-coefficient segment: backward sweep, x written over z
    template <bool STAGED, bool SPK>
    static PADO_HD PADO_INLINE void bwd_fast(const KParams &kp, const Smem &sm, double *p, long long rs, int l, int s,
                                             int a, double P1, double P2, double E1, double E2, double &x1, double &x2)
    {
        const double ga = kp.kc[3], d1 = kp.kc[4], d2 = kp.kc[5];
        using SR = SpikeRows<STAGED>;
        const double *tbs = SPK ? SR::rows(kp, sm, s, a) : nullptr;
#pragma unroll
        for (int t = M - 1; t >= 0; --t) {
            double z = p[(long long)t * rs] + P1 * kp.pu[t];
            if (ORDER2) z += P2 * kp.pv[t];
            double x = ga * z;
            if (SPK) {
                const double *tr = tbs + (size_t)t * SR::STRIDE;
                x -= tld<STAGED>(tr + SR::E1) * E1;
                if (ORDER2) x -= tld<STAGED>(tr + SR::E2) * E2;
            }
            if (ORDER2) x -= d2 * x2;
            x -= d1 * x1;
            p[(long long)t * rs] = x;
            x2 = x1;
            x1 = x;
        }
    }

    // ---- edge pieces of exactly E rows (edge_piece_rows; the layout cuts the rows
    // outside the constant-coefficient block into such pieces): the per-row
    // table path fully unrolled, every tile and table offset an immediate, no
    // per-row bounds; the same arithmetic as the generic per-row loop.
    static constexpr int E = edge_piece_rows(RK, PER, M);
    static_assert(E >= 5, "the unrolled edge path needs pieces of at least 5 rows");

    // the same address, marked for the compiler as shared memory (tile and
    // staged tables), so that the unrolled paths load with shared-space
    // instructions; the identity on the host
    template <typename T>
    static PADO_HD PADO_INLINE T *in_shared(T *q)
    {
#ifdef __CUDA_ARCH__
        return reinterpret_cast<T *>(__cvta_shared_to_generic(__cvta_generic_to_shared(q)));
#else
        return q;
#endif
    }

    // stencil + forward sweep of an edge piece (len == E); lenb < E only on
    // the last segment of a cyclic line (its last nbord rows are the border)
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fwd_tab(const KParams &kp, const Smem &sm, double *p, long long rs, int l, int s,
                                            int lenb, double (&w)[9], const Halo &h)
    {
        const bool first = !PER && s == 0, last = !PER && s == kp.S - 1;  // last: the piece ends at row n
        p = in_shared(p);
        if (!ADJ) {
#pragma unroll
            for (int k = 0; k < 5; ++k) w[4 + k] = p[(long long)k * rs];
        }
        const double *tb = in_shared(seg_etab(sm, s));
        double cst[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) cst[k] = kp.rc.c[k];
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0, rb0 = 0.0, rb1 = 0.0;
#pragma unroll
        for (int t = 0; t < E; ++t) {
            double r;
            if (ADJ) {
                r = p[(long long)t * rs];
            } else {
                r = rhs_interior_fma(RK, PER, cst, w);
                if (t < CR && first) r = h.cv[t < CR ? t : 0];
                if (t >= E - CR && last) r = h.cl[t >= E - CR ? t - (E - CR) : 0];
            }
            if (!CYC || t < E - 2 || t < lenb) {
                const double *tr = tb + (size_t)t * E_NF;
                const Dbl2 cc = tld2<STAGED>(tr + E_C1);
                const Dbl2 ak = (HAS_ALPHA || CYC) ? tld2<STAGED>(tr + E_ALPHA) : Dbl2{1.0, 0.0};
                double z = HAS_ALPHA ? ak.x * r : r;
                if (ORDER2) z -= cc.y * z2;
                z -= cc.x * z1;
                p[(long long)t * rs] = z;
                if (CYC) {
                    s1 += ak.y * z;
                    if (ORDER2) s2 += tld<STAGED>(tr + E_K2) * z;
                }
                z2 = z1;
                z1 = z;
            } else {
                // border rows of a cyclic line: right-hand sides only
                if (t == lenb) rb0 = r;
                else rb1 = r;
            }
            if (!ADJ) {
#pragma unroll
                for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
                if (t + 5 < E) w[8] = p[(long long)(t + 5 < E ? t + 5 : 0) * rs];
                else if (t + 5 - E < 4) w[8] = h.hn[t + 5 - E < 4 ? t + 5 - E : 0];
            }
        }
        LK::template summarize_fwd<STAGED>(kp, sm, l, s, z1, z2, s1, s2);
        if (CYC && s == kp.S - 1) {
            sm.eb[(size_t)l * 4 + 2] = rb0;
            sm.eb[(size_t)l * 4 + 3] = rb1;
        }
    }

    // backward sweep of an edge piece, x written over z; returns the piece's
    // first two x
    template <bool STAGED>
    static PADO_HD PADO_INLINE Dbl2 bwd_tab(const Smem &sm, double *p, long long rs, int s, int lenb, double P1,
                                            double P2)
    {
        double x1 = 0.0, x2 = 0.0;
        p = in_shared(p);
        const double *tb = in_shared(seg_etab(sm, s));
#pragma unroll
        for (int t = E - 1; t >= 0; --t) {
            if (CYC && t >= E - 2 && t >= lenb) continue;  // border rows
            const double *tr = tb + (size_t)t * E_NF;
            const Dbl2 uv = tld2<STAGED>(tr + E_U);
            const Dbl2 gd = tld2<STAGED>(tr + E_GAMMA);
            double z = p[(long long)t * rs] + P1 * uv.x;
            if (ORDER2) z += P2 * uv.y;
            double x = gd.x * z;
            if (ORDER2) x -= tld<STAGED>(tr + E_D2) * x2;
            x -= gd.y * x1;
            p[(long long)t * rs] = x;
            x2 = x1;
            x1 = x;
        }
        return Dbl2{x1, x2};
    }

    // corrected x of an edge piece -> out
    template <bool STAGED, bool XF>
    static PADO_HD PADO_INLINE void fin_tab(const KParams &kp, const Smem &sm, const double *p, long long rs, double *q,
                                            long long os, int a, int s, int lenb, double Q1, double Q2, double E1,
                                            double E2, bool spike_rows)
    {
        p = in_shared(p);
        const double *tb = in_shared(seg_etab(sm, s));
        const double *rtab = in_shared(sm.rtab);
#pragma unroll
        for (int t = 0; t < E; ++t) {
            if (CYC && t >= E - 2 && t >= lenb) continue;  // border rows
            const Dbl2 stt = tld2<STAGED>(tb + (size_t)t * E_NF + E_S);
            double x = p[(long long)t * rs] + Q1 * stt.x;
            if (ORDER2) x += Q2 * stt.y;
            if (spike_rows && (a + t < kp.ie || a + t >= kp.je)) {
                const double *rr = resp_row(kp, rtab, a + t);
                x += E1 * rr[0];
                if (ORDER2) x += E2 * rr[1];
            }
            if (HAS_DELTA) x *= tld<STAGED>(tb + (size_t)t * E_NF + E_DELTA);
            if (XF) out_put(kp, q + (long long)t * os, x);
            else q[(long long)t * os] = x;
        }
    }

    // ---- fwd: stencil + local forward sweep, z written over f ---------------
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fwd(const KParams &kp, const Smem &sm, double *line, long long rs, int l, int s,
                                        const Halo &h)
    {
        const int n = kp.n, nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        double *p = line + (long long)a * rs;
        double w[9];
        if (!ADJ) {
#pragma unroll
            for (int k = 0; k < 4; ++k) w[k] = h.hp[k];
        }
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0;
        if (fast(kp, s)) {
            // len == M, every window row inside the line; the spike terms of
            // a cyclic line's first segments are a separate instantiation so
            // that the common path carries no per-row predicates
            if (CYC && ((kp.spk_mask >> s) & 1u)) fwd_fast<STAGED, true>(kp, sm, p, rs, l, s, a, w, h);
            else fwd_fast<STAGED, false>(kp, sm, p, rs, l, s, a, w, h);
            return;
        }
        if (len == E) {
            fwd_tab<STAGED>(kp, sm, p, rs, l, s, lenb, w, h);
            return;
        }
        if (!ADJ) {
#pragma unroll
            for (int k = 0; k < 5; ++k) w[4 + k] = k < len ? p[(long long)k * rs] : pick4(h.hn, k - len);
        }
        const double *tb = seg_etab(sm, s);
        const bool first = !PER && s == 0, last = !PER && s == kp.S - 1;
        double rb0 = 0.0, rb1 = 0.0;
        // per-row table path, eight rows per iteration: the window shift is
        // then register renaming inside the body
        double cst[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) cst[k] = kp.rc.c[k];
#pragma unroll 8
        for (int t = 0; t < len; ++t) {
            double r;
            if (ADJ) {
                r = p[(long long)t * rs];
            } else {
                r = rhs_interior_fma(RK, PER, cst, w);
                if (first && t < CR) r = pick4(h.cv, t);
                if (last && a + t >= n - CR) r = pick4(h.cl, a + t - (n - CR));
            }
            if (t < lenb) {
                const double *tr = tb + (size_t)t * E_NF;
                const Dbl2 cc = tld2<STAGED>(tr + E_C1);
                const Dbl2 ak = (HAS_ALPHA || CYC) ? tld2<STAGED>(tr + E_ALPHA) : Dbl2{1.0, 0.0};
                double z = HAS_ALPHA ? ak.x * r : r;
                if (ORDER2) z -= cc.y * z2;
                z -= cc.x * z1;
                p[(long long)t * rs] = z;
                if (CYC) {
                    s1 += ak.y * z;
                    if (ORDER2) s2 += tld<STAGED>(tr + E_K2) * z;
                }
                z2 = z1;
                z1 = z;
            } else {
                // border rows of a cyclic line: right-hand sides only
                if (t == lenb) rb0 = r;
                else rb1 = r;
            }
            if (!ADJ) {
#pragma unroll
                for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
                const int nx = t + 5;
                if (nx < len) w[8] = p[(long long)nx * rs];
                else if (nx - len < 4) w[8] = pick4(h.hn, nx - len);
            }
        }
        LK::template summarize_fwd<STAGED>(kp, sm, l, s, z1, z2, s1, s2);
        if (CYC && s == kp.S - 1) {
            sm.eb[(size_t)l * 4 + 2] = rb0;
            sm.eb[(size_t)l * 4 + 3] = rb1;
        }
    }

    // ---- incoming states and border unknowns (read the other segments'
    // summaries; called after the barrier that ends the phase writing them)
    static PADO_HD PADO_INLINE void incoming_fwd(const KParams &kp, const Smem &sm, int l, int s, double &P1,
                                                 double &P2)
    {
        const int L = kp.L, wf = kp.wf[s];
        double a1 = 0.0, a2 = 0.0, b1 = 0.0, b2 = 0.0;
        const double *xt = sm.xtab + (size_t)kp.xof[s] * 4;
        int d = 1;
        for (; d + 1 <= wf; d += 2) {
            const double *y = sum4(sm, L, s - d, l), *yb = sum4(sm, L, s - d - 1, l);
            const double *ph = xt + (size_t)(d - 1) * 4;
            const double y0 = y[0], y1 = y[L], z0 = yb[0], z1 = yb[L];
            a1 += ph[0] * y0 + ph[1] * y1;
            a2 += ph[2] * y0 + ph[3] * y1;
            b1 += ph[4] * z0 + ph[5] * z1;
            b2 += ph[6] * z0 + ph[7] * z1;
        }
        if (d <= wf) {
            const double *y = sum4(sm, L, s - d, l);
            const double *ph = xt + (size_t)(d - 1) * 4;
            const double y0 = y[0], y1 = y[L];
            a1 += ph[0] * y0 + ph[1] * y1;
            a2 += ph[2] * y0 + ph[3] * y1;
        }
        P1 = a1 + b1;
        P2 = a2 + b2;
    }
    static PADO_HD PADO_INLINE void border(const KParams &kp, const Smem &sm, int l, double &E1, double &E2)
    {
        const int L = kp.L;
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
        const double *eb = sm.eb + (size_t)l * 4;
        const double u0 = eb[2] - sg1, u1 = eb[3] - sg2;
        if (kp.nbord == 1) {
            E1 = kp.mb[0] * u0;
            E2 = 0.0;
        } else {
            E1 = kp.mb[0] * u0 + kp.mb[1] * u1;
            E2 = kp.mb[2] * u0 + kp.mb[3] * u1;
        }
    }
    static PADO_HD PADO_INLINE void incoming_bwd(const KParams &kp, const Smem &sm, int l, int s, double &Q1,
                                                 double &Q2)
    {
        const int L = kp.L, wb = kp.wb[s];
        double a1 = 0.0, a2 = 0.0, b1 = 0.0, b2 = 0.0;
        const double *xt = sm.xtab + (size_t)kp.xob[s] * 4;
        int d = 1;
        for (; d + 1 <= wb; d += 2) {
            const double *w = sum2(sm, L, s + d, l), *wn = sum2(sm, L, s + d + 1, l);
            const double *ps_ = xt + (size_t)(d - 1) * 4;
            const double w0 = w[0], w1 = w[L], v0 = wn[0], v1 = wn[L];
            a1 += ps_[0] * w0 + ps_[1] * w1;
            a2 += ps_[2] * w0 + ps_[3] * w1;
            b1 += ps_[4] * v0 + ps_[5] * v1;
            b2 += ps_[6] * v0 + ps_[7] * v1;
        }
        if (d <= wb) {
            const double *w = sum2(sm, L, s + d, l);
            const double *ps_ = xt + (size_t)(d - 1) * 4;
            const double w0 = w[0], w1 = w[L];
            a1 += ps_[0] * w0 + ps_[1] * w1;
            a2 += ps_[2] * w0 + ps_[3] * w1;
        }
        Q1 = a1 + b1;
        Q2 = a2 + b2;
    }

    // the border unknowns of line l, for fin (the backward sweeps run with
    // E = 0); by an idle slot's threads where the warps are padded, else by
    // segment 0's threads
    static PADO_HD PADO_INLINE void border_only(const KParams &kp, const Smem &sm, int l)
    {
        double E1, E2;
        border(kp, sm, l, E1, E2);
        sm.eb[(size_t)l * 4 + 0] = E1;
        sm.eb[(size_t)l * 4 + 1] = E2;
    }

    // ---- bwd: local backward sweep, x written over z ------------------------
    template <bool STAGED>
    static PADO_HD PADO_INLINE void bwd(const KParams &kp, const Smem &sm, double *line, long long rs, int l, int s)
    {
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        double *p = line + (long long)a * rs;
        double P1, P2;
        incoming_fwd(kp, sm, l, s, P1, P2);
        double x1 = 0.0, x2 = 0.0;
        if (CYC && s == 0 && kp.border_slot < 0) border_only(kp, sm, l);
        if (fast(kp, s)) {
            bwd_fast<STAGED, false>(kp, sm, p, rs, l, s, a, P1, P2, 0.0, 0.0, x1, x2);
        } else if (len == E) {
            const Dbl2 xx = bwd_tab<STAGED>(sm, p, rs, s, lenb, P1, P2);
            x1 = xx.x;
            x2 = xx.y;
        } else {
            const double *tb = seg_etab(sm, s);
#pragma unroll 1
            for (int t = lenb - 1; t >= 0; --t) {
                const double *tr = tb + (size_t)t * E_NF;
                const Dbl2 uv = tld2<STAGED>(tr + E_U);
                const Dbl2 gd = tld2<STAGED>(tr + E_GAMMA);
                const double d2r = tld<STAGED>(tr + E_D2);
                double z = p[(long long)t * rs] + P1 * uv.x;
                if (ORDER2) z += P2 * uv.y;
                double x = gd.x * z;
                if (ORDER2) x -= d2r * x2;
                x -= gd.y * x1;
                p[(long long)t * rs] = x;
                x2 = x1;
                x1 = x;
            }
        }
        double *o = sum2(sm, kp.L, s, l);
        o[0] = x1;     // x at the segment's first row
        o[kp.L] = x2;  // and the second
    }

    // constant-coefficient segment: corrected x -> out; RSP: the rows also
    // take the border unknowns' response E1 R1 + E2 R2
    template <bool RSP, bool XF>
    static PADO_HD PADO_INLINE void fin_fast(const KParams &kp, const Smem &sm, const double *p, long long rs, double *q,
                                             long long os, int a, double Q1, double Q2, double E1, double E2)
    {
        // response rows: t < tl (first region, rows a + t) and t >= tr (last
        // region, packed after the first one), each at a fixed offset from a
        // per-segment base
        const int tl = RSP ? kp.ie - a : 0, tr = RSP ? kp.je - a : M;
        const double *rl = RSP ? sm.rtab + (long long)a * 2 : nullptr;
        const double *rr_ = RSP ? sm.rtab + (long long)(kp.ie - kp.je + a) * 2 : nullptr;
#pragma unroll
        for (int t = 0; t < M; ++t) {
            double x = p[(long long)t * rs] + Q1 * kp.ps[t];
            if (ORDER2) x += Q2 * kp.pt[t];
            if (RSP && (t < tl || t >= tr)) {
                const double *rr = (t < tl ? rl : rr_) + 2 * t;
                x += E1 * rr[0];
                if (ORDER2) x += E2 * rr[1];
            }
            if (HAS_DELTA) x *= kp.kc[6];
            if (XF) out_put(kp, q + (long long)t * os, x);
            else q[(long long)t * os] = x;
        }
    }

    // ---- fin: corrected x -> out (row r at out[r * os]); out_df: out is df
    // itself, so the launch's output mode applies (else the tile).  The
    // scaled / accumulating form runs out of line (fin_out_mode), so that the
    // common form keeps its register allocation.
    template <bool STAGED>
    static PADO_HD PADO_INLINE void fin(const KParams &kp, const Smem &sm, const double *line, long long rs, int l,
                                        int s, double *out, long long os, bool live, bool out_df = false)
    {
        if (!live) return;
        if (out_df && kp.out_mode != OUT_STORE) {
            fin_out_mode<RK, PER, M, ADJ, STAGED>(kp, sm, line, rs, l, s, out, os);
            return;
        }
        fin_body<STAGED, false>(kp, sm, line, rs, l, s, out, os);
    }

    template <bool STAGED, bool XF>
    static PADO_HD PADO_INLINE void fin_body(const KParams &kp, const Smem &sm, const double *line, long long rs, int l,
                                             int s, double *out, long long os)
    {
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        const double *p = line + (long long)a * rs;
        double *q = out + (long long)a * os;
        double Q1, Q2;
        incoming_bwd(kp, sm, l, s, Q1, Q2);
        double E1 = 0.0, E2 = 0.0;
        // rows that take the border unknowns' response
        const bool spike_rows = CYC && (a < kp.ie || a + len > kp.je);
        if (spike_rows) {
            E1 = sm.eb[(size_t)l * 4 + 0];
            E2 = sm.eb[(size_t)l * 4 + 1];
        }
        if (fast(kp, s)) {
            if (spike_rows) fin_fast<true, XF>(kp, sm, p, rs, q, os, a, Q1, Q2, E1, E2);
            else fin_fast<false, XF>(kp, sm, p, rs, q, os, a, Q1, Q2, 0.0, 0.0);
            return;
        }
        const double *tb = seg_etab(sm, s);
        if (len == E) {
            fin_tab<STAGED, XF>(kp, sm, p, rs, q, os, a, s, lenb, Q1, Q2, E1, E2, spike_rows);
        } else {
#pragma unroll 2
        for (int t = 0; t < lenb; ++t) {
            const Dbl2 stt = tld2<STAGED>(tb + (size_t)t * E_NF + E_S);
            double x = p[(long long)t * rs] + Q1 * stt.x;
            if (ORDER2) x += Q2 * stt.y;
            if (spike_rows && a + t < nb && (a + t < kp.ie || a + t >= kp.je)) {
                const double *rr = resp_row(kp, sm.rtab, a + t);
                x += E1 * rr[0];
                if (ORDER2) x += E2 * rr[1];
            }
            if (HAS_DELTA) x *= tld<STAGED>(tb + (size_t)t * E_NF + E_DELTA);
            if (XF) out_put(kp, q + (long long)t * os, x);
            else q[(long long)t * os] = x;
        }
        }
        if (CYC && s == kp.S - 1) {
            if (XF) {
                out_put(kp, out + (long long)nb * os, sm.eb[(size_t)l * 4 + 0]);
                if (kp.nbord == 2) out_put(kp, out + (long long)(nb + 1) * os, sm.eb[(size_t)l * 4 + 1]);
            } else {
                out[(long long)nb * os] = sm.eb[(size_t)l * 4 + 0];
                if (kp.nbord == 2) out[(long long)(nb + 1) * os] = sm.eb[(size_t)l * 4 + 1];
            }
        }
    }

    // column j of B^T at a bounded line's end (explicit blocks; every row of
    // the line when n <= 32), rows read with stride rs
    static PADO_HD PADO_INLINE double bt_column(const double *bt, const double *line, long long rs, int n, int j)
    {
        double acc = 0.0;
        if (n <= 32) {
            const double *w = bt + (size_t)j * n;
            for (int i = 0; i < n; ++i) acc += PADO_LDG(w + i) * line[(long long)i * rs];
            return acc;
        }
        const int i0 = j < 8 ? 0 : n - 12;
        const double *w = bt + (size_t)(j < 8 ? j : 8 + j - (n - 8)) * 12;
        for (int i = 0; i < 12; ++i) acc += PADO_LDG(w + i) * line[(long long)(i0 + i) * rs];
        return acc;
    }

    // ---- adjoint, in place (x lines: the tile then goes out by bulk copy) ----
    // Columns of B^T at a bounded line's ends go through a small scratch: slot
    // j (first columns) or zone + j - (n - zone) (last ones), zone = n <= 32 ?
    // n : 8, value for line l at scratch[slot * L + l].
    static PADO_HD PADO_INLINE int adj_scratch_slots(int n) { return n <= 32 ? n : 16; }
    // phase A (z final in the tile): the 4 rows on each side of the segment,
    // and the end columns of B^T among the segment's rows
    static PADO_HD PADO_INLINE void adj_gather(const KParams &kp, const double *line, long long rs, int l, int s,
                                               double *scratch, Halo &h)
    {
        const int n = kp.n, a = seg_start(kp, s), len = seg_len(kp, s);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            h.hp[k] = row_or_zero(line, rs, a - 4 + k, n);
            h.hn[k] = row_or_zero(line, rs, a + len + k, n);
        }
        if (PER) return;
        const int zone = n <= 32 ? n : 8;
        for (int t = 0; t < len; ++t) {
            const int j = a + t;
            if (j < zone) scratch[(size_t)j * kp.L + l] = bt_column(kp.bt, line, rs, n, j);
            else if (j >= n - zone && n > 32) scratch[(size_t)(8 + j - (n - 8)) * kp.L + l] = bt_column(kp.bt, line, rs, n, j);
        }
    }
    // phase B (after a barrier): fbar = B^T z over the segment's rows, written
    // over z; the 9-row window runs ahead of the writes
    static PADO_HD PADO_INLINE void adj_inplace(const KParams &kp, double *line, long long rs, int l, int s,
                                                const double *scratch, const Halo &h)
    {
        const int n = kp.n, a = seg_start(kp, s), len = seg_len(kp, s);
        double tp[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) tp[k] = kp.taps[k];
        double *p = line + (long long)a * rs;
        double w[9];
#pragma unroll
        for (int k = 0; k < 4; ++k) w[k] = h.hp[k];
#pragma unroll
        for (int k = 0; k < 4; ++k) w[4 + k] = k < len ? p[(long long)k * rs] : pick4(h.hn, k - len);
        const int zone = n <= 32 ? n : 8;
        const bool edge = !PER && (a < zone || a + len > n - zone);
#pragma unroll 4
        for (int t = 0; t < len; ++t) {
            const int nx = t + 4;
            w[8] = nx < len ? p[(long long)nx * rs] : pick4(h.hn, nx - len);
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 9; ++k) acc += tp[k] * w[k];
            const int j = a + t;
            if (edge) {
                if (j < zone) acc = scratch[(size_t)j * kp.L + l];
                else if (j >= n - zone) acc = scratch[(size_t)(8 + j - (n - 8)) * kp.L + l];
            }
            p[(long long)t * rs] = acc;
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
        }
    }

    // ---- adjoint: fbar = B^T z, z in the tile (every segment's fin done) ----
    static PADO_HD PADO_INLINE void adj_out(const KParams &kp, const double *line, long long rs, int s, double *out,
                                            long long os, bool live)
    {
        if (!live) return;
        const int n = kp.n, a = seg_start(kp, s), len = seg_len(kp, s);
        double tp[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) tp[k] = kp.taps[k];
        double w[9];
#pragma unroll
        for (int k = 0; k < 8; ++k) w[k] = row_or_zero(line, rs, a - 4 + k, n);
        const int zone = n <= 32 ? n : 8;
        const bool edge = !PER && (a < zone || a + len > n - zone);
#pragma unroll 4
        for (int t = 0; t < len; ++t) {
            w[8] = row_or_zero(line, rs, a + t + 4, n);
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 9; ++k) acc += tp[k] * w[k];
            const int j = a + t;
            if (edge && (j < zone || j >= n - zone)) acc = bt_column(kp.bt, line, rs, n, j);
            out[(long long)j * os] = acc;
#pragma unroll
            for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
        }
    }
};

template <int RK, bool PER, int M, bool ADJ, bool STAGED>
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
    void
    fin_out_mode(const KParams &kp, const Smem sm, const double *line, long long rs, int l, int s, double *out,
                 long long os)
{
    ResidentLine<RK, PER, M, ADJ>::template fin_body<STAGED, true>(kp, sm, line, rs, l, s, out, os);
}

}  // namespace pado

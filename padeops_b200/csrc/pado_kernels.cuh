// pado_kernels.cuh -- the line kernel: explicit stencil fused with the banded
// solve, for one line family (all lines of a field along one axis).
//
// A CTA owns a tile of L lines (lanes) and cuts every line into S segments
// (thread (l, s) = lane l, segment s).  Per tile:
//
//   load     the L x n tile into shared memory (pitch P = odd, so lane-strided
//            accesses are bank-conflict free)
//   fwd      stencil rows of the segment (reference grouping), then the local
//            forward recurrence with zero incoming state, kept in registers
//   chainF   one thread per line walks the S segments: incoming states,
//            cyclic border unknowns
//   bwd      local backward recurrence (forward values corrected on the fly)
//   chainB   one thread per line walks the segments backwards
//   fin      x = local + incoming-state corrections -> tile -> global
//
// The adjoint kernel runs the transposed sweep first and the transposed
// stencil last.  Each phase is a __host__ __device__ function so tests can
// run the same code on the CPU.
#pragma once

#include "pado_common.h"

namespace pado {

// Parameters of one launch (passed by value).
struct KParams {
    const double *in;
    double *out;
    long long nlines;      // lines in the family
    long long line_ia;     // base(q) = (q % line_ia) + (q / line_ia) * line_oc
    long long line_oc;
    long long stride;      // element stride along a line
    int n, nb, nbord, P;   // line length, banded rows, border rows, tile pitch
    int S, base, rem;      // segment layout over [0, n)
    int L;                 // lines per CTA
    int bc1, bcn;
    const double *tab;     // [nb][T_NF]
    const double *segsum;  // [S][4]
    const double *bt;      // adjoint: transposed stencil blocks (bounded)
    double mb[4];
    double taps[9];        // adjoint: interior transposed taps
    RhsCoef rc;
};

PADO_HD PADO_INLINE int seg_start(const KParams &kp, int s) { return s * kp.base + (s < kp.rem ? s : kp.rem); }
PADO_HD PADO_INLINE int seg_len(const KParams &kp, int s) { return kp.base + (s < kp.rem ? 1 : 0); }
PADO_HD PADO_INLINE long long line_base(const KParams &kp, long long q)
{
    return (q % kp.line_ia) + (q / kp.line_ia) * kp.line_oc;
}

// Shared-memory carve-up (doubles).
struct Smem {
    double *tile;  // [L][P]
    double *buf4;  // [S][L][4]  forward summaries, later backward summaries
    double *buf2;  // [S][L][2]  forward incoming states, later backward ones
    double *eb;    // [L][4]     border unknowns E (0..1) and border rhs (2..3)
};

PADO_HD PADO_INLINE size_t smem_doubles(int L, int P, int S) { return (size_t)L * P + (size_t)S * L * 6 + (size_t)L * 4; }

PADO_HD PADO_INLINE Smem carve(double *base, int L, int P, int S)
{
    Smem sm;
    sm.tile = base;
    sm.buf4 = sm.tile + (size_t)L * P;
    sm.buf2 = sm.buf4 + (size_t)S * L * 4;
    sm.eb = sm.buf2 + (size_t)S * L * 2;
    return sm;
}

template <int M>
struct Regs {
    double r[M];
};

#ifdef __CUDA_ARCH__
#define PADO_LDG(p) __ldg(p)
#else
#define PADO_LDG(p) (*(p))
#endif

// ---------------------------------------------------------------------------
// Tile load / store (cooperative over the CTA's nthreads threads).
// ---------------------------------------------------------------------------
PADO_HD PADO_INLINE void tile_load(const KParams &kp, const Smem &sm, long long q0, int tid, int nthreads)
{
    const int n = kp.n, L = kp.L, P = kp.P;
    if (kp.stride == 1) {
        // lines contiguous: stream each line with all threads
        for (int l = 0; l < L; ++l) {
            const long long q = q0 + l;
            if (q >= kp.nlines) break;
            const double *src = kp.in + line_base(kp, q);
            double *dst = sm.tile + (size_t)l * P;
            for (int r = tid; r < n; r += nthreads) dst[r] = src[r];
        }
    } else {
        // strided lines: lanes read consecutive lines (coalesced) row by row
        const int l = tid % L, s = tid / L, S = nthreads / L;
        const long long q = q0 + l;
        if (s < S && q < kp.nlines) {
            const double *src = kp.in + line_base(kp, q);
            double *dst = sm.tile + (size_t)l * P;
            for (int r = s; r < n; r += S) dst[r] = src[(long long)r * kp.stride];
        }
    }
}

PADO_HD PADO_INLINE void tile_store(const KParams &kp, const Smem &sm, long long q0, int tid, int nthreads)
{
    const int n = kp.n, L = kp.L, P = kp.P;
    if (kp.stride == 1) {
        for (int l = 0; l < L; ++l) {
            const long long q = q0 + l;
            if (q >= kp.nlines) break;
            double *dst = kp.out + line_base(kp, q);
            const double *src = sm.tile + (size_t)l * P;
            for (int r = tid; r < n; r += nthreads) dst[r] = src[r];
        }
    } else {
        const int l = tid % L, s = tid / L, S = nthreads / L;
        const long long q = q0 + l;
        if (s < S && q < kp.nlines) {
            double *dst = kp.out + line_base(kp, q);
            const double *src = sm.tile + (size_t)l * P;
            for (int r = s; r < n; r += S) dst[(long long)r * kp.stride] = src[r];
        }
    }
}

// Closure rows are rare (first/last few rows of a bounded line): evaluate
// them out of line from the tile.
#ifdef __CUDA_ARCH__
__device__ __noinline__
#else
inline
#endif
    double
    closure_row_noinline(const RhsCoef &rc, const double *line, int n, int row, int bc1, int bcn)
{
    return rhs_closure_row(rc.rk, rc.c, line, n, row, bc1, bcn);
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

template <int RK, bool PER, bool ADJ, int M>
struct LineKernel {
    static constexpr bool CYC = PER;

    // value of the tile line at row (wrapped when periodic, 0 outside when bounded)
    static PADO_HD PADO_INLINE double tv(const double *line, int n, int row)
    {
        if (PER) {
            row = row < 0 ? row + n : (row >= n ? row - n : row);
            return line[row];
        }
        return (row >= 0 && row < n) ? line[row] : 0.0;
    }

    // ---- phase fwd: right-hand side (primal) + local forward sweep ---------
    static PADO_HD PADO_INLINE void fwd(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int n = kp.n, nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;  // banded rows of this segment
        const double *line = sm.tile + (size_t)l * kp.P;
        if (!ADJ) {
            // sliding 9-point window over the tile row
            double v[9];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k + 1] = tv(line, n, a - 4 + k);
            const int cr = closure_rows(RK);
#pragma unroll
            for (int t = 0; t < M; ++t) {
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = v[k + 1];
                v[8] = t < len ? tv(line, n, a + t + 4) : 0.0;
                if (t < len) {
                    const int row = a + t;
                    if (!PER && (row < cr || row >= n - cr))
                        R.r[t] = closure_row_noinline(kp.rc, line, n, row, kp.bc1, kp.bcn);
                    else
                        R.r[t] = rhs_interior(RK, PER, kp.rc.c, v);
                }
            }
        } else {
#pragma unroll
            for (int t = 0; t < M; ++t)
                if (t < len) R.r[t] = line[a + t];
        }
        // local forward sweep with zero incoming state
        double z1 = 0.0, z2 = 0.0, s1 = 0.0, s2 = 0.0;
        const double *tb = kp.tab + (size_t)a * T_NF;
#pragma unroll
        for (int t = 0; t < M; ++t) {
            if (t < lenb) {
                const double *tr = tb + (size_t)t * T_NF;
                const double c1 = PADO_LDG(tr + T_C1), c2 = PADO_LDG(tr + T_C2), al = PADO_LDG(tr + T_ALPHA);
                const double z = (al * R.r[t] - c2 * z2) - c1 * z1;
                R.r[t] = z;
                if (CYC) {
                    s1 += PADO_LDG(tr + T_K1) * z;
                    s2 += PADO_LDG(tr + T_K2) * z;
                }
                z2 = z1;
                z1 = z;
            }
        }
        double *o = sm.buf4 + ((size_t)s * kp.L + l) * 4;
        o[0] = z1;  // z at the last banded row of the segment
        o[1] = z2;  // and the one before
        o[2] = s1;
        o[3] = s2;
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
    static PADO_HD PADO_INLINE void chain_fwd(const KParams &kp, const Smem &sm, int l)
    {
        double P1 = 0.0, P2 = 0.0, sg1 = 0.0, sg2 = 0.0;
        for (int s = 0; s < kp.S; ++s) {
            const double *in4 = sm.buf4 + ((size_t)s * kp.L + l) * 4;
            const double zl = in4[0], zl2 = in4[1], ps1 = in4[2], ps2 = in4[3];
            double *st = sm.buf2 + ((size_t)s * kp.L + l) * 2;
            st[0] = P1;
            st[1] = P2;
            if (CYC) {
                const double *ss = kp.segsum + (size_t)s * 4;
                sg1 += ps1 + P1 * PADO_LDG(ss + 0) + P2 * PADO_LDG(ss + 1);
                sg2 += ps2 + P1 * PADO_LDG(ss + 2) + P2 * PADO_LDG(ss + 3);
            }
            if (s + 1 < kp.S) {
                const int a = seg_start(kp, s), len = seg_len(kp, s);
                const int b = (a + len <= kp.nb) ? a + len : kp.nb;
                const double *t1 = kp.tab + (size_t)(b - 1) * T_NF, *t2 = kp.tab + (size_t)(b - 2) * T_NF;
                const double n1 = zl + P1 * PADO_LDG(t1 + T_U) + P2 * PADO_LDG(t1 + T_V);
                const double n2 = zl2 + P1 * PADO_LDG(t2 + T_U) + P2 * PADO_LDG(t2 + T_V);
                P1 = n1;
                P2 = n2;
            }
        }
        if (CYC) {
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
    static PADO_HD PADO_INLINE void bwd(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        const double *st = sm.buf2 + ((size_t)s * kp.L + l) * 2;
        const double P1 = st[0], P2 = st[1];
        double E1 = 0.0, E2 = 0.0;
        if (CYC) {
            E1 = sm.eb[(size_t)l * 4 + 0];
            E2 = sm.eb[(size_t)l * 4 + 1];
        }
        const double *tb = kp.tab + (size_t)a * T_NF;
        double x1 = 0.0, x2 = 0.0;
#pragma unroll
        for (int t = M - 1; t >= 0; --t) {
            if (t < lenb) {
                const double *tr = tb + (size_t)t * T_NF;
                const double z = R.r[t] + P1 * PADO_LDG(tr + T_U) + P2 * PADO_LDG(tr + T_V);
                double x = PADO_LDG(tr + T_GAMMA) * z;
                if (CYC) x = x - PADO_LDG(tr + T_E2) * E2 - PADO_LDG(tr + T_E1) * E1;
                x = x - PADO_LDG(tr + T_D2) * x2 - PADO_LDG(tr + T_D1) * x1;
                R.r[t] = x;
                x2 = x1;
                x1 = x;
            }
        }
        double *o = sm.buf4 + ((size_t)s * kp.L + l) * 4;
        o[0] = x1;  // x at the segment's first row
        o[1] = x2;  // and the second
    }

    // ---- phase chainB: backward incoming states ---------------------------
    static PADO_HD PADO_INLINE void chain_bwd(const KParams &kp, const Smem &sm, int l)
    {
        double Q1 = 0.0, Q2 = 0.0;
        for (int s = kp.S - 1; s >= 0; --s) {
            const double *in4 = sm.buf4 + ((size_t)s * kp.L + l) * 4;
            double *st = sm.buf2 + ((size_t)s * kp.L + l) * 2;
            st[0] = Q1;
            st[1] = Q2;
            if (s > 0) {
                const int a = seg_start(kp, s);
                const double *t0 = kp.tab + (size_t)a * T_NF, *t1 = kp.tab + (size_t)(a + 1) * T_NF;
                const double n1 = in4[0] + Q1 * PADO_LDG(t0 + T_S) + Q2 * PADO_LDG(t0 + T_T);
                const double n2 = in4[1] + Q1 * PADO_LDG(t1 + T_S) + Q2 * PADO_LDG(t1 + T_T);
                Q1 = n1;
                Q2 = n2;
            }
        }
    }

    // ---- phase fin: corrected values -> tile ------------------------------
    static PADO_HD PADO_INLINE void fin(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int nb = kp.nb;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const int lenb = (a + len <= nb) ? len : nb - a;
        const double *st = sm.buf2 + ((size_t)s * kp.L + l) * 2;
        const double Q1 = st[0], Q2 = st[1];
        const double *tb = kp.tab + (size_t)a * T_NF;
        double *line = sm.tile + (size_t)l * kp.P;
#pragma unroll
        for (int t = 0; t < M; ++t) {
            if (t < lenb) {
                const double *tr = tb + (size_t)t * T_NF;
                double x = R.r[t] + Q1 * PADO_LDG(tr + T_S) + Q2 * PADO_LDG(tr + T_T);
                if (ADJ) x = PADO_LDG(tr + T_DELTA) * x;
                line[a + t] = x;
            }
        }
        if (CYC && s == kp.S - 1) {
            line[nb] = sm.eb[(size_t)l * 4 + 0];
            if (kp.nbord == 2) line[nb + 1] = sm.eb[(size_t)l * 4 + 1];
        }
    }

    // ---- phase adjoint stencil: tile (A^{-T} g) -> registers (B^T ...) ----
    static PADO_HD PADO_INLINE void adj_stencil(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int n = kp.n;
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        const double *line = sm.tile + (size_t)l * kp.P;
        double v[9];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k + 1] = tv(line, n, a - 4 + k);
        const int zone = n <= 32 ? n : 8;
#pragma unroll
        for (int t = 0; t < M; ++t) {
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = v[k + 1];
            v[8] = t < len ? tv(line, n, a + t + 4) : 0.0;
            if (t < len) {
                const int j = a + t;
                if (!PER && (j < zone || j >= n - zone)) {
                    R.r[t] = bt_column_noinline(kp.bt, line, n, j);
                } else {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < 9; ++k) acc += kp.taps[k] * v[k];
                    R.r[t] = acc;
                }
            }
        }
    }

    static PADO_HD PADO_INLINE void adj_write(const KParams &kp, const Smem &sm, Regs<M> &R, int l, int s)
    {
        const int a = seg_start(kp, s), len = seg_len(kp, s);
        double *line = sm.tile + (size_t)l * kp.P;
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < len) line[a + t] = R.r[t];
    }
};

// One tile of kp.L lines on a CTA of nthreads threads (nthreads >= L*S;
// the extra threads only help with the tile load/store).
template <int RK, bool PER, bool ADJ, int M>
PADO_HD PADO_INLINE void tile_phase(int phase, const KParams &kp, const Smem &sm, Regs<M> &R, long long q0, int tid,
                                    int nthreads)
{
    using K = LineKernel<RK, PER, ADJ, M>;
    const int l = tid % kp.L, s = tid / kp.L;
    const bool active = s < kp.S;
    switch (phase) {
    case 0: tile_load(kp, sm, q0, tid, nthreads); break;
    case 1: if (active) K::fwd(kp, sm, R, l, s); break;
    case 2: if (s == 0) K::chain_fwd(kp, sm, l); break;
    case 3: if (active) K::bwd(kp, sm, R, l, s); break;
    case 4: if (s == 0) K::chain_bwd(kp, sm, l); break;
    case 5: if (active) K::fin(kp, sm, R, l, s); break;
    case 6: if (ADJ && active) K::adj_stencil(kp, sm, R, l, s); break;
    case 7: if (ADJ && active) K::adj_write(kp, sm, R, l, s); break;
    default: tile_store(kp, sm, q0, tid, nthreads); break;
    }
}
constexpr int NPHASES = 9;

#ifdef __CUDACC__
template <int RK, bool PER, bool ADJ, int M>
__device__ __forceinline__ void run_tile(const KParams &kp, const Smem &sm, long long q0)
{
    Regs<M> R;
    const int tid = threadIdx.x, nthreads = blockDim.x;
#pragma unroll
    for (int ph = 0; ph < NPHASES; ++ph) {
        if (!ADJ && (ph == 6 || ph == 7)) continue;
        tile_phase<RK, PER, ADJ, M>(ph, kp, sm, R, q0, tid, nthreads);
        if (ph + 1 < NPHASES) __syncthreads();
    }
}

// One CTA = one tile of kp.L lines; blockDim.x >= kp.L * kp.S.
template <int RK, bool PER, bool ADJ, int M>
__global__ void __launch_bounds__(M <= 8 ? 1024 : (M <= 32 ? 512 : 256)) line_kernel(const KParams kp)
{
    extern __shared__ double smem_raw[];
    const Smem sm = carve(smem_raw, kp.L, kp.P, kp.S);
    run_tile<RK, PER, ADJ, M>(kp, sm, (long long)blockIdx.x * kp.L);
}
#endif

// Host emulation of one tile (tests): the phases in kernel order over all
// threads of the CTA.
template <int RK, bool PER, bool ADJ, int M>
inline void emulate_tile(const KParams &kp, double *smem, long long q0, int nthreads)
{
    const Smem sm = carve(smem, kp.L, kp.P, kp.S);
    Regs<M> *R = new Regs<M>[nthreads];
    for (int ph = 0; ph < NPHASES; ++ph) {
        if (!ADJ && (ph == 6 || ph == 7)) continue;
        for (int tid = 0; tid < nthreads; ++tid) tile_phase<RK, PER, ADJ, M>(ph, kp, sm, R[tid], q0, tid, nthreads);
    }
    delete[] R;
}

}  // namespace pado

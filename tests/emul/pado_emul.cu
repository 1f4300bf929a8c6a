// pado_emul.cu -- TEST ONLY.  Runs the device kernel's phase functions
// (padeops_b200/csrc/pado_kernels.cuh) on the CPU, tile by tile, with the
// product's host-side tables (pado_tables.cpp).  Lets the CPU test suite
// check the partitioned sweep, the tables and the adjoint without a GPU.
#include <cstring>
#include <vector>

#include "../../padeops_b200/csrc/pado_kernels.cuh"
#include "../../padeops_b200/csrc/pado_params.h"
#include "../../padeops_b200/csrc/pado_stream.cuh"
#include "../../padeops_b200/csrc/pado_tables.h"

using namespace pado;

// Every input path the library uses: strided lines through the cp.async
// rows tile (primal) or straight from global memory (adjoint); contiguous
// lines through the [L][P] tile.
template <int RK, bool PER, bool ADJ, int M>
static void run_all(const KParams &kp, int nthreads)
{
    const bool strided = kp.stride != 1;
    const size_t tile = (ADJ || !strided) ? (size_t)kp.L * kp.P : (size_t)kp.n * kp.L;
    std::vector<double> smem(smem_doubles(kp.L, kp.S, kp.xd, tile), 0.0);
    for (long long q0 = 0; q0 < kp.nlines; q0 += kp.L) {
        if (!strided) emulate_tile<RK, PER, ADJ, M, IN_LINES>(kp, smem.data(), q0, nthreads);
        else if (ADJ) emulate_tile<RK, PER, ADJ, M, IN_GLOBAL>(kp, smem.data(), q0, nthreads);
        else emulate_tile<RK, PER, ADJ, M, IN_ROWS>(kp, smem.data(), q0, nthreads);
    }
}

template <int RK, bool PER, bool ADJ>
static int pick_m(const KParams &kp, int m, int nthreads)
{
    switch (m) {
    case 16: run_all<RK, PER, ADJ, 16>(kp, nthreads); return 0;
    case 32: run_all<RK, PER, ADJ, 32>(kp, nthreads); return 0;
    case 64: run_all<RK, PER, ADJ, 64>(kp, nthreads); return 0;
    }
    return -1;
}

template <int RK>
static int pick(const KParams &kp, bool per, bool adj, int m, int nthreads)
{
    if (per) return adj ? pick_m<RK, true, true>(kp, m, nthreads) : pick_m<RK, true, false>(kp, m, nthreads);
    return adj ? pick_m<RK, false, true>(kp, m, nthreads) : pick_m<RK, false, false>(kp, m, nthreads);
}

extern "C" int emul_apply(int scheme, int kind, int n, double dx, int periodic, int bc1, int bcn, int m, int lines,
                          int extra_threads, int adjoint, int axis, const double *f, double *df, long na, long nb,
                          int fast)
{
    const OpTables ot = make_op_tables(scheme, kind, n, dx, periodic, bc1, bcn, m, adjoint != 0);
    const Layout &lay = ot.lay;
    KParams kp{};
    fill_params(kp, ot, n, bc1, bcn);
    kp.in = f;
    kp.out = df;
    set_geometry(kp, axis, n, na, nb);
    kp.L = lines;
    kp.tab = ot.tab.data();
    const ChainTables &ch = fast ? ot.chain : ot.chain_exact;
    kp.ctab = ch.ctab.data();
    kp.xtab = ch.xtab.data();
    set_chain(kp, ch);
    kp.bt = ot.bt.empty() ? nullptr : ot.bt.data();
    if (!fast) {
        kp.int_mask = 0u;
        kp.spk_mask = 0u;
        for (int i = 0; i < 32; ++i) kp.sperm[i] = (unsigned char)i;
        kp.nslots = kp.S;
    }
    const int nthreads = lines * lay.S + extra_threads;
    switch (ot.rc.rk) {
    case RHS_CD06_D1: return pick<RHS_CD06_D1>(kp, periodic, adjoint, m, nthreads);
    case RHS_CD10_D1: return pick<RHS_CD10_D1>(kp, periodic, adjoint, m, nthreads);
    case RHS_CD10_D2: return pick<RHS_CD10_D2>(kp, periodic, adjoint, m, nthreads);
    default: return pick<RHS_CF90>(kp, periodic, adjoint, m, nthreads);
    }
}

// The streaming kernel's tile loop (primal): tiles of `lines` lines, x
// lines through the [L][n+2] tile, y/z lines through the [row][L] tile.
template <int RK, bool PER, bool ADJ>
static int stream_pick_adj(const StreamParams &sp, int m, bool xl, int nthreads)
{
    switch (m * 2 + (xl ? 1 : 0)) {
    case 32: emulate_stream<RK, PER, 16, false, ADJ>(sp, nthreads); return 0;
    case 33: emulate_stream<RK, PER, 16, true, ADJ>(sp, nthreads); return 0;
    case 64: emulate_stream<RK, PER, 32, false, ADJ>(sp, nthreads); return 0;
    case 65: emulate_stream<RK, PER, 32, true, ADJ>(sp, nthreads); return 0;
    case 128: emulate_stream<RK, PER, 64, false, ADJ>(sp, nthreads); return 0;
    case 129: emulate_stream<RK, PER, 64, true, ADJ>(sp, nthreads); return 0;
    }
    return -1;
}

template <int RK, bool PER>
static int stream_pick(const StreamParams &sp, int m, bool xl, int nthreads, bool adj)
{
    return adj ? stream_pick_adj<RK, PER, true>(sp, m, xl, nthreads) : stream_pick_adj<RK, PER, false>(sp, m, xl, nthreads);
}

extern "C" int emul_stream(int scheme, int kind, int n, double dx, int periodic, int bc1, int bcn, int m, int lines,
                           int axis, const double *f, double *df, long na, long nb, int adjoint)
{
    const OpTables ot = make_op_tables(scheme, kind, n, dx, periodic, bc1, bcn, m, adjoint != 0);
    const Layout &lay = ot.lay;
    StreamParams sp;
    std::memset(&sp, 0, sizeof(sp));
    KParams &kp = sp.kp;
    fill_params(kp, ot, n, bc1, bcn);
    kp.in = f;
    kp.out = df;
    set_geometry(kp, axis, n, na, nb);
    kp.L = lines;
    kp.tab = ot.tab.data();
    kp.ctab = ot.chain.ctab.data();
    kp.xtab = ot.chain.xtab.data();
    kp.bt = ot.bt.empty() ? nullptr : ot.bt.data();
    const bool xl = axis == 1;
    sp.axis = axis;
    sp.stages = 1;
    sp.etab_rows = (int)(ot.etab.size() / E_NF);
    sp.etab = ot.etab.data();
    sp.ktab_rows = (int)(ot.ktab.size() / KT_NF);
    sp.ktab = ot.ktab.data();
    sp.rtab = ot.rtab.data();
    sp.toff = ot.toff.data();
    if (xl) {
        kp.P = n + 2;
        sp.tile_doubles = (lines * kp.P + 15) / 16 * 16;
        sp.ntiles = (kp.nlines + lines - 1) / lines;
    } else {
        sp.nbox = (n + 255) / 256;
        sp.box_rows = ((n + sp.nbox - 1) / sp.nbox + 15) / 16 * 16;
        sp.tile_doubles = (sp.nbox * sp.box_rows * lines + 15) / 16 * 16;
        sp.na = (int)na;
        sp.xblocks = (int)((na + lines - 1) / lines);
        sp.ntiles = (long long)sp.xblocks * nb;
        sp.pstride = axis == 2 ? na * (long long)n : na;
    }
    kp.nslots = warp_slots(ot, lines, kp.sperm, KMAXSLOT, true);
    kp.border_slot = first_idle_slot(kp.sperm, kp.nslots);
    const int nthreads = lines * kp.nslots;
    const bool per = periodic != 0;
    switch (ot.rc.rk) {
    case RHS_CD06_D1:
        return per ? stream_pick<RHS_CD06_D1, true>(sp, m, xl, nthreads, adjoint) : stream_pick<RHS_CD06_D1, false>(sp, m, xl, nthreads, adjoint);
    case RHS_CD10_D1:
        return per ? stream_pick<RHS_CD10_D1, true>(sp, m, xl, nthreads, adjoint) : stream_pick<RHS_CD10_D1, false>(sp, m, xl, nthreads, adjoint);
    case RHS_CD10_D2:
        return per ? stream_pick<RHS_CD10_D2, true>(sp, m, xl, nthreads, adjoint) : stream_pick<RHS_CD10_D2, false>(sp, m, xl, nthreads, adjoint);
    default:
        return per ? stream_pick<RHS_CF90, true>(sp, m, xl, nthreads, adjoint) : stream_pick<RHS_CF90, false>(sp, m, xl, nthreads, adjoint);
    }
}

// Dense stencil matrix B (row-major n x n) as the product builds it.
extern "C" int emul_stencil(int scheme, int kind, int n, double dx, int periodic, int bc1, int bcn, double *B)
{
    const RhsCoef rc = make_rhs_coef(scheme, kind, dx, periodic);
    const std::vector<double> b = stencil_matrix(rc, n, bc1, bcn);
    std::memcpy(B, b.data(), sizeof(double) * b.size());
    return 0;
}

// The segment layout and code-path facts of one operator's tables:
// starts[0..S] (S = *nseg), fast[s] (constant-coefficient interior segment),
// *edge (the unrolled edge-piece length), *w (coupling window).
extern "C" int emul_layout(int scheme, int kind, int n, int periodic, int bc1, int bcn, int m, int *starts, int *fast,
                           int *nseg, int *edge, int *w)
{
    const OpTables ot = make_op_tables(scheme, kind, n, 0.1, periodic, bc1, bcn, m, false);
    *nseg = ot.lay.S;
    for (int s = 0; s <= ot.lay.S; ++s) starts[s] = ot.lay.st[s];
    for (int s = 0; s < ot.lay.S; ++s) fast[s] = (int)((ot.interior.mask >> s) & 1u);
    *edge = edge_piece_rows(ot.rc.rk, periodic != 0, m);
    *w = ot.chain.W;
    return 0;
}

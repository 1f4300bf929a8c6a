// pado_emul.cu -- TEST ONLY.  Runs the device kernel's phase functions
// (padeops_b200/csrc/pado_kernels.cuh) on the CPU, tile by tile, with the
// product's host-side tables (pado_tables.cpp).  Lets the CPU test suite
// check the partitioned sweep, the tables and the adjoint without a GPU.
#include <cstring>
#include <vector>

#include "../../padeops_b200/csrc/pado_kernels.cuh"
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
    std::vector<double> smem(smem_doubles(kp.L, kp.S, tile), 0.0);
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
    const Sweep prim = primal_sweep(scheme, kind, n, periodic, bc1, bcn);
    const Sweep sw = adjoint ? adjoint_sweep(prim) : prim;
    const RhsCoef rc = make_rhs_coef(scheme, kind, dx, periodic);
    const Layout lay = make_layout(n, m);
    if ((lay.S > 1 && lay.base + (lay.rem ? 1 : 0) > m) || lay.base + 1 > m + 1) return -6;
    std::vector<double> tab, segsum, bt;
    build_device_table(sw, lay, tab, segsum);
    KParams kp{};
    kp.in = f;
    kp.out = df;
    kp.nlines = (long long)na * nb;
    if (axis == 1) { kp.line_ia = 1; kp.line_oc = n; kp.stride = 1; }
    else if (axis == 2) { kp.line_ia = na; kp.line_oc = (long long)na * n; kp.stride = na; }
    else { kp.line_ia = kp.nlines; kp.line_oc = 0; kp.stride = (long long)na * nb; }
    kp.n = n;
    kp.nb = sw.nb;
    kp.nbord = sw.nbord;
    kp.P = (n % 2 == 0) ? n + 1 : n;
    kp.S = lay.S;
    kp.base = lay.base;
    kp.rem = lay.rem;
    kp.L = lines;
    kp.bc1 = bc1;
    kp.bcn = bcn;
    kp.tab = tab.data();
    kp.segsum = segsum.data();
    std::memcpy(kp.mb, sw.mb, sizeof(kp.mb));
    double taps[9];
    interior_taps(rc, taps);
    for (int k = 0; k < 9; ++k) kp.taps[k] = taps[8 - k];
    if (adjoint && !periodic) {
        bt = transposed_stencil_blocks(rc, n, bc1, bcn);
        kp.bt = bt.data();
    }
    kp.rc = rc;
    const Interior in = interior_info(sw, lay, m);
    kp.int_mask = fast ? in.mask : 0u;
    std::memcpy(kp.kc, in.kc, sizeof(kp.kc));
    std::memcpy(kp.pat, in.pat, sizeof(kp.pat));
    const int nthreads = lines * lay.S + extra_threads;
    switch (rc.rk) {
    case RHS_CD06_D1: return pick<RHS_CD06_D1>(kp, periodic, adjoint, m, nthreads);
    case RHS_CD10_D1: return pick<RHS_CD10_D1>(kp, periodic, adjoint, m, nthreads);
    case RHS_CD10_D2: return pick<RHS_CD10_D2>(kp, periodic, adjoint, m, nthreads);
    default: return pick<RHS_CF90>(kp, periodic, adjoint, m, nthreads);
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

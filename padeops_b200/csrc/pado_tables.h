// pado_tables.h -- host-side construction of the solver tables the device
// kernels consume: the reference's LU / Thomas / penta factorizations, their
// conversion into the unified sweep of pado_common.h, the adjoint (transposed)
// sweep, the segment-partition responses, and the transposed stencil blocks.
#pragma once

#include <vector>

#include "pado_common.h"

namespace pado {

// Unified sweep coefficients for one operator (see the comment block at the
// end of pado_common.h).  Vectors have nb entries.
struct Sweep {
    int n = 0, nb = 0, nbord = 0;
    std::vector<double> alpha, c1, c2, k1, k2, gamma, d1, d2, e1, e2, delta;
    double mb[4] = {0, 0, 0, 0};  // border map, row-major nbord x nbord
};

// Reference factorizations, column-major (n, ncol) like the Fortran arrays.
// cd06.F90:221-262
std::vector<double> cd06_cyclic_lu(int n, double b, double d, double a);
// cd06.F90:264-327
std::vector<double> cd06_tri1(int n, int bc1, int bcn);
// cd10.F90:351-427, cf90.F90:198-274
std::vector<double> penta_cyclic_lu(int n, double e, double a, double d, double c, double f);
// cd10.F90:429-578 (kind D1), :580-709 (D2), cf90.F90:276-418 (filter)
std::vector<double> penta_bounded(int scheme, int kind, int n, int bc1, int bcn);

// The sweep that reproduces the reference's solve for (scheme, kind).
// bc1/bcn: closures of a bounded line (cd06 uses its init closures).
Sweep primal_sweep(int scheme, int kind, int n, int periodic, int bc1, int bcn);
// The sweep of the transposed solve A^{-T}.
Sweep adjoint_sweep(const Sweep &p);

// Cut of [0, n) into S <= 32 segments, segment s = rows [st[s], st[s+1]).
struct Layout {
    int n = 0, S = 1;
    std::vector<int> st{0, 0};
    int start(int s) const { return st[s]; }
    int len(int s) const { return st[s + 1] - st[s]; }
};
// With an interior [i0, i1) (i0 < i1): as many segments of exactly m rows as
// fit in it, and the rows before and after cut into pieces of e_rows rows
// (edge_piece_rows of pado_common.h; 0: m/2), the kernels' fully unrolled
// per-row-table path, when n is a multiple of e_rows, else into near-equal
// pieces of about m/3 rows (the generic per-row loop).
// Without one: ceil(n/m) segments of near-equal length.
constexpr int MAX_SEGMENTS = 32;
Layout make_layout(int n, int m, int i0 = 0, int i1 = 0, int e_rows = 0);
// Banded rows [i0, i1) whose coefficients have settled (see Interior);
// i0 == i1 == 0 when there are none.
void interior_range(const Sweep &sw, int *i0, int *i1);

// Device table: T_NF doubles per banded row (TabField order) with the
// segment responses folded in, plus 4 segment sums per segment
// (k1.U, k1.V, k2.U, k2.V).
void build_device_table(const Sweep &sw, const Layout &lay, std::vector<double> &tab, std::vector<double> &segsum);

// Constant-coefficient interior.  Away from the line ends the factor
// coefficients of every sweep converge to constants (within ~20-90 rows) and
// the cyclic spike terms decay to nothing.  Segments that lie wholly in that
// region, have length m and a full stencil window inside the line run a
// register-only path: constant coefficients, and the inter-segment
// corrections read from the unit responses below.
constexpr int MAXM = 64;  // longest segment a kernel is built for
struct Interior {
    unsigned mask = 0;       // bit s: segment s takes the constant-coefficient path
    unsigned spk_mask = 0;   // bit s: ... and adds the cyclic spike terms of its rows
    double kc[8] = {0};      // alpha, c1, c2, gamma, d1, d2, delta, (unused)
    // responses of a length-m segment, rows t = 0..m-1: forward sweep to the
    // unit incoming states z_{-1} (pu) and z_{-2} (pv); backward sweep to
    // x_m (ps) and x_{m+1} (pt)
    double pu[MAXM] = {0}, pv[MAXM] = {0}, ps[MAXM] = {0}, pt[MAXM] = {0};
    int i0 = 0, i1 = 0;      // banded rows treated as interior
};
Interior interior_info(const Sweep &sw, const Layout &lay, int m);

// Inter-segment coupling.  With A_s = [[U(b-1), V(b-1)], [U(b-2), V(b-2)]]
// the forward transfer of segment s (a, b: first rows of segments s and
// s+1) and B_s = [[S(a), T(a)], [S(a+1), T(a+1)]] the backward one, the
// incoming states are
//   P_s = sum_{j<s} Phi(s,j) y_j,  Phi(s,j) = A_{s-1} ... A_{j+1}
//   Q_s = sum_{j>s} Psi(s,j) w_j,  Psi(s,j) = B_{s+1} ... B_{j-1}
// (y_j, w_j: the local end / first values of segment j).  The products decay
// like the sweep's homogeneous solutions; those below XFER_DROP are dropped,
// which bounds the window W (a dropped product moves the result by less than
// 1e-17 of the coupled segment's end value, far below FP64 rounding).
//   xtab: packed 2x2 blocks (4 doubles, row-major): Phi(s, s-d) for d =
//         1..wf[s] from block xof[s], Psi(s, s+d) for d = 1..wb[s] from xob[s]
//   ctab [S][CT_NF]: G1_s, G2_s with G_s = sum_{t>s} k_t Phi(t, s), k_t the
//                    (k.U, k.V) sums of segment t: the cyclic border sums are
//                    sum_s (local sum_s + G_s . y_s)
// Constant-coefficient segments take the responses of Interior.
constexpr int CT_NF = 4;
constexpr double XFER_DROP = 1e-17;
struct ChainTables {
    std::vector<double> ctab, xtab;
    int W = 0;  // largest window
    unsigned char wf[MAX_SEGMENTS] = {0}, wb[MAX_SEGMENTS] = {0};  // per-segment windows
    unsigned short xof[MAX_SEGMENTS] = {0}, xob[MAX_SEGMENTS] = {0};  // first block of each list
};
ChainTables chain_tables(const std::vector<double> &tab, const std::vector<double> &segsum, const Layout &lay, int nb,
                         const Interior &in, int m);

// Rows of the segments that read the per-row table (every segment not in
// `mask`), packed in segment order (etab, the E_NF fields of EtabField per
// row), and the cyclic sums' spike values (k1, k2) of the rows of the
// segments in `spk` (ktab, 2 per row); toff[s] = first packed row of segment s
// in its table (0 otherwise).  tri: a tridiagonal sweep, whose c2 slot
// carries delta instead (E_DELTA).
constexpr int KT_NF = 2;
void edge_table(const std::vector<double> &tab, const Layout &lay, int nb, unsigned mask, unsigned spk, bool tri,
                std::vector<double> &etab, std::vector<double> &ktab, std::vector<int> &toff);

// Everything a kernel launch reads for one (scheme, kind, closures,
// direction) operator, on the host.
struct OpTables {
    int nb = 0, nbord = 0, m = 0;
    double mb[4] = {0, 0, 0, 0};
    double taps[9] = {0};  // adjoint: transposed interior taps (tap at offset o is c_{-o})
    Layout lay;
    RhsCoef rc{};
    Interior interior;
    std::vector<double> tab, etab, ktab, bt;
    // cyclic lines: responses of the backward sweep to its spike columns,
    // x = x(E = 0) + E1 R1 + E2 R2, kept on rows [0, ie) and [je, nb) (in
    // between they are below 1e-17 of their largest magnitude), stored as
    // (R1, R2) pairs, the rows of [0, ie) first
    std::vector<double> rtab;
    int ie = 0, je = 0;
    ChainTables chain;        // coupling of the segments as the kernels run them
    ChainTables chain_exact;  // with every segment on the per-row table
    std::vector<int> toff;
    unsigned char sperm[32] = {0};  // thread slot -> segment: per-row-table segments first
};
OpTables make_op_tables(int scheme, int kind, int n, double dx, int periodic, int bc1, int bcn, int m, bool adjoint);

// Thread-slot order for kernels whose threads are (line tid % L, slot
// tid / L): segments grouped by the code path they take -- per-row table;
// constant-coefficient with cyclic spike sums and border responses; with
// spike sums only; with border responses only; plain constant-coefficient --
// each group padded with idle slots (0xff) to whole warps (32 / L slots per
// warp), so that no warp runs two paths one after the other.  border_warp:
// one warp of idle slots first (cyclic lines), whose first slot -- the
// first idle one -- solves the border unknowns while the others sweep.  Returns the slot count, or the
// unpadded order's S when the padded one needs more than max_slots.
int warp_slots(const OpTables &ot, int L, unsigned char *sperm, int max_slots, bool border_warp = false);
// First idle slot of a slot order (-1: none).
inline int first_idle_slot(const unsigned char *sperm, int nslots)
{
    for (int k = 0; k < nslots; ++k)
        if (sperm[k] == 0xff) return k;
    return -1;
}

// Transposed stencil of a bounded line: B^T rows for the first and last
// ZB columns.  Dense (n x n) when n <= DENSE_BT_MAX.
constexpr int BT_ZONE = 8, BT_WIN = 12, DENSE_BT_MAX = 32;
std::vector<double> transposed_stencil_blocks(const RhsCoef &rc, int n, int bc1, int bcn);

// Dense B (n x n, row-major) of the explicit stencil; used by the builder
// above and by the self-checks.
std::vector<double> stencil_matrix(const RhsCoef &rc, int n, int bc1, int bcn);

}  // namespace pado

// pado_internal.h -- definitions shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/pado.h"
#include "pado_kernels.cuh"
#include "pado_params.h"
#include "pado_stream.cuh"
#include "pado_tables.h"

namespace pado {

extern std::atomic<long long> g_launches;

// Device-resident tables of one (kind, bc1, bcn, direction) operator, and
// the host copy they were uploaded from.
struct DevTables {
    OpTables host;
    double *tab = nullptr;         // [nb][T_NF]
    double *ctab = nullptr;        // [S][CT_NF] border-sum weights
    double *xtab = nullptr;        // [S][W][8] transfer products
    double *ctab_exact = nullptr;  // the same with every segment on the per-row table
    double *xtab_exact = nullptr;
    double *etab = nullptr;        // packed rows of the segments that read the table
    double *ktab = nullptr;        // packed spike values of the spiky interior segments
    double *rtab = nullptr;        // border-unknown responses (cyclic lines)
    int *toff = nullptr;           // [S]
    double *bt = nullptr;          // transposed stencil blocks (adjoint, bounded)
};

using TabKey = std::tuple<int, int, int, int>;  // kind, bc1, bcn, adjoint

// The streaming kernel's tiling for one (tables, line direction, copy path,
// direction of the solve, requested tiling) of a handle, chosen once by the
// planner: lines per tile, stages, CTAs per SM, thread slots and their
// segments.
struct StreamChoice {
    int L = 0, stages = 0, ctas = 0, nslots = 0;
    unsigned char perm[KMAXSLOT] = {0};
};
using PlanKey = std::tuple<const void *, int, int, int, int, int>;  // tables, x lines, async, adjoint, lines, stages

int cuda_fail(cudaError_t e);
bool kind_supported(int scheme, int kind);
bool valid_bc(int bc);

}  // namespace pado

struct pado_op_s {
    int scheme = 0, n = 0, periodic = 1, bc1 = 0, bcn = 0;
    double dx = 1.0;
    int m = 32, lines = 16;
    int variant = 0;  // 0: automatic; 1..3: one-CTA-per-tile / persistent kernels; 4: streaming kernel
    int device = 0;
    int *d_status = nullptr;  // device-side status word (bounded waits)
    int stream_lines = 0, stream_stages = 0;  // streaming kernel tiling (0: chosen by occupancy)
    mutable std::mutex plan_mu;                                      // guards plan_cache
    mutable std::map<pado::PlanKey, pado::StreamChoice> plan_cache;  // the planner's choices
    std::map<pado::TabKey, pado::DevTables> tables;
    std::vector<void *> allocations;
    // host-buffer staging
    std::mutex staging_mu;
    double *stage_f = nullptr, *stage_df = nullptr;
    size_t stage_elems = 0;
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;  // copy streams of the host-buffer pipeline
    std::vector<cudaEvent_t> ev_in, ev_out;          // per chunk: copied in / computed
};

namespace pado {

// Validates an apply request and fills the launch parameters for the given
// lines-per-CTA.  Returns PADO_OK, or an error; *trivial is set when n == 1
// or the field is empty (nothing for a line kernel to do).
// Kernel entry points, one translation unit per stencil (pado_inst.cu built
// with -DPADO_RK=0..3).
using KernelFn = void (*)(const KParams);
KernelFn pick_kernel_rk0(bool per, bool adj, bool contiguous, int m, int variant);
KernelFn pick_kernel_rk1(bool per, bool adj, bool contiguous, int m, int variant);
KernelFn pick_kernel_rk2(bool per, bool adj, bool contiguous, int m, int variant);
KernelFn pick_kernel_rk3(bool per, bool adj, bool contiguous, int m, int variant);
using StreamFn = void (*)(const StreamParams);
// streaming kernels: strided lines are built for 8, 16 or 32 lines per tile
// (`lines`), x lines for any; adj: the adjoint (transposed sweep, then B^T)
StreamFn pick_stream_rk0(bool per, int m, bool xl, int lines, bool adj, bool as);
StreamFn pick_stream_rk1(bool per, int m, bool xl, int lines, bool adj, bool as);
StreamFn pick_stream_rk2(bool per, int m, bool xl, int lines, bool adj, bool as);
StreamFn pick_stream_rk3(bool per, int m, bool xl, int lines, bool adj, bool as);

// no_fast: every segment on the per-row table (for kernels built for a
// segment length other than the handle's).
// solve_bc1/solve_bcn: the closures whose system is solved, when they differ
// from the right-hand side's (bc1, bcn); SAME_BC: the same.
constexpr int SAME_BC = 99;
// Forward apply through the resident tile kernel with plain loads (for fields
// the streaming kernel's copies cannot move); PADO_E_UNSUPPORTED when the
// field does not fit it.  info != nullptr: report the plan, launch nothing.
// out_mode / out_alpha: how results reach df (OutMode of pado_kernels.cuh).
int launch_resident_single(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb,
                           int bc1, int bcn, cudaStream_t st, int *info = nullptr, int out_mode = OUT_STORE,
                           double out_alpha = 1.0);
int prepare_launch(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                   int bcn, bool adjoint, int lines, bool no_fast, KParams *kp, bool *trivial, int solve_bc1 = SAME_BC,
                   int solve_bcn = SAME_BC, int out_mode = OUT_STORE, double out_alpha = 1.0);

}  // namespace pado

// pado_api.cu -- the C ABI of include/pado.h: scheme objects, table upload,
// kernel dispatch and the host-buffer path.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "pado_internal.h"

#include <algorithm>

using namespace pado;

namespace pado {
std::atomic<long long> g_launches{0};
}

namespace pado {

int cuda_fail(cudaError_t e)
{
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? PADO_E_NOMEM : PADO_E_CUDA;
}

bool valid_bc(int bc) { return bc == 0 || bc == 1 || bc == -1; }

bool kind_supported(int scheme, int kind)
{
    if (scheme == CD06) return kind == D1;  // cd06 d2 is "Incomplete" in the reference (cd06.F90:492-513)
    if (scheme == CD10) return kind == D1 || kind == D2;
    return kind == FILTER;
}

}  // namespace pado

namespace {

int max_threads_for_m(int m) { return m >= 64 ? 256 : 512; }

int upload(pado_op_s *op, const std::vector<double> &h, double **d)
{
    if (h.empty()) {
        *d = nullptr;
        return PADO_OK;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, h.size() * sizeof(double));
    if (e != cudaSuccess) return cuda_fail(e);
    op->allocations.push_back(p);
    e = cudaMemcpy(p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e);
    *d = static_cast<double *>(p);
    return PADO_OK;
}

// Default tiling: segment length and lines per CTA for a line of length n.
void default_tiling(int n, int *m, int *lines)
{
    *m = n > 32 * 32 ? 64 : (n >= 96 ? 32 : 16);
    const int S = (n + *m - 1) / *m;
    int L = 32;
    while (L > 8 && L * S > max_threads_for_m(*m)) L /= 2;
    *lines = L;
}

int build_tables(pado_op_s *op)
{
    for (void *p : op->allocations) cudaFree(p);
    op->allocations.clear();
    op->tables.clear();
    const int n = op->n;
    if (n == 1) return PADO_OK;
    std::vector<int> kinds;
    for (int k : {FILTER, D1, D2})
        if (kind_supported(op->scheme, k)) kinds.push_back(k);
    std::vector<std::pair<int, int>> bcs;
    if (op->periodic || op->scheme == CD06) bcs.push_back({0, 0});
    else
        for (int b1 : {0, 1, -1})
            for (int bn : {0, 1, -1}) bcs.push_back({b1, bn});
    for (int kind : kinds) {
        for (auto [b1, bn] : bcs) {
            // cd06 takes its closures from init (cd06.F90:177)
            const int cb1 = op->scheme == CD06 ? op->bc1 : b1, cbn = op->scheme == CD06 ? op->bcn : bn;
            const Sweep prim = primal_sweep(op->scheme, kind, n, op->periodic, cb1, cbn);
            const Sweep adj = adjoint_sweep(prim);
            const RhsCoef rc = make_rhs_coef(op->scheme, kind, op->dx, op->periodic);
            const Layout lay = make_layout(n, op->m);
            for (int dir = 0; dir < 2; ++dir) {
                const Sweep &sw = dir == 0 ? prim : adj;
                DevTables dt;
                dt.nb = sw.nb;
                dt.nbord = sw.nbord;
                dt.lay = lay;
                dt.rc = rc;
                std::memcpy(dt.mb, sw.mb, sizeof(dt.mb));
                std::vector<double> tab, segsum;
                build_device_table(sw, lay, tab, segsum);
                dt.interior = interior_info(sw, lay, op->m);
                int rc_ = upload(op, tab, &dt.tab);
                if (rc_ == PADO_OK) rc_ = upload(op, segsum, &dt.segsum);
                if (rc_ != PADO_OK) return rc_;
                if (dir == 1) {
                    double taps[9];
                    interior_taps(rc, taps);
                    for (int k = 0; k < 9; ++k) dt.taps[k] = taps[8 - k];  // B^T: tap at offset o is c_{-o}
                    if (!op->periodic) {
                        rc_ = upload(op, transposed_stencil_blocks(rc, n, cb1, cbn), &dt.bt);
                        if (rc_ != PADO_OK) return rc_;
                    }
                }
                op->tables[TabKey(kind, b1, bn, dir)] = dt;
            }
        }
    }
    return PADO_OK;
}

KernelFn pick_kernel(int rk, bool per, bool adj, bool contiguous, int m, int variant)
{
    switch (rk) {
    case RHS_CD06_D1: return pick_kernel_rk0(per, adj, contiguous, m, variant);
    case RHS_CD10_D1: return pick_kernel_rk1(per, adj, contiguous, m, variant);
    case RHS_CD10_D2: return pick_kernel_rk2(per, adj, contiguous, m, variant);
    default: return pick_kernel_rk3(per, adj, contiguous, m, variant);
    }
}

// Geometry of the line family for (axis, na, nb).
void set_geometry(KParams &kp, int axis, int n, long long na, long long nb)
{
    kp.nlines = na * nb;
    if (axis == 1) {
        kp.line_ia = 1;
        kp.line_oc = n;
        kp.stride = 1;
    } else if (axis == 2) {
        kp.line_ia = na;
        kp.line_oc = na * (long long)n;
        kp.stride = na;
    } else {
        kp.line_ia = kp.nlines > 0 ? kp.nlines : 1;
        kp.line_oc = 0;
        kp.stride = na * nb;
    }
}

}  // namespace

int pado::prepare_launch(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                         int bcn, bool adjoint, int lines, KParams *kpo, bool *trivial)
{
    *trivial = true;
    if (!op) return PADO_E_NULL;
    if (axis < 1 || axis > 3 || na < 0 || nb < 0) return PADO_E_ARG;
    if (!kind_supported(op->scheme, kind)) return PADO_E_UNSUPPORTED;
    // the reference validates bc before looking at periodicity (cd10.F90:2042-2058)
    if (op->scheme != CD06 && (!valid_bc(bc1) || !valid_bc(bcn))) return PADO_E_BC;
    const int n = op->n;
    const long long total = (long long)n * na * nb;
    if (na > 0 && nb > 0 && total / na / nb != n) return PADO_E_SIZE;
    if (total == 0) return PADO_OK;
    if (!f || !df) return PADO_E_NULL;
    if (f < df + total && df < f + total) return PADO_E_ALIAS;
    if (n == 1) return PADO_OK;
    const bool bounded_bc = !op->periodic && op->scheme != CD06;
    auto it = op->tables.find(TabKey(kind, bounded_bc ? bc1 : 0, bounded_bc ? bcn : 0, adjoint ? 1 : 0));
    if (it == op->tables.end()) return PADO_E_STATE;
    const DevTables &dt = it->second;

    KParams kp{};
    kp.in = f;
    kp.out = df;
    set_geometry(kp, axis, n, na, nb);
    kp.n = n;
    kp.nb = dt.nb;
    kp.nbord = dt.nbord;
    kp.P = (n % 2 == 0) ? n + 1 : n;
    kp.S = dt.lay.S;
    kp.base = dt.lay.base;
    kp.rem = dt.lay.rem;
    kp.L = lines;
    kp.bc1 = op->scheme == CD06 ? op->bc1 : bc1;
    kp.bcn = op->scheme == CD06 ? op->bcn : bcn;
    kp.tab = dt.tab;
    kp.segsum = dt.segsum;
    kp.bt = dt.bt;
    std::memcpy(kp.mb, dt.mb, sizeof(kp.mb));
    std::memcpy(kp.taps, dt.taps, sizeof(kp.taps));
    kp.rc = dt.rc;
    kp.int_mask = dt.interior.mask;
    std::memcpy(kp.kc, dt.interior.kc, sizeof(kp.kc));
    std::memcpy(kp.pat, dt.interior.pat, sizeof(kp.pat));
    *kpo = kp;
    *trivial = false;
    return PADO_OK;
}

namespace {

int launch(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1, int bcn,
           cudaStream_t st, bool adjoint)
{
    KParams kp;
    bool trivial = true;
    int rc = prepare_launch(op, kind, axis, f, df, na, nb, bc1, bcn, adjoint, op ? op->lines : 0, &kp, &trivial);
    if (rc != PADO_OK) return rc;
    if (trivial) {
        const long long total = (long long)op->n * na * nb;
        if (total == 0) return PADO_OK;
        // n == 1: cd06.F90:781-784, cd10.F90:2037-2040 (zero), cf90.F90:1028-1031 (copy)
        cudaError_t e = (kind == FILTER) ? cudaMemcpyAsync(df, f, total * sizeof(double), cudaMemcpyDeviceToDevice, st)
                                         : cudaMemsetAsync(df, 0, total * sizeof(double), st);
        return e == cudaSuccess ? PADO_OK : cuda_fail(e);
    }
    const int threads = kp.L * kp.S;
    if (threads > max_threads_for_m(op->m)) return PADO_E_SIZE;
    const bool contiguous = kp.stride == 1;
    const bool persist = !adjoint && (op->variant == 2 || (op->variant == 3 && !contiguous));
    const size_t tile = (adjoint || contiguous) ? (size_t)kp.L * kp.P : (op->variant == 2 ? (size_t)kp.n * kp.L : 0);
    const size_t smem = smem_doubles(kp.L, kp.S, tile) * sizeof(double);
    if (smem > 227 * 1024) return PADO_E_SIZE;
    KernelFn fn = pick_kernel(kp.rc.rk, op->periodic != 0, adjoint, contiguous, op->m, op->variant);
    int per_sm = 1;
    {
        static std::mutex attr_mu;
        std::lock_guard<std::mutex> g(attr_mu);
        cudaError_t e = cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
        if (e != cudaSuccess) return cuda_fail(e);
        if (per_sm < 1) return PADO_E_SIZE;
    }
    const long long ntiles = (kp.nlines + kp.L - 1) / kp.L;
    long long grid = ntiles;
    if (persist) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        grid = std::min<long long>(ntiles, (long long)per_sm * sms);
    }
    if (grid > 0x7fffffffLL) return PADO_E_SIZE;
    fn<<<(unsigned)grid, threads, smem, st>>>(kp);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

}  // namespace

extern "C" {

int pado_create(pado_op_t *out, int scheme, int n, double dx, int periodic, int bc1, int bcn)
{
    if (!out) return PADO_E_NULL;
    *out = nullptr;
    if (scheme < CD06 || scheme > CF90 || n < 1) return PADO_E_ARG;
    if (scheme != CF90 && !(dx > 0.0 || dx < 0.0)) return PADO_E_ARG;
    periodic = periodic ? 1 : 0;
    // Size checks of the reference's init (cd06.F90:153-183, cd10.F90:219-309, cf90.F90:123-168)
    if (n != 1) {
        if (scheme == CD06 && periodic && n < 6) return 3;
        if (scheme == CD06 && !periodic && n < 8) return 2;
        if (scheme == CD10 && n < 8) return 2;
        if (scheme == CF90 && n < 10) return 7;
    }
    if (n > 32 * 64) return PADO_E_SIZE;
    auto *op = new (std::nothrow) pado_op_s;
    if (!op) return PADO_E_NOMEM;
    op->scheme = scheme;
    op->n = n;
    op->dx = scheme == CF90 ? 1.0 : dx;
    op->periodic = periodic;
    op->bc1 = bc1;
    op->bcn = bcn;
    cudaGetDevice(&op->device);
    default_tiling(n, &op->m, &op->lines);
    int rc = build_tables(op);
    if (rc != PADO_OK) {
        pado_destroy(op);
        return rc;
    }
    *out = op;
    return PADO_OK;
}

int pado_cd06_init(pado_op_t *op, int n, double dx, int periodic, int bc1, int bcn)
{
    return pado_create(op, CD06, n, dx, periodic, bc1, bcn);
}
int pado_cd10_init(pado_op_t *op, int n, double dx, int periodic, int bc1, int bcn)
{
    return pado_create(op, CD10, n, dx, periodic, bc1, bcn);
}
int pado_cf90_init(pado_op_t *op, int n, int periodic) { return pado_create(op, CF90, n, 1.0, periodic, 0, 0); }

void pado_destroy(pado_op_t op)
{
    if (!op) return;
    for (void *p : op->allocations) cudaFree(p);
    if (op->stage_f) cudaFree(op->stage_f);
    if (op->stage_df) cudaFree(op->stage_df);
    delete op;
}

int pado_get_size(pado_op_t op) { return op ? op->n : PADO_E_NULL; }

int pado_apply(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1, int bcn,
               void *stream)
{
    return launch(op, kind, axis, f, df, na, nb, bc1, bcn, (cudaStream_t)stream, false);
}

int pado_apply_adjoint(pado_op_t op, int kind, int axis, const double *g, double *fbar, long na, long nb, int bc1,
                       int bcn, void *stream)
{
    return launch(op, kind, axis, g, fbar, na, nb, bc1, bcn, (cudaStream_t)stream, true);
}

#define PADO_NAMED(name, kind, axis)                                                                        \
    int name(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream)    \
    {                                                                                                        \
        return launch(op, kind, axis, f, df, na, nb, bc1, bcn, (cudaStream_t)stream, false);                 \
    }
PADO_NAMED(pado_dd1, D1, 1)
PADO_NAMED(pado_dd2, D1, 2)
PADO_NAMED(pado_dd3, D1, 3)
PADO_NAMED(pado_d2d1, D2, 1)
PADO_NAMED(pado_d2d2, D2, 2)
PADO_NAMED(pado_d2d3, D2, 3)
PADO_NAMED(pado_filter1, FILTER, 1)
PADO_NAMED(pado_filter2, FILTER, 2)
PADO_NAMED(pado_filter3, FILTER, 3)
#undef PADO_NAMED

int pado_apply_host(pado_op_t op, int kind, int axis, const double *f_host, double *df_host, long na, long nb,
                    int bc1, int bcn, void *stream)
{
    if (!op) return PADO_E_NULL;
    if (na < 0 || nb < 0) return PADO_E_ARG;
    const size_t total = (size_t)op->n * (size_t)na * (size_t)nb;
    if (total == 0) return PADO_OK;
    if (!f_host || !df_host) return PADO_E_NULL;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(op->staging_mu);
    if (op->stage_elems < total) {
        if (op->stage_f) cudaFree(op->stage_f);
        if (op->stage_df) cudaFree(op->stage_df);
        op->stage_f = op->stage_df = nullptr;
        op->stage_elems = 0;
        cudaError_t e = cudaMalloc(&op->stage_f, total * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&op->stage_df, total * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(e);
        op->stage_elems = total;
    }
    cudaError_t e = cudaMemcpyAsync(op->stage_f, f_host, total * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e);
    int rc = launch(op, kind, axis, op->stage_f, op->stage_df, na, nb, bc1, bcn, st, false);
    if (rc != PADO_OK) return rc;
    e = cudaMemcpyAsync(df_host, op->stage_df, total * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

int pado_set_tiling(pado_op_t op, int m, int lines)
{
    if (!op) return PADO_E_NULL;
    if (m != 0 && m != 16 && m != 32 && m != 64) return PADO_E_ARG;
    if (lines != 0 && lines != 8 && lines != 16 && lines != 32) return PADO_E_ARG;
    const int om = op->m, ol = op->lines;
    if (m) op->m = m;
    if (lines) op->lines = lines;
    const int S = (op->n + op->m - 1) / op->m;
    if (S > 32 || op->lines * S > max_threads_for_m(op->m)) {
        op->m = om;
        op->lines = ol;
        return PADO_E_SIZE;
    }
    if (op->m != om) return build_tables(op);
    return PADO_OK;
}

int pado_set_kernel_variant(pado_op_t op, int variant)
{
    if (!op) return PADO_E_NULL;
    if (variant < 0 || variant > 3) return PADO_E_ARG;
    op->variant = variant == 0 ? 1 : variant;
    return PADO_OK;
}

int pado_get_tiling(pado_op_t op, int *m, int *lines)
{
    if (!op) return PADO_E_NULL;
    if (m) *m = op->m;
    if (lines) *lines = op->lines;
    return PADO_OK;
}

const char *pado_strerror(int s)
{
    switch (s) {
    case PADO_OK: return "ok";
    case 2: return "n too small for this scheme (reference ierr 2)";
    case 3: return "n too small for periodic cd06 (reference ierr 3)";
    case 7: return "n too small for cf90 (reference ierr 7)";
    case PADO_E_BC: return "boundary specification must be 0, 1 or -1";
    case PADO_E_NULL: return "null handle or pointer";
    case PADO_E_ALIAS: return "input and output overlap";
    case PADO_E_UNSUPPORTED: return "operator not provided by this scheme";
    case PADO_E_ARG: return "invalid argument";
    case PADO_E_CUDA: return "CUDA runtime error";
    case PADO_E_SIZE: return "size out of the supported range";
    case PADO_E_TIMEOUT: return "bounded device wait expired";
    case PADO_E_NOMEM: return "out of memory";
    case PADO_E_STATE: return "object not in a state that allows the call";
    default: return "unknown status";
    }
}

long long pado_launch_count(void) { return pado::g_launches.load(); }

const char *pado_version(void) { return "padeops_b200 0.1 (sm_100a, FP64)"; }

}  // extern "C"

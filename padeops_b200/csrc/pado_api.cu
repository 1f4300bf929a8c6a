// pado_api.cu -- the C ABI of include/pado.h: scheme objects, table upload,
// kernel dispatch and the host-buffer path.
#include <cuda.h>
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
static_assert(PADO_STATUS_TIMEOUT == PADO_E_TIMEOUT, "device and host timeout codes differ");
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

// host-buffer pipeline: about this many bytes per chunk, at most this many chunks
constexpr size_t HOST_CHUNK_BYTES = size_t(16) << 20;
constexpr size_t HOST_MAX_CHUNKS = 128;

int max_threads_for_m(int m) { return m >= 64 ? 256 : 512; }

// When the streaming kernel cannot run, the automatic choice takes the
// resident tiles with plain loads (variant 5) where they beat the line kernel
// (measured at 511^3): x lines, and the tridiagonal cd06 sweeps on any axis;
// the line kernel elsewhere.
bool resident_fallback(const pado_op_s *op, int axis) { return axis == 1 || op->scheme == CD06; }

// Default tiling: segment length and lines per CTA for a line of length n.
void default_tiling(int n, int *m, int *lines)
{
    *m = n >= 32 * 32 ? 64 : (n >= 96 ? 32 : 16);
    const int S = (n + *m - 1) / *m;
    int L = 32;
    while (L > 8 && L * S > max_threads_for_m(*m)) L /= 2;
    *lines = L;
}

template <typename T>
int upload_vec(pado_op_s *op, const std::vector<T> &h, T **d)
{
    *d = nullptr;
    if (h.empty()) return PADO_OK;
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, h.size() * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e);
    op->allocations.push_back(p);
    e = cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e);
    *d = static_cast<T *>(p);
    return PADO_OK;
}

int build_tables(pado_op_s *op)
{
    for (void *p : op->allocations) cudaFree(p);
    op->allocations.clear();
    op->tables.clear();
    {
        std::lock_guard<std::mutex> g(op->plan_mu);
        op->plan_cache.clear();  // its keys name the tables
    }
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
            for (int dir = 0; dir < 2; ++dir) {
                DevTables dt;
                dt.host = make_op_tables(op->scheme, kind, n, op->dx, op->periodic, cb1, cbn, op->m, dir == 1);
                const OpTables &h = dt.host;
                int rc = upload_vec(op, h.tab, &dt.tab);
                if (rc == PADO_OK) rc = upload_vec(op, h.chain.ctab, &dt.ctab);
                if (rc == PADO_OK) rc = upload_vec(op, h.chain.xtab, &dt.xtab);
                if (rc == PADO_OK) rc = upload_vec(op, h.chain_exact.ctab, &dt.ctab_exact);
                if (rc == PADO_OK) rc = upload_vec(op, h.chain_exact.xtab, &dt.xtab_exact);
                if (rc == PADO_OK) rc = upload_vec(op, h.etab, &dt.etab);
                if (rc == PADO_OK) rc = upload_vec(op, h.ktab, &dt.ktab);
                if (rc == PADO_OK) rc = upload_vec(op, h.rtab, &dt.rtab);
                if (rc == PADO_OK) rc = upload_vec(op, h.toff, &dt.toff);
                if (rc == PADO_OK) rc = upload_vec(op, h.bt, &dt.bt);
                if (rc != PADO_OK) return rc;
                op->tables[TabKey(kind, b1, bn, dir)] = std::move(dt);
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

// cuTensorMapEncodeTiled, from the driver through the runtime (no link
// against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

StreamFn pick_stream(int rk, bool per, int m, bool xl, int lines, bool adj, bool as)
{
    switch (rk) {
    case RHS_CD06_D1: return pick_stream_rk0(per, m, xl, lines, adj, as);
    case RHS_CD10_D1: return pick_stream_rk1(per, m, xl, lines, adj, as);
    case RHS_CD10_D2: return pick_stream_rk2(per, m, xl, lines, adj, as);
    default: return pick_stream_rk3(per, m, xl, lines, adj, as);
    }
}

int round16(long long v) { return (int)((v + 15) / 16 * 16); }

// Pitch of an x-line tile: n + 2 (rows 16-byte aligned) for the bulk copies;
// the odd kp.P (n or n + 1) for per-element copies, so that the threads of a
// warp, which sweep 16 different lines, hit different banks.
int stream_xl_pitch(int n, bool as) { return as ? (n % 2 == 0 ? n + 1 : n) : n + 2; }

// Doubles of one stage buffer: [L][pitch] (x lines), nbox boxes of
// box_rows x L (strided lines, tensor copies) or n x L (strided lines,
// per-element copies), rounded to 128 bytes.
int stream_tile_doubles(bool xl, int n, int L, bool as)
{
    if (xl) return round16((long long)L * stream_xl_pitch(n, as));
    if (as) return round16((long long)n * L);
    const int nbox = (n + 255) / 256, box_rows = ((n + nbox - 1) / nbox + 15) / 16 * 16;
    return round16((long long)nbox * box_rows * L);
}

// Lets a streaming kernel use up to 227 KB of shared memory (once per kernel).
bool grant_smem(StreamFn fn)
{
    static std::mutex mu;
    static std::map<const void *, bool> granted;
    std::lock_guard<std::mutex> g(mu);
    bool &ok = granted[(const void *)fn];
    if (!ok) {
        if (cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) !=
            cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        ok = true;
    }
    return true;
}

// Plan of a streaming launch (primal): lines per tile, stages, shared memory
// and the copy descriptors, chosen for the most resident warps per SM.  False
// when the field or tiling does not fit it (odd strides, unaligned pointers,
// a table too large to stage); the caller then runs the one-CTA-per-tile
// kernel.
// The streaming kernel's tiling for one (tables, direction, copy path).  The
// candidates are tried in order of preference (16 lines and one stage, two
// CTAs per SM, is fastest for every operator at n = 512; a larger tile only
// pays for short lines); the first that fits two CTAs per SM wins, else the
// one with the most resident warps.  One exception, measured on lines of 64
// to 256 points: 32 lines per tile beat 16 by 3-24% (x lines, and y/z lines
// of every operator but bounded cd06, which keeps 16 from n = 256) whenever
// they keep at least as many threads resident (two CTAs or more per SM).
bool choose_stream_tiling(const pado_op_s *op, const DevTables &dt, const KParams &kp0, bool xl, bool as, bool adj,
                          int etab_rows, int ktab_rows, StreamChoice *out)
{
    const int n = op->n, S = kp0.S;
    struct Cand {
        StreamChoice c;
        bool ok = false;
    };
    const int cand[6][2] = {{16, 1}, {32, 1}, {8, 1}, {16, 2}, {32, 2}, {8, 2}};
    Cand res[6];
    for (int i = 0; i < 6; ++i) {
        const int L = cand[i][0], stages = cand[i][1];
        // slots grouped by code path, padded to whole warps
        unsigned char perm[KMAXSLOT];
        int nslots = warp_slots(dt.host, L, perm, KMAXSLOT, true);
        if (L * nslots > 384) nslots = warp_slots(dt.host, L, perm, KMAXSLOT, false);
        if (L * nslots > 384) continue;  // the kernel is built for 384 threads, two CTAs per SM
        if (op->stream_lines && L != op->stream_lines) continue;
        if (op->stream_stages && stages != op->stream_stages) continue;
        StreamFn fn = pick_stream(kp0.rc.rk, op->periodic != 0, op->m, xl, L, adj, as);
        if (!grant_smem(fn)) continue;
        const int tile_doubles = stream_tile_doubles(xl, n, L, as);
        const size_t bytes = stream_smem_bytes(L, S, kp0.xd, stages, tile_doubles, etab_rows, ktab_rows, resp_rows(kp0));
        if (bytes > 227 * 1024) continue;
        int ctas = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, fn, L * nslots, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        if (ctas < 1) continue;
        res[i].ok = true;
        res[i].c.L = L;
        res[i].c.stages = stages;
        res[i].c.ctas = ctas;
        res[i].c.nslots = nslots;
        std::memcpy(res[i].c.perm, perm, sizeof(perm));
    }
    auto resident = [&](int i) { return (long long)res[i].c.ctas * res[i].c.L * res[i].c.nslots; };
    int pick = -1;
    for (int i = 0; i < 6 && pick < 0; ++i)
        if (res[i].ok && res[i].c.ctas >= 2) pick = i;
    const bool keep16 = !xl && op->scheme == CD06 && !op->periodic && n >= 256;  // measured 5% faster at 16
    if (pick == 0 && !keep16 && res[1].ok && res[1].c.ctas >= 2 && resident(1) >= resident(0)) pick = 1;
    if (pick < 0) {
        long long best = -1;
        for (int i = 0; i < 6; ++i)
            if (res[i].ok && resident(i) > best) {
                best = resident(i);
                pick = i;
            }
    }
    if (pick < 0) return false;
    *out = res[pick].c;
    return true;
}

bool plan_stream(const pado_op_s *op, const DevTables &dt, const KParams &kp0, int axis, long long na, long long nb,
                 bool adj, StreamParams *sp, int *threads, size_t *smem, int *ctas_per_sm)
{
    const int n = op->n, S = kp0.S;
    if (op->m != 16 && op->m != 32 && op->m != 64) return false;
    const bool xl = axis == 1;
    const size_t align_bits = reinterpret_cast<size_t>(kp0.in) | reinterpret_cast<size_t>(kp0.out);
    if (na > 0x7fffffffLL || nb > 0x7fffffffLL) return false;
    if (kp0.nlines > 0x7fffffffLL) return false;  // tile indices are 32-bit in the kernel
    // tensor / bulk copies need 16-byte aligned fields and an even extent along
    // the contiguous axis (16-byte row strides); per-element asynchronous
    // copies (variant 6, or the automatic choice when the copy engine cannot
    // move the field) need 8-byte alignment and forward operators
    const bool tma_ok = !(align_bits & 15) && (xl ? n % 2 == 0 : na % 2 == 0);
    // Some x lines run faster from the odd-pitch tile the per-element copies
    // fill (no bank conflicts between the lines a warp sweeps) than from the
    // bulk copies' even pitch.  Measured (B200, lines of 128 to 1024 points):
    // cd06 and the bounded operators for n = 128..512 (2-17% faster; the
    // bounded cd10 d2 only from n = 256); the periodic cd10 and cf90, and
    // every n = 1024, are 0-20% slower with them and keep the bulk copies.
    const bool prefer_async = xl && !adj && n >= 128 && n <= 512 &&
                              (op->scheme == CD06 || (!op->periodic && (kp0.rc.rk != RHS_CD10_D2 || n >= 256)));
    const bool as_ok = !adj && !(align_bits & 7);
    bool as = op->variant == 6 || (op->variant == 0 && (!tma_ok || prefer_async));
    if (as && !as_ok && op->variant == 0 && tma_ok) as = false;
    if (as ? !as_ok : !tma_ok) return false;
    const int etab_rows = (int)(dt.host.etab.size() / E_NF), ktab_rows = (int)(dt.host.ktab.size() / KT_NF);
    const PlanKey pkey(&dt, xl ? 1 : 0, as ? 1 : 0, adj ? 1 : 0, op->stream_lines, op->stream_stages);
    StreamChoice choice;
    bool cached = false;
    {
        std::lock_guard<std::mutex> g(op->plan_mu);
        auto it = op->plan_cache.find(pkey);
        if (it != op->plan_cache.end()) {
            choice = it->second;
            cached = true;
        }
    }
    if (!cached) {
        if (!choose_stream_tiling(op, dt, kp0, xl, as, adj, etab_rows, ktab_rows, &choice)) return false;
        std::lock_guard<std::mutex> g(op->plan_mu);
        op->plan_cache[pkey] = choice;
    }
    const int best_slots = choice.nslots, best_ctas = choice.ctas;
    unsigned char best_perm[KMAXSLOT];
    std::memcpy(best_perm, choice.perm, sizeof(best_perm));
    if (!grant_smem(pick_stream(kp0.rc.rk, op->periodic != 0, op->m, xl, choice.L, adj, as))) return false;
    const int L = choice.L, stages = choice.stages;
    const int tile_doubles = stream_tile_doubles(xl, n, L, as);
    std::memset(sp, 0, sizeof(*sp));
    sp->kp = kp0;
    sp->kp.L = L;
    sp->kp.nslots = best_slots;
    std::memcpy(sp->kp.sperm, best_perm, sizeof(best_perm));
    sp->kp.border_slot = first_idle_slot(best_perm, best_slots);
    sp->kp.P = xl ? stream_xl_pitch(n, as) : kp0.P;
    sp->async_copy = as ? 1 : 0;
    sp->axis = axis;
    sp->stages = stages;
    sp->tile_doubles = tile_doubles;
    sp->etab_rows = etab_rows;
    sp->ktab_rows = ktab_rows;
    sp->etab = dt.etab;
    sp->ktab = dt.ktab;
    sp->rtab = dt.rtab;
    sp->toff = dt.toff;
    sp->status = op->d_status;
    if (xl) {
        sp->ntiles = (kp0.nlines + L - 1) / L;
    } else if (as) {
        sp->na = (int)na;
        sp->xblocks = (int)((na + L - 1) / L);
        sp->ntiles = (long long)sp->xblocks * nb;
        sp->pstride = axis == 2 ? na * (long long)n : na;
    } else {
        // boxes of at most 256 rows; a multiple of 16 rows keeps every box's
        // shared-memory destination 128-byte aligned for any L
        sp->nbox = (n + 255) / 256;
        sp->box_rows = ((n + sp->nbox - 1) / sp->nbox + 15) / 16 * 16;
        sp->na = (int)na;
        sp->xblocks = (int)((na + L - 1) / L);
        sp->ntiles = (long long)sp->xblocks * nb;
        sp->pstride = axis == 2 ? na * (long long)n : na;
        EncodeTiledFn enc = encode_tiled();
        if (!enc) return false;
        const cuuint64_t dims[3] = {(cuuint64_t)na, (cuuint64_t)(axis == 2 ? n : nb), (cuuint64_t)(axis == 2 ? nb : n)};
        const cuuint64_t strides[2] = {(cuuint64_t)na * 8, (cuuint64_t)na * (axis == 2 ? n : nb) * 8};
        const cuuint32_t box[3] = {(cuuint32_t)L, (cuuint32_t)(axis == 2 ? sp->box_rows : 1),
                                   (cuuint32_t)(axis == 2 ? 1 : sp->box_rows)};
        const cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&sp->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(kp0.in), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    *threads = L * best_slots;
    *smem = stream_smem_bytes(L, S, kp0.xd, stages, tile_doubles, etab_rows, ktab_rows, resp_rows(kp0));
    *ctas_per_sm = best_ctas;
    return true;
}

int sm_count()
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

int launch_stream(pado_op_s *op, const StreamParams &sp, bool adj, int threads, size_t smem, int ctas_per_sm,
                  cudaStream_t st)
{
    StreamFn fn = pick_stream(sp.kp.rc.rk, op->periodic != 0, op->m, sp.axis == 1, sp.kp.L, adj, sp.async_copy != 0);
    const long long grid = std::min<long long>(sp.ntiles, (long long)ctas_per_sm * sm_count());
    if (grid < 1) return PADO_OK;
    fn<<<(unsigned)grid, threads, smem, st>>>(sp);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

}  // namespace

int pado::prepare_launch(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                         int bcn, bool adjoint, int lines, bool no_fast, KParams *kpo, bool *trivial, int solve_bc1,
                         int solve_bcn, int out_mode, double out_alpha)
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
    const int sb1 = solve_bc1 == SAME_BC ? bc1 : solve_bc1, sbn = solve_bcn == SAME_BC ? bcn : solve_bcn;
    auto it = op->tables.find(TabKey(kind, bounded_bc ? sb1 : 0, bounded_bc ? sbn : 0, adjoint ? 1 : 0));
    if (it == op->tables.end()) return PADO_E_STATE;
    const DevTables &dt = it->second;

    KParams kp{};
    fill_params(kp, dt.host, n, op->scheme == CD06 ? op->bc1 : bc1, op->scheme == CD06 ? op->bcn : bcn);
    kp.in = f;
    kp.out = df;
    kp.out_mode = out_mode;
    kp.out_alpha = out_alpha;
    set_geometry(kp, axis, n, na, nb);
    kp.L = lines;
    kp.tab = dt.tab;
    kp.ctab = dt.ctab;
    kp.xtab = dt.xtab;
    kp.bt = dt.bt;
    if (no_fast) {
        // every segment on the per-row table (kernels built for another segment length)
        kp.int_mask = 0;
        kp.spk_mask = 0;
        kp.ctab = dt.ctab_exact;
        kp.xtab = dt.xtab_exact;
        set_chain(kp, dt.host.chain_exact);
        for (int i = 0; i < 32; ++i) kp.sperm[i] = (unsigned char)i;
        kp.nslots = kp.S;
    }
    *kpo = kp;
    *trivial = false;
    return PADO_OK;
}

namespace {

// df = alpha * f (+ df) elementwise: the n == 1 filter under a scaled or
// accumulating output mode
__global__ void out_copy_kernel(const double *__restrict__ f, double *__restrict__ df, long long total, int mode,
                                double alpha)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        df[i] = mode == OUT_ACC ? fma(alpha, f[i], df[i]) : alpha * f[i];
}

int launch(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1, int bcn,
           cudaStream_t st, bool adjoint, int solve_bc1 = SAME_BC, int solve_bcn = SAME_BC, int out_mode = OUT_STORE,
           double out_alpha = 1.0)
{
    if (adjoint && out_mode != OUT_STORE) return PADO_E_UNSUPPORTED;
    KParams kp;
    bool trivial = true;
    int rc = prepare_launch(op, kind, axis, f, df, na, nb, bc1, bcn, adjoint, op ? op->lines : 0, false, &kp, &trivial,
                            solve_bc1, solve_bcn, out_mode, out_alpha);
    if (rc != PADO_OK) return rc;
    if (trivial) {
        const long long total = (long long)op->n * na * nb;
        if (total == 0) return PADO_OK;
        // n == 1: cd06.F90:781-784, cd10.F90:2037-2040 (zero), cf90.F90:1028-1031 (copy)
        cudaError_t e = cudaSuccess;
        if (kind != FILTER) {
            if (out_mode != OUT_ACC) e = cudaMemsetAsync(df, 0, total * sizeof(double), st);  // df + alpha * 0 = df
        } else if (out_mode == OUT_STORE) {
            e = cudaMemcpyAsync(df, f, total * sizeof(double), cudaMemcpyDeviceToDevice, st);
        } else {
            const long long blocks = std::min<long long>((total + 255) / 256, 4096);
            out_copy_kernel<<<(unsigned)blocks, 256, 0, st>>>(f, df, total, out_mode, out_alpha);
            g_launches.fetch_add(1, std::memory_order_relaxed);
            e = cudaGetLastError();
        }
        return e == cudaSuccess ? PADO_OK : cuda_fail(e);
    }
    if (op->variant == 0 || op->variant == 4 || op->variant == 6) {
        const bool bounded_bc = !op->periodic && op->scheme != CD06;
        const int sb1 = solve_bc1 == SAME_BC ? bc1 : solve_bc1, sbn = solve_bcn == SAME_BC ? bcn : solve_bcn;
        const DevTables &dt = op->tables.at(TabKey(kind, bounded_bc ? sb1 : 0, bounded_bc ? sbn : 0, adjoint ? 1 : 0));
        StreamParams sp;
        int sthreads = 0, sctas = 0;
        size_t ssmem = 0;
        if (plan_stream(op, dt, kp, axis, na, nb, adjoint, &sp, &sthreads, &ssmem, &sctas))
            return launch_stream(op, sp, adjoint, sthreads, ssmem, sctas, st);
        if (op->variant == 4 || (op->variant == 6 && !adjoint)) return PADO_E_UNSUPPORTED;
    }
    if ((op->variant == 5 || (op->variant == 0 && resident_fallback(op, axis))) && !adjoint && solve_bc1 == SAME_BC) {
        // the same resident tiles, with plain loads
        rc = launch_resident_single(op, kind, axis, f, df, na, nb, bc1, bcn, st, nullptr, out_mode, out_alpha);
        if (rc != PADO_E_UNSUPPORTED || op->variant == 5) return rc;
    }
    // lines per CTA: the handle's choice, halved until the segments fit
    while (kp.L > 1 && kp.L * kp.S > max_threads_for_m(op->m)) kp.L /= 2;
    const int threads = kp.L * kp.S;
    const bool contiguous = kp.stride == 1;
    const bool persist = !adjoint && (op->variant == 2 || (op->variant == 3 && !contiguous));
    const size_t tile = (adjoint || contiguous) ? (size_t)kp.L * kp.P : (op->variant == 2 ? (size_t)kp.n * kp.L : 0);
    const size_t smem = smem_doubles(kp.L, kp.S, kp.xd, tile) * sizeof(double);
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
    {
        cudaError_t e = cudaMalloc(&op->d_status, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(op->d_status, 0, sizeof(int));
        if (e != cudaSuccess) {
            const int rc = cuda_fail(e);
            pado_destroy(op);
            return rc;
        }
    }
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
    for (cudaEvent_t ev : op->ev_in) cudaEventDestroy(ev);
    for (cudaEvent_t ev : op->ev_out) cudaEventDestroy(ev);
    if (op->s_h2d) cudaStreamDestroy(op->s_h2d);
    if (op->s_d2h) cudaStreamDestroy(op->s_d2h);
    if (op->d_status) cudaFree(op->d_status);
    delete op;
}

int pado_get_size(pado_op_t op) { return op ? op->n : PADO_E_NULL; }

int pado_apply(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1, int bcn,
               void *stream)
{
    return launch(op, kind, axis, f, df, na, nb, bc1, bcn, (cudaStream_t)stream, false);
}

int pado_apply_scaled(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                      int bcn, double alpha, double beta, void *stream)
{
    if (beta != 0.0 && beta != 1.0) return PADO_E_ARG;
    const int mode = beta == 1.0 ? OUT_ACC : (alpha == 1.0 ? OUT_STORE : OUT_SCALE);
    return launch(op, kind, axis, f, df, na, nb, bc1, bcn, (cudaStream_t)stream, false, SAME_BC, SAME_BC, mode, alpha);
}

int pado_apply_adjoint(pado_op_t op, int kind, int axis, const double *g, double *fbar, long na, long nb, int bc1,
                       int bcn, void *stream)
{
    return launch(op, kind, axis, g, fbar, na, nb, bc1, bcn, (cudaStream_t)stream, true);
}

int pado_filter3_complex(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn,
                         void *stream)
{
    if (!op) return PADO_E_NULL;
    if (op->scheme != CF90) return PADO_E_UNSUPPORTED;
    if (na < 0 || nb < 0) return PADO_E_ARG;
    // a periodic object has no penta_nn system (cf90.F90:1249 would read an unallocated array)
    if (op->periodic && op->n != 1) return PADO_E_UNSUPPORTED;
    // interleaved (re, im): the real (2 na, nb, n) field, each part filtered alone; the
    // right-hand side takes the closures (bc1, bcn), the solve always the bc (0, 0) system
    return launch(op, FILTER, 3, f, df, 2 * na, nb, bc1, bcn, (cudaStream_t)stream, false, 0, 0);
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
    if (axis < 1 || axis > 3) return PADO_E_ARG;
    const size_t total = (size_t)op->n * (size_t)na * (size_t)nb;
    if (total == 0) return PADO_OK;
    if (!f_host || !df_host) return PADO_E_NULL;
    if (f_host == df_host) return PADO_E_ALIAS;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(op->staging_mu);

    // Chunks: groups of whole lines.  x lines: consecutive lines (contiguous);
    // y lines: consecutive (.., .., k) slabs (contiguous); z lines: a range of
    // the middle index, one strided 2-D copy per chunk.  Each chunk is solved
    // as its own compact field, so its device base is rounded to 32 doubles.
    const size_t n = (size_t)op->n;
    const size_t units = axis == 1 ? (size_t)na * (size_t)nb : (size_t)nb;
    const size_t unit_elems = total / units;
    const size_t target = HOST_CHUNK_BYTES / sizeof(double);
    size_t nch = std::min<size_t>(std::max<size_t>(1, (total + target - 1) / target), HOST_MAX_CHUNKS);
    nch = std::min(nch, units);
    const size_t per = (units + nch - 1) / nch;
    nch = (units + per - 1) / per;
    const size_t slot = (per * unit_elems + 31) / 32 * 32;
    const size_t need = slot * nch;
    if (op->stage_elems < need) {
        if (op->stage_f) cudaFree(op->stage_f);
        if (op->stage_df) cudaFree(op->stage_df);
        op->stage_f = op->stage_df = nullptr;
        op->stage_elems = 0;
        cudaError_t e = cudaMalloc(&op->stage_f, need * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&op->stage_df, need * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(e);
        op->stage_elems = need;
    }
    if (!op->s_h2d) {
        cudaError_t e = cudaStreamCreateWithFlags(&op->s_h2d, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&op->s_d2h, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    while (op->ev_in.size() < nch) {
        cudaEvent_t a = nullptr, b = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e);
        op->ev_in.push_back(a);
        op->ev_out.push_back(b);
    }

    auto copy = [&](size_t c, bool in, cudaStream_t cs) -> cudaError_t {
        const size_t u0 = c * per, cu = std::min(per, units - u0);
        double *dev = (in ? op->stage_f : op->stage_df) + c * slot;
        if (axis == 3) {
            // (na, nb, n): rows of na*cu doubles, one per z plane
            const size_t w = (size_t)na * cu * sizeof(double), hp = (size_t)na * (size_t)nb * sizeof(double);
            const size_t off = u0 * (size_t)na;
            return in ? cudaMemcpy2DAsync(dev, w, f_host + off, hp, w, n, cudaMemcpyHostToDevice, cs)
                      : cudaMemcpy2DAsync(df_host + off, hp, dev, w, w, n, cudaMemcpyDeviceToHost, cs);
        }
        const size_t off = u0 * unit_elems, bytes = cu * unit_elems * sizeof(double);
        return in ? cudaMemcpyAsync(dev, f_host + off, bytes, cudaMemcpyHostToDevice, cs)
                  : cudaMemcpyAsync(df_host + off, dev, bytes, cudaMemcpyDeviceToHost, cs);
    };

    int rc = PADO_OK;
    cudaError_t e = cudaSuccess;
    for (size_t c = 0; c < nch && e == cudaSuccess; ++c) {
        e = copy(c, true, op->s_h2d);
        if (e == cudaSuccess) e = cudaEventRecord(op->ev_in[c], op->s_h2d);
    }
    for (size_t c = 0; c < nch && e == cudaSuccess && rc == PADO_OK; ++c) {
        const size_t cu = std::min(per, units - c * per);
        const long ca = axis == 1 ? (long)cu : na, cb = axis == 1 ? 1L : (long)cu;
        e = cudaStreamWaitEvent(st, op->ev_in[c], 0);
        if (e != cudaSuccess) break;
        rc = launch(op, kind, axis, op->stage_f + c * slot, op->stage_df + c * slot, ca, cb, bc1, bcn, st, false);
        if (rc != PADO_OK) break;
        e = cudaEventRecord(op->ev_out[c], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(op->s_d2h, op->ev_out[c], 0);
        if (e == cudaSuccess) e = copy(c, false, op->s_d2h);
    }
    // every copy that was enqueued ends before the host buffers are handed back
    const cudaError_t e1 = cudaStreamSynchronize(op->s_h2d);
    const cudaError_t e2 = cudaStreamSynchronize(op->s_d2h);
    const cudaError_t e3 = cudaStreamSynchronize(st);
    if (rc != PADO_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e);
    if (e1 != cudaSuccess) return cuda_fail(e1);
    if (e2 != cudaSuccess) return cuda_fail(e2);
    return e3 == cudaSuccess ? PADO_OK : cuda_fail(e3);
}

int pado_apply_host_terms(const double *f_host, long n1, long n2, long n3, const pado_host_term *terms, int nterms,
                          double *const *out_host, int nout, void *stream)
{
    if (!f_host || !terms || !out_host) return PADO_E_NULL;
    if (n1 < 1 || n2 < 1 || n3 < 1 || nterms < 1 || nout < 1) return PADO_E_ARG;
    const long ext[3] = {n1, n2, n3};
    for (int i = 0; i < nterms; ++i) {
        const pado_host_term &t = terms[i];
        if (!t.op) return PADO_E_NULL;
        if (t.axis < 1 || t.axis > 3 || t.op->n != ext[t.axis - 1]) return PADO_E_ARG;
        if (t.beta != 0.0 && t.beta != 1.0) return PADO_E_ARG;
        const int prev = i ? terms[i - 1].out : -1;
        if (t.out != prev && t.out != prev + 1) return PADO_E_ARG;  // outputs in order, terms consecutive
        if (t.out != prev && t.beta != 0.0) return PADO_E_ARG;      // an output starts from its first term
        if (t.out >= nout || !out_host[t.out]) return PADO_E_ARG;
    }
    if (terms[nterms - 1].out != nout - 1) return PADO_E_ARG;
    pado_op_s *op0 = terms[0].op;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(op0->staging_mu);
    const size_t total = (size_t)n1 * (size_t)n2 * (size_t)n3;
    const size_t slot = (total + 31) / 32 * 32;
    // f in stage_f, two output fields in stage_df
    if (op0->stage_elems < 2 * slot) {
        if (op0->stage_f) cudaFree(op0->stage_f);
        if (op0->stage_df) cudaFree(op0->stage_df);
        op0->stage_f = op0->stage_df = nullptr;
        op0->stage_elems = 0;
        cudaError_t e = cudaMalloc(&op0->stage_f, 2 * slot * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&op0->stage_df, 2 * slot * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(e);
        op0->stage_elems = 2 * slot;
    }
    if (!op0->s_h2d) {
        cudaError_t e = cudaStreamCreateWithFlags(&op0->s_h2d, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&op0->s_d2h, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    // events: [0] f arrived, then per output: computed, copied out
    const size_t nev = 1 + 2 * (size_t)nout;
    while (op0->ev_in.size() < nev) {
        cudaEvent_t a = nullptr, b = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e);
        op0->ev_in.push_back(a);
        op0->ev_out.push_back(b);
    }
    const size_t chunk = HOST_CHUNK_BYTES * 4 / sizeof(double);
    int rc = PADO_OK;
    cudaError_t e = cudaSuccess;
    for (size_t o = 0; o < total && e == cudaSuccess; o += chunk)
        e = cudaMemcpyAsync(op0->stage_f + o, f_host + o, std::min(chunk, total - o) * sizeof(double),
                            cudaMemcpyHostToDevice, op0->s_h2d);
    if (e == cudaSuccess) e = cudaEventRecord(op0->ev_in[0], op0->s_h2d);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, op0->ev_in[0], 0);
    int i = 0;
    for (int o = 0; o < nout && e == cudaSuccess && rc == PADO_OK; ++o) {
        double *dev = op0->stage_df + (size_t)(o & 1) * slot;
        // the buffer's previous output has left the device
        if (o >= 2) e = cudaStreamWaitEvent(st, op0->ev_out[1 + 2 * (o - 2) + 1], 0);
        for (; e == cudaSuccess && rc == PADO_OK && i < nterms && terms[i].out == o; ++i) {
            const pado_host_term &t = terms[i];
            const long na = t.axis == 1 ? n2 : n1, nb = t.axis == 3 ? n2 : n3;
            const int mode = t.beta == 1.0 ? OUT_ACC : (t.alpha == 1.0 ? OUT_STORE : OUT_SCALE);
            rc = launch(t.op, t.kind, t.axis, op0->stage_f, dev, na, nb, t.bc1, t.bcn, st, false, SAME_BC, SAME_BC,
                        mode, t.alpha);
        }
        if (rc != PADO_OK || e != cudaSuccess) break;
        e = cudaEventRecord(op0->ev_out[1 + 2 * o], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(op0->s_d2h, op0->ev_out[1 + 2 * o], 0);
        for (size_t c = 0; c < total && e == cudaSuccess; c += chunk)
            e = cudaMemcpyAsync(out_host[o] + c, dev + c, std::min(chunk, total - c) * sizeof(double),
                                cudaMemcpyDeviceToHost, op0->s_d2h);
        if (e == cudaSuccess) e = cudaEventRecord(op0->ev_out[1 + 2 * o + 1], op0->s_d2h);
    }
    // every copy that was enqueued ends before the host buffers are handed back
    const cudaError_t e1 = cudaStreamSynchronize(op0->s_h2d);
    const cudaError_t e2 = cudaStreamSynchronize(op0->s_d2h);
    const cudaError_t e3 = cudaStreamSynchronize(st);
    if (rc != PADO_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e);
    if (e1 != cudaSuccess) return cuda_fail(e1);
    if (e2 != cudaSuccess) return cuda_fail(e2);
    return e3 == cudaSuccess ? PADO_OK : cuda_fail(e3);
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
    if (S > 32) {
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
    if (variant < 0 || variant > 6) return PADO_E_ARG;
    op->variant = variant;
    return PADO_OK;
}

int pado_launch_plan(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                     int bcn, int *info)
{
    if (!info) return PADO_E_NULL;
    for (int i = 0; i < 8; ++i) info[i] = 0;
    KParams kp;
    bool trivial = true;
    int rc = prepare_launch(op, kind, axis, f, df, na, nb, bc1, bcn, false, op ? op->lines : 0, false, &kp, &trivial);
    if (rc != PADO_OK || trivial) return rc;
    info[4] = kp.S;
    info[5] = kp.W;
    if (op->variant == 0 || op->variant == 4 || op->variant == 6) {
        const bool bounded_bc = !op->periodic && op->scheme != CD06;
        const DevTables &dt = op->tables.at(TabKey(kind, bounded_bc ? bc1 : 0, bounded_bc ? bcn : 0, 0));
        StreamParams sp;
        int threads = 0, ctas = 0;
        size_t smem = 0;
        if (plan_stream(op, dt, kp, axis, na, nb, false, &sp, &threads, &smem, &ctas)) {
            info[0] = sp.async_copy ? 6 : 4;
            info[1] = sp.kp.L;
            info[2] = sp.stages;
            info[3] = ctas;
            info[6] = threads;
            info[7] = (int)smem;
            return PADO_OK;
        }
    }
    if ((op->variant == 5 || (op->variant == 0 && resident_fallback(op, axis))) &&
        launch_resident_single(op, kind, axis, f, df, na, nb, bc1, bcn, nullptr, info) == PADO_OK)
        return PADO_OK;
    info[0] = op->variant == 0 ? 1 : op->variant;
    info[1] = kp.L;
    info[6] = kp.L * kp.S;
    return PADO_OK;
}

int pado_set_stream_tiling(pado_op_t op, int lines, int stages)
{
    if (!op) return PADO_E_NULL;
    if ((lines != 0 && lines != 8 && lines != 16 && lines != 32) || stages < 0 || stages > 2) return PADO_E_ARG;
    op->stream_lines = lines;
    op->stream_stages = stages;
    return PADO_OK;
}

int pado_device_status(pado_op_t op, int clear)
{
    if (!op) return PADO_E_NULL;
    if (!op->d_status) return PADO_OK;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, op->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e);
    if (clear && v != 0) {
        const int zero = 0;
        e = cudaMemcpy(op->d_status, &zero, sizeof(int), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    return v;
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
    case PADO_STAGG_E_SHORT: return "cd06stagg needs more than 4 points (reference exit code 21)";
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

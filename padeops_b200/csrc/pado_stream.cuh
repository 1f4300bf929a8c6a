// pado_stream.cuh -- the streaming line kernel: persistent CTAs that stage
// whole tiles of lines in shared memory with the tensor memory accelerator
// (TMA), two tiles ahead, so HBM streams continuously while the CTA runs the
// sweep of the current tile.
//
// Persistent CTAs (as many per SM as fit) walk the tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... through `stages` shared-memory buffers, each
// guarded by an mbarrier.  The sweep runs on the buffer in place
// (pado_resident.cuh):
//
//   wait(full[b])  prep, fwd, bwd, fin (barrier-separated; the chains run
//                  inside bwd and fin)
//   strided lines: results to global memory from fin
//   x lines:       fin writes the buffer; bulk store of each line
//   then the load `stages` tiles ahead is issued into buffer b
//
// Strided lines (y, z): one 3-D tensor copy per box of {L lines, box_rows
// rows} lands as the [row][L] tile.  Contiguous lines (x): one bulk copy per
// line into a [L][P] tile (P = n + 2, rows 16-byte aligned), written back
// by bulk stores.
//
// Fields the copy engine cannot move (an odd extent along the contiguous
// axis, or a pointer that is 8- but not 16-byte aligned) take the same
// kernel with AS = true: every thread issues 8-byte asynchronous copies
// (cp.async) of its share of the next tile and arrives on the stage's
// mbarrier when they land (cp.async.mbarrier.arrive.noinc, one arrival per
// thread), so the copies still run while the other CTAs on the SM compute.
// x-line tiles then use an odd pitch P (no bank conflicts between lines)
// and go back to global memory by coalesced stores from all threads.
//
// The per-row table of the segments that read it and the chain
// coefficients are staged in shared memory once per CTA.  Every wait
// is bounded (2 s); on expiry the CTA records PADO_E_TIMEOUT in *status,
// waits (bounded) for its copies in flight and returns.
#pragma once

#include <cuda.h>

#include <algorithm>
#include <vector>

#include "pado_kernels.cuh"
#include "pado_resident.cuh"

namespace pado {

constexpr int PADO_STATUS_TIMEOUT = -7;  // PADO_E_TIMEOUT of pado.h

struct alignas(64) StreamParams {
    CUtensorMap tmap;   // strided lines: 3-D view of the input field (TMA copies)
    KParams kp;
    int async_copy;     // 1: the tile copies are per-element cp.async (AS kernels)
    long long ntiles;
    long long pstride;  // strided lines: elements between consecutive planes
    int na;             // strided lines: extent of the contiguous axis
    int xblocks;        // strided lines: tiles per plane, ceil(na / L)
    int axis;           // 1, 2, 3
    int stages;
    int box_rows, nbox; // strided lines: rows per tensor copy, copies per tile
    int tile_doubles;   // per stage (a multiple of 16)
    int etab_rows;      // packed table rows staged in shared memory
    int ktab_rows;      // packed spike rows staged in shared memory
    const double *rtab; // [resp_rows][2] border-unknown responses (cyclic lines)
    const double *etab; // [etab_rows][E_NF]
    const double *ktab; // [ktab_rows][2]
    const int *toff;    // [S]
    int *status;        // PADO_E_TIMEOUT on a wait that expired
};

// Shared-memory layout, offsets in doubles from a 1024-byte aligned base.
struct StreamLayout {
    size_t tiles, work, etab, ktab, rtab, toff, bars, total_doubles;
};

PADO_HD PADO_INLINE StreamLayout stream_layout(int L, int S, int xd, int stages, int tile_doubles, int etab_rows,
                                               int ktab_rows, int ie)
{
    StreamLayout o;
    o.tiles = 0;
    o.work = (size_t)stages * tile_doubles;
    o.etab = o.work + smem_doubles(L, S, xd, 0);
    o.ktab = o.etab + (size_t)etab_rows * E_NF;
    o.rtab = o.ktab + (size_t)ktab_rows * 2;
    o.toff = o.rtab + (size_t)ie * 2;
    o.bars = o.toff + (size_t)(S + 1) / 2;
    o.total_doubles = o.bars + (size_t)stages;
    return o;
}

PADO_HD PADO_INLINE size_t stream_smem_bytes(int L, int S, int xd, int stages, int tile_doubles, int etab_rows,
                                             int ktab_rows, int ie)
{
    return stream_layout(L, S, xd, stages, tile_doubles, etab_rows, ktab_rows, ie).total_doubles * sizeof(double) +
           1024;
}

// Line l of strided tile t: plane p, lines x0 .. x0+L-1 of that plane.
// Tile counts fit in 32 bits (the planner checks), and a 32-bit division is
// a few instructions where a 64-bit one is a long software routine.
PADO_HD PADO_INLINE void stream_tile_origin(const StreamParams &sp, long long t, long long *x0, long long *p)
{
    if (sp.axis == 1) {
        *x0 = t * sp.kp.L;
        *p = 0;
    } else {
        const unsigned tu = (unsigned)t, xb = (unsigned)sp.xblocks;
        const unsigned pq = tu / xb;
        *x0 = (long long)(tu - pq * xb) * sp.kp.L;
        *p = pq;
    }
}

PADO_HD PADO_INLINE LineIO stream_line_io_at(const StreamParams &sp, const Smem &sm, int l, long long x0, long long p)
{
    const KParams &kp = sp.kp;
    LineIO io;
    if (sp.axis == 1) {
        io.live = x0 + l < kp.nlines;
        io.src = sm.tile + (size_t)l * kp.P;
        io.ss = 1;
        io.dst = sm.tile + (size_t)l * kp.P;
        io.ds = 1;
    } else {
        const long long x = x0 + l;
        io.live = x < sp.na;
        io.src = sm.tile + l;
        io.ss = kp.L;
        io.dst = kp.out + (io.live ? x + p * sp.pstride : 0);
        io.ds = kp.stride;
    }
    return io;
}

PADO_HD PADO_INLINE LineIO stream_line_io(const StreamParams &sp, const Smem &sm, int l, long long t)
{
    long long x0, p;
    stream_tile_origin(sp, t, &x0, &p);
    return stream_line_io_at(sp, sm, l, x0, p);
}

PADO_HD PADO_INLINE int stream_tile_lines(const StreamParams &sp, long long t)
{
    long long x0, p;
    stream_tile_origin(sp, t, &x0, &p);
    const long long lim = sp.axis == 1 ? sp.kp.nlines : sp.na;
    const long long nl = lim - x0;
    return (int)(nl < sp.kp.L ? nl : sp.kp.L);
}

#ifdef __CUDACC__
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// try_wait with a suspend-time hint: the thread sleeps in hardware until the
// phase completes or about 1 ms passes, instead of spinning on the barrier
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Bounded wait for the phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned long long limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, unsigned long long *bar, int c0, int c1,
                                            int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, const void *src, unsigned bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 8-byte asynchronous copy global -> shared (both addresses 8-byte aligned)
__device__ __forceinline__ void async_copy8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// arrive on the mbarrier once this thread's earlier cp.async copies have
// landed (counts as one of the barrier's expected arrivals)
__device__ __forceinline__ void async_arrive(unsigned long long *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

constexpr unsigned long long STREAM_WAIT_NS = 2000000000ull;  // 2 s
constexpr unsigned long long STREAM_DRAIN_NS = 200000000ull;  // 0.2 s

// Issue the copies of tile t into stage buffer `tile` (one thread).
__device__ __forceinline__ void stream_issue_load(const StreamParams &sp, double *tile, unsigned long long *bar,
                                                  long long t)
{
    const KParams &kp = sp.kp;
    long long x0, p;
    stream_tile_origin(sp, t, &x0, &p);
    if (sp.axis == 1) {
        const int nl = stream_tile_lines(sp, t);
        const unsigned bytes = (unsigned)kp.n * 8u;
        mbar_expect_tx(bar, bytes * (unsigned)nl);
        for (int l = 0; l < nl; ++l)
            bulk_load(tile + (size_t)l * kp.P, kp.in + (x0 + l) * (long long)kp.n, bytes, bar);
    } else {
        mbar_expect_tx(bar, (unsigned)sp.nbox * sp.box_rows * kp.L * 8u);
        for (int b = 0; b < sp.nbox; ++b) {
            const int r0 = b * sp.box_rows;
            double *dst = tile + (size_t)r0 * kp.L;
            if (sp.axis == 2) tma_load_3d(dst, &sp.tmap, bar, (int)x0, r0, (int)p);
            else tma_load_3d(dst, &sp.tmap, bar, (int)x0, (int)p, r0);
        }
    }
}

// The copies of tile t into stage buffer `tile` by every thread of the CTA
// (AS kernels): 8-byte cp.async of the thread's share, then one arrival on
// the stage's mbarrier (initialised to the CTA's thread count).  Strided
// lines: thread tid copies line tid % L, rows tid / L + k * (nthreads / L),
// which lands at tile[tid + k * nthreads]; lines past the field are left
// alone (their results are never stored).  x lines: the tile's lines are
// consecutive in global memory, so element e of the tile's span goes to
// row e % n of line e / n, at tile[(e / n) * P + e % n].
template <bool XL, int LT>
__device__ __forceinline__ void stream_issue_async(const StreamParams &sp, double *tile, unsigned long long *bar,
                                                   long long t, int tid, int nthreads)
{
    const KParams &kp = sp.kp;
    long long x0, p;
    stream_tile_origin(sp, t, &x0, &p);
    if (XL) {
        const int n = kp.n, pad = kp.P - n;
        const int total = stream_tile_lines(sp, t) * n;
        const double *src = kp.in + x0 * (long long)n + tid;
        const int l0 = tid / n;
        int r = tid - l0 * n;
        double *dst = tile + (size_t)l0 * kp.P + r;
        const int dl = nthreads / n, dr = nthreads - dl * n;
        const int dstep = dl * kp.P + dr;
        for (int e = tid; e < total; e += nthreads) {
            async_copy8(dst, src);
            src += nthreads;
            dst += dstep;
            r += dr;
            if (r >= n) {
                r -= n;
                dst += pad;
            }
        }
    } else {
        constexpr int LS = LT > 0 ? LT : 1;  // LT is 0 only in x-line kernels, which never get here
        const int l = tid % LS;
        if (x0 + l < sp.na) {
            const int rstep = nthreads / LS;
            const long long sstep = (long long)rstep * kp.stride;
            const double *src = kp.in + (x0 + l) + p * sp.pstride + (long long)(tid / LS) * kp.stride;
            double *dst = tile + tid;
#pragma unroll 4
            for (int r = tid / LS; r < kp.n; r += rstep) {
                async_copy8(dst, src);
                src += sstep;
                dst += nthreads;
            }
        }
    }
    async_arrive(bar);
}

// LT: lines per tile for strided lines, fixed at compile time so that every
// row offset in the [row][L] tile is an immediate (x lines: 0, L at run time).
// AS: the tile copies are per-element cp.async by all threads (any extent
// and 8-byte alignment) instead of tensor / bulk copies.
template <int RK, bool PER, int M, bool XL, int LT, bool ADJ = false, bool AS = false>
__global__ void __launch_bounds__(384, 2) stream_kernel(const __grid_constant__ StreamParams sp)
{
    static_assert(!(AS && ADJ), "the adjoint streams by tensor / bulk copies only");
    using RL = ResidentLine<RK, PER, M, ADJ>;
    extern __shared__ double smem_raw[];
    // 1024-byte aligned base, by pointer arithmetic on the shared array so
    // that the compiler keeps every access in the shared address space
    double *base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u) / sizeof(double);
    const KParams &kp = sp.kp;
    static_assert(XL || LT > 0, "strided lines need a compile-time tile width");
    const int L = XL ? kp.L : LT, S = kp.S;
    const StreamLayout lay =
        stream_layout(L, S, kp.xd, sp.stages, sp.tile_doubles, sp.etab_rows, sp.ktab_rows, resp_rows(kp));
    Smem sm = carve(base + lay.work, L, kp.P, S, kp.xd);
    double *etab = base + lay.etab;
    double *ktab = base + lay.ktab;
    double *rtab = base + lay.rtab;
    int *toff = reinterpret_cast<int *>(base + lay.toff);
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(base + lay.bars);
    sm.etab = etab;
    sm.toff = toff;
    sm.ktab = ktab;
    sm.rtab = rtab;

    const int tid = threadIdx.x, nthreads = blockDim.x;
    const int l = tid % L, slot = tid / L, s = slot_segment(kp, slot);
    const bool active = s >= 0;
    const long long G = gridDim.x;
    const long long t_first = blockIdx.x;
    const int stages = sp.stages;
    // row r of line l in a stage buffer: [row][L] (y, z) or [L][P] (x)
    constexpr long long rs = XL ? 1 : LT;
    const long long ls = XL ? kp.P : 1;

    if (tid == 0) {
        for (int b = 0; b < stages; ++b) mbar_init(&bars[b], AS ? (unsigned)nthreads : 1u);
        mbar_fence_init();
    }
    stage_chain_table(kp, sm, tid, nthreads);
    for (int i = tid; i < sp.etab_rows * E_NF; i += nthreads) etab[i] = __ldg(sp.etab + i);
    for (int i = tid; i < sp.ktab_rows * 2; i += nthreads) ktab[i] = __ldg(sp.ktab + i);
    for (int i = tid; i < resp_rows(kp) * 2; i += nthreads) rtab[i] = __ldg(sp.rtab + i);
    for (int i = tid; i < S; i += nthreads) toff[i] = __ldg(sp.toff + i);
    __syncthreads();
    if (AS) {
        for (int b = 0; b < stages; ++b) {
            const long long t = t_first + b * G;
            if (t < sp.ntiles)
                stream_issue_async<XL, LT>(sp, base + (size_t)b * sp.tile_doubles, &bars[b], t, tid, nthreads);
        }
    } else if (tid == 0) {
        for (int b = 0; b < stages; ++b) {
            const long long t = t_first + b * G;
            if (t < sp.ntiles) stream_issue_load(sp, base + (size_t)b * sp.tile_doubles, &bars[b], t);
        }
    }

    long long k = 0;
    for (long long t = t_first; t < sp.ntiles; t += G, ++k) {
        const int b = (int)(k % stages);
        const unsigned parity = (unsigned)((k / stages) & 1);
        // warp 0 polls the barrier; the other warps sleep in the CTA barrier
        // (spinning warps would take issue slots from the other CTAs on the SM)
        bool arrived = true;
        if (tid < 32) arrived = mbar_wait(&bars[b], parity, STREAM_WAIT_NS);
        const bool ok = __syncthreads_and(arrived);
        if (!ok) {
            // record, let the copies in flight land, and leave
            if (tid == 0) {
                atomicExch(sp.status, PADO_STATUS_TIMEOUT);
                for (int j = 0; j < stages; ++j) {
                    const long long kk = k + j;
                    if (t + j * G < sp.ntiles)
                        (void)mbar_wait(&bars[kk % stages], (unsigned)((kk / stages) & 1), STREAM_DRAIN_NS);
                }
            }
            if (AS) async_wait_all();
            else if (XL) bulk_wait_all();
            return;
        }
        sm.tile = base + (size_t)b * sp.tile_doubles;
        double *line = sm.tile + l * ls;
        long long x0, p0;
        stream_tile_origin(sp, t, &x0, &p0);
        const LineIO io = stream_line_io_at(sp, sm, l, x0, p0);
        typename RL::Halo h;
        if (!ADJ) {
            if (active) RL::prep(kp, line, rs, s, h);
            __syncthreads();
        }
        if (active) RL::template fwd<true>(kp, sm, line, rs, l, s, h);
        __syncthreads();
        if (active) RL::template bwd<true>(kp, sm, line, rs, l, s);
        else if (PER && slot == kp.border_slot) RL::border_only(kp, sm, l);
        __syncthreads();
        // adjoint x lines: fbar over z in the tile, then the bulk stores, when
        // the end columns of B^T fit the summary buffers (free after fin)
        const bool adj_tile = ADJ && XL && (PER || RL::adj_scratch_slots(kp.n) <= 6 * S + 4);
        if (ADJ) {
            // z = A^{-T} g back into the tile, then fbar = B^T z
            if (active) RL::template fin<true>(kp, sm, line, rs, l, s, line, rs, true);
            __syncthreads();
            if (adj_tile) {
                if (active) RL::adj_gather(kp, line, rs, l, s, sm.buf4, h);
                __syncthreads();
                if (active) RL::adj_inplace(kp, line, rs, l, s, sm.buf4, h);
            } else {
                double *dst = XL ? kp.out + (io.live ? (x0 + l) * (long long)kp.n : 0) : io.dst;
                if (active) RL::adj_out(kp, line, rs, s, dst, XL ? 1 : io.ds, io.live);
            }
        } else {
            if (active) RL::template fin<true>(kp, sm, line, rs, l, s, io.dst, io.ds, io.live, !XL);
        }
        const long long tn = t + (long long)stages * G;  // tile for this buffer next
        if (XL && AS) {
            // the tile's lines are consecutive in global memory: coalesced
            // stores of the whole span by all threads, in the output mode
            __syncthreads();
            const int n = kp.n, pad = kp.P - n;
            const int total = stream_tile_lines(sp, t) * n;
            double *dst = kp.out + x0 * (long long)n + tid;
            const int l0 = tid / n;
            int r = tid - l0 * n;
            const double *src = sm.tile + (size_t)l0 * kp.P + r;
            const int dl = nthreads / n, dr = nthreads - dl * n;
            const int sstep = dl * kp.P + dr;
            if (kp.out_mode == OUT_STORE) {
                for (int e = tid; e < total; e += nthreads) {
                    *dst = *src;
                    dst += nthreads;
                    src += sstep;
                    r += dr;
                    if (r >= n) {
                        r -= n;
                        src += pad;
                    }
                }
            } else {
                for (int e = tid; e < total; e += nthreads) {
                    out_put(kp, dst, *src);
                    dst += nthreads;
                    src += sstep;
                    r += dr;
                    if (r >= n) {
                        r -= n;
                        src += pad;
                    }
                }
            }
        } else if (XL && (!ADJ || adj_tile)) {
            if (!ADJ && kp.out_mode != OUT_STORE) {
                // scaled or accumulated output: the tile's lines take df's values
                // (contiguous, read by whole warps) before they go out
                __syncthreads();
                const long long nl_ = kp.nlines - x0;
                const int nl = (int)(nl_ < L ? nl_ : L);
                const int warp = tid >> 5, lane = tid & 31, nw = nthreads >> 5;
                for (int ll = warp; ll < nl; ll += nw) {
                    double *dl = kp.out + (x0 + ll) * (long long)kp.n;
                    double *tl = sm.tile + (size_t)ll * kp.P;
                    for (int r = lane; r < kp.n; r += 32) {
                        double v = dl[r];
                        if (kp.out_mode == OUT_ACC) v = fma(kp.out_alpha, tl[r], v);
                        else v = kp.out_alpha * tl[r];
                        tl[r] = v;
                    }
                }
            }
            // each line's results -> global memory, then the buffer takes the next load
            fence_proxy_async();
            __syncthreads();
            const long long nl_ = kp.nlines - x0;
            const int nl = (int)(nl_ < L ? nl_ : L);
            if (tid < nl) {
                bulk_store(kp.out + (t * L + tid) * (long long)kp.n, sm.tile + (size_t)tid * kp.P, (unsigned)kp.n * 8u);
                bulk_commit();
                bulk_wait_read();
            }
        }
        __syncthreads();
        if (AS) {
            if (tn < sp.ntiles) stream_issue_async<XL, LT>(sp, sm.tile, &bars[b], tn, tid, nthreads);
        } else if (tid == 0 && tn < sp.ntiles) {
            stream_issue_load(sp, sm.tile, &bars[b], tn);
        }
    }
    if (XL && !AS) bulk_wait_all();
}
#endif  // __CUDACC__

// Host emulation (tests): the kernel's tile loop with plain copies standing
// in for the tensor / bulk copies; phases in kernel order over all threads.
template <int RK, bool PER, int M, bool XL, bool ADJ = false>
inline void emulate_stream(const StreamParams &sp, int nthreads)
{
    using RL = ResidentLine<RK, PER, M, ADJ>;
    const KParams &kp = sp.kp;
    const int L = kp.L, S = kp.S;
    const StreamLayout lay =
        stream_layout(L, S, kp.xd, 1, sp.tile_doubles, sp.etab_rows, sp.ktab_rows, resp_rows(kp));
    std::vector<double> mem(lay.total_doubles, 0.0);
    double *base = mem.data();
    Smem sm = carve(base + lay.work, L, kp.P, S, kp.xd);
    double *etab = base + lay.etab;
    double *ktab = base + lay.ktab;
    double *rtab = base + lay.rtab;
    for (int i = 0; i < sp.ktab_rows * 2; ++i) ktab[i] = sp.ktab[i];
    for (int i = 0; i < resp_rows(kp) * 2; ++i) rtab[i] = sp.rtab[i];
    sm.ktab = ktab;
    sm.rtab = rtab;
    int *toff = reinterpret_cast<int *>(base + lay.toff);
    stage_chain_table(kp, sm, 0, 1);
    for (int i = 0; i < sp.etab_rows * E_NF; ++i) etab[i] = sp.etab[i];
    for (int i = 0; i < S; ++i) toff[i] = sp.toff[i];
    sm.etab = etab;
    sm.toff = toff;
    sm.tile = base;
    const long long rs = XL ? 1 : L, ls = XL ? kp.P : 1;
    std::vector<typename RL::Halo> H(nthreads);
    for (long long t = 0; t < sp.ntiles; ++t) {
        long long x0, p;
        stream_tile_origin(sp, t, &x0, &p);
        const int nl = stream_tile_lines(sp, t);
        // the copy engine's view: full boxes, zero outside the field
        std::fill(sm.tile, sm.tile + sp.tile_doubles, 0.0);
        for (int ll = 0; ll < L; ++ll) {
            if (ll >= nl) continue;
            for (int r = 0; r < kp.n; ++r) {
                if (XL) sm.tile[(size_t)ll * kp.P + r] = kp.in[(x0 + ll) * kp.n + r];
                else sm.tile[(size_t)r * L + ll] = kp.in[x0 + ll + p * sp.pstride + (long long)r * kp.stride];
            }
        }
        const bool adj_tile = ADJ && XL && (PER || RL::adj_scratch_slots(kp.n) <= 6 * S + 4);
        // phases in kernel order, a barrier between consecutive ones
        for (int ph = 0; ph < 6; ++ph) {
            if (ADJ ? ph == 0 : ph >= 4) continue;
            if (ph == 5 && !adj_tile) continue;
            for (int tid = 0; tid < nthreads; ++tid) {
                const int l = tid % L, slot = tid / L, s = slot_segment(kp, slot);
                if (s < 0) {
                    if (PER && ph == 2 && slot == kp.border_slot) RL::border_only(kp, sm, l);
                    continue;
                }
                double *line = sm.tile + l * ls;
                const LineIO io = stream_line_io(sp, sm, l, t);
                switch (ph) {
                case 0: RL::prep(kp, line, rs, s, H[tid]); break;
                case 1: RL::template fwd<true>(kp, sm, line, rs, l, s, H[tid]); break;
                case 2: RL::template bwd<true>(kp, sm, line, rs, l, s); break;
                case 3:
                    if (ADJ) RL::template fin<true>(kp, sm, line, rs, l, s, line, rs, true);
                    else RL::template fin<true>(kp, sm, line, rs, l, s, io.dst, io.ds, io.live, !XL);
                    break;
                case 4:
                    if (adj_tile) RL::adj_gather(kp, line, rs, l, s, sm.buf4, H[tid]);
                    else
                        RL::adj_out(kp, line, rs, s, XL ? kp.out + (io.live ? (x0 + l) * (long long)kp.n : 0) : io.dst,
                                    XL ? 1 : io.ds, io.live);
                    break;
                default: RL::adj_inplace(kp, line, rs, l, s, sm.buf4, H[tid]); break;
                }
            }
        }
        if (XL && (!ADJ || adj_tile))
            for (int ll = 0; ll < nl; ++ll)
                for (int r = 0; r < kp.n; ++r) {
                    double *d = kp.out + (x0 + ll) * kp.n + r;
                    if (ADJ) *d = sm.tile[(size_t)ll * kp.P + r];
                    else out_put(kp, d, sm.tile[(size_t)ll * kp.P + r]);
                }
    }
}

}  // namespace pado

// pado_batch.cuh -- persistent kernel that runs many line families (fields of
// uneven sizes, schemes, boundary types and directions) in one launch.
//
// Work unit = one tile: L consecutive lines of one item (by default as many
// as keep the CTA's 384 threads busy: 384 / segments per line), all rows,
// resident in shared memory while
// the tile-resident sweep of the streaming kernel (pado_resident.cuh) runs on
// it.  Tiles of all items are numbered, most expensive item first; CTAs claim
// tiles from a device counter, BATCH_CLAIM consecutive tiles at a time
// (atomicAdd, no waiting on other CTAs), until the list is exhausted.  A CTA
// claims its next tiles while it solves the current one, and as soon as the current tile's buffer is free every thread issues
// 8-byte asynchronous copies (cp.async) of its share of the next tile, which
// land on an mbarrier (one arrival per thread) while the other CTA on the SM
// computes; the wait on it is bounded.  Results leave straight from the sweep
// (y/z) or from the tile (x).  An item's tables are staged in shared memory
// when a CTA moves to another item.
#pragma once

#include "pado_kernels.cuh"
#include "pado_resident.cuh"
#include "pado_stream.cuh"

namespace pado {

constexpr int BATCH_THREADS = 384;  // threads per CTA: lines per tile x segments per line
#ifndef BATCH_CHUNK
#define BATCH_CHUNK 4
#endif
// tiles a CTA claims at once: consecutive tiles mostly belong to one item, so
// the CTA stages that item's tables once for them
constexpr int BATCH_CLAIM = BATCH_CHUNK;
#ifndef BATCH_MIN_CTAS
#define BATCH_MIN_CTAS 2
#endif

struct BatchItemDev {
    KParams kp;            // geometry and tiling of this item
    const double *etab;    // per-row table of the edge segments
    const double *ktab;    // spike rows of the cyclic sums
    const double *rtab;    // border responses
    const int *toff;       // first table row of each segment
    long long tile0;       // first tile index of this item
    int code;              // ((rk * 2 + periodic) * 2 + x lines) * 4 + (0, 1, 2: segments of 16, 32, 64 rows)
    int etab_rows, ktab_rows, pad;
};

PADO_HD PADO_INLINE int batch_code(int rk, bool periodic, bool xl, int m)
{
    return ((rk * 2 + (periodic ? 1 : 0)) * 2 + (xl ? 1 : 0)) * 4 + (m == 64 ? 2 : (m == 32 ? 1 : 0));
}
PADO_HD PADO_INLINE bool batch_code_xl(int code) { return (code >> 2) & 1; }

// Shared memory of a batch tile (doubles): the item's staged tables (etab,
// ktab, rtab, toff), then the summaries, border slots, border weights,
// transfer products and the tile (carve's layout).
PADO_HD PADO_INLINE size_t batch_table_doubles(int S, int etab_rows, int ktab_rows, int resp_rows)
{
    return (size_t)etab_rows * E_NF + (size_t)ktab_rows * 2 + (size_t)resp_rows * 2 + (size_t)(S + 1) / 2;
}
PADO_HD PADO_INLINE size_t batch_smem_doubles(int L, int S, int n, bool xl, int xd, int etab_rows, int ktab_rows,
                                              int resp_rows)
{
    return batch_table_doubles(S, etab_rows, ktab_rows, resp_rows) +
           smem_doubles(L, S, xd, xl ? (size_t)L * (n | 1) : (size_t)L * n);
}

#ifdef __CUDACC__
PADO_HD PADO_INLINE Smem batch_carve(const BatchItemDev &it, double *smem)
{
    const KParams &kp = it.kp;
    double *p = smem;
    double *etab = p;
    p += (size_t)it.etab_rows * E_NF;
    double *ktab = p;
    p += (size_t)it.ktab_rows * 2;
    double *rtab = p;
    p += (size_t)resp_rows(kp) * 2;
    int *toff = reinterpret_cast<int *>(p);
    p += (size_t)(kp.S + 1) / 2;
    Smem sm = carve(p, kp.L, 0, kp.S, kp.xd);
    sm.etab = etab;
    sm.ktab = ktab;
    sm.rtab = rtab;
    sm.toff = toff;
    return sm;
}

// Copies the item's tables into its shared-memory slots (a CTA does this
// only when its tile belongs to another item than its previous one).
__device__ __forceinline__ void batch_stage(const BatchItemDev &it, const Smem &sm)
{
    const KParams &kp = it.kp;
    const int tid = threadIdx.x, nt = blockDim.x;
    stage_chain_table(kp, sm, tid, nt);
    double *etab = const_cast<double *>(sm.etab), *ktab = const_cast<double *>(sm.ktab);
    double *rtab = const_cast<double *>(sm.rtab);
    int *toff = const_cast<int *>(sm.toff);
    for (int i = tid; i < it.etab_rows * E_NF; i += nt) etab[i] = __ldg(it.etab + i);
    for (int i = tid; i < it.ktab_rows * 2; i += nt) ktab[i] = __ldg(it.ktab + i);
    for (int i = tid; i < resp_rows(kp) * 2; i += nt) rtab[i] = __ldg(it.rtab + i);
    for (int i = tid; i < kp.S; i += nt) toff[i] = __ldg(it.toff + i);
}

// Copies of the tile of item `it` that starts at line q0 into the item's
// tile slot of shared memory, issued by every thread as 8-byte cp.async,
// then one arrival per thread on `bar` (initialised to the CTA's thread
// count).  x lines: the tile's lines are consecutive in global memory and go
// to the [L][n | 1] tile (element e of the span at line e / n, row e % n);
// y/z lines: thread tid copies line tid % L, rows tid / L + k * (threads / L),
// to tile[tid + k * threads] of the [n][L] tile.  Lines past the field's end
// are not copied (their results are never stored).
__device__ __forceinline__ void batch_issue_async(const BatchItemDev &it, double *smem, unsigned long long *bar,
                                                  long long q0)
{
    const KParams &kp = it.kp;
    double *tile = batch_carve(it, smem).tile;
    const int tid = threadIdx.x, nthreads = blockDim.x, L = kp.L, n = kp.n;
    const long long rem = kp.nlines - q0;
    const int nl = (int)(rem < L ? rem : L);
    if (batch_code_xl(it.code)) {
        const int P = n | 1, pad = P - n;
        const int total = nl * n;
        const double *src = kp.in + q0 * (long long)n + tid;
        const int l0 = tid / n;
        int r = tid - l0 * n;
        double *dst = tile + (size_t)l0 * P + r;
        const int dl = nthreads / n, dr = nthreads - dl * n;
        const int dstep = dl * P + dr;
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
        const int l = tid % L;
        if (l < nl) {
            const int rstep = nthreads / L;
            const long long sstep = (long long)rstep * kp.stride;
            const double *src = kp.in + line_base(kp, q0 + l) + (long long)(tid / L) * kp.stride;
            double *dst = tile + tid;
#pragma unroll 4
            for (int r = tid / L; r < n; r += rstep) {
                async_copy8(dst, src);
                src += sstep;
                dst += nthreads;
            }
        }
    }
    async_arrive(bar);
}

// The tile of item `it` starting at line q0 into its shared-memory slot with
// plain coalesced loads (lines past the field's end read as zero).
__device__ __forceinline__ void batch_load_plain(const BatchItemDev &it, double *smem, long long q0)
{
    const KParams &kp = it.kp;
    const int L = kp.L, n = kp.n;
    double *tile = batch_carve(it, smem).tile;
    const int tid = threadIdx.x, nthreads = blockDim.x;
    const long long rem = kp.nlines - q0;
    const int nl = (int)(rem < L ? rem : L);
    if (batch_code_xl(it.code)) {
        const int P = n | 1;
        const int warp = tid >> 5, lane = tid & 31, nw = nthreads >> 5;
        for (int l = warp; l < L; l += nw) {
            const double *src = kp.in + (q0 + l) * (long long)n;
            double *dst = tile + (size_t)l * P;
            for (int r = lane; r < n; r += 32) dst[r] = l < nl ? __ldcs(src + r) : 0.0;
        }
    } else {
        const int l = tid % L, rstep = nthreads / L;
        const double *src = kp.in + (l < nl ? line_base(kp, q0 + l) : 0);
        for (int r = tid / L; r < n; r += rstep)
            tile[(size_t)r * L + l] = l < nl ? __ldcs(src + (long long)r * kp.stride) : 0.0;
    }
}

// The sweep of one tile of one item (tables staged, tile in place).  Not
// inlined: each (stencil, boundary, direction, segment length) gets its own
// register allocation instead of the kernel carrying the union of all of them.
template <int RK, bool PER, int M, bool XL>
__device__ __noinline__ void batch_tile(const BatchItemDev &it, double *smem, long long q0)
{
    using RL = ResidentLine<RK, PER, M>;
    const KParams &kp = it.kp;
    const int L = kp.L, n = kp.n;
    const int P = XL ? (n | 1) : n;  // odd pitch: the lanes (lines) of a warp hit different banks
    const Smem sm = batch_carve(it, smem);
    const int tid = threadIdx.x, nthreads = blockDim.x;
    const long long rem = kp.nlines - q0;
    const int nl = (int)(rem < L ? rem : L);

    const int l = tid % L, slot = tid / L, s = slot_segment(kp, slot);
    const bool active = s >= 0;
    const long long rs = XL ? 1 : (long long)L;
    double *line = sm.tile + (XL ? (size_t)l * P : (size_t)l);
    typename RL::Halo h;
    if (active) RL::prep(kp, line, rs, s, h);
    __syncthreads();
    if (active) RL::template fwd<true>(kp, sm, line, rs, l, s, h);
    __syncthreads();
    if (active) RL::template bwd<true>(kp, sm, line, rs, l, s);
    else if (PER && slot == kp.border_slot) RL::border_only(kp, sm, l);
    __syncthreads();
    if (XL) {
        if (active) RL::template fin<true>(kp, sm, line, rs, l, s, line, 1, true);
        __syncthreads();
        const int warp = tid >> 5, lane = tid & 31, nw = nthreads >> 5;
        for (int ll = warp; ll < nl; ll += nw) {
            double *dst = kp.out + (q0 + ll) * (long long)n;
            const double *src = sm.tile + (size_t)ll * P;
            if (kp.out_mode == OUT_STORE) {
                for (int r = lane; r < n; r += 32) __stcs(dst + r, src[r]);
            } else {
                for (int r = lane; r < n; r += 32) out_put(kp, dst + r, src[r]);
            }
        }
    } else {
        const bool live = l < nl;
        double *dst = kp.out + (live ? line_base(kp, q0 + l) : 0);
        if (active) RL::template fin<true>(kp, sm, line, rs, l, s, dst, kp.stride, live, true);
    }
}

// Runs tile q0 of `it` on the (stencil, boundary, direction, segment length)
// instantiation its code names.
__device__ __forceinline__ void batch_dispatch(const BatchItemDev &it, double *smem, long long q0)
{
    switch (it.code) {
#define PADO_CASE_M(rk, per, xl)                                                             \
    case ((rk * 2 + per) * 2 + xl) * 4 + 0: batch_tile<rk, per, 16, xl>(it, smem, q0); break; \
    case ((rk * 2 + per) * 2 + xl) * 4 + 1: batch_tile<rk, per, 32, xl>(it, smem, q0); break; \
    case ((rk * 2 + per) * 2 + xl) * 4 + 2: batch_tile<rk, per, 64, xl>(it, smem, q0); break;
#define PADO_CASE(rk)                  \
    PADO_CASE_M(rk, false, false)      \
    PADO_CASE_M(rk, false, true)       \
    PADO_CASE_M(rk, true, false)       \
    PADO_CASE_M(rk, true, true)
        PADO_CASE(0)
        PADO_CASE(1)
        PADO_CASE(2)
        PADO_CASE(3)
#undef PADO_CASE
#undef PADO_CASE_M
    default: break;
    }
}

// The item of tile t: the last i with tile0s[i] <= t.
__device__ __forceinline__ int batch_find_item(const long long *__restrict__ tile0s, int nitems, long long t)
{
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tile0s + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// items: descriptors in schedule order; tile0s[i] = items[i].tile0 (compact,
// for the search); counter[0]: tile counter, counter[1]: status word, both
// zeroed before the launch (the status becomes PADO_STATUS_TIMEOUT when a
// CTA's wait for its tile copies expired; that CTA then stops).
__global__ void __launch_bounds__(BATCH_THREADS, BATCH_MIN_CTAS) batch_kernel(const BatchItemDev *__restrict__ items,
                                                                 const long long *__restrict__ tile0s, int nitems,
                                                                 long long ntiles, unsigned long long *counter)
{
    extern __shared__ double smem_raw[];
    __shared__ long long s_tile, s_end, s_next, s_next_end;  // current / next tile and the end of its claim
    __shared__ int s_last;
    __shared__ unsigned long long s_bar;
    // the current item's descriptor, in shared memory: the sweeps read its
    // parameters (segment starts, interior patterns) in their loops
    __shared__ BatchItemDev s_it;
    static_assert(sizeof(BatchItemDev) % sizeof(long long) == 0, "descriptor copy granularity");
    const int tid = threadIdx.x, nthreads = blockDim.x;
    if (tid == 0) {
        s_last = -1;
        s_tile = (long long)atomicAdd(counter, (unsigned long long)BATCH_CLAIM);
        s_end = s_tile + BATCH_CLAIM;
        mbar_init(&s_bar, (unsigned)nthreads);
        mbar_fence_init();
    }
    __syncthreads();
    {
        const long long t = s_tile;
        if (t < ntiles) {
            const BatchItemDev &g = items[batch_find_item(tile0s, nitems, t)];
            batch_issue_async(g, smem_raw, &s_bar, (t - g.tile0) * g.kp.L);
        }
    }
    for (unsigned k = 0;; ++k) {
        const long long t = s_tile;
        if (t >= ntiles) break;
        const int lo = batch_find_item(tile0s, nitems, t);
        // warp 0 waits for the tile's copies; the other warps sleep in the barrier
        bool arrived = true;
        if (tid < 32) arrived = mbar_wait(&s_bar, k & 1u, STREAM_WAIT_NS);
        if (!__syncthreads_and(arrived)) {
            if (tid == 0) atomicExch(counter + 1, (unsigned long long)(long long)PADO_STATUS_TIMEOUT);
            async_wait_all();
            return;
        }
        const bool fresh = lo != s_last;
        if (fresh) {
            const long long *src = reinterpret_cast<const long long *>(items + lo);
            long long *dst = reinterpret_cast<long long *>(&s_it);
            for (int i = tid; i < (int)(sizeof(BatchItemDev) / sizeof(long long)); i += nthreads) dst[i] = src[i];
        }
        __syncthreads();
        if (tid == 0) {
            s_last = lo;
            // the next tile: the rest of this claim, else a new claim, made now
            // so that the atomic's latency hides behind this tile
            if (t + 1 < s_end) {
                s_next = t + 1;
                s_next_end = s_end;
            } else {
                s_next = (long long)atomicAdd(counter, (unsigned long long)BATCH_CLAIM);
                s_next_end = s_next + BATCH_CLAIM;
            }
        }
        if (fresh) {
            // the item's tables into their slots (the tile's slot is disjoint)
            batch_stage(s_it, batch_carve(s_it, smem_raw));
            __syncthreads();
        }
        const BatchItemDev &it = s_it;
        batch_dispatch(it, smem_raw, (t - it.tile0) * it.kp.L);
        __syncthreads();  // the tile's buffer is free, s_next visible
        const long long tn = s_next;
        if (tn < ntiles) {
            const BatchItemDev &g = items[batch_find_item(tile0s, nitems, tn)];
            batch_issue_async(g, smem_raw, &s_bar, (tn - g.tile0) * g.kp.L);
        }
        if (tid == 0) {
            s_tile = tn;
            s_end = s_next_end;
        }
        __syncthreads();
    }
}

// Asks L2 for the lines of the tile starting at line q0 (all threads, one
// request per 128-byte line of memory; nothing waits for them).
__device__ __forceinline__ void prefetch_tile_l2(const KParams &kp, long long q0, bool xl)
{
    const long long rem = kp.nlines - q0;
    if (rem <= 0) return;
    const int nl = (int)(rem < kp.L ? rem : kp.L), n = kp.n;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (xl) {
        const int chunks = (n * 8 + 127) / 128;
        for (int i = tid; i < nl * chunks; i += nt) {
            const double *p = kp.in + (q0 + i / chunks) * (long long)n + (i % chunks) * 16;
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
        }
    } else {
        const double *b0 = kp.in + line_base(kp, q0), *b1 = kp.in + line_base(kp, q0 + nl - 1);
        for (int r = tid; r < n; r += nt) {
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(b0 + (long long)r * kp.stride));
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(b1 + (long long)r * kp.stride));
        }
    }
}

// One field whose lines the streaming kernel's copy engine cannot move (an odd
// extent, an unaligned pointer): the same resident tiles with plain loads,
// the descriptor a kernel parameter, tiles strided over the grid.
__global__ void __launch_bounds__(BATCH_THREADS, BATCH_MIN_CTAS) single_kernel(const __grid_constant__ BatchItemDev it)
{
    extern __shared__ double smem_raw[];
    batch_stage(it, batch_carve(it, smem_raw));
    const long long ntiles = (it.kp.nlines + it.kp.L - 1) / it.kp.L;
    const bool xl = batch_code_xl(it.code);
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        __syncthreads();  // tables staged / the previous tile's buffer free
        const long long q0 = t * it.kp.L;
        batch_load_plain(it, smem_raw, q0);
        // the next tile of this CTA towards L2 while this one is solved
        if (t + gridDim.x < ntiles) prefetch_tile_l2(it.kp, (t + gridDim.x) * it.kp.L, xl);
        __syncthreads();
        batch_dispatch(it, smem_raw, q0);
    }
}
#endif

}  // namespace pado

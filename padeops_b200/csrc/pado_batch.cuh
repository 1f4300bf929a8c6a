// pado_batch.cuh -- persistent kernel that runs many line families (fields of
// uneven sizes, schemes, boundary types and directions) in one launch.
//
// Work unit = one tile (L lines of one field).  Tiles of all items are
// numbered, most expensive item first; CTAs claim tiles from a device
// counter (atomicAdd, no waiting on other CTAs) until the list is exhausted.
#pragma once

#include "pado_kernels.cuh"

namespace pado {

constexpr int BATCH_M = 32;  // segment length of the batched kernel

struct BatchItemDev {
    KParams kp;            // geometry, tables and tiling of this item
    long long tile0;       // first tile index of this item
    int code;              // rk * 4 + periodic * 2 + direct
    int pad;
};

#ifdef __CUDACC__
template <int RK, bool PER, bool STRIDED>
__device__ __forceinline__ void batch_tile(const KParams &kp, double *smem, long long q0)
{
    const Smem sm = carve(smem, kp.L, kp.P, kp.S, kp.xd);
    run_tile<RK, PER, false, BATCH_M, STRIDED ? IN_GLOBAL : IN_LINES>(kp, sm, q0);
}

// counter: tile counter, zeroed before the launch.
__global__ void __launch_bounds__(512) batch_kernel(const BatchItemDev *__restrict__ items, int nitems,
                                                     long long ntiles, unsigned long long *counter)
{
    extern __shared__ double smem_raw[];
    __shared__ long long s_tile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(counter, 1ULL);
        __syncthreads();
        const long long t = s_tile;
        __syncthreads();
        if (t >= ntiles) return;
        int lo = 0, hi = nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].tile0 <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchItemDev &it = items[lo];
        const KParams &kp = it.kp;
        const long long q0 = (t - it.tile0) * kp.L;
        switch (it.code) {
#define PADO_CASE(rk)                                                  \
    case rk * 4 + 0: batch_tile<rk, false, false>(kp, smem_raw, q0); break; \
    case rk * 4 + 1: batch_tile<rk, false, true>(kp, smem_raw, q0); break;  \
    case rk * 4 + 2: batch_tile<rk, true, false>(kp, smem_raw, q0); break;  \
    case rk * 4 + 3: batch_tile<rk, true, true>(kp, smem_raw, q0); break;
            PADO_CASE(0)
            PADO_CASE(1)
            PADO_CASE(2)
            PADO_CASE(3)
#undef PADO_CASE
        default: break;
        }
        __syncthreads();
    }
}
#endif

}  // namespace pado

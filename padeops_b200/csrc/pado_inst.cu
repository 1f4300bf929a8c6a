// pado_inst.cu -- instantiations of the line and streaming kernels for one
// stencil.  The library compiles this file once per stencil with
// -DPADO_RK=0..3 (cd06 d1, cd10 d1, cd10 d2, cf90), so the four instantiation
// sets build in parallel; each defines the entry points pick_kernel_rkN and
// pick_stream_rkN of pado_internal.h.
#include "pado_internal.h"

#ifndef PADO_RK
#error "compile with -DPADO_RK=<stencil 0..3>"
#endif
#define PADO_CAT2(a, b) a##b
#define PADO_CAT(a, b) PADO_CAT2(a, b)

namespace pado {

namespace {

constexpr int RK = PADO_RK;

// variant 1: one CTA per tile; 2: persistent CTAs with cp.async prefetch;
// 3: persistent CTAs reading straight from global memory with an L2 prefetch.
// The adjoint always runs one CTA per tile.
template <bool PER, int M>
KernelFn pick_in(bool adj, bool contiguous, int variant)
{
    if (adj) return contiguous ? line_kernel<RK, PER, true, M, IN_LINES> : line_kernel<RK, PER, true, M, IN_GLOBAL>;
    if (variant == 2)
        return contiguous ? line_kernel_persist<RK, PER, M, IN_LINES> : line_kernel_persist<RK, PER, M, IN_ROWS>;
    if (variant == 3 && !contiguous) return line_kernel_persist<RK, PER, M, IN_GLOBAL>;
    return contiguous ? line_kernel<RK, PER, false, M, IN_LINES> : line_kernel<RK, PER, false, M, IN_GLOBAL>;
}

template <bool PER>
KernelFn pick_m(int m, bool adj, bool contiguous, int variant)
{
    switch (m) {
    case 16: return pick_in<PER, 16>(adj, contiguous, variant);
    case 32: return pick_in<PER, 32>(adj, contiguous, variant);
    default: return pick_in<PER, 64>(adj, contiguous, variant);
    }
}

template <bool PER, bool XL, int LT, bool ADJ, bool AS>
StreamFn pick_stream_m(int m)
{
    switch (m) {
    case 16: return stream_kernel<RK, PER, 16, XL, LT, ADJ, AS>;
    case 32: return stream_kernel<RK, PER, 32, XL, LT, ADJ, AS>;
    default: return stream_kernel<RK, PER, 64, XL, LT, ADJ, AS>;
    }
}

template <bool PER, bool ADJ, bool AS>
StreamFn pick_stream_l(int m, bool xl, int lines)
{
    if (xl) return pick_stream_m<PER, true, 0, ADJ, AS>(m);
    if (lines == 32) return pick_stream_m<PER, false, 32, ADJ, AS>(m);
    return lines == 8 ? pick_stream_m<PER, false, 8, ADJ, AS>(m) : pick_stream_m<PER, false, 16, ADJ, AS>(m);
}

}  // namespace

// as: the tile copies are per-element cp.async (forward operators only)
StreamFn PADO_CAT(pick_stream_rk, PADO_RK)(bool per, int m, bool xl, int lines, bool adj, bool as)
{
    if (adj) return per ? pick_stream_l<true, true, false>(m, xl, lines) : pick_stream_l<false, true, false>(m, xl, lines);
    if (as) return per ? pick_stream_l<true, false, true>(m, xl, lines) : pick_stream_l<false, false, true>(m, xl, lines);
    return per ? pick_stream_l<true, false, false>(m, xl, lines) : pick_stream_l<false, false, false>(m, xl, lines);
}

KernelFn PADO_CAT(pick_kernel_rk, PADO_RK)(bool per, bool adj, bool contiguous, int m, int variant)
{
    return per ? pick_m<true>(m, adj, contiguous, variant) : pick_m<false>(m, adj, contiguous, variant);
}

}  // namespace pado

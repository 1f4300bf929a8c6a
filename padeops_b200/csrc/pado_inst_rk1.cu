// pado_inst_rk1.cu -- instantiations of the line kernels for one stencil
// (cd10 first derivative); split per stencil so the library compiles in parallel.
#include "pado_internal.h"

namespace pado {

namespace {

// variant 1: one CTA per tile; 2: persistent CTAs with cp.async prefetch;
// 3: persistent CTAs reading straight from global memory with an L2 prefetch.
// The adjoint always runs one CTA per tile.
template <bool PER, int M>
KernelFn pick_in(bool adj, bool contiguous, int variant)
{
    constexpr int RK = 1;
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

template <bool PER, bool XL, int LT, bool ADJ>
StreamFn pick_stream_m(int m)
{
    constexpr int RK = 1;
    switch (m) {
    case 16: return stream_kernel<RK, PER, 16, XL, LT, ADJ>;
    case 32: return stream_kernel<RK, PER, 32, XL, LT, ADJ>;
    default: return stream_kernel<RK, PER, 64, XL, LT, ADJ>;
    }
}

template <bool PER, bool ADJ>
StreamFn pick_stream_l(int m, bool xl, int lines)
{
    if (xl) return pick_stream_m<PER, true, 0, ADJ>(m);
    return lines == 8 ? pick_stream_m<PER, false, 8, ADJ>(m) : pick_stream_m<PER, false, 16, ADJ>(m);
}

}  // namespace

StreamFn pick_stream_rk1(bool per, int m, bool xl, int lines, bool adj)
{
    if (adj) return per ? pick_stream_l<true, true>(m, xl, lines) : pick_stream_l<false, true>(m, xl, lines);
    return per ? pick_stream_l<true, false>(m, xl, lines) : pick_stream_l<false, false>(m, xl, lines);
}

KernelFn pick_kernel_rk1(bool per, bool adj, bool contiguous, int m, int variant)
{
    return per ? pick_m<true>(m, adj, contiguous, variant) : pick_m<false>(m, adj, contiguous, variant);
}

}  // namespace pado

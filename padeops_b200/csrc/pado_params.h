// pado_params.h -- fills the table-derived launch parameters of a line
// kernel (everything except pointers and field geometry).  Host only; shared
// by the library and its tests.
#pragma once

#include <cstring>

#include "pado_kernels.cuh"
#include "pado_tables.h"

namespace pado {

static_assert(KMAXM == MAXM && KCT_NF == CT_NF, "kernel and table builder disagree on the table shapes");

inline void set_chain(KParams &kp, const ChainTables &ch);

inline void fill_params(KParams &kp, const OpTables &ot, int n, int bc1, int bcn)
{
    kp.n = n;
    kp.nb = ot.nb;
    kp.nbord = ot.nbord;
    kp.P = (n % 2 == 0) ? n + 1 : n;
    kp.S = ot.lay.S;
    for (int i = 0; i < 33; ++i) kp.sstart[i] = (unsigned short)(i <= ot.lay.S ? ot.lay.st[i] : n);
    kp.bc1 = bc1;
    kp.bcn = bcn;
    std::memcpy(kp.mb, ot.mb, sizeof(kp.mb));
    std::memcpy(kp.taps, ot.taps, sizeof(kp.taps));
    kp.rc = ot.rc;
    const Interior &in = ot.interior;
    kp.int_mask = in.mask;
    kp.spk_mask = in.spk_mask;
    std::memcpy(kp.kc, in.kc, sizeof(kp.kc));
    std::memcpy(kp.pu, in.pu, sizeof(kp.pu));
    std::memcpy(kp.pv, in.pv, sizeof(kp.pv));
    std::memcpy(kp.ps, in.ps, sizeof(kp.ps));
    std::memcpy(kp.pt, in.pt, sizeof(kp.pt));
    std::memcpy(kp.sperm, ot.sperm, sizeof(ot.sperm));
    kp.nslots = kp.S;
    kp.border_slot = -1;
    kp.ie = ot.ie;
    kp.je = ot.nbord > 0 ? ot.je : ot.nb;
    set_chain(kp, ot.chain);
}

// Coupling window of the chain tables in use (the table pointers are set by
// the caller).
inline void set_chain(KParams &kp, const ChainTables &ch)
{
    kp.W = ch.W;
    kp.xd = (int)ch.xtab.size();
    std::memcpy(kp.wf, ch.wf, sizeof(kp.wf));
    std::memcpy(kp.wb, ch.wb, sizeof(kp.wb));
    std::memcpy(kp.xof, ch.xof, sizeof(kp.xof));
    std::memcpy(kp.xob, ch.xob, sizeof(kp.xob));
}

// Field geometry of the line family along `axis` of an (n1, n2, n3) field
// passed as (na, nb) like the reference's dd1/dd2/dd3 (na, nb = the other
// two extents, x first).
inline void set_geometry(KParams &kp, int axis, int n, long long na, long long nb)
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

}  // namespace pado

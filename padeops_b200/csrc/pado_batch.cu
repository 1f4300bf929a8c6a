// pado_batch.cu -- batched execution: one persistent launch over many
// (field, operator) items, its CUDA-graph replay, and the per-item loop it
// replaces.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "pado_batch.cuh"
#include "pado_internal.h"

using namespace pado;

struct pado_batch_s {
    std::vector<pado_batch_item> items;  // as given
    std::vector<BatchItemDev> dev;       // sorted most expensive tile first
    BatchItemDev *d_items = nullptr;
    long long *d_tile0s = nullptr;            // first tile of each item (compact copy for the search)
    unsigned long long *d_counter = nullptr;  // tile counter (device scratch)
    long long ntiles = 0;
    size_t smem = 0;
    int lines = 0, ctas_per_sm = 0;  // lines per tile (0: 16 where it fits, else 8); CTA cap per SM
    int device = 0, num_sms = 0, grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture_stream = nullptr;
    // graph contents: 0 = the persistent launch; k > 0 = one streaming-kernel
    // launch per item, the items dealt round-robin to k concurrent branches
    int branches = 0;
    std::vector<cudaStream_t> branch_streams;
    std::vector<cudaEvent_t> branch_events;  // [0]: fork, [1 + k]: branch k done
};

namespace {

constexpr size_t BATCH_SMEM_CAP = 110 * 1024;  // per CTA, leaves room for 2 CTAs/SM

}  // namespace

namespace pado {

// Descriptor of one item, with the tiling rules shared by batch objects and
// the allocation-free launch.  lines: lines per tile (8, 16, 32 or 64), or 0:
// as many as keep all BATCH_THREADS threads busy (BATCH_THREADS / segments,
// a multiple of 8, at most 64) within the shared-memory cap -- short lines
// have few segments, so their tiles take more lines.  *skip: nothing to do.
int batch_item_descriptor(const pado_batch_item &it, int lines, BatchItemDev *d, long long *tiles, double *cost,
                          size_t *smem, bool *skip)
{
    *skip = false;
    if (!it.op) return PADO_E_NULL;
    if (it.op->m != 16 && it.op->m != 32 && it.op->m != 64) return PADO_E_SIZE;  // the segment lengths built
    if (it.axis < 1 || it.axis > 3 || it.n1 < 0 || it.n2 < 0 || it.n3 < 0) return PADO_E_ARG;
    const long long ext[3] = {it.n1, it.n2, it.n3};
    if (ext[it.axis - 1] != it.op->n) return PADO_E_ARG;
    const long long na = it.axis == 1 ? it.n2 : it.n1;
    const long long nb = it.axis == 3 ? it.n2 : it.n3;
    KParams kp;
    bool trivial = true;
    int rc = prepare_launch(it.op, it.kind, it.axis, it.f, it.df, (long)na, (long)nb, it.bc1, it.bcn, false, 1, false,
                            &kp, &trivial);
    if (rc != PADO_OK) return rc;
    if (trivial) {
        if (it.op->n == 1 && (long long)na * nb > 0) return PADO_E_UNSUPPORTED;  // n == 1 items: use pado_apply
        *skip = true;
        return PADO_OK;
    }
    const bool xl = it.axis == 1;
    const bool bounded_bc = !it.op->periodic && it.op->scheme != CD06;
    const auto tit = it.op->tables.find(TabKey(it.kind, bounded_bc ? it.bc1 : 0, bounded_bc ? it.bcn : 0, 0));
    if (tit == it.op->tables.end()) return PADO_E_STATE;
    const DevTables &dt = tit->second;
    const int erows = (int)(dt.host.etab.size() / E_NF), krows = (int)(dt.host.ktab.size() / KT_NF);
    auto bytes = [&](int L_) {
        return batch_smem_doubles(L_, kp.S, kp.n, xl, kp.xd, erows, krows, resp_rows(kp)) * sizeof(double);
    };
    // the most lines (64, 32, 16, 8) whose slots (grouped by code path,
    // padded to whole warps) fit the CTA and whose tile fits the cap
    int L = 0, nslots = 0;
    unsigned char perm[KMAXSLOT];
    for (int cand : {64, 32, 16, 8}) {
        if (lines && cand != lines) continue;
        int ns = warp_slots(dt.host, cand, perm, KMAXSLOT, true);
        if (cand * ns > BATCH_THREADS) ns = warp_slots(dt.host, cand, perm, KMAXSLOT, false);
        if (cand * ns > BATCH_THREADS || bytes(cand) > BATCH_SMEM_CAP) continue;
        L = cand;
        nslots = ns;
        break;
    }
    if (!L) return PADO_E_SIZE;
    kp.L = L;
    kp.nslots = nslots;
    std::memcpy(kp.sperm, perm, sizeof(perm));
    kp.border_slot = first_idle_slot(perm, nslots);
    std::memset(d, 0, sizeof(*d));
    d->kp = kp;
    d->etab = dt.etab;
    d->ktab = dt.ktab;
    d->rtab = dt.rtab;
    d->toff = dt.toff;
    d->code = batch_code(kp.rc.rk, it.op->periodic != 0, xl, it.op->m);
    d->etab_rows = erows;
    d->ktab_rows = krows;
    *tiles = (kp.nlines + L - 1) / L;
    *cost = (double)L * kp.n;
    *smem = bytes(L);
    return PADO_OK;
}

// The resident single-field kernel (single_kernel) for one apply; returns
// PADO_E_UNSUPPORTED when the field does not fit its rules (segments of 16,
// 32 or 64 rows, the tile within the shared-memory cap), so that the caller can use
// the line kernel instead.  info (not null): fill the launch plan the way
// pado_launch_plan reports it and launch nothing.
int launch_resident_single(pado_op_s *op, int kind, int axis, const double *f, double *df, long na, long nb,
                           int bc1, int bcn, cudaStream_t st, int *info, int out_mode, double out_alpha)
{
    pado_batch_item it{};
    it.op = op;
    it.kind = kind;
    it.axis = axis;
    it.bc1 = bc1;
    it.bcn = bcn;
    it.n1 = axis == 1 ? op->n : na;
    it.n2 = axis == 1 ? na : (axis == 2 ? op->n : nb);
    it.n3 = axis == 3 ? op->n : nb;
    it.f = f;
    it.df = df;
    BatchItemDev d;
    long long tiles = 0;
    double cost = 0;
    size_t smem = 0;
    bool skip = false;
    const int rc = batch_item_descriptor(it, 0, &d, &tiles, &cost, &smem, &skip);
    if (rc == PADO_E_SIZE) return PADO_E_UNSUPPORTED;
    if (rc != PADO_OK || skip) return rc;
    d.tile0 = 0;
    d.kp.out_mode = out_mode;
    d.kp.out_alpha = out_alpha;
    cudaError_t e = cudaFuncSetAttribute((const void *)single_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)BATCH_SMEM_CAP);
    if (e != cudaSuccess) return cuda_fail(e);
    int per_sm = 0, dev = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, single_kernel, BATCH_THREADS, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e);
    if (per_sm < 1) return PADO_E_UNSUPPORTED;
    if (info) {
        info[0] = 5;
        info[1] = d.kp.L;
        info[2] = 1;
        info[3] = per_sm;
        info[6] = d.kp.L * d.kp.nslots;
        info[7] = (int)smem;
        return PADO_OK;
    }
    const long long grid = std::max<long long>(1, std::min<long long>(tiles, (long long)per_sm * sms));
    single_kernel<<<(unsigned)grid, BATCH_THREADS, smem, st>>>(d);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

}  // namespace pado

namespace {

int layout_items(pado_batch_s *b)
{
    struct Pre {
        BatchItemDev d;
        long long tiles;
        double cost;
    };
    std::vector<Pre> pre;
    size_t smem = 0;
    for (const pado_batch_item &it : b->items) {
        Pre p;
        size_t sm = 0;
        bool skip = false;
        const int rc = batch_item_descriptor(it, b->lines, &p.d, &p.tiles, &p.cost, &sm, &skip);
        if (rc != PADO_OK) return rc;
        if (skip) continue;
        smem = std::max(smem, sm);
        pre.push_back(p);
    }
    std::stable_sort(pre.begin(), pre.end(), [](const Pre &x, const Pre &y) { return x.cost > y.cost; });
    b->dev.clear();
    long long t0 = 0;
    for (Pre &p : pre) {
        p.d.tile0 = t0;
        t0 += p.tiles;
        b->dev.push_back(p.d);
    }
    b->ntiles = t0;
    b->smem = smem;
    return PADO_OK;
}

int upload_batch(pado_batch_s *b)
{
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_tile0s) cudaFree(b->d_tile0s);
    b->d_items = nullptr;
    b->d_tile0s = nullptr;
    if (!b->dev.empty()) {
        std::vector<long long> t0(b->dev.size());
        for (size_t i = 0; i < b->dev.size(); ++i) t0[i] = b->dev[i].tile0;
        cudaError_t e = cudaMalloc(&b->d_items, b->dev.size() * sizeof(BatchItemDev));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_tile0s, t0.size() * sizeof(long long));
        if (e != cudaSuccess) return cuda_fail(e);
        e = cudaMemcpy(b->d_items, b->dev.data(), b->dev.size() * sizeof(BatchItemDev), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b->d_tile0s, t0.data(), t0.size() * sizeof(long long), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    if (!b->d_counter) {
        cudaError_t e = cudaMalloc(&b->d_counter, 2 * sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_fail(e);
    }
    // The attribute is per function, shared by every batch: always the cap (every
    // batch's smem is below it), so creating one batch never invalidates another.
    cudaError_t e = cudaFuncSetAttribute((const void *)batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)BATCH_SMEM_CAP);
    if (e != cudaSuccess) return cuda_fail(e);
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, BATCH_THREADS, b->smem);
    if (e != cudaSuccess) return cuda_fail(e);
    if (per_sm < 1) return PADO_E_SIZE;
    if (b->ctas_per_sm > 0) per_sm = std::min(per_sm, b->ctas_per_sm);
    long long grid = (long long)per_sm * b->num_sms;
    if (grid > b->ntiles) grid = b->ntiles;
    b->grid = (int)std::max<long long>(grid, 1);
    return PADO_OK;
}

void drop_graph(pado_batch_s *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

int enqueue_persistent(pado_batch_s *b, cudaStream_t st)
{
    if (b->ntiles == 0) return PADO_OK;
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);
    batch_kernel<<<b->grid, BATCH_THREADS, b->smem, st>>>(b->d_items, b->d_tile0s, (int)b->dev.size(), b->ntiles,
                                                          b->d_counter);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

// Per-item launches on b->branches concurrent branches of stream `st` (fork
// and join by events, so that a stream capture records them as parallel
// branches of one graph), dealt largest first to the least-loaded branch.
int enqueue_branches(pado_batch_s *b, cudaStream_t st)
{
    const int k = b->branches;
    while ((int)b->branch_streams.size() < k) {
        cudaStream_t s = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e);
        b->branch_streams.push_back(s);
    }
    while ((int)b->branch_events.size() < k + 1) {
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e);
        b->branch_events.push_back(ev);
    }
    cudaError_t e = cudaEventRecord(b->branch_events[0], st);
    for (int j = 0; j < k && e == cudaSuccess; ++j) e = cudaStreamWaitEvent(b->branch_streams[j], b->branch_events[0], 0);
    if (e != cudaSuccess) return cuda_fail(e);
    // largest items first, each to the branch with the least work so far
    std::vector<size_t> order(b->items.size());
    std::iota(order.begin(), order.end(), size_t(0));
    auto points = [&](size_t i) { return (double)b->items[i].n1 * b->items[i].n2 * b->items[i].n3; };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return points(x) > points(y); });
    std::vector<double> load(k, 0.0);
    int rc = PADO_OK;
    for (size_t i : order) {
        const pado_batch_item &it = b->items[i];
        const long long na = it.axis == 1 ? it.n2 : it.n1;
        const long long nb = it.axis == 3 ? it.n2 : it.n3;
        const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[j] += points(i);
        rc = pado_apply(it.op, it.kind, it.axis, it.f, it.df, (long)na, (long)nb, it.bc1, it.bcn, b->branch_streams[j]);
        if (rc != PADO_OK) break;
    }
    // join every branch, also after an error, so that a capture can end
    for (int j = 0; j < k && e == cudaSuccess; ++j) {
        e = cudaEventRecord(b->branch_events[1 + j], b->branch_streams[j]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->branch_events[1 + j], 0);
    }
    if (rc != PADO_OK) return rc;
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

}  // namespace

extern "C" {

int pado_batch_set_graph_branches(pado_batch_t b, int branches)
{
    if (!b) return PADO_E_NULL;
    if (branches < 0 || branches > 16) return PADO_E_ARG;
    b->branches = branches;
    drop_graph(b);
    return PADO_OK;
}

int pado_batch_create(pado_batch_t *out, const pado_batch_item *items, int nitems)
{
    if (!out) return PADO_E_NULL;
    *out = nullptr;
    if (nitems < 0 || (nitems > 0 && !items)) return PADO_E_ARG;
    auto *b = new (std::nothrow) pado_batch_s;
    if (!b) return PADO_E_NOMEM;
    b->items.assign(items, items + nitems);
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
    int rc = layout_items(b);
    if (rc == PADO_OK) rc = upload_batch(b);
    if (rc != PADO_OK) {
        pado_batch_destroy(b);
        return rc;
    }
    *out = b;
    return PADO_OK;
}

int pado_batch_set_config(pado_batch_t b, int lines, int ctas_per_sm)
{
    if (!b) return PADO_E_NULL;
    if (lines != 0 && lines != 8 && lines != 16 && lines != 32 && lines != 64) return PADO_E_ARG;
    if (ctas_per_sm < 0) return PADO_E_ARG;
    b->lines = lines;
    b->ctas_per_sm = ctas_per_sm;
    drop_graph(b);
    int rc = layout_items(b);
    if (rc == PADO_OK) rc = upload_batch(b);
    return rc;
}

int pado_batch_run(pado_batch_t b, void *stream)
{
    if (!b) return PADO_E_NULL;
    return enqueue_persistent(b, (cudaStream_t)stream);
}

int pado_batch_run_loop(pado_batch_t b, void *stream)
{
    if (!b) return PADO_E_NULL;
    for (const pado_batch_item &it : b->items) {
        const long long na = it.axis == 1 ? it.n2 : it.n1;
        const long long nb = it.axis == 3 ? it.n2 : it.n3;
        int rc = pado_apply(it.op, it.kind, it.axis, it.f, it.df, (long)na, (long)nb, it.bc1, it.bcn, stream);
        if (rc != PADO_OK) return rc;
    }
    return PADO_OK;
}

int pado_batch_run_graph(pado_batch_t b, void *stream)
{
    if (!b) return PADO_E_NULL;
    if (!b->exec) {
        if (!b->capture_stream) {
            cudaError_t e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return cuda_fail(e);
        }
        if (b->branches > 0) {
            // one uncaptured pass first: the per-item launches set their kernels'
            // attributes on first use, which a capture must not record
            int rc0 = pado_batch_run_loop(b, b->capture_stream);
            if (rc0 != PADO_OK) return rc0;
            cudaError_t e0 = cudaStreamSynchronize(b->capture_stream);
            if (e0 != cudaSuccess) return cuda_fail(e0);
        }
        cudaError_t e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e);
        int rc = b->branches > 0 ? enqueue_branches(b, b->capture_stream) : enqueue_persistent(b, b->capture_stream);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(b->capture_stream, &g);
        if (rc != PADO_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e);
        b->graph = g;
        e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) {
            drop_graph(b);
            return cuda_fail(e);
        }
    }
    cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

void pado_batch_destroy(pado_batch_t b)
{
    if (!b) return;
    drop_graph(b);
    for (cudaStream_t s : b->branch_streams) cudaStreamDestroy(s);
    for (cudaEvent_t ev : b->branch_events) cudaEventDestroy(ev);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_tile0s) cudaFree(b->d_tile0s);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

}  // extern "C"

// ---- the batched launch without device allocation --------------------------
//
// g_static_batch holds the tile counter and the status word (first 256 bytes), the item
// descriptors and their first tiles.  Host code must not use its name as an
// address: the device address comes from cudaGetSymbolAddress, once per
// device.

namespace {

constexpr size_t STATIC_ITEMS_OFFSET = 256;
constexpr size_t STATIC_TILE0_OFFSET = STATIC_ITEMS_OFFSET + (size_t)PADO_STATIC_BATCH_MAX_ITEMS * sizeof(BatchItemDev);
static_assert(STATIC_TILE0_OFFSET % sizeof(long long) == 0, "tile start alignment");
static_assert(STATIC_TILE0_OFFSET + (size_t)PADO_STATIC_BATCH_MAX_ITEMS * sizeof(long long) <=
                  (size_t)PADO_STATIC_BATCH_SCRATCH_BYTES,
              "static batch scratch too small for its item limit");
static_assert(alignof(BatchItemDev) <= STATIC_ITEMS_OFFSET, "descriptor alignment");

constexpr int STATIC_MAX_DEVICES = 64;
constexpr int STATIC_CHUNK = 8;      // descriptors staged per host-to-device copy

std::mutex g_static_mu;
unsigned char *g_static_addr[STATIC_MAX_DEVICES] = {};
// held through a whole pado_batch_run_static call, so that calls from several
// host threads enqueue their copies and launch one after the other
std::mutex g_static_run_mu;

}  // namespace

static __device__ __align__(256) unsigned char g_static_batch[PADO_STATIC_BATCH_SCRATCH_BYTES];

namespace {

// Device address of g_static_batch on device `dev` (the current device).
int static_scratch(int dev, unsigned char **out)
{
    if (dev < 0 || dev >= STATIC_MAX_DEVICES) return PADO_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_batch);
        if (e != cudaSuccess) return cuda_fail(e);
        g_static_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_static_addr[dev];
    return PADO_OK;
}

}  // namespace

extern "C" {

int pado_batch_run_static(const pado_batch_item *items, int nitems, void *stream)
{
    if (nitems < 0 || (nitems > 0 && !items)) return PADO_E_ARG;
    if (nitems > PADO_STATIC_BATCH_MAX_ITEMS) return PADO_E_SIZE;
    if (nitems == 0) return PADO_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e);
    unsigned char *base = nullptr;
    int rc = static_scratch(dev, &base);
    if (rc != PADO_OK) return rc;
    std::lock_guard<std::mutex> run_lock(g_static_run_mu);

    // pass 1: validate, cost and tile count of every item (no descriptor kept)
    double cost[PADO_STATIC_BATCH_MAX_ITEMS];
    long long tiles[PADO_STATIC_BATCH_MAX_ITEMS];
    short order[PADO_STATIC_BATCH_MAX_ITEMS];
    int nvalid = 0;
    size_t smem = 0;
    BatchItemDev chunk[STATIC_CHUNK];
    for (int i = 0; i < nitems; ++i) {
        bool skip = false;
        size_t sm = 0;
        if (items[i].op && items[i].op->device != dev) return PADO_E_ARG;
        rc = batch_item_descriptor(items[i], 0, &chunk[0], &tiles[i], &cost[i], &sm, &skip);
        if (rc != PADO_OK) return rc;
        if (skip) continue;
        smem = std::max(smem, sm);
        // insertion keeps equal costs in item order (most expensive first)
        int j = nvalid++;
        while (j > 0 && cost[order[j - 1]] < cost[i]) {
            order[j] = order[j - 1];
            --j;
        }
        order[j] = (short)i;
    }
    if (nvalid == 0) return PADO_OK;

    // pass 2: descriptors in schedule order, staged a few at a time
    cudaStream_t st = (cudaStream_t)stream;
    BatchItemDev *d_items = reinterpret_cast<BatchItemDev *>(base + STATIC_ITEMS_OFFSET);
    unsigned long long *d_counter = reinterpret_cast<unsigned long long *>(base);
    long long *d_tile0s = reinterpret_cast<long long *>(base + STATIC_TILE0_OFFSET);
    long long starts[PADO_STATIC_BATCH_MAX_ITEMS];
    long long t0 = 0;
    for (int k0 = 0; k0 < nvalid; k0 += STATIC_CHUNK) {
        const int kn = std::min(STATIC_CHUNK, nvalid - k0);
        for (int k = 0; k < kn; ++k) {
            const int i = order[k0 + k];
            bool skip = false;
            size_t sm = 0;
            long long nt = 0;
            double c = 0;
            rc = batch_item_descriptor(items[i], 0, &chunk[k], &nt, &c, &sm, &skip);
            if (rc != PADO_OK) return rc;
            chunk[k].tile0 = t0;
            starts[k0 + k] = t0;
            t0 += nt;
        }
        // pageable source: the copy is staged before the call returns, so the
        // chunk can be refilled right away
        e = cudaMemcpyAsync(d_items + k0, chunk, (size_t)kn * sizeof(BatchItemDev), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    const long long ntiles = t0;
    e = cudaMemcpyAsync(d_tile0s, starts, (size_t)nvalid * sizeof(long long), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e);
    e = cudaMemsetAsync(d_counter, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);

    e = cudaFuncSetAttribute((const void *)batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)BATCH_SMEM_CAP);
    if (e != cudaSuccess) return cuda_fail(e);
    int per_sm = 0, num_sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, BATCH_THREADS, smem);
    if (e != cudaSuccess) return cuda_fail(e);
    if (per_sm < 1) return PADO_E_SIZE;
    e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e);
    const long long grid = std::max<long long>(1, std::min<long long>((long long)per_sm * num_sms, ntiles));
    batch_kernel<<<(unsigned)grid, BATCH_THREADS, smem, st>>>(d_items, d_tile0s, nvalid, ntiles, d_counter);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

int pado_batch_status(pado_batch_t b)
{
    if (!b) return PADO_E_NULL;
    if (!b->d_counter) return PADO_OK;
    unsigned long long v[2] = {0, 0};
    cudaError_t e = cudaMemcpy(v, b->d_counter, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e);
    return (int)(long long)v[1];
}

int pado_batch_info(pado_batch_t b, long long *ntiles, int *grid, int *threads, long long *smem_bytes)
{
    if (!b) return PADO_E_NULL;
    if (ntiles) *ntiles = b->ntiles;
    if (grid) *grid = b->grid;
    if (threads) *threads = BATCH_THREADS;
    if (smem_bytes) *smem_bytes = (long long)b->smem;
    return PADO_OK;
}

}  // extern "C"

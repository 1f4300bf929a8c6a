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
    unsigned long long *d_counter = nullptr;  // tile counter (device scratch)
    long long ntiles = 0;
    size_t smem = 0;
    int threads = 256, ctas_per_sm = 0;
    int device = 0, num_sms = 0, grid = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture_stream = nullptr;
};

namespace {

constexpr size_t BATCH_SMEM_CAP = 110 * 1024;  // per CTA, leaves room for 2 CTAs/SM

int layout_items(pado_batch_s *b)
{
    struct Pre {
        BatchItemDev d;
        double cost;
    };
    std::vector<Pre> pre;
    size_t smem = 0;
    for (const pado_batch_item &it : b->items) {
        if (!it.op) return PADO_E_NULL;
        if (it.op->m > BATCH_M) return PADO_E_SIZE;
        if (it.axis < 1 || it.axis > 3 || it.n1 < 0 || it.n2 < 0 || it.n3 < 0) return PADO_E_ARG;
        const long long ext[3] = {it.n1, it.n2, it.n3};
        if (ext[it.axis - 1] != it.op->n) return PADO_E_ARG;
        const long long na = it.axis == 1 ? it.n2 : it.n1;
        const long long nb = it.axis == 3 ? it.n2 : it.n3;
        const int P = (it.op->n % 2 == 0) ? it.op->n + 1 : it.op->n;
        KParams kp;
        bool trivial = true;
        // the register-only path assumes segments of BATCH_M rows
        int rc = prepare_launch(it.op, it.kind, it.axis, it.f, it.df, (long)na, (long)nb, it.bc1, it.bcn, false, 1,
                                it.op->m != BATCH_M, &kp, &trivial);
        if (rc != PADO_OK) return rc;
        if (trivial) {
            if (it.op->n == 1 && (long long)na * nb > 0) return PADO_E_UNSUPPORTED;  // n == 1 items: use pado_apply
            continue;
        }
        const int S = kp.S;
        int L = b->threads / std::max(S, 1);
        while (L > 1 && smem_doubles(L, S, kp.xd, (size_t)L * P) * sizeof(double) > BATCH_SMEM_CAP) --L;
        if (L < 1 || smem_doubles(L, S, kp.xd, (size_t)L * P) * sizeof(double) > BATCH_SMEM_CAP) return PADO_E_SIZE;
        kp.L = L;
        Pre p{};
        p.d.kp = kp;
        p.d.code = kp.rc.rk * 4 + (it.op->periodic ? 2 : 0) + (kp.stride != 1 ? 1 : 0);
        const long long tiles = (kp.nlines + L - 1) / L;
        p.d.tile0 = tiles;  // temporarily the tile count
        p.cost = (double)L * kp.n;
        smem = std::max(smem, smem_doubles(L, kp.S, kp.xd, kp.stride == 1 ? (size_t)L * P : 0) * sizeof(double));
        pre.push_back(p);
    }
    std::stable_sort(pre.begin(), pre.end(), [](const Pre &x, const Pre &y) { return x.cost > y.cost; });
    b->dev.clear();
    long long t0 = 0;
    for (Pre &p : pre) {
        const long long tiles = p.d.tile0;
        p.d.tile0 = t0;
        t0 += tiles;
        b->dev.push_back(p.d);
    }
    b->ntiles = t0;
    b->smem = smem;
    return PADO_OK;
}

int upload_batch(pado_batch_s *b)
{
    if (b->d_items) cudaFree(b->d_items);
    b->d_items = nullptr;
    if (!b->dev.empty()) {
        cudaError_t e = cudaMalloc(&b->d_items, b->dev.size() * sizeof(BatchItemDev));
        if (e != cudaSuccess) return cuda_fail(e);
        e = cudaMemcpy(b->d_items, b->dev.data(), b->dev.size() * sizeof(BatchItemDev), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    if (!b->d_counter) {
        cudaError_t e = cudaMalloc(&b->d_counter, sizeof(unsigned long long));
        if (e != cudaSuccess) return cuda_fail(e);
    }
    // The attribute is per function, shared by every batch: always the cap (every
    // batch's smem is below it), so creating one batch never invalidates another.
    cudaError_t e = cudaFuncSetAttribute((const void *)batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)BATCH_SMEM_CAP);
    if (e != cudaSuccess) return cuda_fail(e);
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, b->threads, b->smem);
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
    cudaError_t e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);
    batch_kernel<<<b->grid, b->threads, b->smem, st>>>(b->d_items, (int)b->dev.size(), b->ntiles, b->d_counter);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

}  // namespace

extern "C" {

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

int pado_batch_set_config(pado_batch_t b, int threads, int ctas_per_sm)
{
    if (!b) return PADO_E_NULL;
    if (threads != 0 && threads != 128 && threads != 256 && threads != 512) return PADO_E_ARG;
    if (ctas_per_sm < 0) return PADO_E_ARG;
    if (threads) b->threads = threads;
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
        cudaError_t e = cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(e);
        int rc = enqueue_persistent(b, b->capture_stream);
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
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

}  // extern "C"

// ---- the batched launch without device allocation --------------------------
//
// g_static_batch holds the tile counter (first 256 bytes) and the item
// descriptors.  Host code must not use its name as an address: the device
// address comes from cudaGetSymbolAddress, once per device.

namespace {

constexpr size_t STATIC_ITEMS_OFFSET = 256;
static_assert(STATIC_ITEMS_OFFSET + (size_t)PADO_STATIC_BATCH_MAX_ITEMS * sizeof(BatchItemDev) <=
                  (size_t)PADO_STATIC_BATCH_SCRATCH_BYTES,
              "static batch scratch too small for its item limit");
static_assert(alignof(BatchItemDev) <= STATIC_ITEMS_OFFSET, "descriptor alignment");

constexpr int STATIC_MAX_DEVICES = 64;
constexpr int STATIC_THREADS = 256;  // threads per CTA (the batch object's default)
constexpr int STATIC_CHUNK = 8;      // descriptors staged per host-to-device copy

std::mutex g_static_mu;
unsigned char *g_static_addr[STATIC_MAX_DEVICES] = {};

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

// One item's descriptor with the same tiling rules as a batch object
// (STATIC_THREADS threads per CTA).  *skip: nothing to do for this item.
int static_item(const pado_batch_item &it, int dev, BatchItemDev *d, long long *tiles, double *cost, size_t *smem,
                bool *skip)
{
    *skip = false;
    if (!it.op) return PADO_E_NULL;
    if (it.op->device != dev) return PADO_E_ARG;
    if (it.op->m > BATCH_M) return PADO_E_SIZE;
    if (it.axis < 1 || it.axis > 3 || it.n1 < 0 || it.n2 < 0 || it.n3 < 0) return PADO_E_ARG;
    const long long ext[3] = {it.n1, it.n2, it.n3};
    if (ext[it.axis - 1] != it.op->n) return PADO_E_ARG;
    const long long na = it.axis == 1 ? it.n2 : it.n1;
    const long long nb = it.axis == 3 ? it.n2 : it.n3;
    const int P = (it.op->n % 2 == 0) ? it.op->n + 1 : it.op->n;
    KParams kp;
    bool trivial = true;
    int rc = prepare_launch(it.op, it.kind, it.axis, it.f, it.df, (long)na, (long)nb, it.bc1, it.bcn, false, 1,
                            it.op->m != BATCH_M, &kp, &trivial);
    if (rc != PADO_OK) return rc;
    if (trivial) {
        if (it.op->n == 1 && (long long)na * nb > 0) return PADO_E_UNSUPPORTED;  // n == 1 items: use pado_apply
        *skip = true;
        return PADO_OK;
    }
    const int S = kp.S;
    int L = STATIC_THREADS / std::max(S, 1);
    while (L > 1 && smem_doubles(L, S, kp.xd, (size_t)L * P) * sizeof(double) > BATCH_SMEM_CAP) --L;
    if (L < 1 || smem_doubles(L, S, kp.xd, (size_t)L * P) * sizeof(double) > BATCH_SMEM_CAP) return PADO_E_SIZE;
    kp.L = L;
    std::memset(d, 0, sizeof(*d));
    d->kp = kp;
    d->code = kp.rc.rk * 4 + (it.op->periodic ? 2 : 0) + (kp.stride != 1 ? 1 : 0);
    *tiles = (kp.nlines + L - 1) / L;
    *cost = (double)L * kp.n;
    *smem = smem_doubles(L, kp.S, kp.xd, kp.stride == 1 ? (size_t)L * P : 0) * sizeof(double);
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
        rc = static_item(items[i], dev, &chunk[0], &tiles[i], &cost[i], &sm, &skip);
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
    long long t0 = 0;
    for (int k0 = 0; k0 < nvalid; k0 += STATIC_CHUNK) {
        const int kn = std::min(STATIC_CHUNK, nvalid - k0);
        for (int k = 0; k < kn; ++k) {
            const int i = order[k0 + k];
            bool skip = false;
            size_t sm = 0;
            long long nt = 0;
            double c = 0;
            rc = static_item(items[i], dev, &chunk[k], &nt, &c, &sm, &skip);
            if (rc != PADO_OK) return rc;
            chunk[k].tile0 = t0;
            t0 += nt;
        }
        // pageable source: the copy is staged before the call returns, so the
        // chunk can be refilled right away
        e = cudaMemcpyAsync(d_items + k0, chunk, (size_t)kn * sizeof(BatchItemDev), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    const long long ntiles = t0;
    e = cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail(e);

    e = cudaFuncSetAttribute((const void *)batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)BATCH_SMEM_CAP);
    if (e != cudaSuccess) return cuda_fail(e);
    int per_sm = 0, num_sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, STATIC_THREADS, smem);
    if (e != cudaSuccess) return cuda_fail(e);
    if (per_sm < 1) return PADO_E_SIZE;
    e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e);
    const long long grid = std::max<long long>(1, std::min<long long>((long long)per_sm * num_sms, ntiles));
    batch_kernel<<<(unsigned)grid, STATIC_THREADS, smem, st>>>(d_items, nvalid, ntiles, d_counter);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    e = cudaGetLastError();
    return e == cudaSuccess ? PADO_OK : cuda_fail(e);
}

int pado_batch_info(pado_batch_t b, long long *ntiles, int *grid, int *threads, long long *smem_bytes)
{
    if (!b) return PADO_E_NULL;
    if (ntiles) *ntiles = b->ntiles;
    if (grid) *grid = b->grid;
    if (threads) *threads = b->threads;
    if (smem_bytes) *smem_bytes = (long long)b->smem;
    return PADO_OK;
}

}  // extern "C"

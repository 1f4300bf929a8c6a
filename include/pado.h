/*
 * pado.h -- C ABI of padeops_b200, a B200-native (CUDA sm_100a, FP64)
 * implementation of PadeOps' compact-difference operators.
 *
 * Each entry point replaces one type-bound procedure of the reference's
 * Fortran scheme objects (paths relative to the reference project):
 *
 *   cd06stuff  src/derivatives/cd06.F90   init :129, dd1/dd2/dd3 :775/797/819, destroy :203
 *   cd10stuff  src/derivatives/cd10.F90   init :195, dd1/dd2/dd3 :2029/2099/2169,
 *                                         d2d1/d2d2/d2d3 :2239/2309/2379, destroy :317
 *   cf90stuff  src/filters/cf90.F90       init :107, filter1/filter2/filter3 :1020/1090/1160,
 *                                         destroy :177
 *
 * Conventions (the reference's):
 *   - Fields are FP64, column-major f(n1,n2,n3): f[i + n1*(j + n2*k)].
 *   - dd1/d2d1/filter1 act along x on an (n,na,nb) array, dd2/... along y on
 *     (na,n,nb), dd3/... along z on (na,nb,n).
 *   - f is intent(in) and df intent(out); they must not overlap.
 *   - bc1/bcn select the boundary closure of a bounded (non-periodic)
 *     operator: 0 one-sided, 1 symmetric, -1 antisymmetric.  A Fortran caller
 *     that omits the optional arguments passes 0 (the reference's default).
 *     cd06 ignores them (its closures are fixed at init), as do periodic
 *     operators.
 *   - Handles are immutable after init and may be used concurrently from
 *     several host threads and streams -- except through the tuning setters
 *     (pado_set_tiling, pado_set_kernel_variant, pado_set_stream_tiling),
 *     which change the handle and must not overlap other calls on it.
 *
 * Differences from the reference, by design:
 *   - f and df are DEVICE pointers and the work is enqueued on `stream`
 *     (a cudaStream_t, NULL = legacy default stream); the call returns once
 *     enqueued.  pado_apply_host() is the host-buffer variant.
 *   - Errors are returned, never aborted on: a bad bc returns PADO_E_BC
 *     (324, the code the reference passes to GracefulExit), init size errors
 *     return the reference's ierr (2, 3 or 7).
 */
#ifndef PADO_H
#define PADO_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pado_op_s *pado_op_t;

/* schemes */
#define PADO_CD06 0
#define PADO_CD10 1
#define PADO_CF90 2

/* operator kinds */
#define PADO_FILTER 0
#define PADO_D1 1
#define PADO_D2 2

/* status codes (0 and the reference's init ierr values 2, 3, 7 are kept) */
#define PADO_OK 0
#define PADO_E_BC 324          /* bc1/bcn not in {0,1,-1} (cd10.F90:2044-2055)        */
#define PADO_E_NULL (-1)       /* null handle or pointer                               */
#define PADO_E_ALIAS (-2)      /* f and df overlap                                     */
#define PADO_E_UNSUPPORTED (-3)/* operator the reference does not provide (cd06 d2 ...) */
#define PADO_E_ARG (-4)        /* bad axis, kind, scheme, negative size, bad dx        */
#define PADO_E_CUDA (-5)       /* a CUDA runtime call failed                           */
#define PADO_E_SIZE (-6)       /* line longer than the kernels support, or overflow    */
#define PADO_E_TIMEOUT (-7)    /* a bounded device wait expired                        */
#define PADO_E_NOMEM (-8)      /* host or device allocation failed                     */
#define PADO_E_STATE (-9)      /* object used in a state that does not allow the call  */

/* ---- scheme objects ---------------------------------------------------- */

/* cd06%init(n, dx, periodic, bc1, bcn)  -- cd06.F90:129.
 * Returns 0, 3 (periodic, n in 2..5) or 2 (bounded, n in 2..7). */
int pado_cd06_init(pado_op_t *op, int n, double dx, int periodic, int bc1, int bcn);

/* cd10%init(n, dx, periodic, bc1, bcn)  -- cd10.F90:195.  Returns 0 or 2 (n in 2..7). */
int pado_cd10_init(pado_op_t *op, int n, double dx, int periodic, int bc1, int bcn);

/* cf90%init(n, periodic)  -- cf90.F90:107.  Returns 0 or 7 (n in 2..9). */
int pado_cf90_init(pado_op_t *op, int n, int periodic);

/* Generic form of the three inits (scheme = PADO_CD06/CD10/CF90; dx ignored by cf90). */
int pado_create(pado_op_t *op, int scheme, int n, double dx, int periodic, int bc1, int bcn);

/* %destroy  -- cd06.F90:203, cd10.F90:317, cf90.F90:177.  NULL is a no-op. */
void pado_destroy(pado_op_t op);

/* %GetSize  -- cd06.F90:123, cd10.F90:189. */
int pado_get_size(pado_op_t op);

/* ---- operators (device pointers, enqueued on `stream`) ------------------ */

/* cd06%dd1/dd2/dd3 (cd06.F90:775/797/819) and cd10%dd1/dd2/dd3 (cd10.F90:2029/2099/2169). */
int pado_dd1(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_dd2(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_dd3(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);

/* cd10%d2d1/d2d2/d2d3 (cd10.F90:2239/2309/2379). */
int pado_d2d1(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_d2d2(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_d2d3(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);

/* cf90%filter1/filter2/filter3 (cf90.F90:1020/1090/1160, real variant). */
int pado_filter1(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_filter2(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);
int pado_filter3(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn, void *stream);

/* Generic dispatch behind the nine calls above: kind = PADO_D1/D2/FILTER,
 * axis = 1/2/3.  Same semantics as the reference's dd{axis}/d2d{axis}/filter{axis}. */
int pado_apply(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1, int bcn,
               void *stream);

/* Scaled / accumulating form of pado_apply: df = alpha * D f + beta * df,
 * beta 0 or 1 (else PADO_E_ARG).  With beta = 1 a field operator sums its
 * terms straight into its output -- laplacian = d2d1 + d2d2 + d2d3 as three
 * calls (cgrid.F90:480-517), a curl component as a derivative minus another
 * (operators.F90:58-97) -- reading df once per call instead of through a
 * temporary (24 bytes per point instead of 16 + 24).  Same arguments, errors
 * and stream semantics as pado_apply; f and df must not overlap.  No
 * counterpart in the reference (the solver's callers sum derivatives into
 * temporaries). */
int pado_apply_scaled(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                      int bcn, double alpha, double beta, void *stream);

/* Adjoint (transpose) of pado_apply: fbar = D^T g with D = A^{-1} B the
 * operator pado_apply applies, boundary closures included.  No counterpart in
 * the reference; used for reverse-mode differentiation. */
int pado_apply_adjoint(pado_op_t op, int kind, int axis, const double *g, double *fbar, long na, long nb, int bc1,
                       int bcn, void *stream);

/* cf90%filter3 for a complex field -- filter3_CMPLX, cf90.F90:1230-1251.
 * f and df are complex (na,nb,n) arrays: (re, im) pairs of doubles, as the
 * Fortran complex(rkind) type stores them.  As in the reference, the
 * right-hand side takes the closures (bc1, bcn) and the solve always uses the
 * bc (0, 0) system (penta_nn); a Fortran caller passes bc1 = bcn = 0 when it
 * omits bcn_ (the reference reads bc1_ only when bcn_ is present).  A
 * periodic object has no penta_nn system: PADO_E_UNSUPPORTED (the reference
 * indexes an unallocated array there).  n == 1 copies f. */
int pado_filter3_complex(pado_op_t op, const double *f, double *df, long na, long nb, int bc1, int bcn,
                         void *stream);

/* Host-buffer variant of pado_apply for callers whose fields live in host
 * memory (the reference's own calling convention): copies f to the device,
 * applies the operator and copies df back, pipelined in chunks, and returns
 * when df holds the result.  Pinned host memory gives full overlap. */
int pado_apply_host(pado_op_t op, int kind, int axis, const double *f_host, double *df_host, long na, long nb,
                    int bc1, int bcn, void *stream);

/* One term of a host-buffer field operator: output[out] = alpha * D f +
 * beta * output[out], D = op's (kind, axis, bc1, bcn) operator. */
typedef struct {
    pado_op_t op;
    int kind, axis, bc1, bcn;
    double alpha, beta; /* beta 0 or 1; the first term of an output has beta 0 */
    int out;            /* output index; each output's terms are consecutive, outputs in order */
} pado_host_term;

/* Several operators on one host field f(n1,n2,n3), uploading f once: the
 * host-buffer form of gradient (3 outputs, 1 term each), laplacian (1 output,
 * 3 terms summed in the kernels) or any list of terms.  Each output is copied
 * back while the next one is computed; two output fields and f are staged on
 * the device (through terms[0].op's staging buffers and copy streams).
 * Returns when every out_host[k] holds its result.  PADO_E_ARG for terms out
 * of order, a first term with beta != 0 or an op whose n is not the extent
 * along its axis.  No counterpart in the reference, whose solver holds its
 * fields on the host and calls dd* per direction. */
int pado_apply_host_terms(const double *f_host, long n1, long n2, long n3, const pado_host_term *terms, int nterms,
                          double *const *out_host, int nout, void *stream);

/* ---- tuning ------------------------------------------------------------- */

/* Launch shape of the line kernels for this handle: m = segment length
 * (rows one thread solves serially, 8/16/32/64), lines = lines per CTA
 * (8/16/32).  0 keeps the current value.  Rebuilds the handle's tables. */
int pado_set_tiling(pado_op_t op, int m, int lines);
int pado_get_tiling(pado_op_t op, int *m, int *lines);
/* Kernel organisation of the forward operator: 0 = automatic (the
 * streaming kernel: 4 where the copy engine can move the field, else 6;
 * adjoints of fields 4 cannot take run 1; the default),
 * 1 = one CTA per tile of lines, 2 = persistent CTAs that prefetch the next
 * tile with cp.async while the current one is solved, 3 = persistent CTAs
 * that read lines straight into registers and warm L2 with the next tile
 * (strided axes; x lines use 2), 4 = the streaming kernel: persistent CTAs
 * fed by TMA tensor / bulk copies two tiles ahead (needs 16-byte aligned
 * fields, an even x extent for y/z lines and an even n for x lines;
 * PADO_E_UNSUPPORTED otherwise), 5 = the streaming kernel's resident tiles
 * fed by plain loads (any extent and alignment; a tile of 8 lines within
 * 110 KB of shared memory, i.e. n up to about 1300; PADO_E_UNSUPPORTED
 * otherwise), 6 = the streaming kernel fed by per-element asynchronous
 * copies (cp.async, 8 bytes each, landing on the stage's mbarrier): any
 * extent, 8-byte aligned fields, forward operators.  Adjoints follow the
 * same choice (4 runs the transposed sweep in the tile, then B^T); 2, 3, 5
 * and 6 mean 1 for adjoints.
 * No counterpart in the reference (a B200 tuning knob). */
int pado_set_kernel_variant(pado_op_t op, int variant);
/* Tiling of the streaming kernel: lines per tile (8, 16 or 32) and
 * shared-memory stages (1 or 2); 0 leaves the choice to the
 * occupancy-based planner (the default).  A fixed choice that
 * does not fit makes the forward operator fall back to variant 1 (variant 0)
 * or fail with PADO_E_UNSUPPORTED (variant 4).  No counterpart in the
 * reference (a B200 tuning knob). */
int pado_set_stream_tiling(pado_op_t op, int lines, int stages);
/* Device-side status of the handle's kernels: PADO_OK, or PADO_E_TIMEOUT
 * when a streaming kernel's bounded wait for its copies expired (its CTAs
 * then stop early and the output is incomplete).  Synchronous (reads device
 * memory); clear != 0 resets the word.  No counterpart in the reference. */
int pado_device_status(pado_op_t op, int clear);
/* The kernel a forward apply with these arguments would launch (nothing is
 * launched): info[0] kernel variant (1..6), [1] lines per tile, [2] stages,
 * [3] CTAs per SM, [4] segments per line, [5] coupling window, [6] threads
 * per CTA, [7] dynamic shared memory bytes.  No counterpart in the reference. */
int pado_launch_plan(pado_op_t op, int kind, int axis, const double *f, double *df, long na, long nb, int bc1,
                     int bcn, int *info);

/* ---- batched execution (many fields, one persistent launch) ------------ */

typedef struct pado_batch_s *pado_batch_t;

/* One item of a batch: apply `op` (kind, axis, bc1, bcn) to field f of shape
 * (n1,n2,n3) -- the operator's n must equal the extent along `axis` -- writing df. */
typedef struct {
    pado_op_t op;
    int kind, axis, bc1, bcn;
    long n1, n2, n3;
    const double *f;
    double *df;
} pado_batch_item;

/* PADO_E_SIZE when an item's tile of 8 lines does not fit the persistent
 * kernel's 110 KB of shared memory (lines longer than about 1300 points);
 * such fields go through pado_apply. */
int pado_batch_create(pado_batch_t *batch, const pado_batch_item *items, int nitems);
/* Enqueue the whole batch on `stream` as one persistent kernel launch. */
int pado_batch_run(pado_batch_t batch, void *stream);
/* Enqueue the batch as one launch per item (the per-field loop it replaces). */
int pado_batch_run_loop(pado_batch_t batch, void *stream);
/* Capture the batch into a CUDA graph once and replay it on `stream`.  The
 * graph holds the persistent launch of pado_batch_run, or, after
 * pado_batch_set_graph_branches(batch, k) with k > 0, one streaming-kernel
 * launch per item dealt to k concurrent branches (items of different sizes
 * then share the GPU instead of running one after another). */
int pado_batch_run_graph(pado_batch_t batch, void *stream);
/* What pado_batch_run_graph captures: 0 = the persistent launch (default),
 * 1..16 = per-item launches on that many concurrent graph branches.  Drops
 * any captured graph.  Used by the autotuner. */
int pado_batch_set_graph_branches(pado_batch_t batch, int branches);
/* Launch shape of the persistent kernel: lines per tile (8/16/32/64; 0 =
 * enough lines to keep every thread of the CTA busy, 384 / segments per line,
 * within the shared-memory cap) and a cap on resident CTAs per SM (0 = as
 * many as fit).  Used by the autotuner; drops any captured graph. */
int pado_batch_set_config(pado_batch_t batch, int lines, int ctas_per_sm);
/* Tiles, grid size, threads per CTA and dynamic shared memory of the batch. */
int pado_batch_info(pado_batch_t batch, long long *ntiles, int *grid, int *threads, long long *smem_bytes);
/* Device-side status of the batch's last persistent launch: PADO_OK, or
 * PADO_E_TIMEOUT when a CTA's bounded wait for its tile copies expired (that
 * CTA stopped; the outputs are incomplete).  Synchronous.  No counterpart in
 * the reference. */
int pado_batch_status(pado_batch_t batch);
void pado_batch_destroy(pado_batch_t batch);

/* Most items one pado_batch_run_static call accepts. */
#define PADO_STATIC_BATCH_MAX_ITEMS 256
/* Bytes of the library's fixed device scratch array behind pado_batch_run_static. */
#define PADO_STATIC_BATCH_SCRATCH_BYTES (768 * 1024)

/* The batched launch for callers that may not allocate device memory once
 * they are running: a solver that hands all of HBM to its own pool at start-up,
 * or one that builds a different list of fields every time step and may not
 * pay for (or is not allowed) a cudaMalloc/cudaFree per step.  Does what
 * pado_batch_create + pado_batch_run + pado_batch_destroy do, but calls no
 * cudaMalloc or cudaFree: the item descriptors and the tile counter live in
 * a fixed 768 KiB array inside the library (held on every GPU that loads it
 * until the process exits).  The operators' own tables are made by their
 * init, as usual.  The caller passes the inputs and outputs as in
 * pado_batch_item.
 *   - nitems above PADO_STATIC_BATCH_MAX_ITEMS returns PADO_E_SIZE.
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make it before any stream capture.
 *   - All calls on a device share the one array: two calls whose launches
 *     overlap on the GPU race and give wrong results.  Order them on one
 *     stream, or wait for one before starting the next.  Calls made from
 *     several host threads at once are serialized inside the library, so
 *     their copies and launches do not interleave on a shared stream.
 *   - Every item's operator must belong to the current device.
 * No counterpart in the reference. */
int pado_batch_run_static(const pado_batch_item *items, int nitems, void *stream);

/* ---- staggered sixth-order compact scheme (cd06stagg, along z) ---------- */

/* cd06staggstuff (src/derivatives/cd06stagg.F90): first derivatives
 * edge->cell, cell->edge, cell->cell and edge->edge, second derivatives
 * cell->cell and edge->edge, and interpolation edge->cell and cell->edge,
 * along the third index of (n1, n2, nz) column-major fields.  The cell grid
 * has n points, the edge grid n + 1.  Used by the incompressible solver
 * (src/incompressible/PadeDerOps.F90). */
typedef struct pado_stagg_s *pado_stagg_t;

/* Operators, the reference's procedure names in order
 * (ddz_E2C .. InterpZ_C2E, cd06stagg.F90:820-1060). */
#define PADO_STAGG_DDZ_E2C 0
#define PADO_STAGG_DDZ_C2E 1
#define PADO_STAGG_DDZ_C2C 2
#define PADO_STAGG_DDZ_E2E 3
#define PADO_STAGG_D2DZ2_C2C 4
#define PADO_STAGG_D2DZ2_E2E 5
#define PADO_STAGG_INTERPZ_E2C 6
#define PADO_STAGG_INTERPZ_C2E 7
#define PADO_STAGG_NOPS 8
/* nx <= 4: the reference stops with GracefulExit(..., 21) (cd06stagg.F90:183-185). */
#define PADO_STAGG_E_SHORT 21

/* cd06stagg%init_periodic(nx, dx) (cd06stagg.F90:170-195). */
int pado_cd06stagg_init_periodic(pado_stagg_t *stagg, int nx, double dx);
/* cd06stagg%init_nonperiodic(nx, dx, isTopEven, isBotEven, isTopSided,
 * isBotSided) (cd06stagg.F90:197-232); the sided flags are 0 when the
 * reference's optional arguments are absent. */
int pado_cd06stagg_init_nonperiodic(pado_stagg_t *stagg, int nx, double dx, int is_top_even, int is_bot_even,
                                    int is_top_sided, int is_bot_sided);
/* Planes along z read (nin) and written (nout) by operator `op`: n or n + 1.
 * PADO_E_UNSUPPORTED for the C2C / E2E first derivatives of a periodic
 * object (the reference solves them with tables its periodic init never
 * allocates). */
int pado_cd06stagg_sizes(pado_stagg_t stagg, int op, int *nin, int *nout);
/* df(n1, n2, nout) = op applied along z to f(n1, n2, nin): device pointers,
 * enqueued on `stream`; f and df must not overlap.  A complex field is
 * passed as its (re, im) doubles with n1 doubled (the coefficients are
 * real). */
int pado_cd06stagg_apply(pado_stagg_t stagg, int op, const double *f, double *df, long n1, long n2, void *stream);
/* cd06stagg%destroy (cd06stagg.F90:234-243). */
void pado_cd06stagg_destroy(pado_stagg_t stagg);

/* ---- diagnostics -------------------------------------------------------- */

const char *pado_strerror(int status);
/* Number of kernel launches this process has enqueued through the library. */
long long pado_launch_count(void);
/* Library version string. */
const char *pado_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PADO_H */

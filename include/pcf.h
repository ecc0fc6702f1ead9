/*
 * pcf.h -- C ABI of libpcf.so: grid-node pair and triplet counting on one
 * NVIDIA B200 (sm_100a).
 *
 * Every entry point returns a pcf_status (0 on success, a negative code
 * otherwise) and never exits the process; buffers passed in are owned by the
 * caller; grids are owned by the context that built them and must be freed
 * with pcf_grid_free.  One context per host thread; a context serialises its
 * work on one CUDA stream of its own.
 *
 * Reference interfaces replaced (3PCFGPU, paths relative to its root):
 *   pcf_grid_build      open_files/make_nodos + the flattening and H2D copy
 *                       of cuda/create_grid.cuh:35,104 and cuda/main.cu:219-329
 *   pcf_count_pairs     pcf_2iso (cuda/pcf2iso.cuh:11), pcf_2ani
 *                       (cuda/pcf2ani.cuh:5), pcf_2iso_BPC
 *                       (cuda/pcf2isoBPC.cuh:11), pcf_2aniBPC
 *                       (cuda/pcf2aniBPC.cuh:5) -- one histogram per call
 *   pcf_count_triplets  pcf_3iso (cuda/pcf3iso.cuh:10), pcf_3isoBPC
 *                       (cuda/pcf3isoBPC.cuh:10), pcf_3ani
 *                       (cuda/pcf3ani.cuh:10), pcf_3aniBPC
 *                       (cuda/pcf3aniBPC.cuh:10)
 *   pcf_analytic_rr     RR2iso_BPC_analytic path of pcf_2iso_BPCanalytic
 *                       (cuda/pcf2isoBPC.cuh:166)
 *   pcf_analytic_3iso   pcf_3isoBPC_analytic (cuda/pcf3isoBPC.cuh:177)
 *   pcf_batch_pairs     the -rd random-directory loop of pcf_2iso / pcf_2ani
 *                       (cuda/pcf2iso.cuh:96-104, cuda/main.cu:157-192)
 * The legacy C++ signatures themselves are declared in pcf_legacy.h.
 */
#ifndef PCF_H
#define PCF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One catalog point: coordinates and weight, laid out exactly like the
 * reference's PointW3D (cuda/create_grid.cuh:15-20). */
typedef struct pcf_point {
    float x, y, z, w;
} pcf_point;

typedef struct pcf_ctx pcf_ctx;
typedef struct pcf_grid pcf_grid;

typedef enum pcf_status {
    PCF_OK = 0,
    PCF_ERR_INVALID_ARG = -1,  /* a NULL pointer, n < 1, bins < 1, dmax <= 0 ...     */
    PCF_ERR_CUDA = -2,         /* a CUDA runtime call failed (see pcf_last_error)    */
    PCF_ERR_NO_MEMORY = -3,    /* device or host allocation failed                   */
    PCF_ERR_UNSUPPORTED = -4,  /* e.g. periodic boundaries with dmax >= box/2        */
    PCF_ERR_OUT_OF_BOX = -5,   /* a coordinate outside [0, box)                      */
    PCF_ERR_TIMEOUT = -6,      /* a persistent kernel gave up its work queue: abort
                                  requested (pcf_ctx_abort) or iteration cap reached */
    PCF_ERR_IO = -7,           /* catalog / histogram file error                     */
    PCF_ERR_MISMATCH = -8      /* grids of different box or partitions               */
} pcf_status;

/* Histogram kinds.  PCF_BOTH (pair counts only): the isotropic and the
 * anisotropic histogram in one call, written as bins doubles (isotropic)
 * followed by bins*bins doubles (anisotropic).  The call runs the two
 * single-kind launches, or one pass over the candidate pairs for both kinds
 * where pcf_autotune_pairs found that faster for the call's class. */
enum { PCF_ISO = 0, PCF_ANI = 1, PCF_BOTH = 2 };

/* Flags for the counting calls. */
enum {
    PCF_BPC = 1u << 0,         /* periodic box (minimum image; dmax < box/2)            */
    PCF_DS_EXACT = 1u << 1,    /* bin scale bins/dmax (reference 2iso BPC,
                                  2isoBPC_k.cuh:36) instead of floor(bins/dmax*1e6)/1e6 */
    PCF_RULE_CUSTOM = 1u << 2, /* use the two rule bits below instead of the
                                  reference kernel's rule for the variant              */
    PCF_RULE_EXCL_ZERO = 1u << 3, /* require separation > 0                            */
    PCF_RULE_INCLUSIVE = 1u << 4, /* d^2 <= dmax^2 instead of <                        */
    PCF_DEVICE_OUT = 1u << 5,  /* hist points to device memory; the call returns
                                  without synchronising the context stream           */
    PCF_GRAPH = 1u << 7,       /* pcf_batch_pairs: capture the launch in a CUDA graph the
                                  first time and replay it on later calls with the same
                                  grids and parameters                               */
    PCF_REF_NODE_GATES = 1u << 8 /* periodic triplet counts (PCF_BPC): count each ordered
                                  triangle as many times as the reference's periodic CUDA
                                  kernels do (XXX3iso_BPC / XXY3iso_BPC, 3isoBPC_k.cuh:191,940;
                                  XXX3ani_BPC / XXY3ani_BPC, 3aniBPC_k.cuh:210,959) on their
                                  node grid of box / partitions, partitions being the value
                                  given to pcf_grid_build (nonzero, the same for x and y).
                                  Those kernels gate node triples per periodic image case and
                                  five of their 64 gates differ from the geometry, so they
                                  miss some triangles near box edges and count a few twice;
                                  this flag reproduces that count (PCF.out's 3iso / 3ani
                                  -bpc).  Without it every triangle in range is counted once,
                                  as the reference's CPU engines count it.              */
};

/* Counters a counting call can report (any pointer argument may be NULL). */
typedef struct pcf_stats {
    double pairs;          /* in-range units counted: unordered XX pairs, XY pairs,
                              or unordered triangles                               */
    double candidates;     /* pair (or pair-of-pair) tests executed                 */
    double rechecks;       /* tests re-evaluated in FP64 near a bin edge / dmax      */
    float kernel_ms;       /* device time of the counting kernels                   */
    int partitions;        /* cells per box side used                               */
    int work_items;        /* work items in the persistent queue                    */
} pcf_stats;

const char *pcf_status_string(pcf_status s);
/* Text of the last CUDA error seen by this context (empty if none). */
const char *pcf_last_error(const pcf_ctx *ctx);
int pcf_version(void);

pcf_status pcf_ctx_create(int device, pcf_ctx **out);
pcf_status pcf_ctx_destroy(pcf_ctx *ctx);
/* The CUDA stream (cudaStream_t) the context enqueues on. */
void *pcf_ctx_stream(pcf_ctx *ctx);

/*
 * Failure handling without a device fault.  pcf_ctx_abort(ctx, 1) asks the
 * context's persistent kernels (the pair, triplet and batched work queues)
 * to stop taking work at their next work item; any host thread may call it
 * while another thread's call runs (the request is copied, on a stream of the
 * context's own that runs beside the launch in flight, into a device word
 * that the kernels poll; the call returns when the copy has landed).  While
 * it is set, counting calls return
 * PCF_ERR_TIMEOUT without launching, and a call whose kernels gave up
 * returns PCF_ERR_TIMEOUT once its work is complete (partial histograms are
 * not returned).  Every queue also stops at an iteration cap (more tickets
 * than the queue holds) with the same status.  pcf_ctx_abort(ctx, 0) clears
 * the request and the record of kernels that gave up.
 */
pcf_status pcf_ctx_abort(pcf_ctx *ctx, int on);
/* Waits for the context stream; PCF_ERR_TIMEOUT if a kernel of the context
 * gave up its queue since the last clear (device-output calls report it
 * here, as they return before their kernels finish). */
pcf_status pcf_ctx_synchronize(pcf_ctx *ctx);

/*
 * Grid a catalog.  pts may be host or device memory (n points, 16 bytes
 * each).  Every coordinate must lie in [0, box).  partitions = cells per box
 * side (the reference's -p), or 0 to let the library choose.  Pair and
 * triplet counts use the caller's partitions when periodic stencils allow
 * them (2*ceil(dmax/cell) + 2 <= partitions), otherwise the count the
 * library picks for dmax (or the autotuner's, pcf_tune.h); a grid keeps the
 * cell structures of its last few partition counts.  Results do not depend
 * on the partitions.  The points are copied; the caller keeps pts.
 */
pcf_status pcf_grid_build(pcf_ctx *ctx, const pcf_point *pts, int64_t n, float box,
                          int partitions, pcf_grid **out);
pcf_status pcf_grid_free(pcf_ctx *ctx, pcf_grid *g);
pcf_status pcf_grid_info(const pcf_grid *g, int64_t *n, float *box, int *partitions,
                         int64_t *nonempty_cells, int *unit_weights);
/* Copy the cell-ordered points (n) and the cell table (partitions^3 + 1
 * start offsets, cell id = (ix*P + iy)*P + iz) back to host memory. */
pcf_status pcf_grid_download(pcf_ctx *ctx, const pcf_grid *g, pcf_point *pts_out,
                             int32_t *cell_start_out);

/*
 * One pair histogram.  b == NULL: XX (DD or RR) over a, ordered pairs as the
 * reference counts them (each unordered pair twice).  b != NULL: XY (DR),
 * every (a, b) pair once.  kind PCF_ISO: bins doubles; PCF_ANI: bins*bins
 * doubles indexed [bin(|dz|)][bin(r_perp)]; PCF_BOTH: the two, isotropic
 * first (stats count the pairs of both).  hist is overwritten.  stats
 * may be NULL; when given, the call waits for the result and weighted
 * histograms also count their in-range pairs (a little extra kernel work).
 */
pcf_status pcf_count_pairs(pcf_ctx *ctx, int kind, const pcf_grid *a, const pcf_grid *b,
                           int bins, float dmax, uint32_t flags, double *hist,
                           pcf_stats *stats);

/*
 * One triplet histogram.  y == NULL: XXX (DDD / RRR) over x.  y != NULL: XXY
 * with points 1, 2 from x and point 3 from y (DDR: x=D, y=R; DRR: x=R, y=D).
 * PCF_ISO: bins^3 doubles [b(d12)][b(d23)][b(d31)];  PCF_ANI: bins^5 doubles
 * [b(d12)][b(d31)][b(d23)][b(cos12)][b(cos31)].
 */
pcf_status pcf_count_triplets(pcf_ctx *ctx, int kind, const pcf_grid *x, const pcf_grid *y,
                              int bins, float dmax, uint32_t flags, double *hist,
                              pcf_stats *stats);

/* Analytic periodic RR (and DR, which the reference writes as the same
 * histogram): RR[k] = alpha (3k^2 + 3k + 1), constants as the reference
 * computes them.  n = catalog size.  wrap != 0 keeps the reference's 32-bit
 * evaluation of 3k^2+3k+1 (2isoBPC_k.cuh:564). */
pcf_status pcf_analytic_rr(pcf_ctx *ctx, int bins, int64_t n, float box, float dmax, int wrap,
                           double *rr);

/*
 * Analytic 3iso with periodic boundaries: DDD is counted (pass ddd, or NULL
 * to skip it), DDR/DRR and RRR are derived from the fine DD histograms.
 * ptt and bn_ref are the reference's sub-binnings (100 and 200; 0 selects
 * those).  ddr and rrr: bins^3 doubles each.
 */
pcf_status pcf_analytic_3iso(pcf_ctx *ctx, const pcf_grid *d, int bins, float dmax, int ptt,
                             int bn_ref, int wrap, double *ddd, double *ddr, double *rrr,
                             pcf_stats *stats);

/*
 * One data catalog against n_rand random catalogs of any sizes, all in one
 * persistent launch over a (tile, neighbour rows, catalog) work queue.
 * Writes, per random catalog i: rr[i*nb .. ] and dr[i*nb ..] (nb = bins,
 * bins^2, or bins + bins^2 for PCF_BOTH), and dd (nb) once.  Any of dd / rr
 * / dr may be NULL to skip it.
 */
pcf_status pcf_batch_pairs(pcf_ctx *ctx, int kind, const pcf_grid *d, const pcf_grid *const *r,
                           int n_rand, int bins, float dmax, uint32_t flags, double *dd,
                           double *rr, double *dr, pcf_stats *stats);

/*
 * The 3-point analogue of pcf_batch_pairs: one data catalog against n_rand
 * random catalogs, the isotropic triplet histograms in two persistent
 * launches (DDD and every RRR_i; every DDR_i and DRR_i), each over one
 * (anchor, histogram) work queue.  Writes ddd (bins^3) once
 * and, per random catalog i, rrr / ddr / drr at [i*bins^3 ..]; any of them
 * may be NULL to skip it.  Replaces the per-file loop of pcf_3iso /
 * pcf_3isoBPC over the -rd random directory (cuda/pcf3iso.cuh:101-112).
 */
pcf_status pcf_batch_triplets(pcf_ctx *ctx, const pcf_grid *d, const pcf_grid *const *r,
                              int n_rand, int bins, float dmax, uint32_t flags, double *ddd,
                              double *rrr, double *ddr, double *drr, pcf_stats *stats);

/* Cells per side the library would pick for (n, box, dmax, kind). */
int pcf_autotune_partitions(pcf_ctx *ctx, int64_t n, float box, float dmax, int kind,
                            uint32_t flags);

#ifdef __cplusplus
}
#endif

#endif /* PCF_H */

// pcf_internal.cuh -- shared declarations of libpcf (device helpers + host
// structures).  Not part of the public ABI (include/pcf.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pcf.h"

// ---------------------------------------------------------------------------
// Canonical FP64 rule (bit-for-bit the same arithmetic as the CPU oracle):
//   dx = ((double)xj + shift) - (double)xi       exact
//   d2 = (dx*dx + dy*dy) + dz*dz                  rounded per op, no FMA
//   in range: d2 < dd (or <=), d2 > 0 if the rule excludes zero
//   bin = (int)(sqrt(d2) * ds), dropped when >= bins
// References: cuda/kernels/2iso_k.cuh:45-57, 2ani_k.cuh:46-63,
// 2isoBPC_k.cuh:36 (unfloored ds), 2aniBPC_k.cuh:63 (<=).
// ---------------------------------------------------------------------------
#define PCF_RULE_EXCL 1u
#define PCF_RULE_LE 2u

struct PairRule {
    double ds;       // bin scale
    double dd;       // (double)(float)(dmax*dmax)
    int bins;
    unsigned flags;  // PCF_RULE_EXCL | PCF_RULE_LE
};

__device__ __forceinline__ bool rule_in(double d2, const PairRule &r) {
    if ((r.flags & PCF_RULE_EXCL) && !(d2 > 0.0)) return false;
    return (r.flags & PCF_RULE_LE) ? (d2 <= r.dd) : (d2 < r.dd);
}

__device__ __forceinline__ int rule_bin(double d2, const PairRule &r) {
    double s = __dmul_rn(__dsqrt_rn(d2), r.ds);
    int b = (int)s;
    return (b >= 0 && b < r.bins) ? b : -1;
}

// Exact separation components (candidate minus home, candidate shifted).
__device__ __forceinline__ void exact_sep(float hx, float hy, float hz, float cx, float cy,
                                          float cz, float sx, float sy, float sz, double &dx,
                                          double &dy, double &dz) {
    dx = __dsub_rn(__dadd_rn((double)cx, (double)sx), (double)hx);
    dy = __dsub_rn(__dadd_rn((double)cy, (double)sy), (double)hy);
    dz = __dsub_rn(__dadd_rn((double)cz, (double)sz), (double)hz);
}

__device__ __forceinline__ double exact_d2(double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Histogram slot of one pair under the canonical rule, or -1.
template <bool ANI>
__device__ __forceinline__ int exact_slot(double dx, double dy, double dz, const PairRule &r) {
    if (!ANI) {
        double d2 = exact_d2(dx, dy, dz);
        if (!rule_in(d2, r)) return -1;
        return rule_bin(d2, r);
    }
    double zz = __dmul_rn(dz, dz);
    double pp = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    if (!rule_in(zz, r) || !rule_in(pp, r)) return -1;
    int bz = rule_bin(zz, r), bp = rule_bin(pp, r);
    if (bz < 0 || bp < 0) return -1;
    return bz * r.bins + bp;
}

// Queue control.  The abort request is a word in device memory (the host
// sets it by a copy on a stream of its own, which runs beside the kernels),
// read by the persistent kernels at every work ticket through L2; the
// record of a kernel giving up is written, rarely, to mapped host memory.
__device__ __forceinline__ unsigned ctrl_load(const unsigned *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void ctrl_store(unsigned *p, unsigned v) {
    asm volatile("st.relaxed.sys.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
// Status bits a kernel records when it gives up its queue.
#define PCF_GAVE_UP_ABORT 1u
#define PCF_GAVE_UP_CAP 2u

// ---------------------------------------------------------------------------
// Device-side layout.
// ---------------------------------------------------------------------------

// A home tile: a run of cells [z0, z1] of one (ix, iy) column (or a slice of
// one heavy cell), points [start, start+count).
struct TileDesc {
    int start;
    int count;
    int16_t ix, iy, z0, z1;
};

// A neighbour row of the stencil: candidate cells (ix+dx, iy+dy, z0-kz ..
// z1+kz).  kind 1 = the forward half of the home column (XX only): points
// after the tile up to z1+kz.
struct RowDesc {
    int16_t dx, dy, kz, kind;
};

// Device view of a gridded catalog: cell-ordered coordinate planes and the
// cell table (P^3 + 1 starts).
struct GridView {
    const float *x, *y, *z, *w;
    const int *cstart;
};

// The pair kernel's view of a gridded catalog.  Points are pair-packed: the
// cell-ordered points 2k and 2k+1 form one 32-byte block of two float4,
//   pk[2k] = (x_2k, x_2k+1, y_2k, y_2k+1),  pk[2k+1] = (z_2k, z_2k+1, w_2k, w_2k+1),
// so two candidates arrive in two 16-byte loads already laid out for the
// packed f32x2 arithmetic.  qw holds the exact integer weights
// q = w * 2^wshift of a grid whose weights allow it (null otherwise).
struct PairView {
    const float4 *pk;
    const unsigned *qw;
    const int *cstart;
};

// ---------------------------------------------------------------------------
// Host-side objects.
// ---------------------------------------------------------------------------
// Stream-ordered caching allocator of one context: blocks released by a
// grid are reused by later allocations on the same stream, so building and
// freeing grids per request costs no cudaMalloc / cudaFree (each of which
// synchronises the device).
struct MemPool {
    std::multimap<size_t, void *> free_blocks;
    size_t cached = 0;
    cudaError_t get(size_t n, void **p, size_t *got);
    void put(void *p, size_t n);
    void release();
    ~MemPool() { release(); }
};

// Every cudaMalloc / cudaMallocHost of the library goes through these, so
// pcf_alloc_counters can report how many there were and how long they took.
cudaError_t counted_malloc(void **p, size_t n);
cudaError_t counted_malloc_host(void **p, size_t n);

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    std::shared_ptr<MemPool> pool;  // null: plain cudaMalloc / cudaFree
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf();
    cudaError_t ensure(size_t n);  // grow (contents not kept)
    template <class T> T *as() const { return static_cast<T *>(p); }
};

constexpr int kTileCap = 32;  // home points per warp item

// Page-locked host blocks for the grid builds' staging (the cell table read
// back, the tile table sent), reused by size; shared by a context and its
// cell structures, so a structure that outlives its context still returns
// its block.
struct PinnedPool {
    std::mutex mu;
    std::multimap<size_t, void *> free_blocks;
    cudaError_t get(size_t n, void **p, size_t *got);
    void put(void *p, size_t n);
    ~PinnedPool();
};

struct CellGrid {
    int P = 0;
    // a build whose cell table is still on its way to the host (deferred
    // builds): `ready` follows its copy into `stage`; grid_finish completes
    // it.  `stage` (from `pinned`) then feeds the tile table's copy and is
    // returned once `ready`, recorded after that copy, has passed.
    bool pending = false;
    cudaEvent_t ready = nullptr;
    void *stage = nullptr;
    size_t stage_bytes = 0;
    std::shared_ptr<PinnedPool> pinned;
    ~CellGrid();
    uint64_t serial = 0;          // unique per build (keys captured graphs)
    float cell = 0.f;             // box / P
    DevBuf soa;                   // x | y | z | w planes, n + kSoaPad floats each
    size_t plane = 0;             // floats per plane
    DevBuf pk;                    // pair-packed blocks (PairView), pk_blocks(n) x 32 B
    DevBuf qw;                    // exact integer weights (u32 x (n + kSoaPad)), when wfix_ok
    DevBuf cell_start;            // int x (P^3 + 1)
    std::vector<int> h_start;     // host copy of cell_start
    std::vector<TileDesc> tiles;  // home tiles: <= 32 points of one column, <= 2 cells
    DevBuf d_tiles;
    // the same with at most 16 points per tile (an autotuner candidate),
    // built on first use
    std::vector<TileDesc> tiles_half;
    DevBuf d_tiles_half;
    bool have_half = false;
    // largest stencil population of a cell per (dmax, periodic), memoised
    // for the triplet launches (a host pass over every cell and row)
    mutable std::vector<std::pair<std::pair<float, bool>, int64_t>> stencil_memo;
    const std::vector<TileDesc> &tiles_for(int cap) const { return cap == 16 ? tiles_half : tiles; }
    const TileDesc *d_tiles_for(int cap) const {
        return (cap == 16 ? d_tiles_half : d_tiles).as<TileDesc>();
    }
    const float *x() const { return soa.as<float>(); }
    const float *y() const { return soa.as<float>() + plane; }
    const float *z() const { return soa.as<float>() + 2 * plane; }
    const float *w() const { return soa.as<float>() + 3 * plane; }
};
// SoA planes are padded so that a float2 load at the last even index stays
// inside the allocation, and each plane starts 16-byte aligned.
constexpr int kSoaPad = 4;
// Pair-packed blocks of a catalog of n points (one spare block past the end).
inline size_t pk_blocks(int64_t n) { return (size_t)(n / 2) + 2; }

struct pcf_grid {
    std::shared_ptr<MemPool> pool;
    int64_t n = 0;
    float box = 0.f;
    bool unit_weights = true;
    // weight range, for the fixed-point weighted histograms: max |w|, the
    // smallest nonzero |w| (0 if every weight is 0), and whether every
    // weight is finite and >= 0
    float w_absmax = 1.f, w_absmin = 1.f;
    bool w_finite_nonneg = true;
    // exact integer weights q = w * 2^wshift (q < 2^32) exist when every
    // weight is finite, >= 0, and the nonzero ones are normal floats within
    // 8 binades of each other; wqmax = the largest q
    bool wfix_ok = false;
    int wshift = 0;
    unsigned long long wqmax = 0;
    DevBuf raw;                   // float4 x n, input order
    int user_P = 0;               // partitions fixed by the caller at build (0: automatic)
    // cell structures are shared: a captured batch graph keeps the ones it reads alive
    std::shared_ptr<CellGrid> cells;                    // the current cell structure
    std::vector<std::shared_ptr<CellGrid>> cell_cache;  // earlier ones, most recent last
    pcf_ctx *owner = nullptr;       // the context that built it (finishes a deferred build)
    pcf_status bad = PCF_OK;        // set when a deferred build found the catalog invalid
};
constexpr int kCellCache = 2;  // cell structures kept besides the current one

// One of two plan staging slots: while the device runs the kernel of one
// call, the host builds and stages the plan of the next into the other.
struct PlanSlot {
    void *h_pinned = nullptr;
    size_t h_bytes = 0;
    DevBuf d_rows, d_counter;
    cudaEvent_t done = nullptr;  // recorded after the kernel that read this slot
    bool used = false;
};

// Autotuned launch shape of one class of pair histograms.
struct TuneEntry {
    int refine = 0;      // cells per dmax (0: default rule)
    int hist_mode = -1;  // histogram privatisation (-1: default rule)
    float ms = 0.f;      // best kernel time seen while tuning
    int tile = 0;        // home points per tile: 0 or 32 (kTileCap), or 16
    int chunk = 0;       // work items per ticket at most: 0 (the launch rule's 8), 1 or 4
};

// The page-locked staging pool shared by every context of the process: its
// blocks go back only once their copies are done (CellGrid's `ready`), so any
// context may reuse them, and a stream of requests over several contexts
// reaches a steady set of blocks instead of one per context.
std::shared_ptr<PinnedPool> shared_pinned_pool();

struct pcf_ctx {
    std::shared_ptr<MemPool> pool = std::make_shared<MemPool>();
    // the context's own buffers (scratch, histograms, plan slots): reused
    // only by this context's stream, so a block returned while the
    // context's kernels still read it is taken again only after them
    std::shared_ptr<MemPool> scratch_pool = std::make_shared<MemPool>();
    std::map<std::string, TuneEntry> tune;
    TuneEntry tune_override;  // set while the autotuner times a candidate
    bool tune_timing = false; // autotuner: statistics carry kernel time only (no pair
                              // counting), so candidates run the kernels a plain call runs
    PlanSlot slots[2];
    int slot = 0;
    // optional kernel-time log (pcf_ctx_profile)
    bool profile = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    size_t prof_used = 0;
    // the same for grid builds (counting sort + scatter kernels)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_grid_events;
    size_t prof_grid_used = 0;
    int64_t prof_grid_points = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sm_count = 148;
    std::string last_error;
    // scratch reused across calls
    DevBuf scratch_a, scratch_b, scratch_c, d_hist;
    DevBuf d_flag;
    void *h_pinned = nullptr;
    size_t h_pinned_bytes = 0;
    int64_t launches = 0;  // kernels launched by this context
    // Queue control.  d_abort: the abort request in device memory, polled by
    // the persistent kernels at every work item and set by pcf_ctx_abort
    // through ctrl_stream (any host thread).  h_ctrl, mapped page-locked host
    // memory: [0] the host's copy of the request, [1] the record of a kernel
    // that gave up its queue (bit 0: abort request, bit 1: iteration cap),
    // written by the kernel through d_status; [2] = 0 and [3] = 1, the
    // sources of the request copies.
    unsigned *d_abort = nullptr;
    unsigned *h_ctrl = nullptr;
    unsigned *d_status = nullptr;
    cudaStream_t ctrl_stream = nullptr;
    bool abort_host_check = true;  // refuse calls while the request is set
    // adds a triplet kernel's shared u32 histogram absorbs between flushes
    unsigned long long trip_flush_budget = 1ull << 31;
    int pair_variant = 0;  // PCF_OPT_PAIR_VARIANT
    int grid_build = 0;    // PCF_OPT_GRID_BUILD: 0 by size, 1 per-point, 2 bucketed
    bool grid_defer = false;  // PCF_OPT_GRID_DEFER: pcf_grid_build returns once queued
    std::shared_ptr<PinnedPool> pinned = shared_pinned_pool();
    std::map<std::string, std::shared_ptr<struct BatchGraph>> graphs;  // pcf_batch_pairs(PCF_GRAPH)
};

// ---------------------------------------------------------------------------
// Internal host API (implemented in grid.cu / pairs.cu / triplets.cu ...).
// ---------------------------------------------------------------------------
pcf_status pcf_fail(pcf_ctx *ctx, cudaError_t e, const char *what);
// Raises kernel `fn`'s dynamic shared-memory limit on `device` to at least
// `bytes`.  Thread-safe (the request server drives one library from several
// host threads) and monotone: the limit is never lowered, so a launch that
// fits the limit one thread set stays valid while another thread raises it.
cudaError_t ensure_smem_limit(const void *fn, int device, size_t bytes);
#define PCF_CU(ctx, call)                                   \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return pcf_fail(ctx, _e, #call); \
    } while (0)

// defer: return once the build is queued (its cell table read back
// asynchronously); grid_finish then completes it (host cell table, catalog
// checks, tile table).  Every use of a grid's host-side fields goes through
// grid_finish first; it is a no-op for a finished grid.
pcf_status grid_ensure_cells(pcf_ctx *ctx, pcf_grid *g, int P, bool defer = false);
pcf_status grid_finish(pcf_ctx *ctx, const pcf_grid *g);
int choose_partitions(int64_t n, float box, float dmax, int kind, bool bpc, int npoint_kind);

// Stencil of one pair launch (host).  Work items are implicit: item i is
// (tile i / n_chunks, rows [c*rows_per_item, ...) of chunk c = i % n_chunks).
struct PairPlan {
    int P;
    float cell;
    std::vector<RowDesc> rows;
    int rows_per_item = 1;
    int n_chunks = 1;
    int64_t n_items = 0;
};

// Home tiles of a gridded catalog: runs of at most `cap` (<= kTileCap)
// consecutive points of one column within two adjacent cells (pairs.cu).
void build_tiles(const CellGrid &g, int cap, std::vector<TileDesc> &out);
// The 16-point tile table of a cell structure, built and uploaded on first use.
pcf_status ensure_half_tiles(pcf_ctx *ctx, CellGrid &g);
// Stencil rows (dx, dy, kz) of cells that can hold a pair within dmax.
void plan_rows(int P, float box, float dmax, bool ani, bool self, std::vector<RowDesc> &rows);
// Builds the stencil and item shape of one pair launch.  self: XX half shell.
void plan_pairs(const CellGrid &home, float box, float dmax, bool ani, bool self, PairPlan &plan,
                int resident_warps, int tile_cap = kTileCap);

pcf_status pcf_ensure_pinned(pcf_ctx *ctx, size_t bytes);
// PCF_ERR_TIMEOUT if an abort is requested (before a call launches) or if a
// kernel gave up its queue (after the call's work is complete), else PCF_OK.
pcf_status ctx_abort_requested(pcf_ctx *ctx);
pcf_status ctx_queue_status(pcf_ctx *ctx);

// One pair-kernel launch (pairs.cu).
struct PairLaunch {
    bool ani, weighted, bpc, self;
    bool both = false;   // isotropic and anisotropic histograms in one pass (ani set too);
                         // a job slot then holds bins + bins^2 accumulators, iso first
    unsigned flags2 = 0; // both: the anisotropic rule's flags (rule.flags: isotropic)
    PairRule rule;
    double mult;         // 2 for XX (ordered-pair convention), 1 for XY
    int hist_mode = -1;  // 0 lane-private, 1 per-warp shared, 2 global, 3 per-warp
                         // fixed-point (weighted), 4 lane-private fixed-point
                         // (weighted iso); -1 automatic
    bool wfix = false;   // exact integer weight products available (set_weight_fix)
    int wbudget = 0;     // limb adds between flushes of a fixed-point copy
    double wunscale = 0.0;  // single-job launches: weight_unscale(home, cand)
    bool count = true;   // weighted launches: count in-range pairs (statistics)
    // queue control (pcf_ctx_abort): the abort word the kernel polls at every
    // ticket and the status word it sets when it gives up; null: no polling
    const unsigned *ctrl = nullptr;
    unsigned *status = nullptr;
    int variant = 0;     // one-pass kernel variant (PCF_OPT_PAIR_VARIANT; pairs.cu)
    int tile_cap = kTileCap;  // home points per tile (32, or 16 when tuned so)
    int chunk_cap = 0;        // work items per ticket at most (0: the launch rule's 8)
};
// Enables the fixed-point weighted histograms when every grid of the launch
// has exact integer weights and any product fits the three-limb budget.
void set_weight_fix(PairLaunch &pl, const pcf_grid *const *gs, int n);
// 2^-(wshift_home + wshift_cand): converts a fixed-point sum back to w*w units.
double weight_unscale(const pcf_grid *home, const pcf_grid *cand);
std::string tune_key(int kind, bool bpc, bool cross, bool weighted, int bins, int64_t n, float box,
                     float dmax);
pcf_status launch_pairs(pcf_ctx *ctx, const PairPlan &plan, const CellGrid &home,
                        const CellGrid &cand, float box, const PairLaunch &pl,
                        unsigned long long *d_count, double *d_wsum, unsigned long long *d_stats);
pcf_status finalize_hist(pcf_ctx *ctx, const unsigned long long *d_count, const double *d_wsum,
                         bool weighted, double mult, int nb, double *d_out);
// One histogram of a pair launch: home / candidate catalogs, stencil rows,
// and the implicit items [item_begin, item_begin + n_tiles * n_chunks).
struct PairJob {
    PairView home, cand;
    const TileDesc *tiles;
    const RowDesc *rows;
    int n_rows, rows_per_item, n_chunks, slot;
    long long item_begin;
    unsigned rule_flags;  // exact-rule flags of this histogram (XX and XY differ)
    int P;                // cells per side of both grids of this job
    unsigned rule_flags2; // both-kinds launches: the anisotropic histogram's flags
    int pad;
    double wunscale;      // fixed-point launches: weight_unscale(home, cand)
};
PairView pair_view(const CellGrid &g, bool with_q);
void shape_job(PairJob &j, int64_t n_tiles, int n_rows, int64_t total_tile_rows, int sm_count);
// The pair kernel over a device job table (jobs ordered by item_begin);
// counter and the n_jobs * nb accumulators zeroed by the caller.
cudaError_t launch_pair_jobs(const PairJob *d_jobs, int n_jobs, long long n_items, int P, float box,
                             const PairLaunch &pl, unsigned long long *counter,
                             unsigned long long *d_count, double *d_wsum,
                             unsigned long long *d_stats, cudaStream_t st, int sm_count, int device);
// Single-job form on explicit buffers (no context); d_job: device room for
// one PairJob.
cudaError_t launch_pairs_view(const PairView &home, const PairView &cand, const TileDesc *tiles,
                              int64_t n_tiles, const RowDesc *rows, int n_rows, int P, float box,
                              const PairLaunch &pl, unsigned long long *counter,
                              unsigned long long *d_count, double *d_wsum,
                              unsigned long long *d_stats, PairJob *d_job, cudaStream_t st,
                              int sm_count, int device);
cudaError_t launch_finalize(const unsigned long long *d_count, const double *d_wsum, bool weighted,
                            double mult, int nb, double *d_out, cudaStream_t st);
cudaError_t launch_finalize_slots(const unsigned long long *d_count, const double *d_wsum,
                                  bool weighted, const double *d_mult, int nb, int nslots,
                                  double *d_out, cudaStream_t st);
unsigned reference_pair_rule(bool ani, bool bpc, bool cross);
// Counting sort of n points into P^3 cells on explicit buffers; returns the
// number of kernels launched (counts must be zeroed, P^3 + 1 entries).
// soa and qw may be null; pk (pk_blocks(n) blocks, zeroed by the caller) is
// always written, qw only when the weights allow exact integers.  cid, rank
// and perm: n ints of scratch each.
int launch_grid_build(const float4 *raw, int64_t n, int P, float cell, float box, int *cid,
                      int *rank, int *perm, int *counts, int *cell_start, int *scan_tmp, float *soa,
                      size_t plane, float4 *pk, unsigned *qw, int *flags, cudaStream_t st);
// Bucketed counting sort (the build for catalogs of 6M to ~134M points, or
// any size when forced): Q cells per bucket, K buckets; false when the
// catalog needs more buckets than the shared arrays hold (the per-point
// build above then runs).
constexpr int64_t kBucketBuildMin = (int64_t)6 << 20;
bool grid_bucket_plan(int64_t n, int P, int *Q, int *K);
// ints of each of the two CTA x bucket matrices (G CTAs)
size_t grid_bucket_scratch_ints(int G, int K);
cudaError_t grid_bucket_attrs(int device, int K);
// M, Mx: grid_bucket_scratch_ints each; S: n float4 of scratch; flags zeroed.
int launch_grid_build_buckets(const float4 *raw, int64_t n, int P, float cell, float box, int G, int Q,
                              int K, int *M, int *Mx, int *scan_tmp, float4 *S, int *cell_start,
                              float *soa, size_t plane, float4 *pk, unsigned *qw, int *flags,
                              int device, cudaStream_t st);
// Zeroes the padding past point n of the SoA planes, integer weights and pair
// blocks (the builds write entries 0 .. n-1); runs before the build.
int launch_grid_tails(float *soa, size_t plane, int64_t n, float4 *pk, unsigned *qw, cudaStream_t st);
// Host side of the weight scan (flags[0..2] as written by the grid build):
// fills g's weight-range fields, including the integer-weight scale.
void set_weight_range(pcf_grid *g, const unsigned flags[3]);
// Tile table on the device: per cell ceil(count / kTileCap) tiles; tile
// offsets (P^3 + 1) give the total in offsets[P^3].
int launch_tile_build(const int *cell_start, int P, int *tile_counts, int *tile_offsets,
                      int *scan_tmp, TileDesc *tiles, cudaStream_t st);
PairRule make_pair_rule(int bins, float dmax, uint32_t flags, bool ani, bool bpc, bool cross);
pcf_status stage_plan(pcf_ctx *ctx, const PairPlan &plan, PlanSlot **out);
// XX iso pair histogram with an explicit bin scale (analytic path).
pcf_status pcf_count_pairs_ds(pcf_ctx *ctx, const pcf_grid *a, int bins, float dmax, double ds,
                              uint32_t flags, double *hist, pcf_stats *stats);
pcf_status pcf_count_triplets_ani(pcf_ctx *ctx, const pcf_grid *x, const pcf_grid *y, int bins,
                                  float dmax, uint32_t flags, double *hist, pcf_stats *stats);
pcf_status profile_events(pcf_ctx *ctx, cudaEvent_t *a, cudaEvent_t *b);
pcf_status prepare_grids(pcf_ctx *ctx, pcf_grid *a, pcf_grid *b, float dmax, int kind, bool bpc,
                         int *P_out, int refine = 0);

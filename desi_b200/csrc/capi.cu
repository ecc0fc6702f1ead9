// capi.cu -- the extern "C" surface of libpcf.so (include/pcf.h): contexts,
// grids and the pair-histogram entry point.  Triplet / analytic / batched
// entry points live in their own files.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "pcf_internal.cuh"
#include "../../include/pcf_bench.h"


extern "C" {

int pcf_version(void) { return 1; }

const char *pcf_status_string(pcf_status s) {
    switch (s) {
    case PCF_OK: return "ok";
    case PCF_ERR_INVALID_ARG: return "invalid argument";
    case PCF_ERR_CUDA: return "CUDA error";
    case PCF_ERR_NO_MEMORY: return "out of memory";
    case PCF_ERR_UNSUPPORTED: return "unsupported configuration";
    case PCF_ERR_OUT_OF_BOX: return "coordinate outside [0, box)";
    case PCF_ERR_TIMEOUT: return "device wait timed out";
    case PCF_ERR_IO: return "I/O error";
    case PCF_ERR_MISMATCH: return "grids do not share box / partitions";
    }
    return "unknown status";
}

const char *pcf_last_error(const pcf_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

pcf_status pcf_ctx_create(int device, pcf_ctx **out) {
    if (!out) return PCF_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PCF_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return PCF_ERR_INVALID_ARG;
    pcf_ctx *c = new pcf_ctx;
    c->device = device;
    for (DevBuf *b : {&c->scratch_a, &c->scratch_b, &c->scratch_c, &c->d_hist, &c->d_flag})
        b->pool = c->scratch_pool;
    for (PlanSlot &sl : c->slots) sl.d_rows.pool = sl.d_counter.pool = c->scratch_pool;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return PCF_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    void *ctrl = nullptr;
    void *dstatus = nullptr;
    if (cudaHostAlloc(&ctrl, 64, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess ||
        cudaHostGetDevicePointer(&dstatus, ctrl, 0) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void **>(&c->d_abort), 256) != cudaSuccess ||
        cudaMemset(c->d_abort, 0, 256) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->ctrl_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        if (ctrl) cudaFreeHost(ctrl);
        pcf_ctx_destroy(c);
        return PCF_ERR_NO_MEMORY;
    }
    c->h_ctrl = static_cast<unsigned *>(ctrl);
    memset(ctrl, 0, 64);
    c->h_ctrl[3] = 1u;
    c->d_status = static_cast<unsigned *>(dstatus) + 1;
    if (pcf_ensure_pinned(c, (size_t)2 << 20) != PCF_OK) {  // result staging (grows on demand)
        pcf_ctx_destroy(c);
        return PCF_ERR_NO_MEMORY;
    }
    *out = c;
    return PCF_OK;
}

pcf_status pcf_ctx_destroy(pcf_ctx *ctx) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->pool->release();
    ctx->scratch_pool->release();
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->h_ctrl) cudaFreeHost(ctx->h_ctrl);
    if (ctx->d_abort) cudaFree(ctx->d_abort);
    if (ctx->ctrl_stream) cudaStreamDestroy(ctx->ctrl_stream);
    for (auto &sl : ctx->slots) {
        if (sl.h_pinned) cudaFreeHost(sl.h_pinned);
        if (sl.done) cudaEventDestroy(sl.done);
    }
    for (auto &e : ctx->prof_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    for (auto &e : ctx->prof_grid_events) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PCF_OK;
}

void *pcf_ctx_stream(pcf_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

pcf_status pcf_ctx_abort(pcf_ctx *ctx, int on) {
    if (!ctx || !ctx->h_ctrl || !ctx->d_abort) return PCF_ERR_INVALID_ARG;
    volatile unsigned *w = ctx->h_ctrl;
    w[0] = on ? 1u : 0u;
    // the request reaches the device by a copy on the control stream, which
    // runs beside a launch in flight on the context stream
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaMemcpyAsync(ctx->d_abort, ctx->h_ctrl + (on ? 3 : 2), sizeof(unsigned),
                                    cudaMemcpyHostToDevice, ctx->ctrl_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->ctrl_stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return PCF_ERR_CUDA;
    }
    if (!on) w[1] = 0u;
    return PCF_OK;
}

pcf_status pcf_ctx_synchronize(pcf_ctx *ctx) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return ctx_queue_status(ctx);
}

pcf_status pcf_ctx_set_option(pcf_ctx *ctx, int option, int64_t value) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    switch (option) {
    case PCF_OPT_TRIP_FLUSH_BUDGET:
        if (value < 1 || value > ((int64_t)1 << 31)) return PCF_ERR_INVALID_ARG;
        ctx->trip_flush_budget = (unsigned long long)value;
        return PCF_OK;
    case PCF_OPT_ABORT_HOST_CHECK:
        ctx->abort_host_check = value != 0;
        return PCF_OK;
    case PCF_OPT_PAIR_VARIANT:
        if (value < 0 || value > 3) return PCF_ERR_INVALID_ARG;
        ctx->pair_variant = (int)value;
        return PCF_OK;
    case PCF_OPT_GRID_BUILD:
        if (value < 0 || value > 2) return PCF_ERR_INVALID_ARG;
        ctx->grid_build = (int)value;
        return PCF_OK;
    case PCF_OPT_GRID_DEFER:
        ctx->grid_defer = value != 0;
        return PCF_OK;
    }
    return PCF_ERR_INVALID_ARG;
}

int64_t pcf_ctx_launch_count(const pcf_ctx *ctx) { return ctx ? ctx->launches : 0; }

pcf_status pcf_ctx_profile(pcf_ctx *ctx, int enable) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    ctx->profile = enable != 0;
    ctx->prof_used = 0;
    ctx->prof_grid_used = 0;
    ctx->prof_grid_points = 0;
    return PCF_OK;
}

pcf_status pcf_ctx_profile_read_grid(pcf_ctx *ctx, double *total_ms, int64_t *builds, int64_t *points) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    double tot = 0;
    for (size_t i = 0; i < ctx->prof_grid_used; ++i) {
        float ms = 0.f;
        PCF_CU(ctx, cudaEventElapsedTime(&ms, ctx->prof_grid_events[i].first,
                                         ctx->prof_grid_events[i].second));
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (builds) *builds = (int64_t)ctx->prof_grid_used;
    if (points) *points = ctx->prof_grid_points;
    ctx->prof_grid_used = 0;
    ctx->prof_grid_points = 0;
    return PCF_OK;
}

pcf_status pcf_ctx_profile_read(pcf_ctx *ctx, double *total_ms, int64_t *n) {
    if (!ctx) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    double tot = 0;
    for (size_t i = 0; i < ctx->prof_used; ++i) {
        float ms = 0.f;
        PCF_CU(ctx, cudaEventElapsedTime(&ms, ctx->prof_events[i].first, ctx->prof_events[i].second));
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (n) *n = (int64_t)ctx->prof_used;
    ctx->prof_used = 0;
    return PCF_OK;
}

}  // extern "C"

pcf_status ctx_abort_requested(pcf_ctx *ctx) {
    const volatile unsigned *w = ctx->h_ctrl;
    if (ctx->abort_host_check && w && w[0]) {
        ctx->last_error = "abort requested (pcf_ctx_abort)";
        return PCF_ERR_TIMEOUT;
    }
    return PCF_OK;
}

pcf_status ctx_queue_status(pcf_ctx *ctx) {
    const volatile unsigned *w = ctx->h_ctrl;
    if (w && w[1]) {
        ctx->last_error = (w[1] & 2u) ? "a persistent kernel reached its iteration cap"
                                      : "a persistent kernel stopped on the abort request";
        return PCF_ERR_TIMEOUT;
    }
    return PCF_OK;
}

cudaError_t ensure_smem_limit(const void *fn, int device, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> limit;
    std::lock_guard<std::mutex> lk(mu);
    size_t &cur = limit[{fn, device}];
    if (bytes <= cur) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

extern "C" {

static bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

pcf_status pcf_grid_build(pcf_ctx *ctx, const pcf_point *pts, int64_t n, float box,
                          int partitions, pcf_grid **out) {
    if (!ctx || !pts || !out || n < 1 || !(box > 0.f) || partitions < 0 || partitions > 320)
        return PCF_ERR_INVALID_ARG;
    if (n > (int64_t)INT32_MAX / 2) return PCF_ERR_UNSUPPORTED;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    std::unique_ptr<pcf_grid> g(new pcf_grid);
    g->pool = ctx->pool;
    g->raw.pool = ctx->pool;
    g->n = n;
    g->box = box;
    PCF_CU(ctx, g->raw.ensure(sizeof(float4) * (size_t)n));
    PCF_CU(ctx, cudaMemcpyAsync(g->raw.p, pts, sizeof(float4) * (size_t)n,
                                is_device_ptr(pts) ? cudaMemcpyDeviceToDevice
                                                   : cudaMemcpyHostToDevice,
                                ctx->stream));
    g->user_P = partitions;
    int P = partitions > 0 ? partitions : choose_partitions(n, box, box / 8.f, PCF_ISO, false, 4);
    g->owner = ctx;
    pcf_status s = grid_ensure_cells(ctx, g.get(), P, ctx->grid_defer);
    if (s != PCF_OK) return s;
    *out = g.release();
    return PCF_OK;
}

pcf_status pcf_grid_free(pcf_ctx *ctx, pcf_grid *g) {
    if (!g) return PCF_ERR_INVALID_ARG;
    if (ctx) cudaSetDevice(ctx->device);
    // buffers go back to the context's pool; later users of the blocks are
    // ordered after the work already queued on the context stream
    delete g;
    return PCF_OK;
}

pcf_status pcf_grid_info(const pcf_grid *g, int64_t *n, float *box, int *partitions,
                         int64_t *nonempty_cells, int *unit_weights) {
    if (!g) return PCF_ERR_INVALID_ARG;
    if (g->owner) {  // a deferred build completes here
        cudaSetDevice(g->owner->device);
        pcf_status s = grid_finish(g->owner, g);
        if (s != PCF_OK) return s;
    }
    if (n) *n = g->n;
    if (box) *box = g->box;
    if (partitions) *partitions = g->cells ? g->cells->P : 0;
    if (nonempty_cells) {
        int64_t c = 0;
        if (g->cells) {
            const auto &h = g->cells->h_start;
            for (size_t i = 0; i + 1 < h.size(); ++i) c += h[i + 1] > h[i];
        }
        *nonempty_cells = c;
    }
    if (unit_weights) *unit_weights = g->unit_weights ? 1 : 0;
    return PCF_OK;
}

pcf_status pcf_grid_download(pcf_ctx *ctx, const pcf_grid *g, pcf_point *pts_out,
                             int32_t *cell_start_out) {
    if (!ctx || !g || !g->cells) return PCF_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, g);
        if (s0 != PCF_OK) return s0;
    }
    std::vector<float> planes;
    if (pts_out) {  // the cell-ordered SoA planes, interleaved on the host
        const CellGrid &c = *g->cells;
        planes.resize(4 * (size_t)g->n);
        for (int k = 0; k < 4; ++k)
            PCF_CU(ctx, cudaMemcpyAsync(planes.data() + (size_t)k * g->n, c.soa.as<float>() + k * c.plane,
                                        sizeof(float) * (size_t)g->n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (pts_out) {
        float *o = reinterpret_cast<float *>(pts_out);
        const size_t n = (size_t)g->n;
        for (size_t i = 0; i < n; ++i) {
            o[4 * i] = planes[i];
            o[4 * i + 1] = planes[n + i];
            o[4 * i + 2] = planes[2 * n + i];
            o[4 * i + 3] = planes[3 * n + i];
        }
    }
    if (cell_start_out)
        memcpy(cell_start_out, g->cells->h_start.data(), sizeof(int) * g->cells->h_start.size());
    return PCF_OK;
}

int pcf_autotune_partitions(pcf_ctx *ctx, int64_t n, float box, float dmax, int kind,
                            uint32_t flags) {
    (void)ctx;
    return choose_partitions(n, box, dmax, kind, (flags & PCF_BPC) != 0, 0);
}

}  // extern "C"

// Reference rule of a pair variant (see the oracle's reference_rule):
//   iso: XX d>0, XY none (2iso_k.cuh:50,107; 2isoBPC_k.cuh:62,338)
//   ani plain: every component > 0 (2ani_k.cuh:52,121)
//   ani BPC: XX > 0 and <=, XY <= (2aniBPC_k.cuh:63,401)
unsigned reference_pair_rule(bool ani, bool bpc, bool cross) {
    if (!ani) return cross ? 0u : PCF_RULE_EXCL;
    if (!bpc) return PCF_RULE_EXCL;
    return cross ? PCF_RULE_LE : (PCF_RULE_LE | PCF_RULE_EXCL);
}

PairRule make_pair_rule(int bins, float dmax, uint32_t flags, bool ani, bool bpc, bool cross) {
    PairRule r;
    double q = (double)bins / (double)dmax;
    r.ds = (flags & PCF_DS_EXACT) ? q : std::floor(q * 1000000.0) / 1000000.0;
    float ddf = dmax * dmax;
    r.dd = (double)ddf;
    r.bins = bins;
    if (flags & PCF_RULE_CUSTOM) {
        r.flags = ((flags & PCF_RULE_EXCL_ZERO) ? PCF_RULE_EXCL : 0u) |
                  ((flags & PCF_RULE_INCLUSIVE) ? PCF_RULE_LE : 0u);
    } else {
        r.flags = reference_pair_rule(ani, bpc, cross);
    }
    return r;
}

// Shared validation + re-gridding of the counting calls.
pcf_status prepare_grids(pcf_ctx *ctx, pcf_grid *a, pcf_grid *b, float dmax, int kind,
                         bool bpc, int *P_out, int refine) {
    if (b && b->box != a->box) return PCF_ERR_MISMATCH;
    const float box = a->box;
    if (bpc && !(2.0 * (double)dmax < (double)box)) {
        ctx->last_error = "periodic boundaries need dmax < box/2";
        return PCF_ERR_UNSUPPORTED;
    }
    int64_t n = std::max<int64_t>(a->n, b ? b->n : 0);
    // partitions: the autotuner's candidate, else the caller's choice at
    // grid build, else the tuned or default rule
    int P = 0;
    if (ctx->tune_override.refine <= 0) P = a->user_P > 0 ? a->user_P : (b ? b->user_P : 0);
    if (P > 0 && bpc) {  // a periodic stencil must not wrap onto itself: else automatic
        const double cell = (double)box / P;
        const int k = (int)std::ceil(((double)dmax + 1e-4 * cell + 8.0 * box * 1.2e-7) / cell);
        if (2 * k + 2 > P) P = 0;
    }
    if (P <= 0) P = choose_partitions(n, box, dmax, kind, bpc, refine);
    if (bpc) {
        double cell = (double)box / P;
        int k = (int)std::ceil(((double)dmax + 1e-4 * cell + 8.0 * box * 1.2e-7) / cell);
        if (2 * k + 2 > P) {
            ctx->last_error = "dmax too close to box/2 for the periodic stencil";
            return PCF_ERR_UNSUPPORTED;
        }
    }
    // both structures queued before either is completed: a's host work
    // (cell table, tiles) overlaps b's build on the device
    pcf_status s = grid_ensure_cells(ctx, a, P, b != nullptr);
    if (s != PCF_OK) return s;
    if (b) {
        s = grid_ensure_cells(ctx, b, P, true);
        if (s == PCF_OK) s = grid_finish(ctx, a);
        if (s == PCF_OK) s = grid_finish(ctx, b);
        if (s != PCF_OK) return s;
    }
    *P_out = P;
    return PCF_OK;
}

// Device scratch for one histogram: [u64 counts nb][f64 sums nb][u64 stats 8][f64 out nb]
static pcf_status hist_scratch(pcf_ctx *ctx, int nb, unsigned long long **cnt, double **ws,
                               unsigned long long **stats, double **out) {
    size_t bytes = (size_t)nb * 8 * 3 + 64;
    PCF_CU(ctx, ctx->d_hist.ensure(bytes));
    char *p = ctx->d_hist.as<char>();
    *cnt = reinterpret_cast<unsigned long long *>(p);
    *ws = reinterpret_cast<double *>(p + (size_t)nb * 8);
    *stats = reinterpret_cast<unsigned long long *>(p + (size_t)nb * 16);
    *out = reinterpret_cast<double *>(p + (size_t)nb * 16 + 64);
    PCF_CU(ctx, cudaMemsetAsync(p, 0, (size_t)nb * 16 + 64, ctx->stream));
    return PCF_OK;
}

// One pair histogram; ds_override > 0 replaces the bin scale (the fine
// histograms of the analytic path use (float)bins / dmax).
static pcf_status count_pairs_impl(pcf_ctx *ctx, int kind, const pcf_grid *a_, const pcf_grid *b_,
                                   int bins, float dmax, uint32_t flags, double *hist,
                                   pcf_stats *stats, double ds_override) {
    if (!ctx || !a_ || !hist || bins < 1 || !(dmax > 0.f) ||
        (kind != PCF_ISO && kind != PCF_ANI && kind != PCF_BOTH))
        return PCF_ERR_INVALID_ARG;
    if (kind != PCF_ISO && (int64_t)bins * bins > (1 << 24)) return PCF_ERR_UNSUPPORTED;
    if (kind == PCF_BOTH && ds_override > 0) return PCF_ERR_INVALID_ARG;
    if (ctx_abort_requested(ctx) != PCF_OK) return PCF_ERR_TIMEOUT;
    {
        pcf_status s0 = grid_finish(ctx, a_);
        if (s0 == PCF_OK && b_) s0 = grid_finish(ctx, b_);
        if (s0 != PCF_OK) return s0;
    }
    cudaSetDevice(ctx->device);
    pcf_grid *a = const_cast<pcf_grid *>(a_);
    pcf_grid *b = const_cast<pcf_grid *>(b_);
    const bool ani = kind != PCF_ISO, both = kind == PCF_BOTH;
    const bool bpc = (flags & PCF_BPC) != 0, cross = b != nullptr;
    const bool weighted = !(a->unit_weights && (!cross || b->unit_weights));
    TuneEntry te;
    if (ctx->tune_override.refine > 0 || ctx->tune_override.hist_mode >= 0 || ctx->tune_override.tile ||
        ctx->tune_override.chunk) {
        te = ctx->tune_override;
    } else if (!ctx->tune.empty()) {
        auto it = ctx->tune.find(tune_key(kind, bpc, cross, weighted, bins,
                                          std::max<int64_t>(a->n, cross ? b->n : 0), a->box, dmax));
        if (it != ctx->tune.end()) te = it->second;
    }
    // Both kinds run as the two single-kind launches written into one layout
    // unless the autotuner found one pass faster for this call class (a
    // tuned or forced scheme).  One pass saves the isotropic launch's
    // candidate tests, but its isotropic copy takes the anisotropic copy's
    // per-warp scheme, where lanes contend for few hot bins, and its extra
    // shared memory can cost resident CTAs.  Measured (200k x 32 randoms,
    // dmax 120, one batch each): exact weights, 40 bins: one pass 273 ms vs
    // 74 + 146 ms; 48 bins: 500 vs 68 + 267 ms; signed weights (per-warp FP64
    // copies either way), 40 bins: 381 vs 133 + 216 ms.
    if (both && te.hist_mode < 0) {
        pcf_stats si{}, sa{};
        pcf_status s = count_pairs_impl(ctx, PCF_ISO, a_, b_, bins, dmax, flags, hist,
                                        stats ? &si : nullptr, 0.0);
        if (s == PCF_OK)
            s = count_pairs_impl(ctx, PCF_ANI, a_, b_, bins, dmax, flags, hist + bins,
                                 stats ? &sa : nullptr, 0.0);
        if (s == PCF_OK && stats) {
            stats->pairs = si.pairs + sa.pairs;
            stats->candidates = si.candidates + sa.candidates;
            stats->rechecks = si.rechecks + sa.rechecks;
            stats->kernel_ms = si.kernel_ms + sa.kernel_ms;
            stats->partitions = sa.partitions;
            stats->work_items = (int)std::min<int64_t>((int64_t)si.work_items + sa.work_items, INT32_MAX);
        }
        return s;
    }
    int P = 0;
    pcf_status s = prepare_grids(ctx, a, b, dmax, kind, bpc, &P, te.refine);
    if (s != PCF_OK) return s;
    const int tile_cap = te.tile == 16 ? 16 : kTileCap;
    if (tile_cap == 16) {
        s = ensure_half_tiles(ctx, *a->cells);
        if (s != PCF_OK) return s;
    }
    PairPlan plan;
    plan_pairs(*a->cells, a->box, dmax, ani, !cross, plan, ctx->sm_count * 24, tile_cap);
    const int nb = both ? bins + bins * bins : ani ? bins * bins : bins;
    unsigned long long *d_cnt, *d_stats;
    double *d_ws, *d_out;
    s = hist_scratch(ctx, nb, &d_cnt, &d_ws, &d_stats, &d_out);
    if (s != PCF_OK) return s;
    PairLaunch pl;
    pl.ani = ani;
    pl.both = both;
    pl.bpc = bpc;
    pl.self = !cross;
    pl.weighted = weighted;
    pl.hist_mode = te.hist_mode;
    pl.rule = make_pair_rule(bins, dmax, flags, ani && !both, bpc, cross);
    if (both) pl.flags2 = make_pair_rule(bins, dmax, flags, true, bpc, cross).flags;
    if (ds_override > 0) pl.rule.ds = ds_override;
    pl.mult = cross ? 1.0 : 2.0;
    {
        const pcf_grid *gs[2] = {a, cross ? b : a};
        set_weight_fix(pl, gs, 2);
        pl.wunscale = weight_unscale(a, cross ? b : a);
    }
    pl.count = stats != nullptr && !ctx->tune_timing;
    pl.ctrl = ctx->d_abort;
    pl.status = ctx->d_status;
    pl.variant = ctx->pair_variant;
    pl.tile_cap = tile_cap;
    pl.chunk_cap = te.chunk;
    s = launch_pairs(ctx, plan, *a->cells, cross ? *b->cells : *a->cells, a->box, pl, d_cnt, d_ws,
                     d_stats);
    if (s != PCF_OK) return s;
    const bool dev_out = (flags & PCF_DEVICE_OUT) != 0;
    s = finalize_hist(ctx, d_cnt, d_ws, pl.weighted, pl.mult, nb, dev_out ? hist : d_out);
    if (s != PCF_OK) return s;
    if (stats || !dev_out) {
        // results come back through the context's page-locked buffer: copies
        // into pageable memory go through the driver's staging, where the
        // request server's concurrent slots were seen to stall one another
        const size_t hb = dev_out ? 0 : sizeof(double) * nb;
        const size_t cb = (stats && !pl.weighted) ? sizeof(unsigned long long) * nb : 0;
        s = pcf_ensure_pinned(ctx, hb + cb + 64);
        if (s != PCF_OK) return s;
        char *hp = static_cast<char *>(ctx->h_pinned);
        if (hb) PCF_CU(ctx, cudaMemcpyAsync(hp, d_out, hb, cudaMemcpyDeviceToHost, ctx->stream));
        if (cb) PCF_CU(ctx, cudaMemcpyAsync(hp + hb, d_cnt, cb, cudaMemcpyDeviceToHost, ctx->stream));
        PCF_CU(ctx, cudaMemcpyAsync(hp + hb + cb, d_stats, 32, cudaMemcpyDeviceToHost, ctx->stream));
        PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
        s = ctx_queue_status(ctx);
        if (s != PCF_OK) return s;
        if (hb) memcpy(hist, hp, hb);
        unsigned long long hs[4];
        memcpy(hs, hp + hb + cb, sizeof(hs));
        if (cb) {  // unit weights: pairs = sum of the counts
            const unsigned long long *cnt = reinterpret_cast<const unsigned long long *>(hp + hb);
            hs[2] = 0;
            for (int q = 0; q < nb; ++q) hs[2] += cnt[q];
        }
        if (stats) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            stats->rechecks = (double)hs[0];
            stats->candidates = (double)hs[1];
            stats->pairs = (double)hs[2];
            stats->kernel_ms = ms;
            stats->partitions = P;
            stats->work_items = (int)std::min<int64_t>(plan.n_items, INT32_MAX);
        }
    }
    return PCF_OK;
}

extern "C" pcf_status pcf_count_pairs(pcf_ctx *ctx, int kind, const pcf_grid *a, const pcf_grid *b,
                                      int bins, float dmax, uint32_t flags, double *hist,
                                      pcf_stats *stats) {
    return count_pairs_impl(ctx, kind, a, b, bins, dmax, flags, hist, stats, 0.0);
}

pcf_status pcf_count_pairs_ds(pcf_ctx *ctx, const pcf_grid *a, int bins, float dmax, double ds,
                              uint32_t flags, double *hist, pcf_stats *stats) {
    return count_pairs_impl(ctx, PCF_ISO, a, nullptr, bins, dmax, flags, hist, stats, ds);
}

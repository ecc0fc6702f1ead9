// batch.cu -- pcf_batch_pairs: one data catalog against many random
// catalogs of any sizes in ONE persistent launch.
//
// Reference: the -rd mode of cuda/main.cu:157-192 with pcf_2iso /
// pcf_2ani launching two kernels per random file on separate streams
// (pcf2iso.cuh:96-104), all random files forced to the same size.  Here the
// histograms DD, RR_i and DR_i are jobs of one work queue (items laid out
// job after job, each warp flushing its private histogram when it crosses
// into the next job), so small catalogs fill the gaps that large ones leave
// and the whole batch is a single kernel.  With PCF_GRAPH the device side
// of a batch (clears, kernel, finalize) is captured in a CUDA graph the
// first time and replayed on later calls with the same grids.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <sstream>

#include "pcf_internal.cuh"

struct BatchGraph {
    DevBuf plan;   // rows | jobs | mults
    DevBuf accum;  // counts | sums | stats | counter | out
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int nslots = 0, nb = 0;
    double *d_out = nullptr;
    unsigned long long *d_stats = nullptr;
    std::vector<double> mult;  // per slot: 2 for XX, 1 for XY
    std::vector<std::shared_ptr<CellGrid>> keep;  // cell structures the jobs read
    ~BatchGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// Both kinds as two single-kind batches, interleaved into the both-kinds
// layout: per histogram bins isotropic doubles, then bins^2 anisotropic.
// (One pass over the candidates for both kinds is slower: the measurements
// sit beside count_pairs_impl in capi.cu.)
static pcf_status batch_both_split(pcf_ctx *ctx, const pcf_grid *d, const pcf_grid *const *r,
                                   int n_rand, int bins, float dmax, uint32_t flags, double *dd,
                                   double *rr, double *dr, pcf_stats *stats) {
    const size_t b1 = (size_t)bins, b2 = (size_t)bins * bins, nb = b1 + b2, nr = (size_t)n_rand;
    std::vector<double> h[2][3];  // [kind][dd, rr, dr]
    pcf_stats st[2] = {};
    for (int k = 0; k < 2; ++k) {
        const size_t w = k ? b2 : b1;
        if (dd) h[k][0].resize(w);
        if (rr) h[k][1].resize(w * nr);
        if (dr) h[k][2].resize(w * nr);
        auto ptr = [&](int i, bool want) { return want ? h[k][i].data() : nullptr; };
        const pcf_status s = pcf_batch_pairs(ctx, k ? PCF_ANI : PCF_ISO, d, r, n_rand, bins, dmax, flags,
                                             ptr(0, dd != nullptr), ptr(1, rr != nullptr),
                                             ptr(2, dr != nullptr), stats ? &st[k] : nullptr);
        if (s != PCF_OK) return s;
    }
    auto put = [&](double *out, int i, size_t j) {
        memcpy(out + j * nb, h[0][i].data() + j * b1, sizeof(double) * b1);
        memcpy(out + j * nb + b1, h[1][i].data() + j * b2, sizeof(double) * b2);
    };
    if (dd) put(dd, 0, 0);
    for (size_t j = 0; j < nr; ++j) {
        if (rr) put(rr, 1, j);
        if (dr) put(dr, 2, j);
    }
    if (stats) {
        stats->pairs = st[0].pairs + st[1].pairs;
        stats->candidates = st[0].candidates + st[1].candidates;
        stats->rechecks = st[0].rechecks + st[1].rechecks;
        stats->kernel_ms = st[0].kernel_ms + st[1].kernel_ms;
        stats->partitions = st[1].partitions;
        stats->work_items = st[0].work_items + st[1].work_items;
    }
    return PCF_OK;
}

extern "C" pcf_status pcf_batch_pairs(pcf_ctx *ctx, int kind, const pcf_grid *d_,
                                      const pcf_grid *const *r_, int n_rand, int bins, float dmax,
                                      uint32_t flags, double *dd, double *rr, double *dr,
                                      pcf_stats *stats) {
    if (!ctx || !d_ || bins < 1 || !(dmax > 0.f) || n_rand < 0 || (n_rand > 0 && !r_) ||
        (kind != PCF_ISO && kind != PCF_ANI && kind != PCF_BOTH) || (!dd && !rr && !dr))
        return PCF_ERR_INVALID_ARG;
    if (kind == PCF_BOTH) return batch_both_split(ctx, d_, r_, n_rand, bins, dmax, flags, dd, rr, dr, stats);
    if (ctx_abort_requested(ctx) != PCF_OK) return PCF_ERR_TIMEOUT;
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, d_);
        for (int i = 0; s0 == PCF_OK && i < n_rand; ++i)
            if (r_[i]) s0 = grid_finish(ctx, r_[i]);
        if (s0 != PCF_OK) return s0;
    }
    const bool ani = kind == PCF_ANI, bpc = (flags & PCF_BPC) != 0;
    pcf_grid *D = const_cast<pcf_grid *>(d_);
    std::vector<pcf_grid *> R((size_t)n_rand);
    int64_t nmax = D->n;
    for (int i = 0; i < n_rand; ++i) {
        R[i] = const_cast<pcf_grid *>(r_[i]);
        if (!R[i]) return PCF_ERR_INVALID_ARG;
        if (R[i]->box != D->box) return PCF_ERR_MISMATCH;
        nmax = std::max<int64_t>(nmax, R[i]->n);
    }
    const float box = D->box;
    if (bpc && !(2.0 * (double)dmax < (double)box)) return PCF_ERR_UNSUPPORTED;
    // The jobs: DD, then RR_i and DR_i per random catalog.  Each job gets the
    // partition count a single call would use for its catalogs (small
    // catalogs get coarser cells), and holds the cell structures at that
    // count (a grid keeps several).
    struct J {
        pcf_grid *h, *c;
        bool self;
        double mult;
        int P;
        std::shared_ptr<CellGrid> hc, cc;
    };
    std::vector<J> js;
    auto add_job = [&](pcf_grid *h, pcf_grid *c, bool self, double mult) {
        const int64_t n = std::max<int64_t>(h->n, c->n);
        js.push_back({h, c, self, mult, choose_partitions(n, box, dmax, kind, bpc, 0), nullptr, nullptr});
    };
    if (dd) add_job(D, D, true, 2.0);
    for (int i = 0; i < n_rand; ++i) {
        if (rr) add_job(R[i], R[i], true, 2.0);
        if (dr) add_job(D, R[i], false, 1.0);
    }
    pcf_status s = PCF_OK;
    // every structure queued before the first is completed, so the builds'
    // host work overlaps the device; each job holds its structures, and a
    // structure that a later job's partition count replaces is completed at
    // that point, the grids' current ones after the loop
    for (auto &j : js) {
        if ((s = grid_ensure_cells(ctx, j.h, j.P, true)) != PCF_OK) return s;
        j.hc = j.h->cells;
        if ((s = grid_ensure_cells(ctx, j.c, j.P, true)) != PCF_OK) return s;
        j.cc = j.c->cells;
    }
    for (auto &j : js) {
        if ((s = grid_finish(ctx, j.h)) != PCF_OK || (s = grid_finish(ctx, j.c)) != PCF_OK) return s;
    }
    const int nb = ani ? bins * bins : bins;
    bool weighted = !D->unit_weights;
    for (auto *g : R) weighted = weighted || !g->unit_weights;

    // cache key of the captured graph: grids (by cell buffers) and parameters
    std::string key;
    const bool use_graph = (flags & PCF_GRAPH) != 0;
    if (use_graph) {
        std::ostringstream os;
        os << kind << ':' << bins << ':' << dmax << ':' << (flags & ~PCF_GRAPH) << ':' << (dd != nullptr)
           << (rr != nullptr) << (dr != nullptr);
        for (auto &j : js) os << ',' << j.hc->serial << '/' << j.cc->serial;
        key = os.str();
    }
    std::shared_ptr<BatchGraph> bg;
    if (use_graph) {
        auto it = ctx->graphs.find(key);
        if (it != ctx->graphs.end()) bg = it->second;
    }
    cudaStream_t st = ctx->stream;
    PairLaunch pl;
    pl.ani = ani;
    pl.bpc = bpc;
    pl.self = false;
    pl.weighted = weighted;
    pl.rule = make_pair_rule(bins, dmax, flags, ani, bpc, false);
    pl.mult = 1.0;
    pl.ctrl = ctx->d_abort;
    pl.status = ctx->d_status;
    {
        std::vector<const pcf_grid *> gs(R.begin(), R.end());
        gs.push_back(D);
        set_weight_fix(pl, gs.data(), (int)gs.size());
    }
    if (!bg) {
        bg = std::make_shared<BatchGraph>();
        bg->plan.pool = ctx->pool;
        bg->accum.pool = ctx->pool;
        // stencil rows per distinct partition count: [P] -> (self, cross)
        std::map<int, std::pair<std::vector<RowDesc>, std::vector<RowDesc>>> rows;
        for (auto &j : js) {
            if (rows.count(j.P)) continue;
            auto &rp = rows[j.P];
            plan_rows(j.P, box, dmax, ani, true, rp.first);
            plan_rows(j.P, box, dmax, ani, false, rp.second);
        }
        const int nslots = (int)js.size();
        int64_t total = 0;
        for (auto &j : js) {
            const auto &rp = rows[j.P];
            total += (int64_t)j.hc->tiles.size() * (int64_t)(j.self ? rp.first.size() : rp.second.size());
        }
        // plan buffer: row tables | jobs | mults
        std::map<int, std::pair<size_t, size_t>> roff;  // [P] -> (self, cross) byte offsets
        size_t off = 0;
        for (auto &kv : rows) {
            const size_t a = off;
            off = (off + kv.second.first.size() * sizeof(RowDesc) + 255) & ~(size_t)255;
            roff[kv.first] = {a, off};
            off = (off + kv.second.second.size() * sizeof(RowDesc) + 255) & ~(size_t)255;
        }
        const size_t off_j = off;
        const size_t off_m = (off_j + sizeof(PairJob) * nslots + 255) & ~(size_t)255;
        const size_t plan_bytes = off_m + sizeof(double) * nslots;
        PCF_CU(ctx, bg->plan.ensure(plan_bytes));
        char *dp = bg->plan.as<char>();
        std::vector<PairJob> jobs((size_t)nslots);
        std::vector<double> mult((size_t)nslots);
        long long item = 0;
        // exact-rule flags per job
        const unsigned rXX = reference_pair_rule(ani, bpc, false), rXY = reference_pair_rule(ani, bpc, true);
        for (int k = 0; k < nslots; ++k) {
            const CellGrid &h = *js[k].hc, &c = *js[k].cc;
            const auto &rp = rows[js[k].P];
            PairJob &j = jobs[k];
            j.home = pair_view(h, pl.wfix);
            j.cand = pair_view(c, pl.wfix);
            j.wunscale = weight_unscale(js[k].h, js[k].c);
            j.tiles = h.d_tiles.as<TileDesc>();
            j.rows = reinterpret_cast<const RowDesc *>(dp + (js[k].self ? roff[js[k].P].first : roff[js[k].P].second));
            shape_job(j, (int64_t)h.tiles.size(), (int)(js[k].self ? rp.first.size() : rp.second.size()),
                      total, ctx->sm_count);
            j.slot = k;
            j.item_begin = item;
            const unsigned custom = ((flags & PCF_RULE_EXCL_ZERO) ? PCF_RULE_EXCL : 0u) |
                                    ((flags & PCF_RULE_INCLUSIVE) ? PCF_RULE_LE : 0u);
            j.rule_flags = (flags & PCF_RULE_CUSTOM) ? custom : (js[k].self ? rXX : rXY);
            j.rule_flags2 = 0;  // single-kind jobs
            j.pad = 0;
            j.P = js[k].P;
            item += (long long)h.tiles.size() * j.n_chunks;
            mult[k] = js[k].mult;
            bg->keep.push_back(js[k].hc);
            bg->keep.push_back(js[k].cc);
        }
        std::vector<char> host(plan_bytes, 0);
        for (auto &kv : rows) {
            memcpy(host.data() + roff[kv.first].first, kv.second.first.data(),
                   kv.second.first.size() * sizeof(RowDesc));
            memcpy(host.data() + roff[kv.first].second, kv.second.second.data(),
                   kv.second.second.size() * sizeof(RowDesc));
        }
        memcpy(host.data() + off_j, jobs.data(), sizeof(PairJob) * nslots);
        memcpy(host.data() + off_m, mult.data(), sizeof(double) * nslots);
        PCF_CU(ctx, cudaMemcpyAsync(dp, host.data(), plan_bytes, cudaMemcpyHostToDevice, st));
        PCF_CU(ctx, cudaStreamSynchronize(st));  // host staging buffer goes out of scope
        // accumulators: counts | sums | stats(64B) | counter(64B) | out
        const size_t nacc = (size_t)nb * nslots;
        PCF_CU(ctx, bg->accum.ensure(nacc * 24 + 256));
        char *ap = bg->accum.as<char>();
        unsigned long long *cnt = reinterpret_cast<unsigned long long *>(ap);
        double *ws = reinterpret_cast<double *>(ap + nacc * 8);
        unsigned long long *stt = reinterpret_cast<unsigned long long *>(ap + nacc * 16);
        unsigned long long *counter = stt + 8;
        double *out = reinterpret_cast<double *>(ap + nacc * 16 + 128);
        bg->nslots = nslots;
        bg->nb = nb;
        bg->mult = mult;
        bg->d_out = out;
        bg->d_stats = stt;
        auto enqueue = [&]() -> cudaError_t {
            cudaError_t e = cudaMemsetAsync(ap, 0, nacc * 16 + 128, st);
            if (e != cudaSuccess) return e;
            e = launch_pair_jobs(reinterpret_cast<const PairJob *>(dp + off_j), nslots, item, js[0].P, box, pl,
                                 counter, cnt, ws, stt, st, ctx->sm_count, ctx->device);
            if (e != cudaSuccess) return e;
            return launch_finalize_slots(cnt, ws, weighted, reinterpret_cast<const double *>(dp + off_m),
                                         nb, nslots, out, st);
        };
        if (use_graph) {
            // make sure the kernel attributes are set outside the capture
            PCF_CU(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue();
            cudaGraph_t g = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess) return pcf_fail(ctx, e, "batch capture");
            if (e2 != cudaSuccess) return pcf_fail(ctx, e2, "cudaStreamEndCapture");
            bg->graph = g;
            PCF_CU(ctx, cudaGraphInstantiate(&bg->exec, g, 0));
            ctx->graphs[key] = bg;
        } else {
            PCF_CU(ctx, cudaEventRecord(ctx->ev0, st));
            PCF_CU(ctx, enqueue());
            PCF_CU(ctx, cudaEventRecord(ctx->ev1, st));
            ctx->launches += 2;
        }
    }
    if (use_graph) {
        PCF_CU(ctx, cudaEventRecord(ctx->ev0, st));
        PCF_CU(ctx, cudaGraphLaunch(bg->exec, st));
        PCF_CU(ctx, cudaEventRecord(ctx->ev1, st));
        ctx->launches += 2;
    }
    // results
    std::vector<double> host((size_t)bg->nb * bg->nslots);
    unsigned long long hs[4] = {0, 0, 0, 0};
    PCF_CU(ctx, cudaMemcpyAsync(host.data(), bg->d_out, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaMemcpyAsync(hs, bg->d_stats, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaStreamSynchronize(st));
    s = ctx_queue_status(ctx);
    if (s != PCF_OK) return s;
    int k = 0;
    if (dd) memcpy(dd, host.data() + (size_t)(k++) * nb, sizeof(double) * nb);
    for (int i = 0; i < n_rand; ++i) {
        if (rr) memcpy(rr + (size_t)i * nb, host.data() + (size_t)(k++) * nb, sizeof(double) * nb);
        if (dr) memcpy(dr + (size_t)i * nb, host.data() + (size_t)(k++) * nb, sizeof(double) * nb);
    }
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        double pairs = 0;
        if (!weighted) {
            for (int s2 = 0; s2 < bg->nslots; ++s2) {
                double sm = 0;
                for (int q = 0; q < nb; ++q) sm += host[(size_t)s2 * nb + q];
                pairs += sm / bg->mult[s2];  // unordered XX pairs, XY pairs
            }
        }
        stats->pairs = weighted ? (double)hs[2] : pairs;
        stats->rechecks = (double)hs[0];
        stats->candidates = (double)hs[1];
        stats->kernel_ms = ms;
        stats->partitions = js.empty() ? 0 : js[0].P;  // the DD job's (or first job's)
        stats->work_items = bg->nslots;
    }
    if (!use_graph) bg.reset();
    return PCF_OK;
}

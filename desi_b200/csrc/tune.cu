// tune.cu -- autotuner of the pair launch shape (include/pcf_tune.h).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

#include "../../include/pcf_tune.h"
#include "pcf_internal.cuh"

std::string tune_key(int kind, bool bpc, bool cross, bool weighted, int bins, int64_t n, float box,
                     float dmax) {
    // expected neighbours within dmax of a point, in half-octave buckets
    const double nbar = (double)n * 4.18879 * (double)dmax * dmax * dmax / ((double)box * box * box);
    const int bucket = (int)std::lround(2.0 * std::log2(nbar + 1.0));
    std::ostringstream os;
    os << (kind == PCF_BOTH ? "both" : kind == PCF_ANI ? "ani" : "iso") << (bpc ? "-bpc" : "")
       << (cross ? "-xy" : "-xx")
       << (weighted ? "-w" : "-u") << "-b" << bins << "-n" << bucket;
    return os.str();
}

extern "C" pcf_status pcf_autotune_pairs(pcf_ctx *ctx, int kind, const pcf_grid *a,
                                         const pcf_grid *b, int bins, float dmax, uint32_t flags,
                                         pcf_tune_result *res) {
    if (!ctx || !a || bins < 1 || !(dmax > 0.f)) return PCF_ERR_INVALID_ARG;
    {
        cudaSetDevice(ctx->device);
        pcf_status s0 = grid_finish(ctx, a);
        if (s0 == PCF_OK && b) s0 = grid_finish(ctx, b);
        if (s0 != PCF_OK) return s0;
    }
    const bool ani = kind != PCF_ISO, cross = b != nullptr;
    const bool weighted = !(a->unit_weights && (!cross || b->unit_weights));
    const std::string key = tune_key(kind, (flags & PCF_BPC) != 0, cross, weighted, bins,
                                     std::max<int64_t>(a->n, cross ? b->n : 0), a->box, dmax);
    const int nb = kind == PCF_BOTH ? bins + bins * bins : ani ? bins * bins : bins;
    DevBuf out;
    out.pool = ctx->pool;
    PCF_CU(ctx, out.ensure(sizeof(double) * nb));
    const int refines[] = {0, 3, 4, 5, 6, 8};
    const int modes[] = {-1, 0, 1, 3, 4};  // 3, 4: fixed-point weighted sums (weighted only)
    TuneEntry best;
    best.ms = 1e30f;
    float default_ms = 0.f;
    int tried = 0;
    ctx->tune.erase(key);
    ctx->tune_timing = true;
    for (int r : refines) {
        // partitions fixed by the caller: tune the histogram scheme only
        if ((a->user_P > 0 || (b && b->user_P > 0)) && r != 0) continue;
        for (int m : modes) {
            if (((m == 0 || m == 4) && ani) || ((m == 3 || m == 4) && !weighted)) continue;
            ctx->tune_override.refine = r;
            ctx->tune_override.hist_mode = m;
            float ms = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {  // the first run also re-grids
                pcf_stats st{};
                pcf_status s = pcf_count_pairs(ctx, kind, a, b, bins, dmax, flags | PCF_DEVICE_OUT,
                                               out.as<double>(), &st);
                if (s == PCF_ERR_UNSUPPORTED) { ms = 1e30f; break; }
                if (s != PCF_OK) {
                    ctx->tune_override = TuneEntry();
                    ctx->tune_timing = false;
                    return s;
                }
                ms = std::min(ms, st.kernel_ms);
            }
            ++tried;
            if (r == 0 && m == -1) default_ms = ms;
            if (ms < best.ms) {
                best.ms = ms;
                best.refine = r;
                best.hist_mode = m;
            }
        }
    }
    // home tiles of 16 points instead of 32 at the best shape (twice the
    // candidate streams per warp, half the home points per item)
    if (best.ms < 1e30f) {
        ctx->tune_override.refine = best.refine;
        ctx->tune_override.hist_mode = best.hist_mode;
        ctx->tune_override.tile = 16;
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            pcf_stats st{};
            pcf_status s = pcf_count_pairs(ctx, kind, a, b, bins, dmax, flags | PCF_DEVICE_OUT,
                                           out.as<double>(), &st);
            if (s != PCF_OK) { ms = 1e30f; break; }
            ms = std::min(ms, st.kernel_ms);
        }
        ++tried;
        if (ms < best.ms) {
            best.ms = ms;
            best.tile = 16;
        }
        // work items per ticket: runs of up to 8 (the launch rule), 4, or
        // one item per ticket, at the best shape so far
        ctx->tune_override.tile = best.tile;
        for (int c : {4, 1}) {
            ctx->tune_override.chunk = c;
            ms = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {
                pcf_stats st{};
                pcf_status s = pcf_count_pairs(ctx, kind, a, b, bins, dmax, flags | PCF_DEVICE_OUT,
                                               out.as<double>(), &st);
                if (s != PCF_OK) { ms = 1e30f; break; }
                ms = std::min(ms, st.kernel_ms);
            }
            ++tried;
            if (ms < best.ms) {
                best.ms = ms;
                best.chunk = c;
            }
        }
    }
    ctx->tune_override = TuneEntry();
    ctx->tune_timing = false;
    ctx->tune[key] = best;
    if (res) {
        res->refine = best.refine;
        res->hist_mode = best.hist_mode;
        res->tile = best.tile ? best.tile : kTileCap;
        res->chunk = best.chunk ? best.chunk : 8;
        res->best_ms = best.ms;
        res->default_ms = default_ms;
        res->tried = tried;
    }
    return PCF_OK;
}

extern "C" pcf_status pcf_tune_save(const pcf_ctx *ctx, const char *path) {
    if (!ctx || !path) return PCF_ERR_INVALID_ARG;
    std::ofstream f(path);
    if (!f) return PCF_ERR_IO;
    for (const auto &kv : ctx->tune)
        f << kv.first << ' ' << kv.second.refine << ' ' << kv.second.hist_mode << ' ' << kv.second.ms
          << ' ' << (kv.second.tile ? kv.second.tile : kTileCap) << ' '
          << (kv.second.chunk ? kv.second.chunk : 8) << '\n';
    return f ? PCF_OK : PCF_ERR_IO;
}

extern "C" pcf_status pcf_tune_load(pcf_ctx *ctx, const char *path) {
    if (!ctx || !path) return PCF_ERR_INVALID_ARG;
    std::ifstream f(path);
    if (!f) return PCF_ERR_IO;
    std::string line;
    while (std::getline(f, line)) {  // "key refine hist_mode ms [tile [chunk]]"
        std::istringstream is(line);
        std::string key;
        TuneEntry e;
        if (!(is >> key >> e.refine >> e.hist_mode >> e.ms)) continue;
        int tile = 0, chunk = 0;
        if (is >> tile) e.tile = tile == 16 ? 16 : 0;
        if (is >> chunk) e.chunk = (chunk == 1 || chunk == 4) ? chunk : 0;
        ctx->tune[key] = e;
    }
    return PCF_OK;
}

extern "C" int pcf_tune_size(const pcf_ctx *ctx) { return ctx ? (int)ctx->tune.size() : 0; }

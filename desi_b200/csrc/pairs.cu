// pairs.cu -- pair histograms (DD / RR / DR, isotropic and anisotropic,
// plain or periodic) on the CUDA cores.
//
// Reference kernels replaced: XX2iso/XY2iso (cuda/kernels/2iso_k.cuh:8,63),
// XX2ani/XY2ani (2ani_k.cuh:7,70), XX2iso_BPC/XY2iso_BPC (2isoBPC_k.cuh:8,284),
// XX2ani_BPC/XY2ani_BPC (2aniBPC_k.cuh:8,345).  The reference runs one
// thread per (cell, cell) pair with a global FP64 atomic per pair and 8
// image passes for periodic boxes; here:
//
//  * Work = (home tile, stencil rows) items in a persistent queue.  A home
//    tile is <= 128 cell-ordered points of one (ix,iy) column; a stencil row
//    (dx,dy) names the neighbour column, whose cells z0-kz..z1+kz are one
//    contiguous point range (or two when the periodic box wraps in z).  XX
//    uses the half shell (each unordered pair once, histogram doubled at the
//    end, matching the reference's ordered-pair convention).
//  * Periodic boxes: the neighbour column index wraps and the home point is
//    shifted by the image offset once per range, so no image passes.
//  * Separations in FP32 (3 FADD + FMUL + 2 FFMA); the bin comes from
//    r = d2*rsqrt(d2)*ds read out in 15-bit fixed point; any pair whose r is
//    within a proven error window of a bin edge, or whose d2 is near dmax^2
//    or 0, is re-evaluated with the canonical FP64 rule (pcf_internal.cuh),
//    so bin membership equals the FP64 oracle's exactly.
//  * Histograms: per-warp copies in shared memory (u32 counts for unit
//    weights, FP64 sums otherwise), merged once per CTA into global u64 /
//    FP64 and finalised to double (x2 for XX).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "pcf_internal.cuh"

namespace {

constexpr int kThreads = 128;  // 4 warps
constexpr int kWarps = kThreads / 32;
constexpr float kMagic = 256.0f;  // r + 256 -> mantissa = round(r * 2^15)
constexpr int kFracBits = 15;
constexpr unsigned kFracMask = (1u << kFracBits) - 1u;

// Fast-path cut constants for one range type (0: unshifted, 1: image-shifted).
struct FastCuts {
    float dsf;        // (float)ds
    float lo[2];      // d2 below lo (and >= tiny) is safely inside dmax
    float hi[2];      // d2 at or above hi is safely outside dmax
    unsigned w[2];    // edge window in 2^-15 units of r
    float tiny;
    int fast_bins;    // bins the fixed-point path may produce (<= 255)
};

struct PairStats {
    unsigned long long rechecks;
    unsigned long long candidates;
};

// Shared-memory histogram accumulators.
template <bool W>
struct Acc;
template <>
struct Acc<false> {
    typedef unsigned int T;
    __device__ static void add(T *h, int slot, float, float) { atomicAdd(h + slot, 1u); }
};
template <>
struct Acc<true> {
    typedef double T;
    __device__ static void add(T *h, int slot, float wa, float wb) {
        atomicAdd(h + slot, (double)wa * (double)wb);
    }
};

// Slow path: canonical FP64 decision for one pair.
template <bool ANI>
__device__ __noinline__ int slow_slot(float hx, float hy, float hz, float4 c, float sx, float sy,
                                      float sz, PairRule rule) {
    double dx, dy, dz;
    exact_sep(hx, hy, hz, c.x, c.y, c.z, sx, sy, sz, dx, dy, dz);
    return exact_slot<ANI>(dx, dy, dz, rule);
}

// Fixed-point bin of r (>= 0, < 256) with the edge test.  Returns the bin,
// or -1 when r lies within the window of an edge (caller rechecks).
__device__ __forceinline__ int fixed_bin(float r, unsigned w) {
    float a = r + kMagic;
    unsigned q = __float_as_uint(a) & 0x7FFFFFu;  // round(r * 2^15)
    unsigned f = (q - w) & kFracMask;              // frac - w (mod 1)
    bool edge = f >= (kFracMask + 1u - 2u * w);
    return edge ? -1 : (int)(q >> kFracBits);
}

template <bool ANI, bool WEIGHTED, bool GLOBAL_HIST>
__global__ void __launch_bounds__(kThreads) k_pairs(
    const float4 *__restrict__ hpts, const float4 *__restrict__ cpts,
    const int *__restrict__ cstart, const TileDesc *__restrict__ tiles,
    const RowDesc *__restrict__ rows, const WorkItem *__restrict__ items, int n_items,
    int *__restrict__ counter, int P, float box, int bpc, PairRule rule, FastCuts fc,
    unsigned long long *__restrict__ g_count, double *__restrict__ g_wsum,
    unsigned long long *__restrict__ g_stats) {
    typedef typename Acc<WEIGHTED>::T HT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HT *hist_all = reinterpret_cast<HT *>(smem_raw);
    __shared__ int s_item;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nb = ANI ? rule.bins * rule.bins : rule.bins;
    if (!GLOBAL_HIST) {
        for (int k = tid; k < nb * kWarps; k += kThreads) hist_all[k] = (HT)0;
    }
    HT *hist = GLOBAL_HIST ? nullptr : hist_all + warp * nb;
    unsigned long long n_recheck = 0, n_cand = 0, n_pairs = 0;
    __syncthreads();

    for (;;) {
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it_idx = s_item;
        __syncthreads();
        if (it_idx >= n_items) break;
        const WorkItem it = items[it_idx];
        const TileDesc t = tiles[it.tile];
        const int H = t.count;
        const int hw = H <= 32 ? 1 : (H <= 64 ? 2 : 4);  // warps per home set
        const int G = kWarps / hw;                        // candidate split
        const int g = warp / hw;
        const int h = (warp % hw) * 32 + lane;
        const bool valid = h < H;
        const int hidx = t.start + h;
        float4 hp = valid ? hpts[hidx] : make_float4(__int_as_float(0x7fc00000),
                                                     __int_as_float(0x7fc00000),
                                                     __int_as_float(0x7fc00000), 0.f);
        for (int r = it.row_begin; r < it.row_end; ++r) {
            const RowDesc rw = rows[r];
            int nx = t.ix + rw.dx, ny = t.iy + rw.dy;
            float sx = 0.f, sy = 0.f;
            if (bpc) {
                if (nx < 0) { nx += P; sx = -box; } else if (nx >= P) { nx -= P; sx = box; }
                if (ny < 0) { ny += P; sy = -box; } else if (ny >= P) { ny -= P; sy = box; }
            } else if (nx < 0 || nx >= P || ny < 0 || ny >= P) {
                continue;
            }
            const int col = (nx * P + ny) * P;
            // up to two ranges per row
            int a0, b0, a1 = 0, b1 = 0;
            float sz1 = 0.f;
            const int zhi = t.z1 + rw.kz;
            if (rw.kind == 1) {  // forward half of the home column (XX)
                a0 = t.start;    // intra-tile pairs use j > home index
                b0 = cstart[col + min(zhi, P - 1) + 1];
                if (bpc && zhi >= P) { a1 = cstart[col]; b1 = cstart[col + zhi - P + 1]; sz1 = box; }
            } else {
                const int zlo = t.z0 - rw.kz;
                a0 = cstart[col + max(zlo, 0)];
                b0 = cstart[col + min(zhi, P - 1) + 1];
                if (bpc) {
                    if (zlo < 0) { a1 = cstart[col + zlo + P]; b1 = cstart[col + P]; sz1 = -box; }
                    else if (zhi >= P) { a1 = cstart[col]; b1 = cstart[col + zhi - P + 1]; sz1 = box; }
                }
            }
            #pragma unroll 1
            for (int seg = 0; seg < 2; ++seg) {
                const int a = seg ? a1 : a0, b = seg ? b1 : b0;
                if (a >= b) continue;
                const float ssx = sx, ssy = sy, ssz = seg ? sz1 : 0.f;
                const int sh = (ssx != 0.f || ssy != 0.f || ssz != 0.f) ? 1 : 0;
                const float lo = fc.lo[sh], hi = fc.hi[sh];
                const unsigned w = fc.w[sh];
                const float hx = hp.x - ssx, hy = hp.y - ssy, hz = hp.z - ssz;
                const int jmin = (rw.kind == 1 && seg == 0) ? hidx : -1;
                if (tid == 0) n_cand += (unsigned long long)(b - a) * (unsigned long long)H;
                #pragma unroll 4
                for (int j = a + g; j < b; j += G) {
                    const float4 c = __ldg(cpts + j);
                    const float dx = c.x - hx, dy = c.y - hy, dz = c.z - hz;
                    if (!ANI) {
                        const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (d2 < hi && j > jmin) {
                            int slot = -1;
                            bool fast = !GLOBAL_HIST && (d2 < lo) && (d2 >= fc.tiny);
                            if (fast) {
                                float rr = d2 * (rsqrtf(d2) * fc.dsf);
                                slot = fixed_bin(rr, w);
                                fast = slot >= 0 && slot < fc.fast_bins;
                            }
                            if (!fast) {
                                ++n_recheck;
                                slot = slow_slot<false>(hp.x, hp.y, hp.z, c, ssx, ssy, ssz, rule);
                            }
                            if (slot >= 0) {
                                ++n_pairs;
                                if (GLOBAL_HIST) {
                                    if (WEIGHTED) atomicAdd(g_wsum + slot, (double)hp.w * (double)c.w);
                                    else atomicAdd(g_count + slot, 1ull);
                                } else {
                                    Acc<WEIGHTED>::add(hist, slot, hp.w, c.w);
                                }
                            }
                        }
                    } else {
                        const float zz = dz * dz;
                        const float pp = fmaf(dy, dy, dx * dx);
                        if (fmaxf(zz, pp) < hi && j > jmin) {
                            int slot = -1;
                            bool fast = !GLOBAL_HIST && (zz < lo) && (pp < lo) && (zz >= fc.tiny) &&
                                        (pp >= fc.tiny);
                            if (fast) {
                                float rz = fabsf(dz) * fc.dsf;
                                float rp = pp * (rsqrtf(pp) * fc.dsf);
                                int bz = fixed_bin(rz, w), bp = fixed_bin(rp, w);
                                fast = (bz >= 0) && (bp >= 0) && bz < fc.fast_bins && bp < fc.fast_bins;
                                slot = bz * rule.bins + bp;
                            }
                            if (!fast) {
                                ++n_recheck;
                                slot = slow_slot<true>(hp.x, hp.y, hp.z, c, ssx, ssy, ssz, rule);
                            }
                            if (slot >= 0) {
                                ++n_pairs;
                                if (GLOBAL_HIST) {
                                    if (WEIGHTED) atomicAdd(g_wsum + slot, (double)hp.w * (double)c.w);
                                    else atomicAdd(g_count + slot, 1ull);
                                } else {
                                    Acc<WEIGHTED>::add(hist, slot, hp.w, c.w);
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if (!GLOBAL_HIST) {
        for (int k = tid; k < nb; k += kThreads) {
            HT s = 0;
            #pragma unroll
            for (int q = 0; q < kWarps; ++q) s += hist_all[q * nb + k];
            if (s != (HT)0) {
                if (WEIGHTED) atomicAdd(g_wsum + k, (double)s);
                else atomicAdd(g_count + k, (unsigned long long)s);
            }
        }
    }
    // stats
    for (int off = 16; off > 0; off >>= 1) {
        n_recheck += __shfl_down_sync(0xffffffffu, n_recheck, off);
        n_pairs += __shfl_down_sync(0xffffffffu, n_pairs, off);
    }
    if (lane == 0 && n_recheck) atomicAdd(g_stats + 0, n_recheck);
    if (lane == 0 && n_pairs) atomicAdd(g_stats + 2, n_pairs);
    if (tid == 0 && n_cand) atomicAdd(g_stats + 1, n_cand);
}

// out[k] = mult * hist[k] (u64 counts or FP64 sums).
__global__ void k_finalize(const unsigned long long *__restrict__ cnt, const double *__restrict__ ws,
                           int weighted, double mult, int nb, double *__restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    double v = weighted ? ws[k] : (double)cnt[k];
    out[k] = mult * v;
}

}  // namespace

// ---------------------------------------------------------------------------
// Host planning.
// ---------------------------------------------------------------------------
void plan_pairs(const CellGrid &home, const CellGrid *cand, float box, float dmax, bool ani,
                bool bpc, bool self, int tile_cap, int cat, PairPlan &plan, int sm_count) {
    const int P = home.P;
    const double cell = (double)box / P;
    const double R = (double)dmax;
    // margin for points that sit a rounding step outside their cell
    const double margin = 1e-4 * cell + 8.0 * (double)box * 1.2e-7;
    const double Rm = R + margin;
    const int k = (int)std::ceil(Rm / cell);
    plan.P = P;
    plan.cell = (float)cell;
    plan.rows.clear();
    int kz_max = 0;
    for (int dx = -k; dx <= k; ++dx) {
        for (int dy = -k; dy <= k; ++dy) {
            double mx = std::max(std::abs(dx) - 1, 0) * cell;
            double my = std::max(std::abs(dy) - 1, 0) * cell;
            double mxy2 = mx * mx + my * my;
            if (mxy2 >= Rm * Rm) continue;
            int kz;
            if (ani) {
                kz = k;
            } else {
                double rem = std::sqrt(std::max(Rm * Rm - mxy2, 0.0));
                kz = (int)std::ceil(rem / cell);  // max(|dz|-1,0)*cell < rem
                kz = std::min(kz, k);
            }
            kz_max = std::max(kz_max, kz);
            RowDesc r;
            r.dx = (int16_t)dx;
            r.dy = (int16_t)dy;
            r.kz = (int16_t)kz;
            r.kind = 0;
            if (self) {
                if (dx == 0 && dy == 0) {
                    r.kind = 1;
                    plan.rows.insert(plan.rows.begin(), r);
                    continue;
                }
                if (!(dx > 0 || (dx == 0 && dy > 0))) continue;
            }
            plan.rows.push_back(r);
        }
    }
    // tiles
    plan.tiles.clear();
    const std::vector<int> &hs = home.h_start;
    const int span_cap = bpc ? std::max(1, std::min(P - 2 * kz_max - 1, std::max(1, k / 2) + 1))
                             : std::max(1, k / 2 + 1);
    for (int ix = 0; ix < P; ++ix) {
        for (int iy = 0; iy < P; ++iy) {
            const int col = (ix * P + iy) * P;
            int cur_start = -1, cur_cnt = 0, z0 = 0, zlast = 0;
            auto emit = [&](int start, int count, int za, int zb) {
                TileDesc t;
                t.start = start;
                t.count = count;
                t.ix = (int16_t)ix;
                t.iy = (int16_t)iy;
                t.z0 = (int16_t)za;
                t.z1 = (int16_t)zb;
                plan.tiles.push_back(t);
            };
            auto flush = [&]() {
                if (cur_start >= 0 && cur_cnt > 0) emit(cur_start, cur_cnt, z0, zlast);
                cur_start = -1;
                cur_cnt = 0;
            };
            for (int iz = 0; iz < P; ++iz) {
                const int s = hs[col + iz], c = hs[col + iz + 1] - s;
                if (c == 0) continue;
                if (cur_start >= 0 && (cur_cnt + c > tile_cap || iz - z0 + 1 > span_cap)) flush();
                if (c > tile_cap) {  // heavy cell: slices of tile_cap points
                    for (int o = 0; o < c; o += tile_cap) emit(s + o, std::min(tile_cap, c - o), iz, iz);
                    continue;
                }
                if (cur_start < 0) {
                    cur_start = s;
                    z0 = iz;
                }
                cur_cnt += c;
                zlast = iz;
            }
            flush();
        }
    }
    // cost of (tile, row) = H * candidates in the row's ranges
    const std::vector<int> &cs = cand ? cand->h_start : home.h_start;
    auto row_cost = [&](const TileDesc &t, const RowDesc &rw) -> double {
        int nx = t.ix + rw.dx, ny = t.iy + rw.dy;
        if (bpc) {
            nx = (nx % P + P) % P;
            ny = (ny % P + P) % P;
        } else if (nx < 0 || nx >= P || ny < 0 || ny >= P) {
            return 0.0;
        }
        const int col = (nx * P + ny) * P;
        int zlo = t.z0 - rw.kz, zhi = t.z1 + rw.kz;
        if (rw.kind == 1) zlo = t.z0;
        double n = 0;
        if (bpc) {
            for (int z = zlo; z <= zhi; ++z) {
                int zz = (z % P + P) % P;
                n += cs[col + zz + 1] - cs[col + zz];
            }
        } else {
            zlo = std::max(zlo, 0);
            zhi = std::min(zhi, P - 1);
            if (zlo <= zhi) n = cs[col + zhi + 1] - cs[col + zlo];
        }
        return n * t.count;
    };
    double total = 0;
    std::vector<std::vector<double>> rc(plan.tiles.size());
    for (size_t ti = 0; ti < plan.tiles.size(); ++ti) {
        rc[ti].resize(plan.rows.size());
        for (size_t ri = 0; ri < plan.rows.size(); ++ri) {
            rc[ti][ri] = row_cost(plan.tiles[ti], plan.rows[ri]);
            total += rc[ti][ri];
        }
    }
    const double target = std::max(total / (double)(sm_count * 16 * 4), 4096.0);
    struct CI { WorkItem w; double c; };
    std::vector<CI> items;
    for (size_t ti = 0; ti < plan.tiles.size(); ++ti) {
        int rb = 0;
        double acc = 0;
        for (size_t ri = 0; ri < plan.rows.size(); ++ri) {
            acc += rc[ti][ri];
            if (acc >= target || ri + 1 == plan.rows.size()) {
                if (acc > 0) items.push_back({{(int)ti, rb, (int)ri + 1, cat}, acc});
                rb = (int)ri + 1;
                acc = 0;
            }
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const CI &a, const CI &b) { return a.c > b.c; });
    plan.items.clear();
    plan.items.reserve(items.size());
    for (auto &c : items) plan.items.push_back(c.w);
}

// ---------------------------------------------------------------------------
// Launch one pair histogram (device side; result left in d_out as doubles).
// ---------------------------------------------------------------------------
static FastCuts make_cuts(const PairRule &rule, float box, float dmax, bool ani) {
    FastCuts fc;
    fc.dsf = (float)rule.ds;
    const double dd = rule.dd;
    const double rmax = (double)dmax * rule.ds + 1.0;  // r units
    // relative FP32 error of d2 (subtraction, 3 products/sums) <= ~2^-21:
    // windows carry an 8x-16x margin.
    const double e_plain_d2 = dd * std::ldexp(1.0, -17);
    const double w_plain = rmax * std::ldexp(1.0, -17);
    // image-shifted home point: |error of dx| <= L*2^-23 per axis
    const double e_shift_d2 = e_plain_d2 + (double)dmax * (double)box * std::ldexp(1.0, -19);
    const double w_shift = w_plain + rule.ds * (double)box * std::ldexp(1.0, -19);
    fc.lo[0] = (float)(dd - e_plain_d2);
    fc.hi[0] = (float)(dd + e_plain_d2);
    fc.lo[1] = (float)(dd - e_shift_d2);
    fc.hi[1] = (float)(dd + e_shift_d2);
    // fixed-point quantisation adds 2^-16
    fc.w[0] = (unsigned)std::ceil((w_plain + std::ldexp(1.0, -16)) * 32768.0) + 1u;
    fc.w[1] = (unsigned)std::ceil((w_shift + std::ldexp(1.0, -16)) * 32768.0) + 1u;
    fc.w[0] = std::min(fc.w[0], 8000u);
    fc.w[1] = std::min(fc.w[1], 8000u);
    fc.tiny = 1e-30f;
    fc.fast_bins = std::min(rule.bins, 255);
    (void)ani;
    return fc;
}

// Launches the pair kernel for one (home, cand) plan into d_count/d_wsum.
pcf_status launch_pairs(pcf_ctx *ctx, const PairPlan &plan, const CellGrid &home,
                        const CellGrid &cand, float box, const PairLaunch &pl,
                        unsigned long long *d_count, double *d_wsum,
                        unsigned long long *d_stats) {
    cudaStream_t st = ctx->stream;
    if (plan.items.empty()) return PCF_OK;
    size_t tb = plan.tiles.size() * sizeof(TileDesc);
    size_t rb = plan.rows.size() * sizeof(RowDesc);
    size_t ib = plan.items.size() * sizeof(WorkItem);
    PCF_CU(ctx, ctx->d_tiles.ensure(tb));
    PCF_CU(ctx, ctx->d_rows.ensure(rb));
    PCF_CU(ctx, ctx->d_items.ensure(ib));
    PCF_CU(ctx, ctx->d_counter.ensure(sizeof(int) * 16));
    pcf_status s = pcf_ensure_pinned(ctx, tb + rb + ib + 64);
    if (s != PCF_OK) return s;
    // stage through pinned memory (the stream may still read the previous plan,
    // so wait for it first)
    PCF_CU(ctx, cudaStreamSynchronize(st));
    char *hp = static_cast<char *>(ctx->h_pinned);
    memcpy(hp, plan.tiles.data(), tb);
    memcpy(hp + tb, plan.rows.data(), rb);
    memcpy(hp + tb + rb, plan.items.data(), ib);
    PCF_CU(ctx, cudaMemcpyAsync(ctx->d_tiles.p, hp, tb, cudaMemcpyHostToDevice, st));
    PCF_CU(ctx, cudaMemcpyAsync(ctx->d_rows.p, hp + tb, rb, cudaMemcpyHostToDevice, st));
    PCF_CU(ctx, cudaMemcpyAsync(ctx->d_items.p, hp + tb + rb, ib, cudaMemcpyHostToDevice, st));
    PCF_CU(ctx, cudaMemsetAsync(ctx->d_counter.p, 0, sizeof(int), st));

    FastCuts fc = make_cuts(pl.rule, box, std::sqrt((float)pl.rule.dd), pl.ani);
    const int nb = pl.ani ? pl.rule.bins * pl.rule.bins : pl.rule.bins;
    const size_t hbytes = (size_t)nb * kWarps * (pl.weighted ? 8 : 4);
    const bool global_hist = hbytes > 160 * 1024 || pl.rule.bins > 255;
    const int grid = std::max(1, std::min((int)plan.items.size(), ctx->sm_count * 8));
    const size_t smem = global_hist ? 0 : hbytes;
    int *counter = ctx->d_counter.as<int>();
    const int bpc = pl.bpc ? 1 : 0;
    PCF_CU(ctx, cudaEventRecord(ctx->ev0, st));
#define PCF_LAUNCH(A, W, G)                                                                      \
    do {                                                                                         \
        auto kfn = k_pairs<A, W, G>;                                                             \
        if (smem > 48 * 1024)                                                                    \
            PCF_CU(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                             (int)smem));                                        \
        kfn<<<grid, kThreads, smem, st>>>(home.pts.as<float4>(), cand.pts.as<float4>(),          \
                                          cand.cell_start.as<int>(), ctx->d_tiles.as<TileDesc>(), \
                                          ctx->d_rows.as<RowDesc>(), ctx->d_items.as<WorkItem>(), \
                                          (int)plan.items.size(), counter, plan.P, box, bpc,     \
                                          pl.rule, fc, d_count, d_wsum, d_stats);                \
    } while (0)
    if (global_hist) {
        // wide histograms (e.g. the fine DD of the analytic path): every
        // in-range pair takes the FP64 rule, accumulated in global memory
        if (pl.ani) {
            if (pl.weighted) PCF_LAUNCH(true, true, true);
            else PCF_LAUNCH(true, false, true);
        } else {
            if (pl.weighted) PCF_LAUNCH(false, true, true);
            else PCF_LAUNCH(false, false, true);
        }
    } else if (pl.ani) {
        if (pl.weighted) PCF_LAUNCH(true, true, false);
        else PCF_LAUNCH(true, false, false);
    } else {
        if (pl.weighted) PCF_LAUNCH(false, true, false);
        else PCF_LAUNCH(false, false, false);
    }
#undef PCF_LAUNCH
    PCF_CU(ctx, cudaGetLastError());
    PCF_CU(ctx, cudaEventRecord(ctx->ev1, st));
    ++ctx->launches;
    return PCF_OK;
}

pcf_status finalize_hist(pcf_ctx *ctx, const unsigned long long *d_count, const double *d_wsum,
                         bool weighted, double mult, int nb, double *d_out) {
    k_finalize<<<(nb + 255) / 256, 256, 0, ctx->stream>>>(d_count, d_wsum, weighted ? 1 : 0, mult,
                                                          nb, d_out);
    PCF_CU(ctx, cudaGetLastError());
    ++ctx->launches;
    return PCF_OK;
}

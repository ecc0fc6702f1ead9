// grid.cu -- GPU counting sort of a catalog into a uniform cell grid.
//
// Replaces the host grid builder of the reference (open_files/make_nodos/add
// in cuda/create_grid.cuh:35-139 and the flattening in cuda/main.cu:248-329,
// an O(sum len^2) reallocation per insert followed by a serial copy): three
// HBM-bound passes over the points --
//   1. cell id + per-cell count (atomic), with out-of-box / weight checks,
//   2. exclusive scan of the counts into the dense cell table,
//   3. the destination of every point (a 4-byte scattered write),
//   4. a gather in destination order that writes the cell-ordered copies
//      (SoA planes, pair-packed blocks, integer weights) coalesced.
// Cell id = (ix*P + iy)*P + iz with ix = (int)(x / cell), the reference's
// binning (create_grid.cuh:131-133) clamped to [0, P-1].
#include <algorithm>
#include <atomic>
#include <map>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "pcf_internal.cuh"

// The smallest cached block that holds n bytes is reused if it is at most
// 8n + 1 MB: a cudaMalloc can stall other threads' work on the device (the
// request server's slots), so a moderately oversized block beats a new one.
cudaError_t MemPool::get(size_t n, void **p, size_t *got) {
    auto it = free_blocks.lower_bound(n);
    if (it != free_blocks.end() && it->first <= 8 * n + (1u << 20)) {
        *p = it->second;
        *got = it->first;
        cached -= it->first;
        free_blocks.erase(it);
        return cudaSuccess;
    }
    size_t want = std::max<size_t>(256, (n + 255) & ~(size_t)255);
    cudaError_t e = cudaMalloc(p, want);
    if (e == cudaErrorMemoryAllocation && !free_blocks.empty()) {
        cudaGetLastError();
        release();
        e = cudaMalloc(p, want);
    }
    if (e == cudaSuccess) *got = want;
    return e;
}

void MemPool::put(void *p, size_t n) {
    free_blocks.emplace(n, p);
    cached += n;
}

void MemPool::release() {
    for (auto &kv : free_blocks) cudaFree(kv.second);
    free_blocks.clear();
    cached = 0;
}

DevBuf::~DevBuf() {
    if (!p) return;
    if (pool) pool->put(p, bytes);
    else cudaFree(p);
}

cudaError_t DevBuf::ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    if (p) {
        if (pool) pool->put(p, bytes);
        else cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
    if (pool) return pool->get(std::max<size_t>(n, 256), &p, &bytes);
    size_t want = std::max<size_t>(n, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
}

namespace {

constexpr int kScanItems = 1024;  // per block (256 threads x 4)

// flags[0] |= 1: a coordinate outside [0, box); |= 2: a weight != 1; |= 4: a
// negative or non-finite weight.  flags[1] = max |w| (float bits), flags[2] =
// ~(bits of the smallest nonzero |w|) -- both by atomicMax, after a warp
// reduction, so a launch makes one atomic per warp, not per point.
__global__ void k_cell_ids(const float4 *__restrict__ pts, int64_t n, int P, float cell, float box,
                           int *__restrict__ cid, int *__restrict__ rank,
                           int *__restrict__ counts, int *__restrict__ flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned f = 0u, wmax = 0u, wminc = 0u;
    if (i < n) {
        const float4 p = pts[i];
        const bool ok = (p.x >= 0.f) && (p.x < box) && (p.y >= 0.f) && (p.y < box) && (p.z >= 0.f) &&
                        (p.z < box);
        if (!ok) f |= 1u;
        if (p.w != 1.0f) f |= 2u;
        if (!(p.w >= 0.f) || !(p.w < INFINITY)) {
            f |= 4u;
        } else {
            wmax = __float_as_uint(p.w);
            if (p.w > 0.f) wminc = ~__float_as_uint(p.w);
        }
        int ix = (int)__fdiv_rn(p.x, cell), iy = (int)__fdiv_rn(p.y, cell),
            iz = (int)__fdiv_rn(p.z, cell);
        ix = min(max(ix, 0), P - 1);
        iy = min(max(iy, 0), P - 1);
        iz = min(max(iz, 0), P - 1);
        const int c = (ix * P + iy) * P + iz;
        cid[i] = c;
        rank[i] = atomicAdd(&counts[c], 1);
    }
    // one update of the three flag words per block, and only when it changes
    // them: every block targets the same three addresses, which would
    // otherwise serialise millions of atomics in L2
    f = __reduce_or_sync(0xffffffffu, f);
    wmax = __reduce_max_sync(0xffffffffu, wmax);
    wminc = __reduce_max_sync(0xffffffffu, wminc);
    __shared__ unsigned s_f, s_max, s_minc;
    if (threadIdx.x == 0) s_f = s_max = s_minc = 0u;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        if (f) atomicOr(&s_f, f);
        if (wmax) atomicMax(&s_max, wmax);
        if (wminc) atomicMax(&s_minc, wminc);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned *uf = reinterpret_cast<unsigned *>(flags);
        const volatile unsigned *vf = uf;
        if (s_f && (vf[0] & s_f) != s_f) atomicOr(uf, s_f);
        if (s_max > vf[1]) atomicMax(uf + 1, s_max);
        if (s_minc > vf[2]) atomicMax(uf + 2, s_minc);
    }
}

// Exclusive scan of one 1024-element chunk per block; the chunk total goes to
// sums[blockIdx.x].
__global__ void __launch_bounds__(256) k_scan_chunk(const int *__restrict__ in, int *__restrict__ out,
                                                   int *__restrict__ sums, int64_t n) {
    __shared__ int s[256];
    const int t = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * kScanItems + t * 4;
    int v0 = base + 0 < n ? in[base + 0] : 0;
    int v1 = base + 1 < n ? in[base + 1] : 0;
    int v2 = base + 2 < n ? in[base + 2] : 0;
    int v3 = base + 3 < n ? in[base + 3] : 0;
    int tot = v0 + v1 + v2 + v3;
    s[t] = tot;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        int x = t >= off ? s[t - off] : 0;
        __syncthreads();
        s[t] += x;
        __syncthreads();
    }
    int ex = s[t] - tot;
    if (base + 0 < n) out[base + 0] = ex;
    if (base + 1 < n) out[base + 1] = ex + v0;
    if (base + 2 < n) out[base + 2] = ex + v0 + v1;
    if (base + 3 < n) out[base + 3] = ex + v0 + v1 + v2;
    if (t == 255) sums[blockIdx.x] = s[255];
}

__global__ void k_scan_add(int *__restrict__ out, const int *__restrict__ offs, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * kScanItems + threadIdx.x;
    int add = offs[blockIdx.x];
    for (int k = 0; k < 4; ++k, i += 256)
        if (i < n) out[i] += add;
}

// Biased exponents of the weight range (flags[1] = bits of max |w|, flags[2]
// = ~bits of the smallest nonzero |w|) and whether the weights have exact
// integer images q = w * 2^(150 - emin) below 2^32: every weight finite and
// >= 0, the nonzero ones normal and within 8 binades of each other.
__host__ __device__ inline bool weight_fix_range(unsigned f0, unsigned wmaxb, unsigned wminc, int *emin,
                                                 int *emax) {
    *emin = (int)((~wminc >> 23) & 0xFFu);
    *emax = (int)((wmaxb >> 23) & 0xFFu);
    return !(f0 & 4u) && wminc != 0u && *emin >= 1 && *emax - *emin <= 8;
}

// Destination of every point: perm[start[cid] + rank] = i (one scattered
// 4-byte write per point).
__global__ void k_perm(int64_t n, const int *__restrict__ cid, const int *__restrict__ rank,
                       const int *__restrict__ start, int *__restrict__ perm) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[start[cid[i]] + rank[i]] = (int)i;
}

// Cell-ordered copies, one thread per destination d: a random 16-byte read
// of the source point, then coalesced writes of the SoA planes, the integer
// weight and the pair-packed blocks (an even lane writes block d/2 with its
// odd neighbour's values).
__global__ void k_gather(const float4 *__restrict__ pts, int64_t n, const int *__restrict__ perm,
                         float *__restrict__ soa, size_t plane, float4 *__restrict__ pk,
                         unsigned *__restrict__ qw, const int *__restrict__ flags) {
    const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    if (d < n) p = pts[perm[d]];
    const float nx = __shfl_down_sync(0xffffffffu, p.x, 1), ny = __shfl_down_sync(0xffffffffu, p.y, 1);
    const float nz = __shfl_down_sync(0xffffffffu, p.z, 1), nw = __shfl_down_sync(0xffffffffu, p.w, 1);
    if (d >= n) return;
    if (soa) {
        soa[d] = p.x;
        soa[plane + d] = p.y;
        soa[2 * plane + d] = p.z;
        soa[3 * plane + d] = p.w;
    }
    if (!(d & 1)) {  // block d/2: (x_d x_d+1 y_d y_d+1)(z_d z_d+1 w_d w_d+1); d+1 >= n gives 0
        const bool has = d + 1 < n;
        pk[d] = make_float4(p.x, has ? nx : 0.f, p.y, has ? ny : 0.f);
        pk[d + 1] = make_float4(p.z, has ? nz : 0.f, p.w, has ? nw : 0.f);
    }
    if (qw) {
        int emin, emax;
        const unsigned *uf = reinterpret_cast<const unsigned *>(flags);
        unsigned q = 0u;
        if (weight_fix_range(uf[0], uf[1], uf[2], &emin, &emax)) {
            const unsigned b = __float_as_uint(p.w) & 0x7FFFFFFFu;  // +0 and -0 give 0
            if (b) q = ((b & 0x7FFFFFu) | 0x800000u) << ((int)(b >> 23) - emin);
        }
        qw[d] = q;
    }
}

// Exclusive scan of n ints, in -> out, using tmp for the per-chunk sums
// (recursive on the sums).  tmp must hold ceil(n/1024) * 2 + ... ints; the
// caller passes a buffer of at least n/512 + 64 ints.
int scan_exclusive(const int *in, int *out, int64_t n, int *tmp, cudaStream_t st) {
    int64_t nb = (n + kScanItems - 1) / kScanItems;
    int *sums = tmp;
    int *sums_ex = tmp + nb;
    int launches = 1;
    k_scan_chunk<<<(unsigned)nb, 256, 0, st>>>(in, out, sums, n);
    if (nb > 1) {
        launches += scan_exclusive(sums, sums_ex, nb, tmp + 2 * nb, st);
        k_scan_add<<<(unsigned)nb, 256, 0, st>>>(out, sums_ex, n);
        ++launches;
    }
    return launches;
}

__global__ void k_tile_counts(const int *__restrict__ start, int ncell, int *__restrict__ tc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > ncell) return;
    tc[c] = c < ncell ? (start[c + 1] - start[c] + kTileCap - 1) / kTileCap : 0;
}

__global__ void k_tile_emit(const int *__restrict__ start, const int *__restrict__ toff, int P,
                            TileDesc *__restrict__ tiles) {
    const int ncell = P * P * P;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int s0 = start[c], n = start[c + 1] - s0;
    const int iz = c % P, iy = (c / P) % P, ix = c / (P * P);
    int o = toff[c];
    for (int k = 0; k < n; k += kTileCap, ++o) {
        TileDesc t;
        t.start = s0 + k;
        t.count = min(kTileCap, n - k);
        t.ix = (int16_t)ix;
        t.iy = (int16_t)iy;
        t.z0 = t.z1 = (int16_t)iz;
        tiles[o] = t;
    }
}

}  // namespace

int launch_grid_build(const float4 *raw, int64_t n, int P, float cell, float box, int *cid,
                      int *rank, int *perm, int *counts, int *cell_start, int *scan_tmp, float *soa,
                      size_t plane, float4 *pk, unsigned *qw, int *flags, cudaStream_t st) {
    const int64_t ncell = (int64_t)P * P * P;
    const int thr = 256;
    const unsigned blocks = (unsigned)((n + thr - 1) / thr);
    k_cell_ids<<<blocks, thr, 0, st>>>(raw, n, P, cell, box, cid, rank, counts, flags);
    int launches = 1 + scan_exclusive(counts, cell_start, ncell + 1, scan_tmp, st);
    k_perm<<<blocks, thr, 0, st>>>(n, cid, rank, cell_start, perm);
    k_gather<<<blocks, thr, 0, st>>>(raw, n, perm, soa, plane, pk, qw, flags);
    return launches + 2;
}

void set_weight_range(pcf_grid *g, const unsigned hf[3]) {
    g->unit_weights = (hf[0] & 2u) == 0;
    g->w_finite_nonneg = (hf[0] & 4u) == 0;
    std::memcpy(&g->w_absmax, &hf[1], sizeof(float));
    const unsigned mn = ~hf[2];
    if (hf[2]) std::memcpy(&g->w_absmin, &mn, sizeof(float));
    else g->w_absmin = 0.f;
    int emin = 0, emax = 0;
    g->wfix_ok = weight_fix_range(hf[0], hf[1], hf[2], &emin, &emax);
    g->wshift = 150 - emin;
    g->wqmax = g->wfix_ok ? (unsigned long long)((hf[1] & 0x7FFFFFu) | 0x800000u) << (emax - emin) : 0ull;
}

int launch_tile_build(const int *cell_start, int P, int *tile_counts, int *tile_offsets,
                      int *scan_tmp, TileDesc *tiles, cudaStream_t st) {
    const int ncell = P * P * P;
    k_tile_counts<<<(ncell + 1 + 255) / 256, 256, 0, st>>>(cell_start, ncell, tile_counts);
    int launches = 1 + scan_exclusive(tile_counts, tile_offsets, ncell + 1, scan_tmp, st);
    k_tile_emit<<<(ncell + 255) / 256, 256, 0, st>>>(cell_start, tile_offsets, P, tiles);
    return launches + 1;
}

pcf_status pcf_fail(pcf_ctx *ctx, cudaError_t e, const char *what) {
    if (ctx) {
        ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
    }
    cudaGetLastError();  // clear a sticky-free error so the context stays usable
    return e == cudaErrorMemoryAllocation ? PCF_ERR_NO_MEMORY : PCF_ERR_CUDA;
}

// The context's page-locked staging buffer, grown to at least `bytes`.  A
// copy queued from it may still be in flight: growing waits for the stream.
pcf_status pcf_ensure_pinned(pcf_ctx *ctx, size_t bytes) {
    if (ctx->h_pinned_bytes >= bytes) return PCF_OK;
    if (ctx->h_pinned) {
        PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFreeHost(ctx->h_pinned);
    }
    ctx->h_pinned = nullptr;
    ctx->h_pinned_bytes = 0;
    size_t want = std::max<size_t>(bytes, 1 << 20);
    PCF_CU(ctx, cudaMallocHost(&ctx->h_pinned, want));
    ctx->h_pinned_bytes = want;
    return PCF_OK;
}

// Build (or rebuild) the cell structure of g for P cells per side.
// A grid keeps the cell structures of the last few partition counts it was
// counted at, so classes of histograms tuned to different partitions do not
// rebuild (and synchronise) on every switch.
pcf_status grid_ensure_cells(pcf_ctx *ctx, pcf_grid *g, int P) {
    if (g->cells && g->cells->P == P) return PCF_OK;
    if (P < 1 || P > 320) return PCF_ERR_INVALID_ARG;
    for (size_t i = 0; i < g->cell_cache.size(); ++i) {
        if (g->cell_cache[i]->P != P) continue;
        std::shared_ptr<CellGrid> hit = std::move(g->cell_cache[i]);
        g->cell_cache.erase(g->cell_cache.begin() + (long)i);
        if (g->cells) g->cell_cache.push_back(std::move(g->cells));
        g->cells = std::move(hit);
        return PCF_OK;
    }
    static std::atomic<uint64_t> next_serial{0};  // contexts on several host threads build grids
    std::shared_ptr<CellGrid> cg(new CellGrid);
    cg->serial = ++next_serial;
    cg->soa.pool = cg->cell_start.pool = g->pool;
    cg->P = P;
    cg->cell = g->box / (float)P;
    const int64_t n = g->n;
    const int64_t ncell = (int64_t)P * P * P;
    cudaStream_t st = ctx->stream;
    cg->plane = ((size_t)n + kSoaPad + 3) & ~(size_t)3;
    PCF_CU(ctx, cg->soa.ensure(sizeof(float) * cg->plane * 4));
    PCF_CU(ctx, cudaMemsetAsync(cg->soa.p, 0, sizeof(float) * cg->plane * 4, ctx->stream));
    cg->pk.pool = cg->qw.pool = g->pool;
    PCF_CU(ctx, cg->pk.ensure(32 * pk_blocks(n)));
    PCF_CU(ctx, cudaMemsetAsync(cg->pk.p, 0, 32 * pk_blocks(n), ctx->stream));
    PCF_CU(ctx, cg->qw.ensure(sizeof(unsigned) * cg->plane));
    PCF_CU(ctx, cudaMemsetAsync(cg->qw.p, 0, sizeof(unsigned) * cg->plane, ctx->stream));
    PCF_CU(ctx, cg->cell_start.ensure(sizeof(int) * (size_t)(ncell + 1)));
    // scratch: cid, rank (n each); counts (ncell + 1); scan tmp.
    PCF_CU(ctx, ctx->scratch_a.ensure(sizeof(int) * (size_t)n * 3));
    PCF_CU(ctx, ctx->scratch_b.ensure(sizeof(int) * (size_t)(ncell + 1)));
    PCF_CU(ctx, ctx->scratch_c.ensure(sizeof(int) * (size_t)((ncell + 1) / 256 + 256)));
    PCF_CU(ctx, ctx->d_flag.ensure(sizeof(int) * 4));
    int *cid = ctx->scratch_a.as<int>();
    int *rank = cid + n;
    int *perm = rank + n;
    int *counts = ctx->scratch_b.as<int>();
    int *flags = ctx->d_flag.as<int>();
    PCF_CU(ctx, cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)(ncell + 1), st));
    PCF_CU(ctx, cudaMemsetAsync(flags, 0, sizeof(int) * 3, st));
    cudaEvent_t pg0 = nullptr, pg1 = nullptr;  // kernel-time log of grid builds
    if (ctx->profile) {
        if (ctx->prof_grid_used == ctx->prof_grid_events.size()) {
            cudaEvent_t e0, e1;
            PCF_CU(ctx, cudaEventCreate(&e0));
            PCF_CU(ctx, cudaEventCreate(&e1));
            ctx->prof_grid_events.push_back({e0, e1});
        }
        pg0 = ctx->prof_grid_events[ctx->prof_grid_used].first;
        pg1 = ctx->prof_grid_events[ctx->prof_grid_used].second;
        ++ctx->prof_grid_used;
        ctx->prof_grid_points += n;
        PCF_CU(ctx, cudaEventRecord(pg0, st));
    }
    ctx->launches += launch_grid_build(g->raw.as<float4>(), n, P, cg->cell, g->box, cid, rank, perm,
                                       counts, cg->cell_start.as<int>(), ctx->scratch_c.as<int>(),
                                       cg->soa.as<float>(), cg->plane, cg->pk.as<float4>(),
                                       cg->qw.as<unsigned>(), flags, st);
    PCF_CU(ctx, cudaGetLastError());
    if (pg1) PCF_CU(ctx, cudaEventRecord(pg1, st));
    // cell table and flags come back through the context's page-locked
    // buffer (pageable copies go through the driver's staging, where
    // concurrent contexts were seen to stall one another)
    const size_t sb = sizeof(int) * (size_t)(ncell + 1);
    pcf_status ps = pcf_ensure_pinned(ctx, sb + 64);
    if (ps != PCF_OK) return ps;
    char *hp = static_cast<char *>(ctx->h_pinned);
    PCF_CU(ctx, cudaMemcpyAsync(hp, cg->cell_start.p, sb, cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaMemcpyAsync(hp + sb, flags, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaStreamSynchronize(st));
    cg->h_start.assign(reinterpret_cast<const int *>(hp), reinterpret_cast<const int *>(hp) + ncell + 1);
    unsigned hf[3];
    memcpy(hf, hp + sb, sizeof(hf));
    const int hflags = (int)hf[0];
    if (hflags & 1) {
        ctx->last_error = "a coordinate lies outside [0, box)";
        return PCF_ERR_OUT_OF_BOX;
    }
    set_weight_range(g, hf);
    build_tiles(*cg, kTileCap, cg->tiles);
    cg->d_tiles.pool = g->pool;
    PCF_CU(ctx, cg->d_tiles.ensure(sizeof(TileDesc) * std::max<size_t>(1, cg->tiles.size())));
    if (!cg->tiles.empty()) {
        // staged in the page-locked buffer: every later host write to it
        // follows a synchronisation of this stream
        const size_t tb = sizeof(TileDesc) * cg->tiles.size();
        if ((ps = pcf_ensure_pinned(ctx, tb)) != PCF_OK) return ps;
        memcpy(ctx->h_pinned, cg->tiles.data(), tb);
        PCF_CU(ctx, cudaMemcpyAsync(cg->d_tiles.p, ctx->h_pinned, tb, cudaMemcpyHostToDevice, st));
    }
    if (g->cells) {
        g->cell_cache.push_back(std::move(g->cells));
        if ((int)g->cell_cache.size() > kCellCache) g->cell_cache.erase(g->cell_cache.begin());
    }
    g->cells = std::move(cg);
    return PCF_OK;
}

// Cells per side for a counting call: cell size about dmax/4 (so the
// stencil hugs the dmax sphere), coarsened while cells would hold fewer
// than ~6 points on average, and kept so that a periodic stencil never
// wraps onto itself (2k+1 <= P).
int choose_partitions(int64_t n, float box, float dmax, int kind, bool bpc, int refine) {
    if (refine <= 0) {
        const char *e = getenv("PCF_REFINE");  // experiment / autotuner override
        refine = e ? atoi(e) : 4;
        if (refine < 1 || refine > 16) refine = 4;
    }
    double L = box, R = dmax;
    int P = (int)std::floor(L / (R / refine));
    // mean occupancy floor
    while (P > 1) {
        double occ = (double)n / ((double)P * P * P);
        if (occ >= 6.0) break;
        int nr = refine - 1;
        if (nr < 1) break;
        refine = nr;
        P = (int)std::floor(L / (R / refine));
    }
    P = std::max(1, std::min(P, 256));
    if (bpc) {
        // need 2k+1 <= P with k = ceil(R / (L/P)) (+1 for the tile span)
        for (;;) {
            double cell = L / P;
            int k = (int)std::ceil((R + 1e-4 * cell + 8.0 * L * 1.2e-7) / cell);
            if (2 * k + 2 <= P || P >= 256) break;
            ++P;
        }
    }
    (void)kind;
    return P;
}

pcf_status ensure_half_tiles(pcf_ctx *ctx, CellGrid &g) {
    if (g.have_half) return PCF_OK;
    build_tiles(g, 16, g.tiles_half);
    g.d_tiles_half.pool = g.d_tiles.pool;
    PCF_CU(ctx, g.d_tiles_half.ensure(sizeof(TileDesc) * std::max<size_t>(1, g.tiles_half.size())));
    if (!g.tiles_half.empty()) {
        // the page-locked buffer may still feed an earlier copy: wait first
        PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
        const size_t tb = sizeof(TileDesc) * g.tiles_half.size();
        pcf_status ps = pcf_ensure_pinned(ctx, tb);
        if (ps != PCF_OK) return ps;
        memcpy(ctx->h_pinned, g.tiles_half.data(), tb);
        PCF_CU(ctx, cudaMemcpyAsync(g.d_tiles_half.p, ctx->h_pinned, tb, cudaMemcpyHostToDevice,
                                    ctx->stream));
    }
    g.have_half = true;
    return PCF_OK;
}

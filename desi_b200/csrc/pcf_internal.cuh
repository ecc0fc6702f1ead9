// pcf_internal.cuh -- shared declarations of libpcf (device helpers + host
// structures).  Not part of the public ABI (include/pcf.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
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

// One unit of the persistent work queue.
struct WorkItem {
    int tile;       // index into the tile table
    int row_begin;  // rows [row_begin, row_end) of the stencil
    int row_end;
    int cat;        // catalog slot (batched launches), else 0
};

// Device view of a gridded catalog.
struct CatView {
    const float4 *pts;      // cell-ordered points
    const int *cell_start;  // P^3 + 1
};

// ---------------------------------------------------------------------------
// Host-side objects.
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf();
    cudaError_t ensure(size_t n);  // grow (contents not kept)
    template <class T> T *as() const { return static_cast<T *>(p); }
};

struct CellGrid {
    int P = 0;
    float cell = 0.f;             // box / P
    DevBuf pts;                   // float4 x n, cell order
    DevBuf soa;                   // x | y | z | w planes, n + kSoaPad floats each
    size_t plane = 0;             // floats per plane
    DevBuf cell_start;            // int x (P^3 + 1)
    std::vector<int> h_start;     // host copy of cell_start
    const float *x() const { return soa.as<float>(); }
    const float *y() const { return soa.as<float>() + plane; }
    const float *z() const { return soa.as<float>() + 2 * plane; }
    const float *w() const { return soa.as<float>() + 3 * plane; }
};
// SoA planes are padded so that a float2 load at the last even index stays
// inside the allocation, and each plane starts 16-byte aligned.
constexpr int kSoaPad = 4;

struct pcf_grid {
    int64_t n = 0;
    float box = 0.f;
    bool unit_weights = true;
    DevBuf raw;                   // float4 x n, input order
    std::unique_ptr<CellGrid> cells;
};

struct pcf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sm_count = 148;
    std::string last_error;
    // scratch reused across calls
    DevBuf scratch_a, scratch_b, scratch_c, d_hist, d_items, d_tiles, d_rows, d_counter;
    DevBuf d_flag;
    void *h_pinned = nullptr;
    size_t h_pinned_bytes = 0;
    int64_t launches = 0;  // kernels launched by this context
};

// ---------------------------------------------------------------------------
// Internal host API (implemented in grid.cu / pairs.cu / triplets.cu ...).
// ---------------------------------------------------------------------------
pcf_status pcf_fail(pcf_ctx *ctx, cudaError_t e, const char *what);
#define PCF_CU(ctx, call)                                   \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return pcf_fail(ctx, _e, #call); \
    } while (0)

pcf_status grid_ensure_cells(pcf_ctx *ctx, pcf_grid *g, int P);
int choose_partitions(int64_t n, float box, float dmax, int kind, bool bpc, int npoint_kind);

// Stencil / tiles / work-list construction (host).
struct PairPlan {
    int P;
    float cell;
    std::vector<TileDesc> tiles;
    std::vector<RowDesc> rows;
    std::vector<WorkItem> items;
};

// Builds the work plan of one pair launch.  self: XX half shell.
void plan_pairs(const CellGrid &home, const CellGrid *cand, float box, float dmax, bool ani,
                bool bpc, bool self, int tile_cap, int cat, PairPlan &plan, int sm_count);

pcf_status pcf_ensure_pinned(pcf_ctx *ctx, size_t bytes);

// One pair-kernel launch (pairs.cu).
struct PairLaunch {
    bool ani, weighted, bpc, self;
    PairRule rule;
    double mult;  // 2 for XX (ordered-pair convention), 1 for XY
};
pcf_status launch_pairs(pcf_ctx *ctx, const PairPlan &plan, const CellGrid &home,
                        const CellGrid &cand, float box, const PairLaunch &pl,
                        unsigned long long *d_count, double *d_wsum, unsigned long long *d_stats);
pcf_status finalize_hist(pcf_ctx *ctx, const unsigned long long *d_count, const double *d_wsum,
                         bool weighted, double mult, int nb, double *d_out);
PairRule make_pair_rule(int bins, float dmax, uint32_t flags, bool ani, bool bpc, bool cross);
pcf_status prepare_grids(pcf_ctx *ctx, pcf_grid *a, pcf_grid *b, float dmax, int kind, bool bpc,
                         int *P_out);

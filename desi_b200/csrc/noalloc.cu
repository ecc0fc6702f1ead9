// noalloc.cu -- pcf_count_pairs_noalloc (include/pcf_noalloc.h): the pair
// histogram with every scratch buffer carved out of one fixed device array,
// for callers that cannot allocate device memory.
//
// The array below is a file-scope __device__ object: host code cannot use
// its name as a device address (taking it on the host yields a host-side
// stand-in), so each device's address is looked up once with
// cudaGetSymbolAddress, with that device current, and passed to the kernels.
#include <mutex>

#include "../../include/pcf_noalloc.h"
#include "pcf_internal.cuh"

static __device__ __align__(256) unsigned char g_pcf_noalloc_scratch[PCF_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_base[kMaxDevices];
int g_sms[kMaxDevices];

// Per-device set-up (first call on a device): address of the scratch array.
cudaError_t scratch_base(int dev, unsigned char **base, int *sms) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_pcf_noalloc_scratch);
        if (e != cudaSuccess) return e;
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        g_base[dev] = static_cast<unsigned char *>(p);
        g_sms[dev] = n;
    }
    *base = g_base[dev];
    *sms = g_sms[dev];
    return cudaSuccess;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carve {
    unsigned char *base;
    size_t used = 0;
    template <class T> T *take(size_t count) {
        T *p = reinterpret_cast<T *>(base + used);
        used += (count * sizeof(T) + 255) & ~(size_t)255;
        return p;
    }
};

struct CatBufs {
    int *cid, *rank, *perm, *counts, *start;
    float4 *pk;  // pair-packed points (PairView)
};

pcf_status fail(cudaError_t e) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? PCF_ERR_NO_MEMORY : PCF_ERR_CUDA;
}

}  // namespace

extern "C" pcf_status pcf_count_pairs_noalloc(const pcf_point *a, int64_t na, const pcf_point *b,
                                              int64_t nb, float box, int kind, int bins, float dmax,
                                              uint32_t flags, double *hist, void *stream) {
    if (!a || na < 1 || (b && nb < 1) || !(box > 0.f) || bins < 1 || !(dmax > 0.f) || !hist ||
        (kind != PCF_ISO && kind != PCF_ANI))
        return PCF_ERR_INVALID_ARG;
    const bool ani = kind == PCF_ANI, bpc = (flags & PCF_BPC) != 0, cross = b != nullptr;
    if (bpc && !(2.0 * (double)dmax < (double)box)) return PCF_ERR_UNSUPPORTED;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(e);
    unsigned char *base = nullptr;
    int sms = 0;
    e = scratch_base(dev, &base, &sms);
    if (e != cudaSuccess) return fail(e);

    const int64_t nmax = std::max<int64_t>(na, cross ? nb : 0);
    const int P = choose_partitions(nmax, box, dmax, kind, bpc, 0);
    if (bpc) {
        const double cell = (double)box / P;
        const int k = (int)std::ceil(((double)dmax + 1e-4 * cell + 8.0 * box * 1.2e-7) / cell);
        if (2 * k + 2 > P) return PCF_ERR_UNSUPPORTED;
    }
    const int64_t ncell = (int64_t)P * P * P;
    // the same bound as pcf_count_pairs (bins^2 accumulators at most 2^24)
    if (ani && (int64_t)bins * bins > (1 << 24)) return PCF_ERR_UNSUPPORTED;
    const int nbins = ani ? bins * bins : bins;
    std::vector<RowDesc> rows;
    plan_rows(P, box, dmax, ani, !cross, rows);

    // layout (checked against the array size before anything runs)
    Carve cv{base};
    auto carve_cat = [&](int64_t n) {
        CatBufs c;
        c.cid = cv.take<int>((size_t)n);
        c.rank = cv.take<int>((size_t)n);
        c.perm = cv.take<int>((size_t)n);
        c.counts = cv.take<int>((size_t)ncell + 1);
        c.start = cv.take<int>((size_t)ncell + 1);
        c.pk = cv.take<float4>(2 * pk_blocks(n));
        return c;
    };
    CatBufs A = carve_cat(na);
    CatBufs B = cross ? carve_cat(nb) : A;
    int *tile_counts = cv.take<int>((size_t)ncell + 1);
    int *tile_offsets = cv.take<int>((size_t)ncell + 1);
    TileDesc *tiles = cv.take<TileDesc>((size_t)na);
    int *scan_tmp = cv.take<int>((size_t)(ncell + 1) / 256 + 256);
    RowDesc *d_rows = cv.take<RowDesc>(rows.size());
    unsigned long long *counter = cv.take<unsigned long long>(8);
    unsigned long long *d_cnt = cv.take<unsigned long long>((size_t)nbins);
    double *d_ws = cv.take<double>((size_t)nbins);
    unsigned long long *d_stats = cv.take<unsigned long long>(8);
    int *d_flags = cv.take<int>(8);
    PairJob *d_job = cv.take<PairJob>(1);
    if (cv.used > PCF_NOALLOC_SCRATCH_BYTES) return PCF_ERR_UNSUPPORTED;

    // everything that accumulates starts at zero (the array keeps the last
    // call's contents)
    if ((e = cudaMemsetAsync(A.counts, 0, sizeof(int) * (ncell + 1), st)) != cudaSuccess) return fail(e);
    if (cross && (e = cudaMemsetAsync(B.counts, 0, sizeof(int) * (ncell + 1), st)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemsetAsync(A.pk, 0, 32 * pk_blocks(na), st)) != cudaSuccess) return fail(e);
    if (cross && (e = cudaMemsetAsync(B.pk, 0, 32 * pk_blocks(nb), st)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(counter, 0, 64, st)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * nbins, st)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(d_ws, 0, sizeof(double) * nbins, st)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(d_stats, 0, 64, st)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(d_flags, 0, 32, st)) != cudaSuccess) return fail(e);

    const float cell = box / (float)P;
    launch_grid_build(reinterpret_cast<const float4 *>(a), na, P, cell, box, A.cid, A.rank, A.perm,
                      A.counts, A.start, scan_tmp, nullptr, 0, A.pk, nullptr, d_flags, st);
    if (cross)
        launch_grid_build(reinterpret_cast<const float4 *>(b), nb, P, cell, box, B.cid, B.rank,
                          B.perm, B.counts, B.start, scan_tmp, nullptr, 0, B.pk, nullptr, d_flags, st);
    launch_tile_build(A.start, P, tile_counts, tile_offsets, scan_tmp, tiles, st);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpyAsync(d_rows, rows.data(), sizeof(RowDesc) * rows.size(),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return fail(e);
    int h_tiles = 0, h_flags = 0;
    if ((e = cudaMemcpyAsync(&h_tiles, tile_offsets + ncell, sizeof(int), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
        return fail(e);
    if ((e = cudaMemcpyAsync(&h_flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return fail(e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e);
    if (h_flags & 1) return PCF_ERR_OUT_OF_BOX;

    PairLaunch pl;
    pl.ani = ani;
    pl.bpc = bpc;
    pl.self = !cross;
    pl.weighted = (h_flags & 2) != 0;
    pl.rule = make_pair_rule(bins, dmax, flags, ani, bpc, cross);
    pl.mult = cross ? 1.0 : 2.0;
    const PairView hv{A.pk, nullptr, A.start};
    const PairView cvw{B.pk, nullptr, B.start};
    e = launch_pairs_view(hv, cvw, tiles, h_tiles, d_rows, (int)rows.size(), P, box, pl, counter,
                          d_cnt, d_ws, d_stats, d_job, st, sms, dev);
    if (e != cudaSuccess) return fail(e);
    e = launch_finalize(d_cnt, d_ws, pl.weighted, pl.mult, nbins, hist, st);
    if (e != cudaSuccess) return fail(e);
    return PCF_OK;
}

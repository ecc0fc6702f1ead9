// grid.cu -- GPU counting sort of a catalog into a uniform cell grid.
//
// Replaces the host grid builder of the reference (open_files/make_nodos/add
// in cuda/create_grid.cuh:35-139 and the flattening in cuda/main.cu:248-329,
// an O(sum len^2) reallocation per insert followed by a serial copy).
// Cell id = (ix*P + iy)*P + iz with ix = (int)(x / cell), the reference's
// binning (create_grid.cuh:131-133) clamped to [0, P-1].
//
// Catalogs of 6M to ~134M points take a bucketed build (runs of cells):
// three streaming passes with shared-memory histograms and no per-point
// global atomic:
//   1. per CTA, a histogram of its slice of the input over the buckets, with
//      the out-of-box / weight checks;
//   2. a scan of the CTA x bucket matrix, then a scatter of the points into
//      bucket order (each CTA into its own exact ranges);
//   3. per bucket, a counting sort by cell in shared memory that writes the
//      bucket's cell table and the cell-ordered copies (SoA planes,
//      pair-packed blocks, integer weights) coalesced.
// Other catalogs take the per-point build: cell id + per-cell count
// (atomic), a scan, the destination of every point (a scattered write) and a
// gather in destination order; below 6M points its atomics and gathers stay
// in L2 and it is the faster of the two.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include <cooperative_groups.h>

#include "pcf_internal.cuh"

namespace {
std::atomic<unsigned long long> g_alloc[6];  // device n, bytes, ns; host n, bytes, ns

template <class F>
cudaError_t counted(int slot, size_t n, F call) {
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = call();
    const auto t1 = std::chrono::steady_clock::now();
    if (e == cudaSuccess) {
        g_alloc[slot].fetch_add(1);
        g_alloc[slot + 1].fetch_add(n);
    }
    g_alloc[slot + 2].fetch_add(
        (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    return e;
}
}  // namespace

cudaError_t counted_malloc(void **p, size_t n) {
    return counted(0, n, [&] { return cudaMalloc(p, n); });
}

cudaError_t counted_malloc_host(void **p, size_t n) {
    return counted(3, n, [&] { return cudaHostAlloc(p, n, cudaHostAllocPortable); });
}

std::shared_ptr<PinnedPool> shared_pinned_pool() {
    // never destroyed: its blocks are released by the process's exit, after
    // which the CUDA runtime can no longer be called from a destructor
    static std::shared_ptr<PinnedPool> *pool = new std::shared_ptr<PinnedPool>(std::make_shared<PinnedPool>());
    return *pool;
}

namespace {
// Size classes of the device pool: four per power of two above 4 KB, so
// catalogs of nearby sizes reuse one another's blocks.
size_t pool_class(size_t n) {
    if (n <= 4096) return 4096;
    const int k = 63 - __builtin_clzll((unsigned long long)(n - 1));
    const size_t base = (size_t)1 << k, step = base >> 2;
    return base + (n - base + step - 1) / step * step;
}
}  // namespace

extern "C" pcf_status pcf_alloc_counters(uint64_t out[6]) {
    if (!out) return PCF_ERR_INVALID_ARG;
    for (int k = 0; k < 6; ++k) out[k] = g_alloc[k].load();
    return PCF_OK;
}

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
    const size_t want = pool_class(n);
    cudaError_t e = counted_malloc(p, want);
    if (e == cudaErrorMemoryAllocation && !free_blocks.empty()) {
        cudaGetLastError();
        release();
        e = counted_malloc(p, want);
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

// Blocks come in power-of-two sizes from 64 KB, so a freed block serves any
// later request of its size class: pinning new pages (cudaMallocHost) is slow
// and serialises the threads that share the device.
cudaError_t PinnedPool::get(size_t n, void **p, size_t *got) {
    size_t want = 64u << 10;
    while (want < n) want <<= 1;
    std::lock_guard<std::mutex> lk(mu);
    auto it = free_blocks.find(want);
    if (it != free_blocks.end()) {
        *p = it->second;
        *got = it->first;
        free_blocks.erase(it);
        return cudaSuccess;
    }
    cudaError_t e = counted_malloc_host(p, want);
    if (e == cudaSuccess) *got = want;
    return e;
}

void PinnedPool::put(void *p, size_t n) {
    std::lock_guard<std::mutex> lk(mu);
    free_blocks.insert({n, p});
}

PinnedPool::~PinnedPool() {
    for (auto &kv : free_blocks) cudaFreeHost(kv.second);
}

CellGrid::~CellGrid() {
    if (ready) {  // the stage may still feed the tile table's copy
        cudaEventSynchronize(ready);
        cudaEventDestroy(ready);
    }
    if (stage && pinned) pinned->put(stage, stage_bytes);
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
    cudaError_t e = counted_malloc(&p, want);
    if (e == cudaSuccess) bytes = want;
    return e;
}

namespace {

constexpr int kScanItems = 1024;  // per block (256 threads x 4)

// (int)(x / cell) with the division correctly rounded, as the reference's
// host code computes it.  x * (1/cell) is within 2^-23 (relative) of the
// exact quotient, i.e. within 6.2e-5 for quotients below 512 (P <= 320), and
// the rounded quotient within half an ulp (3.1e-5) of it; so when the
// product lies more than 2.4e-4 from every integer both truncate alike, and
// only the rare quotients near a cell face take the division.  Negative,
// infinite and NaN coordinates all take the division.
__device__ __forceinline__ int cell_axis(float x, float cell, float rcell) {
    const float q = x * rcell;
    const int k = (int)q;
    const float fr = q - (float)k;
    if (fr > 2.4e-4f && fr < 1.0f - 2.4e-4f) return k;
    return (int)__fdiv_rn(x, cell);
}

// Cell of a point: ix = (int)(x / cell) clamped to [0, P-1] per axis, the
// reference's binning (create_grid.cuh:131-133).  Every pass of both builds
// computes it with this one function, so a point's cell never differs
// between passes.
__device__ __forceinline__ int cell_of_point(const float4 &p, int P, float cell) {
    const float rcell = 1.0f / cell;
    int ix = cell_axis(p.x, cell, rcell), iy = cell_axis(p.y, cell, rcell), iz = cell_axis(p.z, cell, rcell);
    ix = min(max(ix, 0), P - 1);
    iy = min(max(iy, 0), P - 1);
    iz = min(max(iz, 0), P - 1);
    return (ix * P + iy) * P + iz;
}

// c / Q for c < K * Q with K <= 2^14: the float estimate is within 0.003 of
// the quotient, so one correction step makes it exact.
__device__ __forceinline__ int div_q(int c, int Q, float rq) {
    int k = (int)((float)c * rq);
    const int r = c - k * Q;
    k += (r >= Q) - (r < 0);
    return k;
}

// flags[0] |= 1: a coordinate outside [0, box); |= 2: a weight != 1; |= 4: a
// negative or non-finite weight.  flags[1] = max |w| (float bits), flags[2] =
// ~(bits of the smallest nonzero |w|).
__device__ __forceinline__ void point_flags(const float4 &p, float box, unsigned &f, unsigned &wmax,
                                            unsigned &wminc) {
    const bool ok = (p.x >= 0.f) && (p.x < box) && (p.y >= 0.f) && (p.y < box) && (p.z >= 0.f) &&
                    (p.z < box);
    if (!ok) f |= 1u;
    if (p.w != 1.0f) f |= 2u;
    if (!(p.w >= 0.f) || !(p.w < INFINITY)) {
        f |= 4u;
    } else {
        wmax = max(wmax, __float_as_uint(p.w));
        if (p.w > 0.f) wminc = max(wminc, ~__float_as_uint(p.w));
    }
}

// One update of the three flag words per block (after a warp reduction), and
// only when it changes them: every block targets the same three addresses,
// which would otherwise serialise millions of atomics in L2.  Called by every
// thread of the block.
__device__ __forceinline__ void flush_flags(unsigned f, unsigned wmax, unsigned wminc, int *flags) {
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

__global__ void k_cell_ids(const float4 *__restrict__ pts, int64_t n, int P, float cell, float box,
                           int *__restrict__ cid, int *__restrict__ rank,
                           int *__restrict__ counts, int *__restrict__ flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned f = 0u, wmax = 0u, wminc = 0u;
    if (i < n) {
        const float4 p = pts[i];
        point_flags(p, box, f, wmax, wminc);
        const int c = cell_of_point(p, P, cell);
        cid[i] = c;
        rank[i] = atomicAdd(&counts[c], 1);
    }
    flush_flags(f, wmax, wminc, flags);
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

// ---- bucketed build -------------------------------------------------------
// Buckets are runs of Q consecutive cells (at most kBktMaxCells), about
// kBktTarget points each.  The count pass gives every CTA a shared histogram
// of its own contiguous slice of the input; one scan of the CTA x bucket
// matrix (bucket-major) hands each CTA a private, exact write range per
// bucket.  The scatter pass then sorts each 8192-point chunk of its slice by
// bucket in shared memory and writes every bucket's run of the chunk to the
// front of its range, so stores leave as coalesced runs instead of one random
// 16-byte store per point (those ran at ~6e10/s: partial sectors scattered
// over the whole scratch array).  No pass makes a per-point global atomic.
// The sort pass takes one bucket per cluster of kCluster CTAs: the CTAs count
// their shares of the bucket per cell, merge the counts through distributed
// shared memory into the bucket's cell table, place every point into the
// shared memory of the CTA that owns its destination, and write the
// cell-ordered copies (SoA planes, pair-packed blocks, integer weights)
// coalesced.
constexpr int kBktThreads = 1024;                   // count and scatter CTAs, one per SM
constexpr int kBktUnroll = 8;                       // loads in flight per thread in every pass
constexpr int kChunk = kBktThreads * kBktUnroll;    // points per scatter round
constexpr int kBktTarget = 32768;                   // mean points per bucket
constexpr int kBktMinBuckets = 128;                 // buckets of a small catalog (sort-pass parallelism)
constexpr int kBktMaxCells = 4096;                  // cells per bucket (the sort's counters)
constexpr int kBktMaxBuckets = 4096;                // buckets (count / scatter shared arrays)
constexpr int kCluster = 4;                         // CTAs sorting one bucket
constexpr int kSortThreads = 1024;
constexpr int kSortUnroll = 4;         // loads in flight per thread in the sort (its shares are prefetched into L2)
constexpr int kClusterCap = 11264;                  // points staged per CTA of a sorting cluster
constexpr size_t kSortSmem = (size_t)kClusterCap * sizeof(float4) + 2 * (size_t)kBktMaxCells * sizeof(int);
inline size_t scatter_smem(int K) {
    return (size_t)kChunk * (sizeof(float4) + sizeof(unsigned short)) + 2 * sizeof(int) * (size_t)K;
}

__device__ __forceinline__ unsigned weight_q(float w, int emin) {
    const unsigned b = __float_as_uint(w) & 0x7FFFFFFFu;  // +0 and -0 give 0
    return b ? ((b & 0x7FFFFFu) | 0x800000u) << ((int)(b >> 23) - emin) : 0u;
}

// This point's half of pair block d/2 (components d & 1 of its two float4s).
__device__ __forceinline__ void pk_put(float4 *pk, int64_t d, const float4 &p) {
    const int h = (int)(d & 1);
    float *a = reinterpret_cast<float *>(pk + (d - h));
    float *b = a + 4;
    a[h] = p.x;
    a[2 + h] = p.y;
    b[h] = p.z;
    b[2 + h] = p.w;
}

// Asks L2 to fetch [p, p + bytes) (p 16-byte aligned) ahead of its use, in
// bulk requests of at most 64 KB; no shared memory or registers are held.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const char *c = static_cast<const char *>(p);
    bytes &= ~(size_t)15;
    while (bytes) {
        const unsigned sz = (unsigned)min(bytes, (size_t)65536);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c), "r"(sz) : "memory");
        c += sz;
        bytes -= sz;
    }
}

// Exclusive scan of a[0..q) in place, q <= 4 * blockDim.x, blockDim.x a
// multiple of 32 and at most 1024.  Called by every thread of the block;
// ends with the block synchronised.
__device__ void block_excl_scan4(int *a, int q, int *wsum) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int v[4], s = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = 4 * t + u;
        v[u] = i < q ? a[i] : 0;
        s += v[u];
    }
    int x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        const int ws = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        int z = ws;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        wsum[lane] = z - ws;
    }
    __syncthreads();
    int e = wsum[w] + x - s;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = 4 * t + u;
        if (i < q) a[i] = e;
        e += v[u];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kBktThreads) k_bkt_count(const float4 *__restrict__ pts, int64_t n,
                                                           int64_t span, int P, float cell, float box,
                                                           int Q, float rq, int K, int *__restrict__ M,
                                                           int *__restrict__ flags) {
    extern __shared__ int hist[];
    for (int k = threadIdx.x; k < K; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int64_t i0 = (int64_t)blockIdx.x * span, i1 = min(n, i0 + span);
    const int64_t T = blockDim.x;
    unsigned f = 0u, wmax = 0u, wminc = 0u;
    int64_t i = i0 + threadIdx.x;
    for (; i + (kBktUnroll - 1) * T < i1; i += kBktUnroll * T) {
        if (threadIdx.x == 0) {  // the next block of the slice into L2 meanwhile
            const int64_t nb = i + kBktUnroll * T, ne = min(i1, nb + kBktUnroll * T);
            if (nb < ne) prefetch_l2(pts + nb, (size_t)(ne - nb) * sizeof(float4));
        }
        float4 p[kBktUnroll];
#pragma unroll
        for (int u = 0; u < kBktUnroll; ++u) p[u] = pts[i + u * T];
#pragma unroll
        for (int u = 0; u < kBktUnroll; ++u) {
            point_flags(p[u], box, f, wmax, wminc);
            atomicAdd(&hist[div_q(cell_of_point(p[u], P, cell), Q, rq)], 1);
        }
    }
    for (; i < i1; i += T) {
        const float4 p = pts[i];
        point_flags(p, box, f, wmax, wminc);
        atomicAdd(&hist[div_q(cell_of_point(p, P, cell), Q, rq)], 1);
    }
    flush_flags(f, wmax, wminc, flags);  // ends with the block's histogram complete
    const int64_t G = gridDim.x;
    for (int k = threadIdx.x; k < K; k += blockDim.x) M[k * G + blockIdx.x] = hist[k];
}

// Rounds of kChunk points: the round's count per bucket (shared counters), a
// scan of the counts into run starts, each point staged in its bucket's run
// (a second shared atomic hands out the slots), then each staged point stored
// at its bucket's cursor + its offset in the run.
__global__ void __launch_bounds__(kBktThreads) k_bkt_scatter(const float4 *__restrict__ pts, int64_t n,
                                                             int64_t span, int P, float cell, int Q,
                                                             float rq, int K, const int *__restrict__ base,
                                                             float4 *__restrict__ S) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4 *stg = reinterpret_cast<float4 *>(smem);
    int *cur = reinterpret_cast<int *>(smem + (size_t)kChunk * sizeof(float4));  // K write cursors
    int *cnt = cur + K;                                                            // K: counts, then run starts
    unsigned short *skb = reinterpret_cast<unsigned short *>(cnt + K);            // bucket of each staged point
    __shared__ int wsum[32];
    const int64_t G = gridDim.x;
    const int T = blockDim.x;
    for (int k = threadIdx.x; k < K; k += T) cur[k] = base[k * G + blockIdx.x];
    const int64_t i0 = (int64_t)blockIdx.x * span, i1 = min(n, i0 + span);
    for (int64_t r0 = i0; r0 < i1; r0 += kChunk) {
        if (threadIdx.x == 0) {  // the next round's points into L2 while this one runs
            const int64_t nb = r0 + kChunk, ne = min(i1, nb + kChunk);
            if (nb < ne) prefetch_l2(pts + nb, (size_t)(ne - nb) * sizeof(float4));
        }
        for (int k = threadIdx.x; k < K; k += T) cnt[k] = 0;
        __syncthreads();
        float4 p[kBktUnroll];
        int kbs[kBktUnroll];  // bucket, or -1 past the slice
#pragma unroll
        for (int u = 0; u < kBktUnroll; ++u) {
            const int64_t i = r0 + u * T + threadIdx.x;
            if (i < i1) p[u] = pts[i];
        }
#pragma unroll
        for (int u = 0; u < kBktUnroll; ++u) {
            const int64_t i = r0 + u * T + threadIdx.x;
            kbs[u] = -1;
            if (i < i1) {
                kbs[u] = div_q(cell_of_point(p[u], P, cell), Q, rq);
                atomicAdd(&cnt[kbs[u]], 1);
            }
        }
        __syncthreads();
        block_excl_scan4(cnt, K, wsum);  // run starts; the slots below turn each into its run's end
#pragma unroll
        for (int u = 0; u < kBktUnroll; ++u) {
            if (kbs[u] < 0) continue;
            const int s = atomicAdd(&cnt[kbs[u]], 1);
            stg[s] = p[u];
            skb[s] = (unsigned short)kbs[u];
        }
        __syncthreads();
        const int cn = (int)min((int64_t)kChunk, i1 - r0);
        for (int t = threadIdx.x; t < cn; t += T) {
            const int kb = skb[t];
            S[cur[kb] + (t - (kb ? cnt[kb - 1] : 0))] = stg[t];
        }
        __syncthreads();
        for (int k = threadIdx.x; k < K; k += T) cur[k] += cnt[k] - (k ? cnt[k - 1] : 0);
        __syncthreads();
    }
}

// Cell-ordered copies of point d = b0 + t of a CTA's output share [t0, t1)
// (ord holds the share).  A pair block whose partner lies in another share,
// bucket or nowhere (the catalog's last point) is written half by half.
__device__ __forceinline__ void emit_point(const float4 *ord, int t, int t0, int t1, int64_t d, int64_t n,
                                           float *soa, size_t plane, float4 *pk, unsigned *qw, bool fix,
                                           int emin) {
    const float4 p = ord[t - t0];
    if (soa) {
        soa[d] = p.x;
        soa[plane + d] = p.y;
        soa[2 * plane + d] = p.z;
        soa[3 * plane + d] = p.w;
    }
    if (qw) qw[d] = fix ? weight_q(p.w, emin) : 0u;
    if (!(d & 1)) {
        if (t + 1 < t1) {  // block d/2 lies inside the share
            const float4 o = ord[t + 1 - t0];
            pk[d] = make_float4(p.x, o.x, p.y, o.y);
            pk[d + 1] = make_float4(p.z, o.z, p.w, o.w);
        } else if (d + 1 >= n) {
            pk[d] = make_float4(p.x, 0.f, p.y, 0.f);
            pk[d + 1] = make_float4(p.z, 0.f, p.w, 0.f);
        } else {
            pk_put(pk, d, p);  // the partner opens the next share
        }
    } else if (t == t0) {
        pk_put(pk, d, p);  // the partner closes an earlier share
    }
}

// Buckets k = c, c + C, ... for cluster c of C (persistent: a cluster's
// launch and barriers are paid once, and while a bucket's copies are written
// the next bucket's share is prefetched into L2).  Per bucket, CTA r of the
// cluster reads the r-th share of the bucket's points in S and writes the
// r-th share of its cell-ordered output.  A bucket above kCluster *
// kClusterCap points (a very dense region) takes the same counting sort with
// each point's copies written where they land.
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kSortThreads) k_bkt_sort(
    const float4 *__restrict__ S, const int *__restrict__ base, int G, int K, int n, int P, float cell,
    int Q, int ncell, int *__restrict__ cell_start, float *__restrict__ soa, size_t plane,
    float4 *__restrict__ pk, unsigned *__restrict__ qw, const int *__restrict__ flags) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem[];
    float4 *ord = reinterpret_cast<float4 *>(smem);
    int *cnt = reinterpret_cast<int *>(smem + (size_t)kClusterCap * sizeof(float4));  // own counts per cell
    int *off = cnt + kBktMaxCells;                      // this CTA's next slot per cell
    int *tot = reinterpret_cast<int *>(smem);           // cluster counts, then cell starts (in ord's space)
    __shared__ int wsum[32];
    const int r = (int)cl.block_rank();
    const int T = blockDim.x;
    const int C = gridDim.x / kCluster;
    int emin, emax;
    const unsigned *uf = reinterpret_cast<const unsigned *>(flags);
    const bool fix = weight_fix_range(uf[0], uf[1], uf[2], &emin, &emax);
    // the r-th share [j0, j1) of bucket k: offset b0, m points, per per CTA
    auto share = [&](int k, int &b0, int &m, int &per, int &j0, int &j1) {
        b0 = base[(int64_t)k * G];
        m = (k + 1 < K ? base[(int64_t)(k + 1) * G] : n) - b0;
        per = (m + kCluster - 1) / kCluster;
        j0 = min(m, r * per);
        j1 = min(m, j0 + per);
    };
    for (int k = blockIdx.x / kCluster; k < K; k += C) {
        int b0, m, per, j0, j1;
        share(k, b0, m, per, j0, j1);
        const int c0 = k * Q, q = min(Q, ncell - c0);
        for (int i = threadIdx.x; i < q; i += T) cnt[i] = 0;
        __syncthreads();
        for (int j = j0 + threadIdx.x; j < j1; j += kSortUnroll * T) {
            float4 p[kSortUnroll];
#pragma unroll
            for (int u = 0; u < kSortUnroll; ++u)
                if (j + u * T < j1) p[u] = S[b0 + j + u * T];
#pragma unroll
            for (int u = 0; u < kSortUnroll; ++u) {
                if (j + u * T >= j1) break;
                const int lc = cell_of_point(p[u], P, cell) - c0;
                if ((unsigned)lc < (unsigned)q) atomicAdd(&cnt[lc], 1);
            }
        }
        cl.sync();  // every CTA's counts are complete (and every CTA is done with the last bucket's ord)
        for (int i = threadIdx.x; i < q; i += T) {
            int t = 0, pre = 0;
#pragma unroll
            for (int r2 = 0; r2 < kCluster; ++r2) {
                const int v = cl.map_shared_rank(cnt, r2)[i];
                pre += r2 < r ? v : 0;
                t += v;
            }
            tot[i] = t;
            off[i] = pre;
        }
        __syncthreads();
        block_excl_scan4(tot, q, wsum);
        for (int i = threadIdx.x; i < q; i += T) {
            off[i] += tot[i];
            if (r == 0) cell_start[c0 + i] = b0 + tot[i];
        }
        if (k == K - 1 && r == 0 && threadIdx.x == 0) cell_start[ncell] = n;
        cl.sync();  // no CTA reads counts any more, and none still uses tot (ord's space)
        if (per <= kClusterCap) {
            for (int j = j0 + threadIdx.x; j < j1; j += kSortUnroll * T) {
                float4 p[kSortUnroll];
#pragma unroll
                for (int u = 0; u < kSortUnroll; ++u)
                    if (j + u * T < j1) p[u] = S[b0 + j + u * T];  // second read of the share: L2
                const float rper = 1.0f / (float)per;
#pragma unroll
                for (int u = 0; u < kSortUnroll; ++u) {
                    if (j + u * T >= j1) break;
                    const int lc = cell_of_point(p[u], P, cell) - c0;
                    if ((unsigned)lc >= (unsigned)q) continue;
                    const int slot = atomicAdd(&off[lc], 1);
                    const int o = div_q(slot, per, rper);
                    cl.map_shared_rank(ord, o)[slot - o * per] = p[u];
                }
            }
            cl.sync();  // every share is in place
            if (threadIdx.x == 0 && k + C < K) {  // the next bucket's share into L2 meanwhile
                int nb0, nm, nper, nj0, nj1;
                share(k + C, nb0, nm, nper, nj0, nj1);
                if (nj1 > nj0) prefetch_l2(S + nb0 + nj0, (size_t)(nj1 - nj0) * sizeof(float4));
            }
            for (int t = j0 + threadIdx.x; t < j1; t += T)
                emit_point(ord, t, j0, j1, (int64_t)b0 + t, n, soa, plane, pk, qw, fix, emin);
        } else {
            for (int j = j0 + threadIdx.x; j < j1; j += T) {
                const float4 p = S[b0 + j];
                const int lc = cell_of_point(p, P, cell) - c0;
                if ((unsigned)lc >= (unsigned)q) continue;
                const int64_t d = (int64_t)b0 + atomicAdd(&off[lc], 1);
                if (soa) {
                    soa[d] = p.x;
                    soa[plane + d] = p.y;
                    soa[2 * plane + d] = p.z;
                    soa[3 * plane + d] = p.w;
                }
                if (qw) qw[d] = fix ? weight_q(p.w, emin) : 0u;
                pk_put(pk, d, p);  // the partner slot of an odd n's last block is zeroed beforehand
            }
        }
        __syncthreads();  // this CTA's emit is done before its counters are zeroed again
    }
}

// Zero the padding past the catalog: the SoA planes' and integer weights'
// entries n .. plane - 1 and the pair blocks from the one holding point n
// (an odd n leaves that block's second half empty).
__global__ void k_tails(float *__restrict__ soa, size_t plane, int64_t n, float4 *__restrict__ pk,
                        int64_t pk_from, int64_t pk_to, unsigned *__restrict__ qw) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (int64_t)plane - n) {
        if (soa)
            for (int a = 0; a < 4; ++a) soa[a * plane + n + t] = 0.f;
        if (qw) qw[n + t] = 0u;
    }
    if (pk_from + t < pk_to) pk[pk_from + t] = make_float4(0.f, 0.f, 0.f, 0.f);
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

bool grid_bucket_plan(int64_t n, int P, int *Q, int *K) {
    const int64_t ncell = (int64_t)P * P * P;
    if (n < 1 || n > ((int64_t)1 << 30)) return false;
    // mean bucket near kBktTarget points, at least kBktMinBuckets buckets (the
    // sort pass fills the GPU for a small catalog), at most kBktMaxCells
    // cells per bucket
    int64_t k = std::max<int64_t>((n + kBktTarget - 1) / kBktTarget, kBktMinBuckets);
    k = std::max<int64_t>(k, (ncell + kBktMaxCells - 1) / kBktMaxCells);
    k = std::max<int64_t>(1, std::min<int64_t>(k, ncell));
    const int64_t q = (ncell + k - 1) / k;
    k = (ncell + q - 1) / q;
    if (k > kBktMaxBuckets || q > kBktMaxCells) return false;
    *Q = (int)q;
    *K = (int)k;
    return true;
}

size_t grid_bucket_scratch_ints(int G, int K) { return (size_t)G * K + 1; }

cudaError_t grid_bucket_attrs(int device, int K) {
    cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(k_bkt_count), device,
                                      sizeof(int) * (size_t)K);
    if (e == cudaSuccess)
        e = ensure_smem_limit(reinterpret_cast<const void *>(k_bkt_scatter), device, scatter_smem(K));
    if (e == cudaSuccess)
        e = ensure_smem_limit(reinterpret_cast<const void *>(k_bkt_sort), device, kSortSmem);
    return e;
}

// Clusters of the sort that the device runs at once (persistent grid size),
// per device, after the kernel's shared-memory limit is raised.
static int sort_clusters(int device) {
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(device);
    if (it != cache.end()) return it->second;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kCluster * 256);
    cfg.blockDim = dim3(kSortThreads);
    cfg.dynamicSmemBytes = kSortSmem;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, reinterpret_cast<const void *>(k_bkt_sort), &cfg) != cudaSuccess ||
        num < 1) {
        cudaGetLastError();
        num = 16;
    }
    cache[device] = num;
    return num;
}

int launch_grid_build_buckets(const float4 *raw, int64_t n, int P, float cell, float box, int G, int Q,
                              int K, int *M, int *Mx, int *scan_tmp, float4 *S, int *cell_start,
                              float *soa, size_t plane, float4 *pk, unsigned *qw, int *flags,
                              int device, cudaStream_t st) {
    const int ncell = P * P * P;
    const int64_t span = (n + G - 1) / G;
    const size_t hs = sizeof(int) * (size_t)K;
    const float rq = 1.0f / (float)Q;
    k_bkt_count<<<G, kBktThreads, hs, st>>>(raw, n, span, P, cell, box, Q, rq, K, M, flags);
    int launches = 1 + scan_exclusive(M, Mx, (int64_t)G * K, scan_tmp, st);
    k_bkt_scatter<<<G, kBktThreads, scatter_smem(K), st>>>(raw, n, span, P, cell, Q, rq, K, Mx, S);
    const int nclus = std::min(K, sort_clusters(device));
    k_bkt_sort<<<nclus * kCluster, kSortThreads, kSortSmem, st>>>(S, Mx, G, K, (int)n, P, cell, Q, ncell,
                                                              cell_start, soa, plane, pk, qw, flags);
    return launches + 2;
}

int launch_grid_tails(float *soa, size_t plane, int64_t n, float4 *pk, unsigned *qw, cudaStream_t st) {
    const int64_t from = 2 * (n / 2), to = 2 * (int64_t)pk_blocks(n);
    const int64_t m = std::max<int64_t>((int64_t)plane - n, to - from);
    k_tails<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(soa, plane, n, pk, from, to, qw);
    return 1;
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
    PCF_CU(ctx, counted_malloc_host(&ctx->h_pinned, want));
    ctx->h_pinned_bytes = want;
    return PCF_OK;
}

// Build (or rebuild) the cell structure of g for P cells per side.
// A grid keeps the cell structures of the last few partition counts it was
// counted at, so classes of histograms tuned to different partitions do not
// rebuild (and synchronise) on every switch.
pcf_status grid_ensure_cells(pcf_ctx *ctx, pcf_grid *g, int P, bool defer) {
    if (g->cells && g->cells->P == P) return defer ? PCF_OK : grid_finish(ctx, g);
    pcf_status s0 = grid_finish(ctx, g);  // the current structure, before it is replaced
    if (s0 != PCF_OK) return s0;
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
    cg->pk.pool = cg->qw.pool = g->pool;
    PCF_CU(ctx, cg->pk.ensure(32 * pk_blocks(n)));
    PCF_CU(ctx, cg->qw.ensure(sizeof(unsigned) * cg->plane));
    PCF_CU(ctx, cg->cell_start.ensure(sizeof(int) * (size_t)(ncell + 1)));
    int Q = 0, K = 0;
    const int G = ctx->sm_count;
    // the bucketed build pays a fixed cost per bucket (a cluster of four
    // CTAs and three cluster barriers): below ~6M points the per-point build,
    // whose atomics and gathers then stay in L2, is faster (32768 points: 22
    // vs 46 us; 8.4M: 0.36 vs 0.35 ms; 33.5M: 2.04 vs 1.31 ms)
    const bool want_buckets = ctx->grid_build == 2 || (ctx->grid_build == 0 && n >= kBucketBuildMin);
    const bool buckets = want_buckets && grid_bucket_plan(n, P, &Q, &K);
    const size_t mat = buckets ? grid_bucket_scratch_ints(G, K) : 0;
    if (buckets) {
        // scratch: the bucketed copy of the catalog (n float4); the CTA x
        // bucket counts and their scan; scan tmp.
        PCF_CU(ctx, ctx->scratch_a.ensure(sizeof(float4) * (size_t)n));
        PCF_CU(ctx, ctx->scratch_b.ensure(sizeof(int) * 2 * mat));
        PCF_CU(ctx, ctx->scratch_c.ensure(sizeof(int) * (mat / 256 + 256)));
        PCF_CU(ctx, grid_bucket_attrs(ctx->device, K));
    } else {
        // scratch: cid, rank, perm (n each); counts (ncell + 1); scan tmp.
        PCF_CU(ctx, ctx->scratch_a.ensure(sizeof(int) * (size_t)n * 3));
        PCF_CU(ctx, ctx->scratch_b.ensure(sizeof(int) * (size_t)(ncell + 1)));
        PCF_CU(ctx, ctx->scratch_c.ensure(sizeof(int) * (size_t)((ncell + 1) / 256 + 256)));
    }
    PCF_CU(ctx, ctx->d_flag.ensure(sizeof(int) * 4));
    int *flags = ctx->d_flag.as<int>();
    if (!buckets) PCF_CU(ctx, cudaMemsetAsync(ctx->scratch_b.p, 0, sizeof(int) * (size_t)(ncell + 1), st));
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
    ctx->launches += launch_grid_tails(cg->soa.as<float>(), cg->plane, n, cg->pk.as<float4>(),
                                       cg->qw.as<unsigned>(), st);
    if (buckets) {
        int *M = ctx->scratch_b.as<int>();
        ctx->launches += launch_grid_build_buckets(
            g->raw.as<float4>(), n, P, cg->cell, g->box, G, Q, K, M, M + mat, ctx->scratch_c.as<int>(),
            ctx->scratch_a.as<float4>(), cg->cell_start.as<int>(), cg->soa.as<float>(), cg->plane,
            cg->pk.as<float4>(), cg->qw.as<unsigned>(), flags, ctx->device, st);
    } else {
        int *cid = ctx->scratch_a.as<int>();
        ctx->launches += launch_grid_build(g->raw.as<float4>(), n, P, cg->cell, g->box, cid, cid + n,
                                           cid + 2 * n, ctx->scratch_b.as<int>(), cg->cell_start.as<int>(),
                                           ctx->scratch_c.as<int>(), cg->soa.as<float>(), cg->plane,
                                           cg->pk.as<float4>(), cg->qw.as<unsigned>(), flags, st);
    }
    PCF_CU(ctx, cudaGetLastError());
    if (pg1) PCF_CU(ctx, cudaEventRecord(pg1, st));
    // this build's own page-locked block: the cell table and flags come back
    // into it, and the tile table later goes out from it (pageable copies go
    // through the driver's staging, where concurrent contexts were seen to
    // stall one another); sized for both (tiles <= n / kTileCap + the
    // non-empty cells + 1)
    const size_t sb = sizeof(int) * (size_t)(ncell + 1);
    const size_t tile_max = sizeof(TileDesc) * (size_t)(std::min<int64_t>(ncell, n) + n / kTileCap + 2);
    cg->pinned = ctx->pinned;
    PCF_CU(ctx, ctx->pinned->get(std::max(sb + 64, tile_max), &cg->stage, &cg->stage_bytes));
    char *hp = static_cast<char *>(cg->stage);
    PCF_CU(ctx, cudaMemcpyAsync(hp, cg->cell_start.p, sb, cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaMemcpyAsync(hp + sb, flags, 3 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    PCF_CU(ctx, cudaEventCreateWithFlags(&cg->ready, cudaEventDisableTiming));
    PCF_CU(ctx, cudaEventRecord(cg->ready, st));
    cg->pending = true;
    if (g->cells) {
        g->cell_cache.push_back(std::move(g->cells));
        if ((int)g->cell_cache.size() > kCellCache) g->cell_cache.erase(g->cell_cache.begin());
    }
    g->cells = std::move(cg);
    return defer ? PCF_OK : grid_finish(ctx, g);
}

// Completes a queued build: waits for its cell table, checks the catalog's
// flags, sets the weight range and sends the tile table.  A catalog found
// invalid stays marked, so every later use reports it.
pcf_status grid_finish(pcf_ctx *ctx, const pcf_grid *g_) {
    pcf_grid *g = const_cast<pcf_grid *>(g_);
    if (g->bad != PCF_OK) {
        ctx->last_error = "a coordinate lies outside [0, box)";
        return g->bad;
    }
    CellGrid *cg = g->cells.get();
    if (!cg || !cg->pending) return PCF_OK;
    cg->pending = false;
    PCF_CU(ctx, cudaEventSynchronize(cg->ready));
    const int64_t ncell = (int64_t)cg->P * cg->P * cg->P;
    const size_t sb = sizeof(int) * (size_t)(ncell + 1);
    const char *hp = static_cast<const char *>(cg->stage);
    cg->h_start.assign(reinterpret_cast<const int *>(hp), reinterpret_cast<const int *>(hp) + ncell + 1);
    unsigned hf[3];
    memcpy(hf, hp + sb, sizeof(hf));
    if (hf[0] & 1u) {
        g->bad = PCF_ERR_OUT_OF_BOX;
        ctx->last_error = "a coordinate lies outside [0, box)";
        return PCF_ERR_OUT_OF_BOX;
    }
    set_weight_range(g, hf);
    build_tiles(*cg, kTileCap, cg->tiles);
    cg->d_tiles.pool = g->pool;
    PCF_CU(ctx, cg->d_tiles.ensure(sizeof(TileDesc) * std::max<size_t>(1, cg->tiles.size())));
    if (!cg->tiles.empty()) {
        const size_t tb = sizeof(TileDesc) * cg->tiles.size();
        if (tb > cg->stage_bytes) {  // cannot happen: the staging is sized by the bound above
            ctx->last_error = "tile table larger than its staging block";
            return PCF_ERR_CUDA;
        }
        memcpy(cg->stage, cg->tiles.data(), tb);  // the cell table's copy into it has completed
        PCF_CU(ctx, cudaMemcpyAsync(cg->d_tiles.p, cg->stage, tb, cudaMemcpyHostToDevice, ctx->stream));
        PCF_CU(ctx, cudaEventRecord(cg->ready, ctx->stream));
    }
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

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
#include <type_traits>

#include "pcf_internal.cuh"

namespace {

constexpr int kThreads = 128;  // 4 independent warps per CTA
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr float kMagic = 256.0f;  // r + 256 -> low mantissa bits = round(r * 2^15)
constexpr int kFracBits = 15;
constexpr unsigned kFracMask = (1u << kFracBits) - 1u;

enum { H_LANE = 0, H_WARP = 1, H_GLOBAL = 2, H_WFIX = 3 };

// H_WFIX (weighted, per-warp copy): each product w_a*w_b is rounded to an
// integer v = round(w_a*w_b * 2^s) < 2^64 and added as four 16-bit limbs, each
// with a 32-bit shared reduction (several times faster than a 64-bit one).
// A limb counter absorbs kWfixBudget adds of < 2^16 before it could wrap, so a
// warp flushes its copy after at most that many pair tests.
constexpr int kWfixBudget = 65536;
constexpr int kWfixChunk = kWfixBudget / 32;  // candidates per budget check (<= 32 homes each)

// Fast-path cut constants for one range type (0: unshifted, 1: image-shifted).
struct FastCuts {
    float dsf;        // (float)ds
    float ds2;        // dsf * dsf
    float lo[2];      // d2 below lo (and >= tiny) is safely inside dmax
    float hi[2];      // d2 at or above hi is safely outside dmax
    unsigned w[2];    // edge window in 2^-15 units of r
    float tiny;
};

struct PairArgs {
    const PairJob *jobs;  // histograms of this launch, items laid out job after job
    int n_jobs;
    long long n_items;
    unsigned long long *counter;
    int P;
    float box;
    int bpc;
    PairRule rule;
    FastCuts fc;
    unsigned long long *g_count;
    double *g_wsum;
    unsigned long long *g_stats;
    float wscale;     // H_WFIX: 2^s, applied to the home weight
    double wunscale;  // H_WFIX: 2^-s
    int wlimbs;       // H_WFIX: limbs per bin (3: v < 2^48, 4: v < 2^64)
};

__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Fixed-point readout of r in [0, 256): q = round(r * 2^15).  The bin
// (q >> 15) is exact unless r is within w/2^15 of an integer.
__device__ __forceinline__ bool fix_safe(unsigned q, unsigned w) {
    return ((q + w) & kFracMask) >= 2u * w;
}

// Predicated shared / global reductions (one instruction, no branch).
__device__ __forceinline__ void red_s_u32(const void *p, unsigned v, bool pred) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q red.shared.add.u32 [%0], %1;\n\t}"
                 :: "r"(a), "r"(v), "r"((unsigned)pred) : "memory");
}
__device__ __forceinline__ void red_s_f64(const void *p, double v, bool pred) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t@q red.shared.add.f64 [%0], %1;\n\t}"
                 :: "r"(a), "d"(v), "r"((unsigned)pred) : "memory");
}

// Histogram sinks.  H_LANE: one u32 / f64 column per lane (iso, few bins),
// no contention; H_WARP: one copy per warp with shared atomics; H_GLOBAL:
// global atomics (very wide histograms).  add() is predicated on `pred`.
template <bool WEIGHTED, int HM>
struct Sink {
    void *base;  // shared: this warp's region (lane column folded in); global: g_count / g_wsum
    int plane;   // H_WFIX: u32 words between limb planes (bins of the histogram)
    bool four;   // H_WFIX: the top limb is in use
    __device__ __forceinline__ void add(int slot, float wa, float wb, bool pred) const {
        if (HM == H_WFIX) {  // wa carries the 2^s scale; w_a*w_b is exact in FP64
            const unsigned long long v = __double2ull_rn((double)wa * (double)wb);
            unsigned *b = static_cast<unsigned *>(base) + slot;
            const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
            red_s_u32(b, lo & 0xFFFFu, pred);
            red_s_u32(b + plane, lo >> 16, pred);
            red_s_u32(b + 2 * plane, hi & 0xFFFFu, pred);
            red_s_u32(b + 3 * plane, hi >> 16, pred && four);
        } else if (HM == H_LANE) {
            if (WEIGHTED) {  // lane-private column: unconditional add of 0 or w_a*w_b,
                // so a lane without a pair (its slot undefined) adds 0 to slot 0
                double *h = static_cast<double *>(base) + (pred ? slot : 0) * 32;
                *h += pred ? (double)wa * (double)wb : 0.0;
            } else {
                red_s_u32(static_cast<unsigned *>(base) + slot * 32, 1u, pred);
            }
        } else if (HM == H_WARP) {
            if (WEIGHTED) red_s_f64(static_cast<double *>(base) + slot, (double)wa * (double)wb, pred);
            else red_s_u32(static_cast<unsigned *>(base) + slot, 1u, pred);
        } else if (pred) {
            if (WEIGHTED) atomicAdd(static_cast<double *>(base) + slot, (double)wa * (double)wb);
            else atomicAdd(static_cast<unsigned long long *>(base) + slot, 1ull);
        }
    }
};

struct Home {
    float x, y, z, w;  // original coordinates
};

struct Seg {
    float sx, sy, sz;  // image shift of the candidates
    float lo, hi;
    unsigned w;
    unsigned rule_flags;
};

// Canonical FP64 decision for one pair (rare path): histogram slot or -1.
template <bool ANI>
__device__ __noinline__ int slow_slot(float hx, float hy, float hz, float cx, float cy, float cz,
                                      float sx, float sy, float sz, PairRule rule) {
    double dx, dy, dz;
    exact_sep(hx, hy, hz, cx, cy, cz, sx, sy, sz, dx, dy, dz);
    return exact_slot<ANI>(dx, dy, dz, rule);
}

template <bool ANI, bool WEIGHTED, int HM>
__device__ __forceinline__ void slow_pair(const PairArgs &A, const GridView &C, const Home &h,
                                          const Seg &sg, int j, const Sink<WEIGHTED, HM> &sink,
                                          unsigned &n_pairs) {
    PairRule rule = A.rule;
    rule.flags = sg.rule_flags;
    const int slot = slow_slot<ANI>(h.x, h.y, h.z, __ldg(C.x + j), __ldg(C.y + j), __ldg(C.z + j),
                                    sg.sx, sg.sy, sg.sz, rule);
    if (slot >= 0) {
        sink.add(slot, h.w, WEIGHTED ? __ldg(C.w + j) : 1.f, true);
        if (WEIGHTED) ++n_pairs;
    }
}

// Adds this warp's histogram copy into histogram `slot` of the launch and
// clears it (job change or end of the queue).
template <bool WEIGHTED, int HM>
__device__ __forceinline__ void flush_hist(typename std::conditional<WEIGHTED, double, unsigned>::type *mine,
                                           int nb, int per_warp, int lane, const PairArgs &A,
                                           int slot) {
    typedef typename std::conditional<WEIGHTED, double, unsigned>::type HT;
    if (HM == H_GLOBAL) return;
    __syncwarp();
    const size_t off = (size_t)slot * nb;
    if (HM == H_LANE) {
        for (int k = 0; k < nb; ++k) {
            HT s = mine[k * 32 + lane];
            mine[k * 32 + lane] = (HT)0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
            if (lane == 0 && s != (HT)0) {
                if (WEIGHTED) atomicAdd(A.g_wsum + off + k, (double)s);
                else atomicAdd(A.g_count + off + k, (unsigned long long)s);
            }
        }
    } else {
        for (int k = lane; k < nb; k += 32) {
            const HT s = mine[k];
            mine[k] = (HT)0;
            if (s != (HT)0) {
                if (WEIGHTED) atomicAdd(A.g_wsum + off + k, (double)s);
                else atomicAdd(A.g_count + off + k, (unsigned long long)s);
            }
        }
    }
    __syncwarp();
    (void)per_warp;
}

__device__ __forceinline__ void flush_wfix(unsigned *mine, int nb, int limbs, int lane,
                                           const PairArgs &A, int slot);
template <bool WEIGHTED, int HM, typename HT>
__device__ __forceinline__ void flush_any(HT *mine, int nb, int per_warp, int lane, const PairArgs &A,
                                          int slot) {
    if (HM == H_WFIX) flush_wfix(reinterpret_cast<unsigned *>(mine), nb, A.wlimbs, lane, A, slot);
    else flush_hist<WEIGHTED, HM>(reinterpret_cast<typename std::conditional<WEIGHTED, double, unsigned>::type *>(mine),
                                  nb, per_warp, lane, A, slot);
}

// H_WFIX flush: limbs -> FP64 sum * 2^-s into histogram `slot`; clears the copy.
__device__ __forceinline__ void flush_wfix(unsigned *mine, int nb, int limbs, int lane,
                                           const PairArgs &A, int slot) {
    __syncwarp();
    const size_t off = (size_t)slot * nb;
    for (int k = lane; k < nb; k += 32) {
        const unsigned l0 = mine[k], l1 = mine[nb + k], l2 = mine[2 * nb + k];
        const unsigned l3 = limbs == 4 ? mine[3 * nb + k] : 0u;
        mine[k] = 0u;
        mine[nb + k] = 0u;
        mine[2 * nb + k] = 0u;
        if (limbs == 4) mine[3 * nb + k] = 0u;
        if (l0 | l1 | l2 | l3) {
            // each term is exact; the sum of the four rounds once or twice
            const double v = ((double)l3 * 0x1p48 + (double)l2 * 0x1p32) + ((double)l1 * 0x1p16 + (double)l0);
            atomicAdd(A.g_wsum + off + k, v * A.wunscale);
        }
    }
    __syncwarp();
}

// One candidate pair of elements (packed): distance test, fixed-point bin,
// predicated accumulate.  Pairs within the edge window of a bin, near dmax,
// or at zero separation (frac(r) = 0 fails the window test) go to the FP64
// rule, behind one warp-uniform branch.
template <bool ANI, bool WEIGHTED, int HM>
__device__ __forceinline__ void take2(const PairArgs &A, const GridView &C, float2 DX, float2 DY,
                                      float2 DZ, bool v0,
                                      bool v1, int j, float2 Wt, const Home &h, const Seg &sg,
                                      const Sink<WEIGHTED, HM> &sink, unsigned &n_pairs,
                                      unsigned &n_rechk) {
    const FastCuts &fc = A.fc;
    const float2 DS2 = make_float2(fc.ds2, fc.ds2);
    const float2 MG = make_float2(kMagic, kMagic);
    bool f0 = false, f1 = false;
    float m0, m1;  // largest squared component, for the recheck test
    if (!ANI) {
        float2 D2 = __fmul2_rn(DX, DX);
        D2 = __ffma2_rn(DY, DY, D2);
        D2 = __ffma2_rn(DZ, DZ, D2);
        m0 = D2.x;
        m1 = D2.y;
        if (HM != H_GLOBAL) {
            const float2 U = __fmul2_rn(D2, DS2);
            const float2 Q = __fadd2_rn(make_float2(sqrt_approx(U.x), sqrt_approx(U.y)), MG);
            const unsigned q0 = __float_as_uint(Q.x) & 0x7FFFFFu;
            const unsigned q1 = __float_as_uint(Q.y) & 0x7FFFFFu;
            f0 = v0 && (D2.x < sg.lo) && fix_safe(q0, sg.w);
            f1 = v1 && (D2.y < sg.lo) && fix_safe(q1, sg.w);
            // f0 / f1 imply r < bins away from an edge, so q >> 15 <= bins - 1
            sink.add((int)(q0 >> kFracBits), h.w, Wt.x, f0);
            sink.add((int)(q1 >> kFracBits), h.w, Wt.y, f1);
        }
    } else {
        const float2 ZZ = __fmul2_rn(DZ, DZ);
        const float2 PP = __ffma2_rn(DY, DY, __fmul2_rn(DX, DX));
        m0 = fmaxf(ZZ.x, PP.x);
        m1 = fmaxf(ZZ.y, PP.y);
        if (HM != H_GLOBAL) {
            const float2 RZ = __fmul2_rn(DZ, make_float2(fc.dsf, fc.dsf));
            const float2 U = __fmul2_rn(PP, DS2);
            const float2 QZ = __fadd2_rn(make_float2(fabsf(RZ.x), fabsf(RZ.y)), MG);
            const float2 QP = __fadd2_rn(make_float2(sqrt_approx(U.x), sqrt_approx(U.y)), MG);
            const unsigned z0 = __float_as_uint(QZ.x) & 0x7FFFFFu, z1 = __float_as_uint(QZ.y) & 0x7FFFFFu;
            const unsigned p0 = __float_as_uint(QP.x) & 0x7FFFFFu, p1 = __float_as_uint(QP.y) & 0x7FFFFFu;
            f0 = v0 && (m0 < sg.lo) && fix_safe(z0, sg.w) && fix_safe(p0, sg.w);
            f1 = v1 && (m1 < sg.lo) && fix_safe(z1, sg.w) && fix_safe(p1, sg.w);
            const int B = A.rule.bins;
            sink.add((int)(z0 >> kFracBits) * B + (int)(p0 >> kFracBits), h.w, Wt.x, f0);
            sink.add((int)(z1 >> kFracBits) * B + (int)(p1 >> kFracBits), h.w, Wt.y, f1);
        }
    }
    if (WEIGHTED) n_pairs += (unsigned)f0 + (unsigned)f1;
    const bool r0 = !f0 && v0 && m0 < sg.hi;
    const bool r1 = !f1 && v1 && m1 < sg.hi;
    // Lanes of different candidate streams leave the stream loop after
    // different trip counts, so vote only among the lanes that are here.
    if (__any_sync(__activemask(), r0 || r1)) {
        if (r0) {
            ++n_rechk;
            slow_pair<ANI, WEIGHTED, HM>(A, C, h, sg, j, sink, n_pairs);
        }
        if (r1) {
            ++n_rechk;
            slow_pair<ANI, WEIGHTED, HM>(A, C, h, sg, j + 1, sink, n_pairs);
        }
    }
}

#ifndef PCF_PAIR_MINB
#define PCF_PAIR_MINB 6
#endif
template <bool ANI, bool WEIGHTED, int HM>
// H_WFIX copies take 3-4x the shared memory of a u32 copy, which already
// holds those launches to ~5 CTAs per SM: let them use the registers of 5.
__global__ void __launch_bounds__(kThreads, HM == H_WFIX ? 5 : PCF_PAIR_MINB) k_pairs(const PairArgs A) {
    typedef typename std::conditional<WEIGHTED && HM != H_WFIX, double, unsigned>::type HT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HT *hist_all = reinterpret_cast<HT *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int bins = A.rule.bins;
    const int nb = ANI ? bins * bins : bins;
    const int per_warp = HM == H_LANE ? nb * 32 : (HM == H_WARP ? nb : (HM == H_WFIX ? nb * A.wlimbs : 0));
    HT *mine = hist_all + warp * per_warp;
    for (int k = lane; k < per_warp; k += 32) mine[k] = (HT)0;
    __syncwarp();
    Sink<WEIGHTED, HM> sink;
    if (HM != H_GLOBAL) sink.base = HM == H_LANE ? (void *)(mine + lane) : (void *)mine;
    sink.plane = nb;
    sink.four = A.wlimbs == 4;
    int wfix_since = 0;  // H_WFIX: pair tests since this warp's last flush
    unsigned n_pairs = 0, n_rechk = 0;
    unsigned long long n_cand = 0;
    // current job (items of one warp arrive in increasing order), kept in
    // shared memory to spare registers
    __shared__ PairJob s_job[kWarps];
    PairJob &J = s_job[warp];
    int cj = -1, slot = 0;
    long long job_end = -1;

    long long next = 0;
    if (lane == 0) next = (long long)atomicAdd(A.counter, 1ull);
    next = __shfl_sync(kFull, next, 0);
    while (next < A.n_items) {
        const long long it_idx = next;
        if (lane == 0) next = (long long)atomicAdd(A.counter, 1ull);  // prefetch the next item
        if (it_idx >= job_end) {  // entering another job: flush this one's histogram
            if (cj >= 0) flush_any<WEIGHTED, HM>(mine, nb, per_warp, lane, A, slot);
            wfix_since = 0;
            do {
                ++cj;
                job_end = cj + 1 < A.n_jobs ? A.jobs[cj + 1].item_begin : A.n_items;
            } while (it_idx >= job_end);
            {
                static_assert(sizeof(PairJob) % 4 == 0, "PairJob words");
                const int *src = reinterpret_cast<const int *>(A.jobs + cj);
                int *dst = reinterpret_cast<int *>(&J);
                for (int q = lane; q < (int)(sizeof(PairJob) / 4); q += 32) dst[q] = src[q];
                __syncwarp();
            }
            slot = J.slot;
            if (HM == H_GLOBAL)
                sink.base = WEIGHTED ? (void *)(A.g_wsum + (size_t)slot * nb)
                                     : (void *)(A.g_count + (size_t)slot * nb);
        }
        const long long loc = it_idx - J.item_begin;
        const int tile = (int)(loc / J.n_chunks);
        const int chunk = (int)(loc - (long long)tile * J.n_chunks);
        const int row_begin = chunk * J.rows_per_item;
        const int row_end = min(row_begin + J.rows_per_item, J.n_rows);
        const TileDesc t = J.tiles[tile];
        const int H = t.count;                 // 1..32 home points
        const int S = 32 / H;                  // candidate streams per warp
        const int sidx = lane / H;             // this lane's stream
        const int hl = lane - sidx * H;        // this lane's home point
        const bool valid = sidx < S;
        const int hidx = t.start + hl;
        Home h;
        if (valid) {
            h.x = J.home.x[hidx]; h.y = J.home.y[hidx]; h.z = J.home.z[hidx]; h.w = J.home.w[hidx];
            if (HM == H_WFIX) h.w *= A.wscale;  // exact: a power of two, range checked by the host
        } else {
            h.x = h.y = h.z = __int_as_float(0x7fc00000);  // NaN: never in range
            h.w = 0.f;
        }
        // Candidate ranges of all rows of the item, one row per lane, so the
        // dependent cell-table loads of different rows overlap.
        const int nrows = row_end - row_begin;  // <= 32 (planner)
        int ra0 = 0, rb0 = 0, ra1 = 0, rb1 = 0, rkind = 0;
        float rsx = 0.f, rsy = 0.f, rsz1 = 0.f;
        if (lane < nrows) {
            const RowDesc rw = J.rows[row_begin + lane];
            int nx = t.ix + rw.dx, ny = t.iy + rw.dy;
            const int P = A.P;
            bool ok = true;
            if (A.bpc) {
                if (nx < 0) { nx += P; rsx = -A.box; } else if (nx >= P) { nx -= P; rsx = A.box; }
                if (ny < 0) { ny += P; rsy = -A.box; } else if (ny >= P) { ny -= P; rsy = A.box; }
            } else if (nx < 0 || nx >= P || ny < 0 || ny >= P) {
                ok = false;
            }
            if (ok) {
                const int col = (nx * P + ny) * P;
                const int zhi = t.z1 + rw.kz;
                rkind = rw.kind;
                const int *cs = J.cand.cstart;
                if (rw.kind == 1) {  // forward half of the home column (XX): j > home index
                    ra0 = t.start;
                    rb0 = cs[col + min(zhi, P - 1) + 1];
                    if (A.bpc && zhi >= P) { ra1 = cs[col]; rb1 = cs[col + zhi - P + 1]; rsz1 = A.box; }
                } else {
                    const int zlo = t.z0 - rw.kz;
                    ra0 = cs[col + max(zlo, 0)];
                    rb0 = cs[col + min(zhi, P - 1) + 1];
                    if (A.bpc) {
                        if (zlo < 0) { ra1 = cs[col + zlo + P]; rb1 = cs[col + P]; rsz1 = -A.box; }
                        else if (zhi >= P) { ra1 = cs[col]; rb1 = cs[col + zhi - P + 1]; rsz1 = A.box; }
                    }
                }
            }
        }
        for (int r = 0; r < nrows; ++r) {
            const int a0 = __shfl_sync(kFull, ra0, r), b0 = __shfl_sync(kFull, rb0, r);
            const int a1 = __shfl_sync(kFull, ra1, r), b1 = __shfl_sync(kFull, rb1, r);
            const int kind = __shfl_sync(kFull, rkind, r);
            const float sx = __shfl_sync(kFull, rsx, r), sy = __shfl_sync(kFull, rsy, r);
            const float sz1 = __shfl_sync(kFull, rsz1, r);
            #pragma unroll 1
            for (int seg = 0; seg < 2; ++seg) {
                const int a = seg ? a1 : a0, b = seg ? b1 : b0;
                if (a >= b) continue;
                Seg sg;
                sg.sx = sx; sg.sy = sy; sg.sz = seg ? sz1 : 0.f;
                const int sh = (sg.sx != 0.f || sg.sy != 0.f || sg.sz != 0.f) ? 1 : 0;
                sg.lo = A.fc.lo[sh];
                sg.hi = A.fc.hi[sh];
                sg.w = A.fc.w[sh];
                sg.rule_flags = J.rule_flags;
                const float2 NHX = make_float2(sg.sx - h.x, sg.sx - h.x);
                const float2 NHY = make_float2(sg.sy - h.y, sg.sy - h.y);
                const float2 NHZ = make_float2(sg.sz - h.z, sg.sz - h.z);
                const int jmin = (kind == 1 && seg == 0) ? hidx : a - 1;
                if (lane == 0) n_cand += (unsigned long long)(b - a) * (unsigned long long)H;
                // one aligned pair of candidates (p, p+1); v0 / v1 say which are real
                auto step = [&](int p, bool v0, bool v1) {
                    const float2 X = __ldg(reinterpret_cast<const float2 *>(J.cand.x + p));
                    const float2 Y = __ldg(reinterpret_cast<const float2 *>(J.cand.y + p));
                    const float2 Z = __ldg(reinterpret_cast<const float2 *>(J.cand.z + p));
                    float2 Wt = make_float2(1.f, 1.f);
                    if (WEIGHTED) Wt = __ldg(reinterpret_cast<const float2 *>(J.cand.w + p));
                    // (x_j + shift) - x_home, rounded once: same value as the
                    // scalar (x_j - (x_home - shift)) up to the bound in make_cuts
                    const float2 DX = __fadd2_rn(X, NHX);
                    const float2 DY = __fadd2_rn(Y, NHY);
                    const float2 DZ = __fadd2_rn(Z, NHZ);
                    take2<ANI, WEIGHTED, HM>(A, J.cand, DX, DY, DZ, v0, v1, p, Wt, h, sg, sink,
                                             n_pairs, n_rechk);
                };
                // head: pairs that start before a, or that reach into the home
                // tile of a forward row (j > home index per lane); body: pairs
                // fully inside (a, b) past the tile, no checks; tail: the last
                // pair when it ends at b
                const int chk = (kind == 1 && seg == 0) ? t.start + H : a + 1;
                const int a2 = a & ~1;
                const int stride = 2 * S;
                // candidates [lo, hi) (lo even; hi even or b)
                auto run = [&](int lo, int hi) {
                    int p = lo + 2 * sidx;
                    for (; p < hi && p < chk; p += stride)
                        step(p, p > jmin && p >= a, (p + 1 < b) && (p + 1 > jmin));
                    #pragma unroll 2
                    for (; p + 1 < hi; p += stride) step(p, true, true);
                    if (p < hi) step(p, true, false);
                };
                if (HM == H_WFIX) {  // flush before a limb counter could wrap
                    for (int lo = a2; lo < b; lo += kWfixChunk) {
                        const int hi = min(b, lo + kWfixChunk);
                        const int tests = (hi - lo) * H;
                        if (wfix_since + tests > kWfixBudget) {
                            flush_any<WEIGHTED, HM>(mine, nb, per_warp, lane, A, slot);
                            wfix_since = 0;
                        }
                        wfix_since += tests;
                        run(lo, hi);
                    }
                } else {
                    run(a2, b);
                }
            }
        }
        next = __shfl_sync(kFull, next, 0);
    }
    // per-warp flush (no CTA barrier: warps leave as the queue drains)
    __syncwarp();
    if (cj >= 0) flush_any<WEIGHTED, HM>(mine, nb, per_warp, lane, A, slot);
    unsigned long long rp = n_pairs, rr = n_rechk;
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(kFull, rr, off);
        rp += __shfl_down_sync(kFull, rp, off);
    }
    if (lane == 0) {
        if (rr) atomicAdd(A.g_stats + 0, rr);
        if (n_cand) atomicAdd(A.g_stats + 1, n_cand);
        if (rp) atomicAdd(A.g_stats + 2, rp);
    }
}

// Several histograms: out[s*nb + k] = mult[s] * hist[s*nb + k].
__global__ void k_finalize_slots(const unsigned long long *__restrict__ cnt,
                                 const double *__restrict__ ws, int weighted,
                                 const double *__restrict__ mult, int nb, int nslots,
                                 double *__restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * nslots) return;
    const int s = (int)(t / nb);
    out[t] = mult[s] * (weighted ? ws[t] : (double)cnt[t]);
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
void build_tiles(CellGrid &g) {
    const int P = g.P;
    const std::vector<int> &hs = g.h_start;
    g.tiles.clear();
    for (int ix = 0; ix < P; ++ix)
        for (int iy = 0; iy < P; ++iy)
            for (int iz = 0; iz < P; ++iz) {
                const int c = (ix * P + iy) * P + iz;
                const int s0 = hs[c], n = hs[c + 1] - s0;
                for (int o = 0; o < n; o += kTileCap) {
                    TileDesc t;
                    t.start = s0 + o;
                    t.count = std::min(kTileCap, n - o);
                    t.ix = (int16_t)ix;
                    t.iy = (int16_t)iy;
                    t.z0 = t.z1 = (int16_t)iz;
                    g.tiles.push_back(t);
                }
            }
}

void plan_rows(int P, float box, float dmax, bool ani, bool self, std::vector<RowDesc> &rows) {
    const double cell = (double)box / P;
    const double R = (double)dmax;
    // margin for points that sit a rounding step outside their cell
    const double margin = 1e-4 * cell + 8.0 * (double)box * 1.2e-7;
    const double Rm = R + margin;
    const int k = (int)std::ceil(Rm / cell);
    rows.clear();
    for (int dx = -k; dx <= k; ++dx) {
        for (int dy = -k; dy <= k; ++dy) {
            const double mx = std::max(std::abs(dx) - 1, 0) * cell;
            const double my = std::max(std::abs(dy) - 1, 0) * cell;
            const double mxy2 = mx * mx + my * my;
            if (mxy2 >= Rm * Rm) continue;
            int kz = k;  // ani: cylinder |dz| < dmax
            if (!ani) {  // iso: max(|dz|-1,0)*cell < sqrt(R^2 - mxy^2)
                const double rem = std::sqrt(std::max(Rm * Rm - mxy2, 0.0));
                kz = std::min(k, (int)std::ceil(rem / cell));
            }
            RowDesc r;
            r.dx = (int16_t)dx;
            r.dy = (int16_t)dy;
            r.kz = (int16_t)kz;
            r.kind = 0;
            if (self) {
                if (dx == 0 && dy == 0) {
                    r.kind = 1;  // forward half of the home column
                    rows.insert(rows.begin(), r);
                    continue;
                }
                if (!(dx > 0 || (dx == 0 && dy > 0))) continue;  // half shell
            }
            rows.push_back(r);
        }
    }
}

void plan_pairs(const CellGrid &home, float box, float dmax, bool ani, bool self, PairPlan &plan,
                int resident_warps) {
    const int P = home.P;
    plan.P = P;
    plan.cell = (float)((double)box / P);
    plan_rows(P, box, dmax, ani, self, plan.rows);
    // ~16 items per resident warp keeps the tail short; at most 32 rows each
    const int64_t nt = (int64_t)home.tiles.size();
    const int64_t nr = (int64_t)plan.rows.size();
    const int64_t want = std::max<int64_t>(1, (int64_t)resident_warps * 16);
    int rpi = (int)std::min<int64_t>(32, std::max<int64_t>(1, (nt * nr) / want));
    plan.rows_per_item = rpi;
    plan.n_chunks = (int)((nr + rpi - 1) / rpi);
    plan.n_items = nt * plan.n_chunks;
}

// ---------------------------------------------------------------------------
// Launch one pair histogram (device side; result left in d_out as doubles).
// ---------------------------------------------------------------------------
static FastCuts make_cuts(const PairRule &rule, float box, float dmax) {
    FastCuts fc;
    fc.dsf = (float)rule.ds;
    fc.ds2 = fc.dsf * fc.dsf;
    const double dd = rule.dd;
    const double rmax = (double)dmax * rule.ds + 1.0;  // r units
    // Relative FP32 error of d2 (one rounding in each difference, then the
    // FMA chain) stays below ~2^-21, and of r = sqrt.approx(d2*ds^2) below
    // ~2^-20: the windows below keep an 8x margin over those bounds.
    const double e_plain_d2 = dd * std::ldexp(1.0, -17);
    const double w_plain = rmax * std::ldexp(1.0, -17);
    // image-shifted home point: |error of dx| <= L*2^-23 per axis
    const double e_shift_d2 = e_plain_d2 + (double)dmax * (double)box * std::ldexp(1.0, -19);
    const double w_shift = w_plain + rule.ds * (double)box * std::ldexp(1.0, -19);
    fc.lo[0] = (float)(dd - e_plain_d2);
    fc.hi[0] = (float)(dd + e_plain_d2);
    fc.lo[1] = (float)(dd - e_shift_d2);
    fc.hi[1] = (float)(dd + e_shift_d2);
    // + quantisation of the fixed-point readout (2^-16)
    fc.w[0] = std::min(8000u, (unsigned)std::ceil((w_plain + std::ldexp(1.0, -16)) * 32768.0) + 1u);
    fc.w[1] = std::min(8000u, (unsigned)std::ceil((w_shift + std::ldexp(1.0, -16)) * 32768.0) + 1u);
    fc.tiny = 1e-30f;
    return fc;
}

template <bool ANI, bool W, int HM>
static cudaError_t launch_one(const PairArgs &A, size_t smem, long long n_items, cudaStream_t st,
                              int sm_count, int device) {
    auto kfn = k_pairs<ANI, W, HM>;
    // attribute / occupancy queries cost microseconds each: do them once per
    // (device, variant, shared-memory size)
    constexpr int kDev = 64;
    static size_t attr_smem[kDev] = {};
    static size_t occ_smem[kDev];
    static int occ_per_sm[kDev];
    static bool init = false;
    if (!init) {
        for (int d = 0; d < kDev; ++d) occ_smem[d] = ~(size_t)0;
        init = true;
    }
    const int dv = (device >= 0 && device < kDev) ? device : 0;
    cudaError_t e;
    if (smem > 48 * 1024 && smem > attr_smem[dv]) {
        e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_smem[dv] = smem;
    }
    if (occ_smem[dv] != smem) {
        int per = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, kThreads, smem);
        if (e != cudaSuccess) return e;
        occ_per_sm[dv] = std::max(1, per);
        occ_smem[dv] = smem;
    }
    const long long want = (n_items + kWarps - 1) / kWarps;
    const int grid = (int)std::max(1LL, std::min<long long>(want, (long long)sm_count * occ_per_sm[dv]));
    kfn<<<grid, kThreads, smem, st>>>(A);
    return cudaGetLastError();
}

// Chooses the histogram mode of one launch and starts the kernel.
static cudaError_t dispatch_pairs(const PairArgs &A, const PairLaunch &pl, cudaStream_t st,
                                  int sm_count, int device) {
    const int nb = pl.ani ? pl.rule.bins * pl.rule.bins : pl.rule.bins;
    const size_t ebytes = pl.weighted ? 8 : 4;
    const size_t lane_bytes = (size_t)nb * 32 * kWarps * ebytes;
    const size_t warp_bytes = (size_t)nb * kWarps * ebytes;
    int hm;
    size_t smem;
    const bool wfix_ok = pl.weighted && pl.wlimbs >= 3 && pl.rule.bins <= 255;
    const size_t wfix_bytes = (size_t)nb * 4 * pl.wlimbs * kWarps;
    if (pl.rule.bins > 255 || warp_bytes > 160 * 1024) { hm = H_GLOBAL; smem = 0; }
    else if (!pl.ani && lane_bytes <= 64 * 1024) { hm = H_LANE; smem = lane_bytes; }
    else { hm = H_WARP; smem = warp_bytes; }
    if (hm == H_WARP && wfix_ok && wfix_bytes <= 160 * 1024) { hm = H_WFIX; smem = wfix_bytes; }
    // an autotuned scheme overrides the rule above when it is valid here
    if (pl.hist_mode == H_GLOBAL) { hm = H_GLOBAL; smem = 0; }
    else if (pl.hist_mode == H_WFIX && wfix_ok && wfix_bytes <= 160 * 1024) {
        hm = H_WFIX; smem = wfix_bytes;
    }
    else if (pl.hist_mode == H_WARP && pl.rule.bins <= 255 && warp_bytes <= 160 * 1024) {
        hm = H_WARP; smem = warp_bytes;
    } else if (pl.hist_mode == H_LANE && !pl.ani && pl.rule.bins <= 255 && lane_bytes <= 64 * 1024) {
        hm = H_LANE; smem = lane_bytes;
    }
    const long long n = A.n_items;
#define PCF_DISPATCH(ANI_)                                                                       \
    if (pl.weighted) {                                                                           \
        if (hm == H_LANE) return launch_one<ANI_, true, H_LANE>(A, smem, n, st, sm_count, device);   \
        if (hm == H_WARP) return launch_one<ANI_, true, H_WARP>(A, smem, n, st, sm_count, device);   \
        if (hm == H_WFIX) return launch_one<ANI_, true, H_WFIX>(A, smem, n, st, sm_count, device);   \
        return launch_one<ANI_, true, H_GLOBAL>(A, smem, n, st, sm_count, device);                 \
    } else {                                                                                     \
        if (hm == H_LANE) return launch_one<ANI_, false, H_LANE>(A, smem, n, st, sm_count, device);  \
        if (hm == H_WARP) return launch_one<ANI_, false, H_WARP>(A, smem, n, st, sm_count, device);  \
        return launch_one<ANI_, false, H_GLOBAL>(A, smem, n, st, sm_count, device);                \
    }
    if (pl.ani) { PCF_DISPATCH(true) } else { PCF_DISPATCH(false) }
#undef PCF_DISPATCH
}

static PairArgs make_args(const PairJob *jobs, int n_jobs, long long n_items,
                          unsigned long long *counter, int P, float box, const PairLaunch &pl,
                          unsigned long long *d_count, double *d_wsum,
                          unsigned long long *d_stats) {
    PairArgs A;
    A.jobs = jobs;
    A.n_jobs = n_jobs;
    A.n_items = n_items;
    A.counter = counter;
    A.P = P;
    A.box = box;
    A.bpc = pl.bpc ? 1 : 0;
    A.rule = pl.rule;
    A.fc = make_cuts(pl.rule, box, std::sqrt((float)pl.rule.dd));
    A.g_count = d_count;
    A.g_wsum = d_wsum;
    A.g_stats = d_stats;
    A.wscale = pl.wscale;
    A.wunscale = pl.wlimbs ? 1.0 / (double)pl.wscale : 0.0;
    A.wlimbs = pl.wlimbs;
    return A;
}

// Scale of the fixed-point weighted histograms of a launch whose points come
// from grids gs[0..n): s such that every nonzero product w_a*w_b is at least
// 2^42 after scaling (rounding it costs at most 2^-43 of its value), with
// the largest below 2^48 (three limbs) or 2^64 (four).  Weights must be
// finite and >= 0, and each weight * 2^s a normal float.  Otherwise the
// launch keeps FP64 shared atomics (wlimbs = 0).
void set_weight_fix(PairLaunch &pl, const pcf_grid *const *gs, int n) {
    pl.wscale = 0.f;
    pl.wlimbs = 0;
    if (!pl.weighted) return;
    double wmin = 0.0, wmax = 0.0;
    for (int i = 0; i < n; ++i) {
        const pcf_grid *g = gs[i];
        if (!g->w_finite_nonneg) return;
        wmax = std::max(wmax, (double)g->w_absmax);
        if (g->w_absmin > 0.f) wmin = wmin > 0.0 ? std::min(wmin, (double)g->w_absmin) : (double)g->w_absmin;
    }
    if (!(wmin > 0.0)) return;
    const double pmin = wmin * wmin, pmax = wmax * wmax;  // exact: 24-bit mantissas
    const int s = 42 - (int)std::floor(std::log2(pmin));
    if (s < -120 || s > 120) return;
    const double top = std::ldexp(pmax, s);
    int limbs;
    if (top < std::ldexp(1.0, 48) - 1.0) limbs = 3;
    else if (top < std::ldexp(1.0, 64) - 4096.0) limbs = 4;
    else return;
    if (std::ldexp(wmin, s) < std::ldexp(1.0, -125) || std::ldexp(wmax, s) >= std::ldexp(1.0, 126)) return;
    pl.wscale = std::ldexp(1.0f, s);
    pl.wlimbs = limbs;
}

cudaError_t launch_pair_jobs(const PairJob *d_jobs, int n_jobs, long long n_items, int P, float box,
                             const PairLaunch &pl, unsigned long long *counter,
                             unsigned long long *d_count, double *d_wsum,
                             unsigned long long *d_stats, cudaStream_t st, int sm_count, int device) {
    if (n_items == 0) return cudaSuccess;
    const PairArgs A = make_args(d_jobs, n_jobs, n_items, counter, P, box, pl, d_count, d_wsum, d_stats);
    return dispatch_pairs(A, pl, st, sm_count, device);
}

// Item shape of one job: rows per item so that the whole launch has ~16
// items per resident warp.
void shape_job(PairJob &j, int64_t n_tiles, int n_rows, int64_t total_tile_rows, int sm_count) {
    const int64_t want = std::max<int64_t>(1, (int64_t)sm_count * 24 * 16);
    const int rpi = (int)std::min<int64_t>(32, std::max<int64_t>(1, total_tile_rows / want));
    j.n_rows = n_rows;
    j.rows_per_item = rpi;
    j.n_chunks = (n_rows + rpi - 1) / rpi;
    (void)n_tiles;
}

cudaError_t launch_pairs_view(const GridView &home, const GridView &cand, const TileDesc *tiles,
                              int64_t n_tiles, const RowDesc *rows, int n_rows, int P, float box,
                              const PairLaunch &pl, unsigned long long *counter,
                              unsigned long long *d_count, double *d_wsum,
                              unsigned long long *d_stats, PairJob *d_job, cudaStream_t st,
                              int sm_count, int device) {
    PairJob j;
    j.home = home;
    j.cand = cand;
    j.tiles = tiles;
    j.rows = rows;
    j.slot = 0;
    j.item_begin = 0;
    j.rule_flags = pl.rule.flags;
    j.pad = 0;
    shape_job(j, n_tiles, n_rows, n_tiles * n_rows, sm_count);
    const long long n_items = (long long)n_tiles * j.n_chunks;
    cudaError_t e = cudaMemcpyAsync(d_job, &j, sizeof(PairJob), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return launch_pair_jobs(d_job, 1, n_items, P, box, pl, counter, d_count, d_wsum, d_stats, st,
                            sm_count, device);
}

// Copies the stencil rows into the next staging slot (pinned host ->
// device).  Waits only for the kernel that used that slot two launches ago.
pcf_status stage_plan(pcf_ctx *ctx, const PairPlan &plan, PlanSlot **out) {
    cudaStream_t st = ctx->stream;
    ctx->slot ^= 1;
    PlanSlot &sl = ctx->slots[ctx->slot];
    if (!sl.done) PCF_CU(ctx, cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    if (sl.used) PCF_CU(ctx, cudaEventSynchronize(sl.done));
    const size_t rb = plan.rows.size() * sizeof(RowDesc);
    const size_t jb = sizeof(PairJob) * 4;
    if (sl.h_bytes < rb + jb + 256) {
        if (sl.h_pinned) cudaFreeHost(sl.h_pinned);
        sl.h_pinned = nullptr;
        sl.h_bytes = 0;
        const size_t want = std::max<size_t>((rb + jb) * 2 + 256, 1 << 16);
        PCF_CU(ctx, cudaMallocHost(&sl.h_pinned, want));
        sl.h_bytes = want;
    }
    PCF_CU(ctx, sl.d_rows.ensure(rb + jb + 256));
    PCF_CU(ctx, sl.d_counter.ensure(64));
    memcpy(sl.h_pinned, plan.rows.data(), rb);
    PCF_CU(ctx, cudaMemcpyAsync(sl.d_rows.p, sl.h_pinned, rb, cudaMemcpyHostToDevice, st));
    PCF_CU(ctx, cudaMemsetAsync(sl.d_counter.p, 0, 64, st));
    sl.used = true;
    *out = &sl;
    return PCF_OK;
}

pcf_status profile_events(pcf_ctx *ctx, cudaEvent_t *a, cudaEvent_t *b) {
    if (ctx->prof_used == ctx->prof_events.size()) {
        cudaEvent_t e0, e1;
        PCF_CU(ctx, cudaEventCreate(&e0));
        PCF_CU(ctx, cudaEventCreate(&e1));
        ctx->prof_events.push_back({e0, e1});
    }
    *a = ctx->prof_events[ctx->prof_used].first;
    *b = ctx->prof_events[ctx->prof_used].second;
    ++ctx->prof_used;
    return PCF_OK;
}

// Launches the pair kernel for one (home, cand) plan into d_count/d_wsum.
pcf_status launch_pairs(pcf_ctx *ctx, const PairPlan &plan, const CellGrid &home,
                        const CellGrid &cand, float box, const PairLaunch &pl,
                        unsigned long long *d_count, double *d_wsum,
                        unsigned long long *d_stats) {
    cudaStream_t st = ctx->stream;
    if (plan.n_items == 0) return PCF_OK;
    PlanSlot *sl = nullptr;
    pcf_status ps = stage_plan(ctx, plan, &sl);
    if (ps != PCF_OK) return ps;
    // the one job of this launch, staged behind the rows in the same slot
    PairJob job;
    job.home = GridView{home.x(), home.y(), home.z(), home.w(), home.cell_start.as<int>()};
    job.cand = GridView{cand.x(), cand.y(), cand.z(), cand.w(), cand.cell_start.as<int>()};
    job.tiles = home.d_tiles.as<TileDesc>();
    job.rows = sl->d_rows.as<RowDesc>();
    job.n_rows = (int)plan.rows.size();
    job.rows_per_item = plan.rows_per_item;
    job.n_chunks = plan.n_chunks;
    job.slot = 0;
    job.item_begin = 0;
    job.rule_flags = pl.rule.flags;
    job.pad = 0;
    const size_t roff = (plan.rows.size() * sizeof(RowDesc) + 255) & ~(size_t)255;
    char *hjob = static_cast<char *>(sl->h_pinned) + roff;
    memcpy(hjob, &job, sizeof(PairJob));
    PairJob *d_job = reinterpret_cast<PairJob *>(sl->d_rows.as<char>() + roff);
    PCF_CU(ctx, cudaMemcpyAsync(d_job, hjob, sizeof(PairJob), cudaMemcpyHostToDevice, st));
    const PairArgs A = make_args(d_job, 1, plan.n_items, sl->d_counter.as<unsigned long long>(),
                                 plan.P, box, pl, d_count, d_wsum, d_stats);
    PCF_CU(ctx, cudaEventRecord(ctx->ev0, st));
    cudaEvent_t pe0 = nullptr, pe1 = nullptr;
    if (ctx->profile) {
        pcf_status q = profile_events(ctx, &pe0, &pe1);
        if (q != PCF_OK) return q;
        PCF_CU(ctx, cudaEventRecord(pe0, st));
    }
    PCF_CU(ctx, dispatch_pairs(A, pl, st, ctx->sm_count, ctx->device));
    PCF_CU(ctx, cudaEventRecord(ctx->ev1, st));
    if (pe1) PCF_CU(ctx, cudaEventRecord(pe1, st));
    PCF_CU(ctx, cudaEventRecord(sl->done, st));
    ++ctx->launches;
    return PCF_OK;
}

cudaError_t launch_finalize_slots(const unsigned long long *d_count, const double *d_wsum,
                                  bool weighted, const double *d_mult, int nb, int nslots,
                                  double *d_out, cudaStream_t st) {
    const long long n = (long long)nb * nslots;
    k_finalize_slots<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_count, d_wsum, weighted ? 1 : 0,
                                                                   d_mult, nb, nslots, d_out);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const unsigned long long *d_count, const double *d_wsum, bool weighted,
                            double mult, int nb, double *d_out, cudaStream_t st) {
    k_finalize<<<(nb + 255) / 256, 256, 0, st>>>(d_count, d_wsum, weighted ? 1 : 0, mult, nb, d_out);
    return cudaGetLastError();
}

pcf_status finalize_hist(pcf_ctx *ctx, const unsigned long long *d_count, const double *d_wsum,
                         bool weighted, double mult, int nb, double *d_out) {
    k_finalize<<<(nb + 255) / 256, 256, 0, ctx->stream>>>(d_count, d_wsum, weighted ? 1 : 0, mult,
                                                          nb, d_out);
    PCF_CU(ctx, cudaGetLastError());
    ++ctx->launches;
    return PCF_OK;
}

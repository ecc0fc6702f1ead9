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
//    tile is <= 32 consecutive cell-ordered points of one (ix,iy) column
//    within two cells, one point per lane (a tile of H points runs 32/H
//    candidate streams); a stencil row
//    (dx,dy) names the neighbour column, whose cells z0-kz..z1+kz are one
//    contiguous point range (or two when the periodic box wraps in z).  XX
//    uses the half shell (each unordered pair once, histogram doubled at the
//    end, matching the reference's ordered-pair convention).
//  * Periodic boxes: the neighbour column index wraps and the home point is
//    shifted by the image offset once per range, so no image passes.
//  * Candidates arrive two at a time as two 16-byte loads of the pair-packed
//    layout (PairView); separations in packed FP32 (3 FADD2, FMUL2, 2 FFMA2
//    per two pairs); the bin comes from r = sqrt.approx(d2*ds^2) read out in
//    15-bit fixed point through r + 256.  A pair whose r is within a proven
//    error window of a bin edge, or whose d2 is near dmax^2 or 0, is
//    re-evaluated with the canonical FP64 rule (pcf_internal.cuh), so bin
//    membership equals the FP64 oracle's exactly.
//  * Histograms: u32 shared-memory copies per lane (iso) or per warp (ani),
//    merged into global u64 counts / FP64 sums and finalised to double (x2
//    for XX).  Weighted sums use exact integer weights: the 64-bit product
//    q_a*q_b goes into three u32 limb counters (16 + 16 + 32 bits), flushed
//    before any could wrap; FP64 shared atomics remain for weights without
//    an exact integer image.
//  * A launch produces the isotropic histogram, the anisotropic one, or both
//    from one pass over the candidates (PCF_BOTH).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
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
// bits(256 + r) >> 15 = kBinBias + floor(r) for r in [0, 256) away from an edge
constexpr unsigned kBinBias = 0x43800000u >> kFracBits;

// Histogram privatisation.  H_LANE: a u32 (or FP64) column per lane (iso);
// H_WARP: one copy per warp with shared atomics; H_GLOBAL: global atomics
// (very wide histograms); H_WFIX: per-warp fixed-point limbs (weighted);
// H_LFIX: per-lane fixed-point limbs (weighted iso); H_WFIX4: per-warp
// fixed-point limbs in four sub-copies, lane l adding to copy l % 4 (the
// isotropic copy of a weighted both-kinds launch: its few bins would
// otherwise take the reductions of all 32 lanes).
enum { H_LANE = 0, H_WARP = 1, H_GLOBAL = 2, H_WFIX = 3, H_LFIX = 4, H_WFIX4 = 5, H_WFIX2 = 6 };
// Variants of the weighted one-pass both-kinds kernel (the isotropic copy
// and the candidate loads), selected by PCF_OPT_PAIR_VARIANT for the A/B of
// shared-memory staging: 0 four isotropic sub-copies, candidates by __ldg
// (the default); 1 two sub-copies (frees 720 B per warp), __ldg; 2 two
// sub-copies, candidates of full tiles staged into shared memory by
// cp.async, in double-buffered windows of 16, in the space the two freed
// sub-copies left (so the CTA count per SM stays at four).
constexpr int kStageCands = 16;
constexpr int kStageBytes = 2 * (kStageCands * 16 + kStageCands * 4);  // per warp
constexpr int kLimbs = 3;
// Candidate steps between recheck votes, per kind: the anisotropic (and
// both-kinds) kernels carry more live state per step and schedule better
// with shorter groups.
#ifndef PCF_GROUP_ISO
#define PCF_GROUP_ISO 4
#endif
#ifndef PCF_GROUP_ANI
#define PCF_GROUP_ANI 2
#endif
constexpr int kChunkMax = 8;            // work items per ticket, at most

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
    unsigned long long *counter;  // work tickets handed out so far
    long long n_chunked;          // items [0, n_chunked) go out `kchunk` per ticket,
    long long t_chunked;          // in t_chunked tickets; later tickets: one item each
    int kchunk;
    float box;
    int bpc;
    float zreach;  // dmax * (1 + 1e-5): the z reach of a home tile's rows
    PairRule rule;
    FastCuts fc;
    unsigned long long *g_count;
    double *g_wsum;
    unsigned long long *g_stats;
    int chunk;   // candidates per budget check (even)
    int budget;  // adds one shared counter absorbs between flushes
    int fast;    // 0: every pair in range takes the FP64 rule (bins > 255: r + 256
                 // no longer has a fixed exponent)
    const unsigned *ctrl;  // abort request polled at every ticket (null: none)
    unsigned *status;      // where a warp that gives up records why (null: none)
    long long max_tickets; // iteration cap: tickets one warp may take
};

__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Fixed-point readout of r in [0, 256): u = bits(r + 256 + w/2^15), so the
// low 15 bits are frac(r) + w in 2^-15 units.  The bin (u >> 15, biased) is
// floor(r) unless r is within w/2^15 of an integer, which this rejects.
__device__ __forceinline__ bool fix_safe(unsigned u, unsigned w2) {
    return (u & kFracMask) >= w2;
}

// Shared reductions on 32-bit shared-window addresses.  They are not
// predicated: a lane without a pair adds 0 to a private dummy slot, which
// keeps the candidate loop free of branches around memory operations.
__device__ __forceinline__ void red_s_u32(unsigned a, unsigned v) {
    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(a), "r"(v));
}
__device__ __forceinline__ void red_s_f64(unsigned a, double v) {
    asm volatile("red.shared.add.f64 [%0], %1;" :: "r"(a), "d"(v));
}
// The three limbs of one product into [a], [a + S], [a + 2S].
template <int S>
__device__ __forceinline__ void red_s_limbs(unsigned a, unsigned long long v) {
    const unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    asm volatile("red.shared.add.u32 [%0], %1;\n\t"
                 "red.shared.add.u32 [%0+%4], %2;\n\t"
                 "red.shared.add.u32 [%0+%5], %3;"
                 :: "r"(a), "r"(lo & 0xFFFFu), "r"(lo >> 16), "r"(hi), "n"(S), "n"(2 * S));
}

// Weight carried per point: the exact integer q (fixed-point modes), the
// float w (FP64 modes) or nothing (unit weights).
template <bool WEIGHTED, int HM>
struct WT {
    typedef typename std::conditional<(HM == H_WFIX || HM == H_LFIX || HM == H_WFIX4 || HM == H_WFIX2),
                                      unsigned, float>::type type;
};

// Histogram sink of one lane.  Slots arrive biased (see kBinBias); `base`
// already subtracts bias * stride, so the address is base + sb * stride.
// `dummy` is this lane's private slot for the adds of 0.
template <bool WEIGHTED, int HM>
struct Sink {
    typedef typename WT<WEIGHTED, HM>::type W;
    unsigned base;      // shared-window address (biased)
    unsigned dummy;     // shared-window address of this lane's dummy slot
    unsigned bias;
    double *lane_col;   // H_LANE FP64: this lane's column (generic)
    void *gbase;        // H_GLOBAL: this job's accumulator
    __device__ __forceinline__ void add(unsigned sb, W wa, W wb, bool pred) const {
        if (HM == H_LFIX) {
            red_s_limbs<128>(pred ? base + sb * (kLimbs * 128u) : dummy,
                             (unsigned long long)(pred ? wa : 0u) * wb);
        } else if (HM == H_WFIX || HM == H_WFIX4 || HM == H_WFIX2) {
            // per-warp copies end in a dummy region that is never read, so a
            // lane without a pair adds its real product there: the product
            // and its limbs are then the same for both copies of a
            // both-kinds pass and computed once
            red_s_limbs<4>(pred ? base + sb * (kLimbs * 4u) : dummy, (unsigned long long)wa * wb);
        } else if (HM == H_LANE) {
            if (WEIGHTED) {  // lane-private FP64 column: add 0 to slot 0 when !pred
                double *h = lane_col + (pred ? (int)(sb - bias) : 0) * 32;
                *h += pred ? (double)wa * (double)wb : 0.0;
            } else {
                red_s_u32(pred ? base + sb * 128u : dummy, (unsigned)pred);
            }
        } else if (HM == H_WARP) {
            if (WEIGHTED) red_s_f64(pred ? base + sb * 8u : dummy, pred ? (double)wa * (double)wb : 0.0);
            else red_s_u32(pred ? base + sb * 4u : dummy, (unsigned)pred);
        } else if (pred) {
            if (WEIGHTED) atomicAdd(static_cast<double *>(gbase) + (sb - bias), (double)wa * (double)wb);
            else atomicAdd(static_cast<unsigned long long *>(gbase) + (sb - bias), 1ull);
        }
    }
};

// Point j of a pair-packed view.
__device__ __forceinline__ void load_point(const float4 *pk, int j, float &x, float &y, float &z, float &w) {
    const float4 a = __ldg(pk + (j & ~1)), b = __ldg(pk + (j & ~1) + 1);
    const bool o = j & 1;
    x = o ? a.y : a.x;
    y = o ? a.w : a.z;
    z = o ? b.y : b.x;
    w = o ? b.w : b.z;
}

// Canonical FP64 decision for one pair (rare path): histogram slot or -1.
template <bool ANI>
__device__ __noinline__ int slow_slot(float hx, float hy, float hz, float cx, float cy, float cz,
                                      float sx, float sy, float sz, PairRule rule) {
    double dx, dy, dz;
    exact_sep(hx, hy, hz, cx, cy, cz, sx, sy, sz, dx, dy, dz);
    return exact_slot<ANI>(dx, dy, dz, rule);
}

// Shared-memory words (of the copy's element type) of one warp's copy.
// Per-warp copies end with a dummy region (never flushed) where each lane
// has its own word: 32 words, or for fixed-point limbs 32 + 2, lane l's
// three limbs at words l, l+1, l+2 of the region (one limb per reduction
// instruction, so the lanes of one instruction never share a word; the adds
// there are of 0).
template <int HM>
__host__ __device__ __forceinline__ int copy_words(int nb) {
    return HM == H_LANE ? nb * 32 : HM == H_WARP ? nb + 32 : HM == H_WFIX ? nb * kLimbs + 32 + kLimbs - 1
         : HM == H_WFIX4 ? 4 * nb * kLimbs + 32 + kLimbs - 1 : HM == H_WFIX2 ? 2 * nb * kLimbs + 32 + kLimbs - 1
         : HM == H_LFIX ? nb * kLimbs * 32 : 0;
}

// Adds this warp's copy (nb bins) into the launch's accumulators at `off`
// and clears it.
template <bool WEIGHTED, int HM, bool XCHG = false>
__device__ void flush_copy(void *mine_v, int nb, int lane, const PairArgs &A, size_t off, double unscale) {
    if (HM == H_GLOBAL) return;
    __syncwarp();
    if (HM == H_LANE && !WEIGHTED) {
        unsigned *mine = static_cast<unsigned *>(mine_v);
        for (int k = 0; k < nb; ++k) {
            unsigned long long s = mine[k * 32 + lane];
            mine[k * 32 + lane] = 0u;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
            if (lane == 0 && s) atomicAdd(A.g_count + off + k, s);
        }
    } else if (HM == H_LANE) {
        double *mine = static_cast<double *>(mine_v);
        for (int k = 0; k < nb; ++k) {
            double s = mine[k * 32 + lane];
            mine[k * 32 + lane] = 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
            if (lane == 0 && s != 0.0) atomicAdd(A.g_wsum + off + k, s);
        }
    } else if (HM == H_WARP) {
        for (int k = lane; k < nb; k += 32) {
            if (WEIGHTED) {
                double *mine = static_cast<double *>(mine_v);
                const double s = mine[k];
                mine[k] = 0.0;
                if (s != 0.0) atomicAdd(A.g_wsum + off + k, s);
            } else {
                unsigned *mine = static_cast<unsigned *>(mine_v);
                const unsigned s = mine[k];
                mine[k] = 0u;
                if (s) atomicAdd(A.g_count + off + k, (unsigned long long)s);
            }
        }
    } else if (HM == H_WFIX) {  // [bin][limb]
        unsigned *mine = static_cast<unsigned *>(mine_v);
        for (int k = lane; k < nb; k += 32) {
            unsigned *c = mine + k * kLimbs;
            unsigned l0, l1, l2;
            if (XCHG) {  // a copy shared with a warp that may be adding: each limb read and cleared at once
                l0 = atomicExch(c, 0u);
                l1 = atomicExch(c + 1, 0u);
                l2 = atomicExch(c + 2, 0u);
            } else {
                l0 = c[0];
                l1 = c[1];
                l2 = c[2];
                c[0] = c[1] = c[2] = 0u;
            }
            if (l0 | l1 | l2) {  // each term exact; the sum rounds at most twice
                const double v = (double)l2 * 0x1p32 + ((double)l1 * 0x1p16 + (double)l0);
                atomicAdd(A.g_wsum + off + k, v * unscale);
            }
        }
    } else if (HM == H_WFIX4 || HM == H_WFIX2) {  // [copy][bin][limb]: limbs summed exactly over the copies
        constexpr int NSUB = HM == H_WFIX4 ? 4 : 2;
        unsigned *mine = static_cast<unsigned *>(mine_v);
        for (int k = lane; k < nb; k += 32) {
            unsigned long long s0 = 0, s1 = 0, s2 = 0;
            #pragma unroll
            for (int q = 0; q < NSUB; ++q) {
                unsigned *c = mine + (q * nb + k) * kLimbs;
                s0 += c[0];
                s1 += c[1];
                s2 += c[2];
                c[0] = c[1] = c[2] = 0u;
            }
            if (s0 | s1 | s2) {  // each term exact (< 2^53); the sum rounds at most twice
                const double v = (double)s2 * 0x1p32 + ((double)s1 * 0x1p16 + (double)s0);
                atomicAdd(A.g_wsum + off + k, v * unscale);
            }
        }
    } else if (HM == H_LFIX) {  // [bin][limb][lane]
        unsigned *mine = static_cast<unsigned *>(mine_v);
        for (int k = 0; k < nb; ++k) {
            unsigned *c = mine + k * kLimbs * 32 + lane;
            const unsigned l0 = c[0], l1 = c[32], l2 = c[64];
            c[0] = c[32] = c[64] = 0u;
            double v = (double)l2 * 0x1p32 + ((double)l1 * 0x1p16 + (double)l0);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
            if (lane == 0 && v != 0.0) atomicAdd(A.g_wsum + off + k, v * unscale);
        }
    }
    __syncwarp();
}

#ifndef PCF_PAIR_MINB
#define PCF_PAIR_MINB 6
#endif
// CTAs per SM the shared-memory footprint allows at 30 / 900 bins (the
// register cap of the launch bounds follows from it)
template <int KIND, int HM, int VAR = 0>
struct MinBlocks {
    static constexpr int value = KIND == 2 ? (HM == H_WFIX ? (VAR == 3 ? 5 : 4) : 5)
                               : HM == H_LFIX ? 4 : HM == H_WFIX ? 5 : PCF_PAIR_MINB;
};

// Kinds of one launch: the isotropic histogram, the anisotropic one, or both
// from one pass over the candidates (the anisotropic stencil covers the
// isotropic one).
enum { K_ISO = 0, K_ANI = 1, K_BOTH = 2 };
// Scheme of the isotropic copy of a K_BOTH launch, given the anisotropic one:
// lane-private counts, four per-warp fixed-point sub-copies, else per-warp
// copies of the same element type.
__host__ __device__ constexpr int iso_scheme(bool weighted, int hm, int var = 0) {
    return hm == H_WARP ? (weighted ? H_WARP : H_LANE)
         : hm == H_WFIX ? ((var == 1 || var == 2) ? H_WFIX2 : H_WFIX4) : hm;
}
template <bool WEIGHTED, int HM, int VAR>
struct IsoScheme {
    static constexpr int value = iso_scheme(WEIGHTED, HM, VAR);
};

// Sets up one lane's sink over a copy at shared address ms (see Sink).
template <bool WEIGHTED, int HM>
__device__ __forceinline__ void setup_sink(Sink<WEIGHTED, HM> &sk, unsigned ms, void *mine, int lane,
                                           unsigned bias, int nb) {
    typedef typename std::conditional<WEIGHTED && !(HM == H_WFIX || HM == H_LFIX || HM == H_WFIX4 || HM == H_WFIX2),
                                      double, unsigned>::type HT;
    sk.bias = bias;
    sk.lane_col = reinterpret_cast<double *>(mine) + lane;
    sk.gbase = nullptr;
    switch (HM) {  // dummy: bin 0 of a lane-private column, else slot nb + lane
    case H_LANE: sk.base = ms + lane * 4u - bias * 128u; sk.dummy = ms + lane * 4u; break;
    case H_WARP:
        sk.base = ms - bias * (unsigned)sizeof(HT);
        sk.dummy = ms + (unsigned)(nb + lane) * (unsigned)sizeof(HT);
        break;
    case H_WFIX:
        sk.base = ms - bias * (kLimbs * 4u);
        sk.dummy = ms + (unsigned)(nb * kLimbs + lane) * 4u;
        break;
    case H_WFIX4:
        sk.base = ms + (unsigned)((lane & 3) * nb * kLimbs) * 4u - bias * (kLimbs * 4u);
        sk.dummy = ms + (unsigned)(4 * nb * kLimbs + lane) * 4u;
        break;
    case H_WFIX2:
        sk.base = ms + (unsigned)((lane & 1) * nb * kLimbs) * 4u - bias * (kLimbs * 4u);
        sk.dummy = ms + (unsigned)(2 * nb * kLimbs + lane) * 4u;
        break;
    case H_LFIX: sk.base = ms + lane * 4u - bias * (kLimbs * 128u); sk.dummy = ms + lane * 4u; break;
    default: sk.base = sk.dummy = 0u;
    }
}

// Candidate ranges of one stencil row for the current home tile: [a0, b0)
// unshifted in z, [a1, b1) image-shifted by sz1 (periodic wrap in z); the
// column's image shift is (sx, sy).  kind 1: forward half of the home column.
struct RowRange {
    int a0, b0, a1, b1;
    float sx, sy, sz1;
    int kind;
};

// Per-warp state kept in shared memory, so the candidate loop has the
// registers to itself.
struct WarpState {
    PairJob job;
    RowRange rows[32];
    float4 home[32];                // this item's home point per lane (x, y, z, w)
    unsigned long long n_cand;      // pair tests (statistics)
    long long job_end;
    int cj, slot;
};

// COUNT: also count the in-range pairs (weighted histograms, statistics on).
// HM is the scheme of the anisotropic copy for K_ANI / K_BOTH launches.
template <int KIND, bool WEIGHTED, int HM, bool COUNT, int VAR = 0>
__global__ void __launch_bounds__(kThreads, MinBlocks<KIND, HM, VAR>::value) k_pairs(const PairArgs A) {
    constexpr bool FIX = HM == H_WFIX || HM == H_LFIX;
    constexpr bool DO_I = KIND != K_ANI, DO_A = KIND != K_ISO;
    constexpr bool kPrefetch = KIND == K_BOTH && HM == H_WFIX;  // measured: helps only here
    constexpr bool kStage = VAR == 2;  // candidates of full tiles through shared memory
    // VAR 3 (single-job launches only): warps 2k and 2k+1 share one
    // anisotropic copy, each with its own dummy region, so a CTA's copies fit
    // five CTAs per SM; a shared copy is flushed by atomic exchange, so
    // either warp may flush while the other adds, and each warp flushes
    // within half the budget
    constexpr bool kPairCopy = VAR == 3 && KIND == K_BOTH && HM == H_WFIX;
    // with the next step's loads in flight, a vote per step ran 1.4% faster
    // than one per two steps (periodic 2iso+2ani step, A/B on one box)
    constexpr int kGroup = kPrefetch ? 1 : KIND == K_ISO ? PCF_GROUP_ISO : PCF_GROUP_ANI;
    constexpr int HMI = KIND == K_BOTH ? IsoScheme<WEIGHTED, HM, VAR>::value : HM;
    typedef typename WT<WEIGHTED, HM>::type W;
    typedef typename std::conditional<WEIGHTED && !FIX, double, unsigned>::type HT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ WarpState s_ws[kWarps];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    WarpState &ws = s_ws[warp];
    PairJob &J = ws.job;
    const int bins = A.rule.bins;
    const int nbi = bins, nba = bins * bins;
    const int nbt = (DO_I ? nbi : 0) + (DO_A ? nba : 0);  // accumulators per job slot
    const int wi = DO_I ? copy_words<HMI>(nbi) : 0, wa = DO_A ? copy_words<HM>(nba) : 0;
    constexpr int kDummy = 32 + kLimbs - 1;  // words of one warp's dummy region (kPairCopy)
    const int wpair = kPairCopy ? nba * kLimbs + 2 * kDummy : 0;  // words of one shared copy
    HT *mine_i = kPairCopy ? reinterpret_cast<HT *>(smem_raw) + warp * wi
                           : reinterpret_cast<HT *>(smem_raw) + warp * (wi + wa);
    HT *mine_a = kPairCopy ? reinterpret_cast<HT *>(smem_raw) + kWarps * wi + (warp >> 1) * wpair
                           : mine_i + wi;
    // staging windows (kStage): two of kStageCands candidates per warp after
    // every warp's copies: pair-packed blocks, then their integer weights
    float4 *stg_f4 = nullptr;
    unsigned *stg_q = nullptr;
    if (kStage) {
        unsigned char *sb = smem_raw + (((size_t)kWarps * (wi + wa) * sizeof(HT) + 15) & ~(size_t)15) +
                            (size_t)warp * kStageBytes;
        stg_f4 = reinterpret_cast<float4 *>(sb);
        stg_q = reinterpret_cast<unsigned *>(sb + 2 * kStageCands * 16);
    }
    if (kPairCopy) {  // both warps of a pair zero the shared copy before either adds
        for (int k = lane; k < wi; k += 32) mine_i[k] = (HT)0;
        for (int k = lane; k < wpair; k += 32) mine_a[k] = (HT)0;
        __syncthreads();
    } else {
        for (int k = lane; k < wi + wa; k += 32) mine_i[k] = (HT)0;
    }
    const unsigned bias_i = kBinBias, bias_a = kBinBias * (unsigned)(bins + 1);
    Sink<WEIGHTED, HMI> sink_i;
    Sink<WEIGHTED, HM> sink_a;
    if (DO_I) setup_sink<WEIGHTED, HMI>(sink_i, (unsigned)__cvta_generic_to_shared(mine_i), mine_i, lane, bias_i, nbi);
    if (DO_A) setup_sink<WEIGHTED, HM>(sink_a, (unsigned)__cvta_generic_to_shared(mine_a), mine_a, lane, bias_a, nba);
    if (kPairCopy)
        sink_a.dummy = (unsigned)__cvta_generic_to_shared(mine_a) +
                       (unsigned)(nba * kLimbs + (warp & 1) * kDummy + lane) * 4u;
    // flushes both copies of this warp into job slot `slot`
    auto flush = [&](int slot, double unscale) {
        const size_t off = (size_t)slot * nbt;
        if (DO_I) flush_copy<WEIGHTED, HMI>(mine_i, nbi, lane, A, off, unscale);
        if (DO_A) flush_copy<WEIGHTED, HM, kPairCopy>(mine_a, nba, lane, A, off + (DO_I ? nbi : 0), unscale);
    };
    const int budget = kPairCopy ? A.budget / 2 : A.budget;
    if (lane == 0) {
        ws.n_cand = 0;
        ws.job_end = -1;
        ws.cj = -1;
        ws.slot = 0;
    }
    __syncwarp();
    int since = 0;  // adds per shared counter since this copy's last flush (bound)
    unsigned n_pairs = 0, n_rechk = 0;
    const FastCuts &fc = A.fc;

    // Work queue of tickets: while a queue holds many items per warp, a
    // ticket is a run of `kchunk` consecutive items (a warp then changes job,
    // and flushes its histogram copy, less often); the last two rounds go out
    // one item per ticket so the tail stays short.
    auto ticket_items = [&](long long t, long long &ib, long long &ie) {
        if (t < A.t_chunked) {
            ib = t * A.kchunk;
            ie = min(ib + A.kchunk, A.n_chunked);
        } else {
            ib = A.n_chunked + (t - A.t_chunked);
            ie = ib + 1;
        }
        ie = min(ie, A.n_items);
    };
    long long tk = 0, ib, ie;
    if (lane == 0) tk = (long long)atomicAdd(A.counter, 1ull);
    tk = __shfl_sync(kFull, tk, 0);
    ticket_items(tk, ib, ie);
    long long taken = 1;  // tickets this warp has taken (iteration cap)
    unsigned stop = 0;    // abort request, read with each ticket
    while (ib < A.n_items) {
      if (lane == 0) {  // prefetch the next ticket (and the abort word with it)
          tk = (long long)atomicAdd(A.counter, 1ull);
          if (A.ctrl) stop = ctrl_load(A.ctrl);
      }
      for (long long it_idx = ib; it_idx < ie; ++it_idx) {
        if (it_idx >= ws.job_end) {  // entering another job: flush this one's histogram
            if (ws.cj >= 0) flush(ws.slot, J.wunscale);
            since = 0;
            int cj = ws.cj;
            long long job_end;
            do {
                ++cj;
                job_end = cj + 1 < A.n_jobs ? A.jobs[cj + 1].item_begin : A.n_items;
            } while (it_idx >= job_end);
            __syncwarp();
            static_assert(sizeof(PairJob) % 4 == 0, "PairJob words");
            const int *src = reinterpret_cast<const int *>(A.jobs + cj);
            int *dst = reinterpret_cast<int *>(&J);
            for (int q = lane; q < (int)(sizeof(PairJob) / 4); q += 32) dst[q] = src[q];
            if (lane == 0) {
                ws.cj = cj;
                ws.job_end = job_end;
            }
            __syncwarp();
            if (lane == 0) ws.slot = J.slot;
            if (HM == H_GLOBAL) {
                const size_t off = (size_t)J.slot * nbt;
                void *g = WEIGHTED ? (void *)(A.g_wsum + off) : (void *)(A.g_count + off);
                sink_i.gbase = g;
                sink_a.gbase = WEIGHTED ? (void *)(A.g_wsum + off + (DO_I ? nbi : 0))
                                        : (void *)(A.g_count + off + (DO_I ? nbi : 0));
            }
            __syncwarp();
        }
        const long long loc = it_idx - J.item_begin;
        const int tile = (int)(loc / J.n_chunks);
        const int chunk = (int)(loc - (long long)tile * J.n_chunks);
        const int row_begin = chunk * J.rows_per_item;
        const int nrows = min(row_begin + J.rows_per_item, J.n_rows) - row_begin;  // <= 32
        const TileDesc t = J.tiles[tile];
        const int H = t.count;                 // 1..32 home points
        const int S = 32 / H;                  // candidate streams per warp
        const int sidx = lane / H;             // this lane's stream
        const int hidx = t.start + (lane - sidx * H);
        W hw = (W)0;
        float zmn, zmx;  // the home points' z extent (NaN lanes drop out of fminf / fmaxf)
        {
            float4 h;
            if (sidx < S) {
                load_point(J.home.pk, hidx, h.x, h.y, h.z, h.w);
                if (FIX) hw = (W)__ldg(J.home.qw + hidx);
                else hw = (W)h.w;
            } else {
                h.x = h.y = h.z = __int_as_float(0x7fc00000);  // NaN: never in range
                h.w = 0.f;
            }
            ws.home[lane] = h;
            zmn = zmx = h.z;
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                zmn = fminf(zmn, __shfl_xor_sync(kFull, zmn, o));
                zmx = fmaxf(zmx, __shfl_xor_sync(kFull, zmx, o));
            }
        }
        // Candidate ranges of all rows of the item, one row per lane, so the
        // dependent cell-table loads of different rows overlap.
        if (lane < nrows) {
            RowRange rr{0, 0, 0, 0, 0.f, 0.f, 0.f, 0};
            const RowDesc rw = J.rows[row_begin + lane];
            int nx = t.ix + rw.dx, ny = t.iy + rw.dy;
            const int P = J.P;
            bool ok = true;
            if (A.bpc) {
                if (nx < 0) { nx += P; rr.sx = -A.box; } else if (nx >= P) { nx -= P; rr.sx = A.box; }
                if (ny < 0) { ny += P; rr.sy = -A.box; } else if (ny >= P) { ny -= P; rr.sy = A.box; }
            } else if (nx < 0 || nx >= P || ny < 0 || ny >= P) {
                ok = false;
            }
            if (ok) {
                const int col = (nx * P + ny) * P;
                // the row's cells, clipped to those the home points reach in z:
                // a candidate within dmax of a home point has z in (zmn - dmax,
                // zmx + dmax), so its cell lies in [zcut_lo, zcut_hi] (with
                // 1e-3 of a cell to spare for the rounding of z / cell here
                // and in the grid build; the tile's own cells always stay);
                // periodic images follow the same cell arithmetic past 0 and P
                const float rcell = (float)P / A.box;
                const int zcut_lo = min((int)floorf((zmn - A.zreach) * rcell - 1e-3f), (int)t.z0);
                const int zcut_hi = max((int)floorf((zmx + A.zreach) * rcell + 1e-3f), (int)t.z1);
                const int zhi = min(t.z1 + rw.kz, zcut_hi);
                rr.kind = rw.kind;
                const int *cs = J.cand.cstart;
                if (rw.kind == 1) {  // forward half of the home column (XX): j > home index
                    rr.a0 = t.start;
                    rr.b0 = cs[col + min(zhi, P - 1) + 1];
                    if (A.bpc && zhi >= P) { rr.a1 = cs[col]; rr.b1 = cs[col + zhi - P + 1]; rr.sz1 = A.box; }
                } else {
                    const int zlo = max(t.z0 - rw.kz, zcut_lo);
                    rr.a0 = cs[col + max(zlo, 0)];
                    rr.b0 = cs[col + min(zhi, P - 1) + 1];
                    if (A.bpc) {
                        if (zlo < 0) { rr.a1 = cs[col + zlo + P]; rr.b1 = cs[col + P]; rr.sz1 = -A.box; }
                        else if (zhi >= P) { rr.a1 = cs[col]; rr.b1 = cs[col + zhi - P + 1]; rr.sz1 = A.box; }
                    }
                }
            }
            ws.rows[lane] = rr;
        }
        __syncwarp();
        const float4 *__restrict__ cpk = J.cand.pk;
        const unsigned *__restrict__ cqw = J.cand.qw;
        const int stride = 2 * S;
        for (int r = 0; r < nrows; ++r) {
            #pragma unroll 1
            for (int seg = 0; seg < 2; ++seg) {
                const RowRange &rg = ws.rows[r];
                const int a = seg ? rg.a1 : rg.a0, b = seg ? rg.b1 : rg.b0;
                if (a >= b) continue;
                const float sx = rg.sx, sy = rg.sy, sz = seg ? rg.sz1 : 0.f;
                const int sh = (sx != 0.f || sy != 0.f || sz != 0.f) ? 1 : 0;
                const float lo = fc.lo[sh], hi = fc.hi[sh];
                // r + 256 + w*2^-15: the window offset rides on the magic
                // constant (exact: a multiple of the ulp at 256)
                const unsigned w2 = 2u * fc.w[sh];
                const float mgw = kMagic + (float)fc.w[sh] * 0x1p-15f;
                // (x_j + shift) - x_home, rounded once: same value as the
                // scalar (x_j - (x_home - shift)) up to the bound in make_cuts
                const float4 h = ws.home[lane];
                const float2 NHX = make_float2(sx - h.x, sx - h.x);
                const float2 NHY = make_float2(sy - h.y, sy - h.y);
                const float2 NHZ = make_float2(sz - h.z, sz - h.z);
                const bool fwd = rg.kind == 1 && seg == 0;
                const int jmin = fwd ? hidx : a - 1;
                if (lane == 0) ws.n_cand += (unsigned long long)(b - a) * (unsigned long long)H;

                // Rare path: the canonical rule for candidate j (reloads what
                // the fast path does not keep in registers), for the kinds
                // whose fast path did not take it.
                auto slow = [&](int j, bool do_i, bool do_a) {
                    const RowRange &rq = ws.rows[r];
                    const float4 hh = ws.home[lane];
                    float cx, cy, cz, cw;
                    load_point(cpk, j, cx, cy, cz, cw);
                    W wj;
                    if (FIX) wj = (W)__ldg(cqw + j);
                    else wj = (W)cw;
                    PairRule rule = A.rule;
                    if (DO_I && do_i) {
                        rule.flags = J.rule_flags;
                        const int s = slow_slot<false>(hh.x, hh.y, hh.z, cx, cy, cz, rq.sx, rq.sy,
                                                       seg ? rq.sz1 : 0.f, rule);
                        if (s >= 0) {
                            sink_i.add((unsigned)s + bias_i, hw, wj, true);
                            if (COUNT) ++n_pairs;
                        }
                    }
                    if (DO_A && do_a) {
                        rule.flags = KIND == K_BOTH ? J.rule_flags2 : J.rule_flags;
                        const int s = slow_slot<true>(hh.x, hh.y, hh.z, cx, cy, cz, rq.sx, rq.sy,
                                                      seg ? rq.sz1 : 0.f, rule);
                        if (s >= 0) {
                            sink_a.add((unsigned)s + bias_a, hw, wj, true);
                            if (COUNT) ++n_pairs;
                        }
                    }
                };
                // One aligned pair of candidates (p, p+1); v0 / v1 say which are
                // real.  Pure arithmetic: per kind the histogram slots (biased),
                // which pairs the fast path takes (f) and which need the FP64
                // rule (r).
                struct Eval {
                    unsigned si0, si1, sa0, sa1;
                    W w0, w1;
                    bool fi0, fi1, fa0, fa1, ri0, ri1, ra0, ra1;
                };
                // The loads of one step (two candidates).
                struct Raw {
                    float4 qa, qb;
                    uint2 q;
                };
                auto load = [&](int p) -> Raw {
                    Raw w;
                    w.qa = __ldg(cpk + p);
                    w.qb = __ldg(cpk + p + 1);
                    if (FIX) w.q = __ldg(reinterpret_cast<const uint2 *>(cqw + p));
                    else w.q = make_uint2(0u, 0u);
                    return w;
                };
                auto eval_raw = [&](const Raw &w, bool v0, bool v1) -> Eval {
                    Eval e;
                    const float4 qa = w.qa, qb = w.qb;
                    e.w0 = e.w1 = (W)1;
                    if (FIX) {
                        e.w0 = (W)w.q.x;
                        e.w1 = (W)w.q.y;
                    } else if (WEIGHTED) {
                        e.w0 = (W)qb.z;
                        e.w1 = (W)qb.w;
                    }
                    const float2 DX = __fadd2_rn(make_float2(qa.x, qa.y), NHX);
                    const float2 DY = __fadd2_rn(make_float2(qa.z, qa.w), NHY);
                    const float2 DZ = __fadd2_rn(make_float2(qb.x, qb.y), NHZ);
                    const float2 PP = __ffma2_rn(DY, DY, __fmul2_rn(DX, DX));
                    e.si0 = e.si1 = e.sa0 = e.sa1 = 0u;
                    e.fi0 = e.fi1 = e.fa0 = e.fa1 = e.ri0 = e.ri1 = e.ra0 = e.ra1 = false;
                    if (DO_I) {  // d2 = (dx^2 + dy^2) + dz^2 with fused adds
                        const float2 D2 = __ffma2_rn(DZ, DZ, PP);
                        const float2 U = __fmul2_rn(D2, make_float2(fc.ds2, fc.ds2));
                        const float2 Q = __fadd2_rn(make_float2(sqrt_approx(U.x), sqrt_approx(U.y)),
                                                    make_float2(mgw, mgw));
                        const unsigned u0 = __float_as_uint(Q.x), u1 = __float_as_uint(Q.y);
                        // f implies r < bins away from an edge: the slot is in range
                        e.fi0 = v0 && (D2.x < lo) && fix_safe(u0, w2);
                        e.fi1 = v1 && (D2.y < lo) && fix_safe(u1, w2);
                        if (HM == H_GLOBAL) { e.fi0 = e.fi0 && A.fast; e.fi1 = e.fi1 && A.fast; }
                        e.si0 = u0 >> kFracBits;
                        e.si1 = u1 >> kFracBits;
                        e.ri0 = v0 && !e.fi0 && D2.x < hi;
                        e.ri1 = v1 && !e.fi1 && D2.y < hi;
                    }
                    if (DO_A) {
                        const float2 ZZ = __fmul2_rn(DZ, DZ);
                        const float m0 = fmaxf(ZZ.x, PP.x), m1 = fmaxf(ZZ.y, PP.y);
                        const float2 RZ = __fmul2_rn(DZ, make_float2(fc.dsf, fc.dsf));
                        const float2 U = __fmul2_rn(PP, make_float2(fc.ds2, fc.ds2));
                        const unsigned z0 = __float_as_uint(fabsf(RZ.x) + mgw);
                        const unsigned z1 = __float_as_uint(fabsf(RZ.y) + mgw);
                        const float2 QP = __fadd2_rn(make_float2(sqrt_approx(U.x), sqrt_approx(U.y)),
                                                     make_float2(mgw, mgw));
                        const unsigned p0 = __float_as_uint(QP.x), p1 = __float_as_uint(QP.y);
                        e.fa0 = v0 && (m0 < lo) && fix_safe(z0, w2) && fix_safe(p0, w2);
                        e.fa1 = v1 && (m1 < lo) && fix_safe(z1, w2) && fix_safe(p1, w2);
                        if (HM == H_GLOBAL) { e.fa0 = e.fa0 && A.fast; e.fa1 = e.fa1 && A.fast; }
                        const unsigned B = (unsigned)bins;
                        e.sa0 = (z0 >> kFracBits) * B + (p0 >> kFracBits);
                        e.sa1 = (z1 >> kFracBits) * B + (p1 >> kFracBits);
                        e.ra0 = v0 && !e.fa0 && m0 < hi;
                        e.ra1 = v1 && !e.fa1 && m1 < hi;
                    }
                    return e;
                };
                auto eval = [&](int p, bool v0, bool v1) -> Eval { return eval_raw(load(p), v0, v1); };
                // Accumulates the fast-path pairs; true if any needs the FP64 rule.
                auto core_raw = [&](const Raw &w, bool v0, bool v1) -> bool {
                    const Eval e = eval_raw(w, v0, v1);
                    if (DO_I) {
                        sink_i.add(e.si0, hw, e.w0, e.fi0);
                        sink_i.add(e.si1, hw, e.w1, e.fi1);
                        if (COUNT) n_pairs += (unsigned)e.fi0 + (unsigned)e.fi1;
                    }
                    if (DO_A) {
                        sink_a.add(e.sa0, hw, e.w0, e.fa0);
                        sink_a.add(e.sa1, hw, e.w1, e.fa1);
                        if (COUNT) n_pairs += (unsigned)e.fa0 + (unsigned)e.fa1;
                    }
                    return e.ri0 || e.ri1 || e.ra0 || e.ra1;
                };
                auto core = [&](int p, bool v0, bool v1) -> bool { return core_raw(load(p), v0, v1); };
                // Rechecks of `n` steps from p: the vote is rare, so the
                // candidates are re-evaluated to find which need the FP64 rule.
                // Lanes of different candidate streams leave the stream loop after
                // different trip counts, so vote only among the lanes that are here.
                auto settle = [&](bool any, int p, int n, bool v0, bool v1) {
                    if (__any_sync(__activemask(), any)) {
                        for (int k = 0; k < n; ++k) {
                            const Eval e = eval(p + k * stride, v0, v1);
                            if (e.ri0 || e.ra0) { ++n_rechk; slow(p + k * stride, e.ri0, e.ra0); }
                            if (e.ri1 || e.ra1) { ++n_rechk; slow(p + k * stride + 1, e.ri1, e.ra1); }
                        }
                    }
                };
                // head: pairs that start before a, or that reach into the home
                // tile of a forward row (j > home index per lane); body: pairs
                // fully inside (a, b) past the tile, no checks; tail: the last
                // pair when it ends at b
                const int chk = fwd ? t.start + H : a + 1;
                auto run = [&](int lo_i, int hi_i) {  // candidates [lo_i, hi_i), lo_i even
                    int p = lo_i + 2 * sidx;
                    for (; p < hi_i && p < chk; p += stride) {
                        const bool v0 = p > jmin, v1 = (p + 1 < b) && (p + 1 > jmin);
                        settle(core(p, v0, v1), p, 1, v0, v1);
                    }
                    // body: kGroup steps per vote.  In the fixed-point
                    // both-kinds pass (register room at four CTAs per SM) the
                    // next group's candidates are loaded before this group is
                    // evaluated, so their latency overlaps this group's
                    // arithmetic and the vote; the single-kind fixed-point
                    // kernels ran 4-6% slower that way.
                    if (!kPrefetch) {
                        for (; p + (kGroup - 1) * stride + 1 < hi_i; p += kGroup * stride) {
                            bool any = false;
                            #pragma unroll
                            for (int k = 0; k < kGroup; ++k) any |= core(p + k * stride, true, true);
                            settle(any, p, kGroup, true, true);
                        }
                    } else if (kStage && H == 32) {
                        // the steps p + 1 < hi_i, in windows of kStageCands
                        // candidates copied into this warp's shared buffers by
                        // cp.async (double-buffered; all lanes walk the same
                        // candidates, so reads broadcast)
                        const int nst = p + 1 < hi_i ? (hi_i - p) / 2 : 0;
                        const int nwin = (nst + kStageCands / 2 - 1) / (kStageCands / 2);
                        const int p0 = p;
                        auto stage = [&](int w) {
                            const int q = p0 + kStageCands * w;
                            float4 *dst = stg_f4 + (w & 1) * kStageCands;
                            if (lane < kStageCands) {
                                // float4 q + lane belongs to the block of point q + (lane & ~1)
                                const bool in = q + (lane & ~1) < hi_i;
                                const unsigned d = (unsigned)__cvta_generic_to_shared(dst + lane);
                                asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;"
                                             :: "r"(d), "l"(cpk + q + lane), "r"(in ? 16 : 0));
                            } else if (FIX && lane < kStageCands + kStageCands / 2) {
                                const int t = 2 * (lane - kStageCands);
                                const bool in = q + t < hi_i;
                                const unsigned d = (unsigned)__cvta_generic_to_shared(
                                    stg_q + (w & 1) * kStageCands + t);
                                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;"
                                             :: "r"(d), "l"(cqw + q + t), "r"(in ? 8 : 0));
                            }
                            asm volatile("cp.async.commit_group;" ::: "memory");
                        };
                        if (nwin > 0) stage(0);
                        if (nwin > 1) stage(1);
                        for (int w = 0; w < nwin; ++w) {
                            if (w + 1 < nwin) asm volatile("cp.async.wait_group 1;" ::: "memory");
                            else asm volatile("cp.async.wait_group 0;" ::: "memory");
                            __syncwarp();
                            const int ns = min(kStageCands / 2, nst - (kStageCands / 2) * w);
                            const float4 *sf = stg_f4 + (w & 1) * kStageCands;
                            const uint2 *sq = reinterpret_cast<const uint2 *>(stg_q + (w & 1) * kStageCands);
                            for (int s = 0; s < ns; ++s) {
                                Raw r;
                                r.qa = sf[2 * s];
                                r.qb = sf[2 * s + 1];
                                r.q = FIX ? sq[s] : make_uint2(0u, 0u);
                                settle(core_raw(r, true, true), p0 + kStageCands * w + 2 * s, 1, true, true);
                            }
                            __syncwarp();  // every lane has read this buffer
                            if (w + 2 < nwin) stage(w + 2);
                        }
                        p = p0 + 2 * nst;
                    } else if (p + (kGroup - 1) * stride + 1 < hi_i) {
                        Raw nx[kGroup];
                        #pragma unroll
                        for (int k = 0; k < kGroup; ++k) nx[k] = load(p + k * stride);
                        for (;;) {
                            Raw cur[kGroup];
                            #pragma unroll
                            for (int k = 0; k < kGroup; ++k) cur[k] = nx[k];
                            const int pn = p + kGroup * stride;
                            const bool more = pn + (kGroup - 1) * stride + 1 < hi_i;
                            if (more) {
                                #pragma unroll
                                for (int k = 0; k < kGroup; ++k) nx[k] = load(pn + k * stride);
                            }
                            bool any = false;
                            #pragma unroll
                            for (int k = 0; k < kGroup; ++k) any |= core_raw(cur[k], true, true);
                            settle(any, p, kGroup, true, true);
                            p = pn;
                            if (!more) break;
                        }
                    }
                    for (; p + 1 < hi_i; p += stride) settle(core(p, true, true), p, 1, true, true);
                    if (p < hi_i) settle(core(p, true, false), p, 1, true, false);
                };
                // flush before a shared counter could wrap: a chunk of c
                // candidates adds at most c * H times to one per-warp counter
                // and at most c / S + 2 times to one per-lane counter
                for (int lo_i = a & ~1; lo_i < b; lo_i += A.chunk) {
                    const int hi_i = min(b, lo_i + A.chunk);
                    if (HM != H_GLOBAL) {
                        const int c = hi_i - lo_i;
                        const int adds = (HM == H_LANE || HM == H_LFIX) ? c / S + 2 : c * H;
                        if (since + adds > budget) {
                            flush(ws.slot, J.wunscale);
                            since = 0;
                        }
                        since += adds;
                    }
                    run(lo_i, hi_i);
                }
            }
        }
        __syncwarp();  // the next item overwrites this item's rows and homes
      }
      tk = __shfl_sync(kFull, tk, 0);
      ticket_items(tk, ib, ie);
      // give up the queue on an abort request or past the iteration cap
      // (the histogram copy is still flushed below; the host discards it)
      stop = __shfl_sync(kFull, stop, 0) ? PCF_GAVE_UP_ABORT : 0u;
      if (++taken > A.max_tickets) stop |= PCF_GAVE_UP_CAP;
      if (stop) {
          if (lane == 0 && A.status) ctrl_store(A.status, stop);
          break;
      }
    }
    // per-warp flush (no CTA barrier: warps leave as the queue drains)
    __syncwarp();
    if (ws.cj >= 0) flush(ws.slot, J.wunscale);
    unsigned long long rp = n_pairs, rr = n_rechk;
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(kFull, rr, off);
        rp += __shfl_down_sync(kFull, rp, off);
    }
    if (lane == 0) {
        if (rr) atomicAdd(A.g_stats + 0, rr);
        if (ws.n_cand) atomicAdd(A.g_stats + 1, ws.n_cand);
        if (COUNT && rp) atomicAdd(A.g_stats + 2, rp);
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
// Home tiles: up to kTileCap consecutive points of one (ix, iy) column,
// spanning at most two adjacent cells [z0, z1], so a warp's lanes stay busy
// when cells hold fewer than 32 points.  Two cells keep a periodic stencil
// within the box: the counts require 2k + 2 <= P for k neighbour cells per
// side, and a row covers z0 - k .. z1 + k.
void build_tiles(const CellGrid &g, int cap, std::vector<TileDesc> &out) {
    const int P = g.P;
    const std::vector<int> &hs = g.h_start;
    out.clear();
    for (int ix = 0; ix < P; ++ix)
        for (int iy = 0; iy < P; ++iy) {
            const int col = (ix * P + iy) * P;
            int iz = 0;
            int p = hs[col];
            const int end = hs[col + P];
            while (p < end) {
                while (hs[col + iz + 1] <= p) ++iz;  // cell of point p
                const int limit = hs[col + std::min(iz + 2, P)];
                const int n = std::min(cap, limit - p);
                int z1 = iz;
                while (hs[col + z1 + 1] < p + n) ++z1;  // cell of the tile's last point
                TileDesc t;
                t.start = p;
                t.count = n;
                t.ix = (int16_t)ix;
                t.iy = (int16_t)iy;
                t.z0 = (int16_t)iz;
                t.z1 = (int16_t)z1;
                out.push_back(t);
                p += n;
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
                int resident_warps, int tile_cap) {
    const int P = home.P;
    plan.P = P;
    plan.cell = (float)((double)box / P);
    plan_rows(P, box, dmax, ani, self, plan.rows);
    // ~16 items per resident warp keeps the tail short; at most 32 rows each
    const int64_t nt = (int64_t)home.tiles_for(tile_cap).size();
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

static int copy_words_host(int hm, int nb) {
    switch (hm) {
    case H_LANE: return copy_words<H_LANE>(nb);
    case H_WARP: return copy_words<H_WARP>(nb);
    case H_WFIX: return copy_words<H_WFIX>(nb);
    case H_LFIX: return copy_words<H_LFIX>(nb);
    case H_WFIX4: return copy_words<H_WFIX4>(nb);
    case H_WFIX2: return copy_words<H_WFIX2>(nb);
    }
    return 0;
}

// The one-pass variant of a launch (PCF_OPT_PAIR_VARIANT): only the weighted
// both-kinds kernel with per-warp fixed-point copies has variants.
static int pair_variant(const PairLaunch &pl, int hm, int n_jobs = 1) {
    const int v = (pl.both && pl.weighted && hm == H_WFIX && !pl.count) ? pl.variant : 0;
    return (v == 3 && n_jobs != 1) ? 0 : v;  // shared copies hold one job's adds only
}

template <int KIND, bool W, int HM, bool C, int VAR = 0>
static cudaError_t launch_one(const PairArgs &A, size_t smem, long long n_items, cudaStream_t st,
                              int sm_count, int device) {
    auto kfn = k_pairs<KIND, W, HM, C, VAR>;
    // occupancy queries cost microseconds: cached per (device, shared-memory
    // size) and instantiation, under a lock (several host threads launch)
    struct Occ {
        std::mutex mu;
        std::map<std::pair<int, size_t>, int> per_sm;
    };
    static Occ occ;
    cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(kfn), device, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(occ.mu);
        auto it = occ.per_sm.find({device, smem});
        if (it != occ.per_sm.end()) {
            per_sm = it->second;
        } else {
            int per = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kfn, kThreads, smem);
            if (e != cudaSuccess) return e;
            per_sm = std::max(1, per);
            occ.per_sm[{device, smem}] = per_sm;
        }
    }
    const long long want = (n_items + kWarps - 1) / kWarps;
    const int grid = (int)std::max(1LL, std::min<long long>(want, (long long)sm_count * per_sm));
    // runs of k items per ticket while a queue holds >= 32 runs per warp (k at
    // most 8, or the tuned cap that A.kchunk carries in)
    PairArgs B = A;
    const long long warps = (long long)grid * kWarps;
    const long long cap = A.kchunk > 0 ? std::min<long long>(A.kchunk, kChunkMax) : kChunkMax;
    B.kchunk = (int)std::max(1LL, std::min<long long>(cap, n_items / (warps * 32)));
    B.n_chunked = B.kchunk > 1 ? std::max(0LL, n_items - 2 * warps) : 0;
    B.t_chunked = (B.n_chunked + B.kchunk - 1) / B.kchunk;
    // a warp can take at most every ticket of the queue plus the one that
    // finds it empty
    B.max_tickets = B.t_chunked + (n_items - B.n_chunked) + 2;
    kfn<<<grid, kThreads, smem, st>>>(B);
    return cudaGetLastError();
}

// Shared-memory bytes per CTA of histogram scheme hm for launch pl (both
// kinds: the anisotropic copy plus the isotropic one).
static size_t scheme_bytes(const PairLaunch &pl, int hm, int n_jobs = 1) {
    const int bins = pl.rule.bins;
    const int nb = pl.ani ? bins * bins : bins;
    const size_t e = (hm == H_WFIX || hm == H_LFIX) ? 4 : (pl.weighted ? 8 : 4);
    const int var = pair_variant(pl, hm, n_jobs);
    if (var == 3)  // per-warp isotropic copies, one anisotropic copy per warp pair
        return e * ((size_t)kWarps * copy_words_host(iso_scheme(pl.weighted, hm, var), bins) +
                    (size_t)(kWarps / 2) * ((size_t)nb * kLimbs + 2 * (32 + kLimbs - 1)));
    size_t w = (size_t)copy_words_host(hm, nb);
    if (pl.both) w += (size_t)copy_words_host(iso_scheme(pl.weighted, hm, var), bins);
    size_t b = w * e * kWarps;
    if (var == 2) b = ((b + 15) & ~(size_t)15) + (size_t)kWarps * kStageBytes;
    return b;
}

static bool scheme_fits(const PairLaunch &pl, int hm) {
    if (pl.rule.bins > 255) return hm == H_GLOBAL;
    switch (hm) {
    case H_LANE: return !pl.ani && scheme_bytes(pl, hm) <= 64 * 1024;
    case H_LFIX: return !pl.ani && pl.weighted && pl.wfix && scheme_bytes(pl, hm) <= 64 * 1024;
    case H_WFIX: return pl.weighted && pl.wfix && scheme_bytes(pl, hm) <= 160 * 1024;
    case H_WARP: return scheme_bytes(pl, hm) <= 160 * 1024;
    case H_GLOBAL: return true;
    }
    return false;
}

// The histogram scheme of one launch: lane-private copies where they fit
// (isotropic), else one copy per warp, else global atomics; an autotuned
// scheme overrides the rule when it is valid for the launch.  For a
// both-kinds launch the scheme is the anisotropic copy's; the isotropic copy
// takes the matching scheme (IsoScheme).
static int pair_scheme(const PairLaunch &pl) {
    int hm;
    if (pl.rule.bins > 255 || !scheme_fits(pl, H_WARP)) hm = H_GLOBAL;
    else if (pl.weighted && scheme_fits(pl, H_LFIX)) hm = H_LFIX;
    else if (pl.weighted && scheme_fits(pl, H_WFIX)) hm = H_WFIX;
    else if (!pl.weighted && scheme_fits(pl, H_LANE)) hm = H_LANE;
    else hm = H_WARP;
    if (pl.hist_mode >= 0 && pl.hist_mode <= H_LFIX && scheme_fits(pl, pl.hist_mode)) hm = pl.hist_mode;
    return hm;
}

// Chooses the histogram mode of one launch and starts the kernel.
static cudaError_t dispatch_pairs(PairArgs A, const PairLaunch &pl, cudaStream_t st,
                                  int sm_count, int device) {
    const int hm = pair_scheme(pl);
    const size_t smem = hm == H_GLOBAL ? 0 : scheme_bytes(pl, hm, A.n_jobs);
    // budget: adds one shared counter absorbs between flushes; chunk:
    // candidates per budget check (one chunk alone stays within the budget)
    if (hm == H_WFIX || hm == H_LFIX) {
        A.budget = pl.wbudget;
        A.chunk = std::max(2, (pl.wbudget / 32) & ~1);
    } else {
        A.budget = 1 << 30;  // u32 counters: flushed long before 2^32
        A.chunk = 1 << 22;
    }
    const long long n = A.n_items;
    const bool C = pl.weighted && pl.count;
#define PCF_LAUNCH(K_, W_, H_)                                                                     \
    return C ? launch_one<K_, W_, H_, true>(A, smem, n, st, sm_count, device)                      \
             : launch_one<K_, W_, H_, false>(A, smem, n, st, sm_count, device)
    if (!pl.ani) {
        if (pl.weighted) {
            if (hm == H_LANE) PCF_LAUNCH(K_ISO, true, H_LANE);
            if (hm == H_WARP) PCF_LAUNCH(K_ISO, true, H_WARP);
            if (hm == H_WFIX) PCF_LAUNCH(K_ISO, true, H_WFIX);
            if (hm == H_LFIX) PCF_LAUNCH(K_ISO, true, H_LFIX);
            PCF_LAUNCH(K_ISO, true, H_GLOBAL);
        }
        if (hm == H_LANE) return launch_one<K_ISO, false, H_LANE, false>(A, smem, n, st, sm_count, device);
        if (hm == H_WARP) return launch_one<K_ISO, false, H_WARP, false>(A, smem, n, st, sm_count, device);
        return launch_one<K_ISO, false, H_GLOBAL, false>(A, smem, n, st, sm_count, device);
    }
    const int var = pair_variant(pl, hm, A.n_jobs);
    if (pl.both && var == 1) return launch_one<K_BOTH, true, H_WFIX, false, 1>(A, smem, n, st, sm_count, device);
    if (pl.both && var == 3) return launch_one<K_BOTH, true, H_WFIX, false, 3>(A, smem, n, st, sm_count, device);
    if (pl.both && var == 2) return launch_one<K_BOTH, true, H_WFIX, false, 2>(A, smem, n, st, sm_count, device);
#define PCF_DISPATCH_A(K_)                                                                         \
    if (pl.weighted) {                                                                             \
        if (hm == H_WARP) PCF_LAUNCH(K_, true, H_WARP);                                            \
        if (hm == H_WFIX) PCF_LAUNCH(K_, true, H_WFIX);                                            \
        PCF_LAUNCH(K_, true, H_GLOBAL);                                                            \
    }                                                                                              \
    if (hm == H_WARP) return launch_one<K_, false, H_WARP, false>(A, smem, n, st, sm_count, device); \
    return launch_one<K_, false, H_GLOBAL, false>(A, smem, n, st, sm_count, device);
    if (pl.both) { PCF_DISPATCH_A(K_BOTH) }
    PCF_DISPATCH_A(K_ANI)
#undef PCF_DISPATCH_A
#undef PCF_LAUNCH
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
    (void)P;  // partitions travel per job (PairJob::P)
    A.box = box;
    A.bpc = pl.bpc ? 1 : 0;
    A.rule = pl.rule;
    A.fc = make_cuts(pl.rule, box, std::sqrt((float)pl.rule.dd));
    A.zreach = (float)(std::sqrt(pl.rule.dd) * (1.0 + 1e-5));
    A.g_count = d_count;
    A.g_wsum = d_wsum;
    A.g_stats = d_stats;
    A.chunk = 1 << 22;
    A.budget = 1 << 30;
    A.fast = pl.rule.bins <= 255 ? 1 : 0;
    A.ctrl = pl.ctrl;
    A.status = pl.status;
    A.max_tickets = n_items + 2;  // refined per launch shape in launch_one
    A.kchunk = pl.chunk_cap;      // a cap here; launch_one sets the run length
    return A;
}

// Fixed-point weighted histograms: every grid has exact integer weights q <
// 2^32 (set_weight_range), so a product q_a*q_b is exact in 64 bits and
// splits into limbs l0 = bits 0-15, l1 = bits 16-31, l2 = bits 32-63.  A u32
// counter absorbs 65536 adds of l0 or l1, and floor((2^32-1) / max l2) adds
// of l2: the smaller is the flush budget.  Launches whose largest product
// would leave a budget under 4096 keep FP64 shared atomics.
void set_weight_fix(PairLaunch &pl, const pcf_grid *const *gs, int n) {
    pl.wfix = false;
    pl.wbudget = 0;
    if (!pl.weighted) return;
    unsigned long long qmax = 0;
    for (int i = 0; i < n; ++i) {
        if (!gs[i]->wfix_ok) return;
        qmax = std::max(qmax, gs[i]->wqmax);
    }
    const unsigned __int128 top = (unsigned __int128)qmax * qmax;
    const unsigned long long hi = (unsigned long long)(top >> 32);
    const unsigned long long budget = hi ? std::min<unsigned long long>(65536, 0xFFFFFFFFull / hi) : 65536;
    if (budget < 4096) return;
    pl.wfix = true;
    pl.wbudget = (int)budget;
}

double weight_unscale(const pcf_grid *home, const pcf_grid *cand) {
    return std::ldexp(1.0, -(home->wshift + cand->wshift));
}

PairView pair_view(const CellGrid &g, bool with_q) {
    return PairView{g.pk.as<float4>(), with_q ? g.qw.as<unsigned>() : nullptr,
                    g.cell_start.as<int>()};
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

cudaError_t launch_pairs_view(const PairView &home, const PairView &cand, const TileDesc *tiles,
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
    j.rule_flags2 = pl.flags2;
    j.pad = 0;
    j.P = P;
    j.wunscale = 0.0;
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
        PCF_CU(ctx, counted_malloc_host(&sl.h_pinned, want));
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
    job.home = pair_view(home, pl.wfix);
    job.cand = pair_view(cand, pl.wfix);
    job.tiles = home.d_tiles_for(pl.tile_cap);
    job.rows = sl->d_rows.as<RowDesc>();
    job.n_rows = (int)plan.rows.size();
    job.rows_per_item = plan.rows_per_item;
    job.n_chunks = plan.n_chunks;
    job.slot = 0;
    job.item_begin = 0;
    job.rule_flags = pl.rule.flags;
    job.rule_flags2 = pl.flags2;
    job.pad = 0;
    job.P = plan.P;
    job.wunscale = pl.wunscale;
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

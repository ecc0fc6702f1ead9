// triplets.cu -- isotropic triplet histograms DDD / RRR / DDR / DRR on the
// CUDA cores.
//
// Reference kernels replaced: XXX3iso / XXY3iso (cuda/kernels/3iso_k.cuh:8,94)
// and the periodic count123 / count123_mixed / XXX3iso_BPC / XXY3iso_BPC
// (cuda/kernels/3isoBPC_k.cuh:8,98,191,940), which run one thread per cell
// *triple* with a global FP64 atomic per triangle and spell out 64 image
// combinations.  Here:
//
//  * A persistent CTA takes one anchor point i at a time.  It scans the
//    anchor's neighbour cells (the pair stencil, periodic images by index
//    wrap) and compacts into shared memory the X neighbours j > i (list J)
//    and, for XXY, all Y neighbours (list K), each with its FP32 image
//    displacement from i and its exact side bin (FP32 fast path + FP64
//    recheck, as in the pair kernel).
//  * It then runs the pairs of that list: XXX pairs (j < k) of J, XXY all of
//    J x K.  The third side is |v_k - v_j| -- the consistent embedding of
//    count123 (3isoBPC_k.cuh:56-75) -- tested and binned in FP32 with the
//    same edge-window recheck.  Each unordered XXX triangle is seen once (i
//    its lowest index), each unordered XX pair of an XXY triangle once.
//  * Counts go to a shared u32 histogram U[b_ij][b_jk][b_ki] (one
//    orientation per triangle); the finalize pass symmetrises it into the
//    reference's ordered-triple histogram: XXX sums the 6 axis
//    permutations, XXY the two orders of the XX pair (b_jk <-> b_ki).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>
#include <type_traits>

#include "pcf_internal.cuh"
#include "node_gates.cuh"

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kTThreads = 512;  // 16 warps, one CTA per SM
constexpr int kTWarps = kTThreads / 32;
constexpr float kMagic = 256.0f;
constexpr int kFracBits = 15;
constexpr unsigned kFracMask = (1u << kFracBits) - 1u;
constexpr unsigned kBinBias = 0x43800000u >> kFracBits;  // bits(256 + r) >> 15 = this + floor(r)
#ifndef PCF_TRIP_GROUP
#define PCF_TRIP_GROUP 2  // third-side steps between recheck votes
#endif

struct TripCuts {
    float dsf, ds2;
    float lo, hi;  // d2 window around dd (image-aware bound for periodic boxes)
    unsigned w;    // edge window, 2^-15 units of r
};

struct Cat {
    const float *x, *y, *z, *w;
    const int *cstart;
};

struct TripArgs {
    Cat X, Y;
    int nX;
    const RowDesc *rows;
    int n_rows;
    int P;
    float cell;
    float box;
    int bpc;
    PairRule rXX, rXY;  // side rules (X-X side, X-Y sides)
    TripCuts fc;
    int capJ, capK;          // shared-memory list capacities (entries)
    float4 *gJ, *gK;         // per-CTA overflow lists in global memory
    float *gwJ, *gwK;        // weights of the overflow lists
    int gcap;                // entries per CTA in the overflow lists
    unsigned long long *counter;
    unsigned long long *g_count;  // bins^3 (unit weights)
    double *g_wsum;               // bins^3 (weighted)
    int hist_in_smem;
    unsigned long long *g_stats;
    // adds the shared u32 histogram absorbs between flushes into g_count
    // (a counter then never wraps: one slot gets at most that many adds)
    unsigned long long flush_budget;
    const unsigned *ctrl;  // abort request, polled with every anchor (null: none)
    unsigned *status;      // where a CTA that gives up records why (null: none)
    // batched launches (k_triplets_batch): this job's anchors are the
    // queue's [anchor_begin, anchor_begin + nX); mixed: XXY
    long long anchor_begin;
    int mixed;
    GateGeom gate;  // the reference's node grid (PCF_REF_NODE_GATES)
};

__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ bool fix_safe(unsigned q, unsigned w) {
    return ((q + w) & kFracMask) >= 2u * w;
}

// Exact FP64 side between two catalog points (minimum image when periodic),
// returned as components.
__device__ __forceinline__ void sep_exact(float ax, float ay, float az, float bx, float by,
                                          float bz, int bpc, double L, double &dx, double &dy,
                                          double &dz) {
    dx = __dsub_rn((double)bx, (double)ax);
    dy = __dsub_rn((double)by, (double)ay);
    dz = __dsub_rn((double)bz, (double)az);
    if (bpc) {
        const double h = 0.5 * L;
        if (dx > h) dx = __dsub_rn(dx, L); else if (dx < -h) dx = __dadd_rn(dx, L);
        if (dy > h) dy = __dsub_rn(dy, L); else if (dy < -h) dy = __dadd_rn(dy, L);
        if (dz > h) dz = __dsub_rn(dz, L); else if (dz < -h) dz = __dadd_rn(dz, L);
    }
}

// Side bin of the anchor -> candidate pair in the canonical FP64 rule.
__device__ __noinline__ int exact_side(float ax, float ay, float az, float bx, float by, float bz,
                                       int bpc, float box, PairRule rule) {
    double dx, dy, dz;
    sep_exact(ax, ay, az, bx, by, bz, bpc, (double)box, dx, dy, dz);
    return exact_slot<false>(dx, dy, dz, rule);
}

// Bin of side j-k in the consistent embedding anchored at i: v_jk = v_ik - v_ij.
__device__ __noinline__ int exact_third(float ix, float iy, float iz, float jx, float jy, float jz,
                                        float kx, float ky, float kz, int bpc, float box,
                                        PairRule rule) {
    double ax, ay, az, bx, by, bz;
    sep_exact(ix, iy, iz, jx, jy, jz, bpc, (double)box, ax, ay, az);
    sep_exact(ix, iy, iz, kx, ky, kz, bpc, (double)box, bx, by, bz);
    return exact_slot<false>(__dsub_rn(bx, ax), __dsub_rn(by, ay), __dsub_rn(bz, az), rule);
}

// FP32 fast-path bin of a squared distance, or -1 (recheck needed), -2 (out).
__device__ __forceinline__ int fast_bin(float d2, const TripCuts &c, int bins) {
    if (!(d2 < c.hi)) return -2;
    const float r = sqrt_approx(d2 * c.ds2);
    const unsigned q = __float_as_uint(r + kMagic) & 0x7FFFFFu;
    if (d2 < c.lo && fix_safe(q, c.w)) return min((int)(q >> kFracBits), bins - 1);
    return -1;
}

// Appends the neighbours of anchor (hx,hy,hz) found in catalog C to a list.
// only_after >= 0 keeps candidates with index > only_after (X list of XXX /
// XXY).  Entries: {dx, dy, dz, bits(idx << 8 | bin)}.
// Angle bin of the anisotropic 3-point histograms for the side anchor->point:
// t = (int)((1 + dz/d) * (float)(bins/2)) (3ani_k.cuh:79-91), dz signed, or
// with periodic boxes dz = |z2-z1| - L*f (3aniBPC_k.cuh:57,73); -1 when >= bins.
__device__ __noinline__ int exact_angle(float ax, float ay, float az, float bx, float by, float bz,
                                        int bpc, float box, int bins, float ds_th) {
    double dx, dy, dz;
    sep_exact(ax, ay, az, bx, by, bz, bpc, (double)box, dx, dy, dz);
    const double d = __dsqrt_rn(exact_d2(dx, dy, dz));
    double dzr = dz;
    if (bpc) {
        const double raw = fabs(__dsub_rn((double)bz, (double)az));
        dzr = raw > 0.5 * (double)box ? __dsub_rn(raw, (double)box) : raw;
    }
    const double c = __dadd_rn(1.0, __ddiv_rn(dzr, d));
    const int t = (int)__dmul_rn(c, (double)ds_th);
    return (t >= 0 && t < bins) ? t : -1;
}

// ginfo (PCF_REF_NODE_GATES): per entry, its node on the reference's grid
// and the axes of its image relative to the anchor (gate_pack).
template <bool ANG>
__device__ void build_list(const TripArgs &A, const Cat &C, float hx, float hy, float hz, int hcell_ix,
                           int hcell_iy, int hcell_iz, int only_after, const PairRule &rule,
                           float4 *list, float *wlist, int cap, int *s_n, unsigned &n_rechk,
                           unsigned short *ang = nullptr, int step = 1, unsigned *ginfo = nullptr) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int P = A.P;
    for (int r = 0; r < A.n_rows; ++r) {
        const RowDesc rw = A.rows[r];
        int nx = hcell_ix + rw.dx, ny = hcell_iy + rw.dy;
        float sx = 0.f, sy = 0.f;
        if (A.bpc) {
            if (nx < 0) { nx += P; sx = -A.box; } else if (nx >= P) { nx -= P; sx = A.box; }
            if (ny < 0) { ny += P; sy = -A.box; } else if (ny >= P) { ny -= P; sy = A.box; }
        } else if (nx < 0 || nx >= P || ny < 0 || ny >= P) {
            continue;
        }
        const int col = (nx * P + ny) * P;
        const int zlo = hcell_iz - rw.kz, zhi = hcell_iz + rw.kz;
        int ra[2], rb[2];
        float rz[2] = {0.f, 0.f};
        ra[0] = C.cstart[col + max(zlo, 0)];
        rb[0] = C.cstart[col + min(zhi, P - 1) + 1];
        ra[1] = rb[1] = 0;
        if (A.bpc) {
            if (zlo < 0) { ra[1] = C.cstart[col + zlo + P]; rb[1] = C.cstart[col + P]; rz[1] = -A.box; }
            else if (zhi >= P) { ra[1] = C.cstart[col]; rb[1] = C.cstart[col + zhi - P + 1]; rz[1] = A.box; }
        }
        for (int sgi = 0; sgi < 2; ++sgi) {
            int a = ra[sgi];
            const int b = rb[sgi];
            if (only_after >= 0) a = max(a, only_after + 1);
            if (a >= b) continue;
            const float ex = hx - sx, ey = hy - sy, ez = hz - rz[sgi];
            // warps take 32-candidate chunks
            for (int base = a + warp * 32; base < b; base += kTWarps * 32) {
                const int c = base + lane;
                int bin = -2;
                float vx = 0.f, vy = 0.f, vz = 0.f;
                if (c < b) {
                    vx = C.x[c] - ex;
                    vy = C.y[c] - ey;
                    vz = C.z[c] - ez;
                    const float d2 = fmaf(vz, vz, fmaf(vy, vy, vx * vx));
                    bin = fast_bin(d2, A.fc, rule.bins);
                    if (bin == -1) {
                        ++n_rechk;
                        bin = exact_side(hx, hy, hz, C.x[c], C.y[c], C.z[c], A.bpc, A.box, rule);
                    }
                }
                int tang = 0;
                if (ANG && bin >= 0) {
                    tang = exact_angle(hx, hy, hz, C.x[c], C.y[c], C.z[c], A.bpc, A.box, rule.bins,
                                       (float)rule.bins / 2.0f);
                    if (tang < 0) bin = -2;  // the side can close no triangle
                }
                const bool keep = bin >= 0;
                const unsigned m = __ballot_sync(kFull, keep);
                int off = 0;
                if (lane == 0 && m) off = atomicAdd(s_n, __popc(m));
                off = __shfl_sync(kFull, off, 0);
                if (keep) {
                    const int pos = off + __popc(m & ((1u << lane) - 1u));
                    if (pos < cap) {  // step -1: the list grows downwards from `list`
                        list[step * pos] = make_float4(vx, vy, vz, __int_as_float((c << 8) | bin));
                        if (wlist) wlist[pos] = C.w[c];
                        if (ANG) ang[pos] = (unsigned short)(bin | (tang << 8));
                        if (ginfo)
                            ginfo[pos] = gate_pack(A.gate, C.x[c], C.y[c], C.z[c],
                                                   (sx != 0.f ? 1u : 0u) | (sy != 0.f ? 2u : 0u) |
                                                       (rz[sgi] != 0.f ? 4u : 0u));
                    }
                }
            }
        }
    }
}

// Adds the shared histogram U (nb3 u32) into the u64 histogram g and clears
// it (whole CTA).
__device__ __forceinline__ void flush_hist(unsigned *U, int nb3, unsigned long long *g) {
    __syncthreads();
    for (int k = threadIdx.x; k < nb3; k += kTThreads) {
        const unsigned v = U[k];
        if (v) {
            atomicAdd(g + k, (unsigned long long)v);
            U[k] = 0u;
        }
    }
    __syncthreads();
}

// Per-CTA state of the anchor loop.
struct TripCta {
    unsigned *U;                      // shared histogram (hist_in_smem)
    unsigned char *lists;             // shared neighbour lists
    int *s_nJ, *s_nK, *s_unit;        // shared counters
    unsigned n_rechk;
    unsigned long long n_tri;
    unsigned long long since;         // pair tests since U's last flush
};

// All triangles of anchor i of job A: pass 1 builds the anchor's
// neighbour lists in shared memory (or, past their capacity, in this CTA's
// global scratch), pass 2 counts the neighbour pairs.
template <bool MIXED, bool WEIGHTED>
__device__ __forceinline__ void tri_anchor(const TripArgs &A, int i, TripCta &C) {
    const int bins = A.rXX.bins;
    const int nb3 = bins * bins * bins;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned *U = C.U;
    int &s_nJ = *C.s_nJ, &s_nK = *C.s_nK, &s_unit = *C.s_unit;
    unsigned &n_rechk = C.n_rechk;
    unsigned long long &n_tri = C.n_tri;
    unsigned long long &since = C.since;
    float4 *sJ = reinterpret_cast<float4 *>(C.lists);
    float4 *sK = sJ + A.capJ;
    float *swJ = reinterpret_cast<float *>(sK + (MIXED ? A.capK : 0));
    float *swK = swJ + (WEIGHTED ? A.capJ : 0);
    float4 *gJ = A.gJ + (size_t)blockIdx.x * A.gcap;
    float4 *gK = A.gK ? A.gK + (size_t)blockIdx.x * A.gcap : nullptr;
    float *gwJ = A.gwJ ? A.gwJ + (size_t)blockIdx.x * A.gcap : nullptr;
    float *gwK = A.gwK ? A.gwK + (size_t)blockIdx.x * A.gcap : nullptr;
    auto flush_u = [&]() { flush_hist(U, nb3, A.g_count); };
        const float hx = A.X.x[i], hy = A.X.y[i], hz = A.X.z[i];
        const float hw = WEIGHTED ? A.X.w[i] : 1.f;
        const int P = A.P;
        const int cix = min(max((int)__fdiv_rn(hx, A.cell), 0), P - 1);
        const int ciy = min(max((int)__fdiv_rn(hy, A.cell), 0), P - 1);
        const int ciz = min(max((int)__fdiv_rn(hz, A.cell), 0), P - 1);
        // pass 1: lists into shared memory (sizes counted even past capacity).
        // Pooled (XXY, unit weights, shared histogram): one buffer of capJ
        // entries, J from the front and K from the back, so the anchor
        // overflows only when both together exceed it.
        const bool pool = MIXED && !WEIGHTED && A.hist_in_smem;
        build_list<false>(A, A.X, hx, hy, hz, cix, ciy, ciz, i, A.rXX, sJ, WEIGHTED ? swJ : nullptr,
                          A.capJ, &s_nJ, n_rechk);
        int capK = A.capK;
        if (pool) {
            __syncthreads();
            capK = max(0, A.capJ - s_nJ);
        }
        if (MIXED)
            build_list<false>(A, A.Y, hx, hy, hz, cix, ciy, ciz, -1, A.rXY, pool ? sJ + A.capJ - 1 : sK,
                              WEIGHTED ? swK : nullptr, capK, &s_nK, n_rechk, nullptr, pool ? -1 : 1);
        __syncthreads();
        int nJ = s_nJ, nK = MIXED ? s_nK : nJ;
        const float4 *LJ = sJ;
        const float4 *LK = MIXED ? sK : sJ;
        const float *WJ = swJ, *WK = MIXED ? swK : swJ;
        if (nJ > A.capJ || (MIXED && nK > capK)) {
            // overflow: rebuild the lists in this CTA's global scratch (L2)
            __syncthreads();
            if (tid == 0) { s_nJ = 0; s_nK = 0; }
            __syncthreads();
            build_list<false>(A, A.X, hx, hy, hz, cix, ciy, ciz, i, A.rXX, gJ,
                              WEIGHTED ? gwJ : nullptr, A.gcap, &s_nJ, n_rechk);
            if (MIXED)
                build_list<false>(A, A.Y, hx, hy, hz, cix, ciy, ciz, -1, A.rXY, gK,
                                  WEIGHTED ? gwK : nullptr, A.gcap, &s_nK, n_rechk);
            __threadfence_block();
            __syncthreads();
            nJ = min(s_nJ, A.gcap);
            nK = MIXED ? min(s_nK, A.gcap) : nJ;
            LJ = gJ;
            LK = MIXED ? gK : gJ;
            WJ = gwJ;
            WK = MIXED ? gwK : gwJ;
        }
        // K entry k is LK[kstepK * k]: the pooled K list grows downwards from
        // the end of the shared buffer
        int kstepK = 1;
        if (pool && LJ == sJ) {
            LK = sJ + A.capJ - 1;
            kstepK = -1;
        }
        // Flush budget of the shared histogram: this anchor adds at most
        // `tests` times.  Flush first if the total could pass the budget; an
        // anchor whose tests alone exceed it counts into global memory.
        bool smem_hist = !WEIGHTED && A.hist_in_smem;
        if (smem_hist) {
            const unsigned long long tests =
                MIXED ? (unsigned long long)nJ * (unsigned long long)nK
                      : (unsigned long long)nJ * (unsigned long long)(nJ > 0 ? nJ - 1 : 0) / 2;
            if (tests > A.flush_budget) {
                smem_hist = false;
            } else {
                if (since + tests > A.flush_budget) {
                    flush_u();
                    since = 0;
                }
                since += tests;
            }
        }
        // pass 2: pairs of neighbours.  Rows j are dealt to warps in the
        // order 0, n-1, 1, n-2, ... (XXX rows shrink with j).
        if (smem_hist) {
            // the lists' address space is fixed per instantiation, so the
            // shared-memory case (all but overflowing anchors) uses shared loads
            // LKx[kstep * k] is K entry k (kstep -1: the pooled, downward K list)
            auto pass2 = [&](const float4 *__restrict__ LJx, const float4 *__restrict__ LKx, int kstep) {
            // Unit weights, shared histogram: two k per lane per step in packed
            // FP32, unpredicated shared reductions (a lane without a triangle
            // adds 0 to its dummy slot past the histogram), one recheck vote
            // per group of steps.
            const PairRule &r3 = MIXED ? A.rXY : A.rXX;
            const unsigned Us = (unsigned)__cvta_generic_to_shared(U);
            const unsigned dummy = Us + (unsigned)(nb3 + lane) * 4u;
            const float lo = A.fc.lo, hi = A.fc.hi;
            const unsigned w2 = 2u * A.fc.w;
            const float mgw = kMagic + (float)A.fc.w * 0x1p-15f;
            const float2 DS2 = make_float2(A.fc.ds2, A.fc.ds2);
            // Work units handed out dynamically (a shared counter), so warps
            // finish together: XXX rows j in order (largest first), XXY rows
            // split into `segs` segments of the K list when rows are few.
            const int segs = (MIXED && nJ < 8 * kTWarps) ? 4 : 1;
            const int units = nJ * segs;
            for (;;) {
                int u = 0;
                if (lane == 0) u = atomicAdd(&s_unit, 1);
                u = __shfl_sync(kFull, u, 0);
                if (u >= units) break;
                const int jj = u / segs, sg = u - jj * segs;
                const int kbeg = MIXED ? (int)((long long)nK * sg / segs) : jj + 1;
                const int kend = MIXED ? (int)((long long)nK * (sg + 1) / segs) : nK;
                const float4 ej = LJx[jj];
                const int bj = __float_as_int(ej.w) & 255;
                const int jidx = (int)((unsigned)__float_as_int(ej.w) >> 8);
                // slot = bj*bins^2 + b_jk*bins + b_k, with bits(r+256..) >> 15 = kBinBias + b_jk
                const unsigned base_j = Us + 4u * (unsigned)(bj * bins * bins - (int)kBinBias * bins);
                const float2 NJX = make_float2(-ej.x, -ej.x), NJY = make_float2(-ej.y, -ej.y),
                             NJZ = make_float2(-ej.z, -ej.z);
                struct Ev {
                    unsigned a0, a1;
                    bool f0, f1, r0, r1;
                };
                // k0 and (if v1) k0 + 32
                auto eval = [&](int k0, bool v1) -> Ev {
                    const float4 e0 = LKx[kstep * k0];
                    const float4 e1 = LKx[kstep * (v1 ? k0 + 32 : k0)];
                    const float2 DX = __fadd2_rn(make_float2(e0.x, e1.x), NJX);
                    const float2 DY = __fadd2_rn(make_float2(e0.y, e1.y), NJY);
                    const float2 DZ = __fadd2_rn(make_float2(e0.z, e1.z), NJZ);
                    float2 D2 = __fmul2_rn(DX, DX);
                    D2 = __ffma2_rn(DY, DY, D2);
                    D2 = __ffma2_rn(DZ, DZ, D2);
                    const float2 UU = __fmul2_rn(D2, DS2);
                    const float2 Q = __fadd2_rn(make_float2(sqrt_approx(UU.x), sqrt_approx(UU.y)),
                                                make_float2(mgw, mgw));
                    const unsigned u0 = __float_as_uint(Q.x), u1 = __float_as_uint(Q.y);
                    Ev e;
                    e.f0 = (D2.x < lo) && (u0 & kFracMask) >= w2;
                    e.f1 = v1 && (D2.y < lo) && (u1 & kFracMask) >= w2;
                    e.r0 = !e.f0 && D2.x < hi;
                    e.r1 = v1 && !e.f1 && D2.y < hi;
                    e.a0 = base_j + 4u * ((u0 >> kFracBits) * (unsigned)bins + (unsigned)(__float_as_int(e0.w) & 255));
                    e.a1 = base_j + 4u * ((u1 >> kFracBits) * (unsigned)bins + (unsigned)(__float_as_int(e1.w) & 255));
                    return e;
                };
                auto core = [&](int k0, bool v1) -> bool {
                    const Ev e = eval(k0, v1);
                    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(e.f0 ? e.a0 : dummy), "r"((unsigned)e.f0));
                    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(e.f1 ? e.a1 : dummy), "r"((unsigned)e.f1));
                    n_tri += (unsigned)e.f0 + (unsigned)e.f1;
                    return e.r0 || e.r1;
                };
                // third side by the canonical FP64 rule
                auto slow = [&](int kk) {
                    ++n_rechk;
                    const float4 ek = LKx[kstep * kk];
                    const int kidx = (int)((unsigned)__float_as_int(ek.w) >> 8);
                    const Cat &CK = MIXED ? A.Y : A.X;
                    const int bjk = exact_third(hx, hy, hz, A.X.x[jidx], A.X.y[jidx], A.X.z[jidx],
                                                CK.x[kidx], CK.y[kidx], CK.z[kidx], A.bpc, A.box, r3);
                    if (bjk >= 0) {
                        atomicAdd(U + bj * bins * bins + bjk * bins + (__float_as_int(ek.w) & 255), 1u);
                        ++n_tri;
                    }
                };
                auto settle = [&](bool any, int k0, int nsteps, bool v1) {
                    if (__any_sync(__activemask(), any)) {
                        for (int q = 0; q < nsteps; ++q) {
                            const Ev e = eval(k0 + 64 * q, v1);
                            if (e.r0) slow(k0 + 64 * q);
                            if (e.r1) slow(k0 + 64 * q + 32);
                        }
                    }
                };
                int kk = kbeg + lane;
                constexpr int G = PCF_TRIP_GROUP;
                for (; kk + 64 * (G - 1) + 32 < kend; kk += 64 * G) {
                    bool any = false;
                    #pragma unroll
                    for (int q = 0; q < G; ++q) any |= core(kk + 64 * q, true);
                    settle(any, kk, G, true);
                }
                for (; kk + 32 < kend; kk += 64) settle(core(kk, true), kk, 1, true);
                if (kk < kend) settle(core(kk, false), kk, 1, false);
            }
            };
            if (LJ == sJ) {
                if (pool) pass2(sJ, sJ + A.capJ - 1, -1);
                else pass2(sJ, MIXED ? sK : sJ, 1);
            } else {
                pass2(gJ, MIXED ? gK : gJ, 1);
            }
        } else {
        for (int rr = warp; rr < nJ; rr += kTWarps) {
            const int half = rr >> 1;
            const int jj = MIXED ? rr : ((rr & 1) ? nJ - 1 - half : half);
            const float4 ej = LJ[jj];
            const int bj = __float_as_int(ej.w) & 255;
            const int jidx = (int)((unsigned)__float_as_int(ej.w) >> 8);
            const double wij = WEIGHTED ? (double)hw * (double)WJ[jj] : 1.0;
            const int ubase = bj * bins * bins;
            const int k0 = MIXED ? 0 : jj + 1;
            for (int kk = k0 + lane; kk < nK; kk += 32) {
                const float4 ek = LK[kstepK * kk];
                const float dx = ek.x - ej.x, dy = ek.y - ej.y, dz = ek.z - ej.z;
                const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const PairRule &r3 = MIXED ? A.rXY : A.rXX;
                int bjk = fast_bin(d2, A.fc, bins);
                if (bjk == -1) {
                    ++n_rechk;
                    const int kidx = (int)((unsigned)__float_as_int(ek.w) >> 8);
                    const Cat &CK = MIXED ? A.Y : A.X;
                    bjk = exact_third(hx, hy, hz, A.X.x[jidx], A.X.y[jidx], A.X.z[jidx],
                                      CK.x[kidx], CK.y[kidx], CK.z[kidx], A.bpc, A.box, r3);
                }
                if (bjk >= 0) {
                    const int bk = __float_as_int(ek.w) & 255;
                    const int slot = ubase + bjk * bins + bk;
                    ++n_tri;
                    if (WEIGHTED) {
                        atomicAdd(A.g_wsum + slot, wij * (double)WK[kk]);
                    } else {  // (the shared histogram took the anchor above if it could)
                        atomicAdd(A.g_count + slot, 1ull);
                    }
                }
            }
        }
        }
}

template <bool MIXED, bool WEIGHTED>
__global__ void __launch_bounds__(kTThreads, 1) k_triplets(const TripArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int bins = A.rXX.bins;
    const int nb3 = bins * bins * bins;
    // histogram + 32 dummy slots (see the unit-weight pass 2)
    const size_t u_bytes = A.hist_in_smem ? (((size_t)(nb3 + 32) * 4 + 15) & ~(size_t)15) : 0;
    __shared__ int s_anchor, s_nJ, s_nK, s_unit;
    __shared__ unsigned s_stop;
    const int tid = threadIdx.x, lane = tid & 31;
    TripCta C{reinterpret_cast<unsigned *>(smem), smem + u_bytes, &s_nJ, &s_nK, &s_unit, 0u, 0ull, 0ull};
    if (A.hist_in_smem)
        for (int k = tid; k < nb3 + 32; k += kTThreads) C.U[k] = 0u;
    long long taken = 0;  // anchors this CTA took (iteration cap: nX + 1)
    __syncthreads();
    for (;;) {
        if (tid == 0) {
            s_anchor = (int)atomicAdd(A.counter, 1ull);
            s_nJ = 0;
            s_nK = 0;
            s_unit = 0;
            unsigned stop = (A.ctrl && ctrl_load(A.ctrl)) ? PCF_GAVE_UP_ABORT : 0u;
            if (++taken > (long long)A.nX + 1) stop |= PCF_GAVE_UP_CAP;
            if (stop && A.status) ctrl_store(A.status, stop);
            s_stop = stop;
        }
        __syncthreads();
        const int i = s_anchor;
        if (i >= A.nX || s_stop) break;
        tri_anchor<MIXED, WEIGHTED>(A, i, C);
        __syncthreads();
    }
    if (A.hist_in_smem) {
        for (int k = tid; k < nb3; k += kTThreads)
            if (C.U[k]) atomicAdd(A.g_count + k, (unsigned long long)C.U[k]);
    }
    unsigned long long rr = C.n_rechk, nt = C.n_tri;
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(kFull, rr, off);
        nt += __shfl_down_sync(kFull, nt, off);
    }
    if (lane == 0) {
        if (rr) atomicAdd(A.g_stats + 0, rr);
        if (nt) atomicAdd(A.g_stats + 2, nt);
    }
}

// The job table of a batched launch, passed as the kernel's parameter (so
// job arguments are read from the parameter constant bank, as a single-job
// launch reads its own; a table in global or shared memory ran the four
// histograms of the 3iso step 8% slower).
constexpr int kBatchJobs = 64;
struct TripBatch {
    TripArgs job[kBatchJobs];
    int n_jobs;
    long long n_anchors;
    unsigned long long *counter;
};

// Several isotropic triplet histograms of one kind (XXX, or XXY) in one
// persistent launch: the jobs' anchors form one queue (job after job); a CTA
// that crosses into another job flushes its shared histogram into the
// previous job's histogram.
template <bool MIXED, bool WEIGHTED>
__global__ void __launch_bounds__(kTThreads, 1) k_triplets_batch(const __grid_constant__ TripBatch B) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long s_anchor;
    __shared__ int s_nJ, s_nK, s_unit;
    __shared__ unsigned s_stop;
    const int tid = threadIdx.x, lane = tid & 31;
    const TripArgs &J0 = B.job[0];
    const int bins = J0.rXX.bins;
    const int nb3 = bins * bins * bins;
    const bool in_smem = J0.hist_in_smem != 0;
    const size_t u_bytes = in_smem ? (((size_t)(nb3 + 32) * 4 + 15) & ~(size_t)15) : 0;
    TripCta C{reinterpret_cast<unsigned *>(smem), smem + u_bytes, &s_nJ, &s_nK, &s_unit, 0u, 0ull, 0ull};
    if (in_smem)
        for (int k = tid; k < nb3 + 32; k += kTThreads) C.U[k] = 0u;
    int cur = -1;  // the CTA's current job (uniform: every thread follows s_anchor)
    long long taken = 0;
    __syncthreads();
    for (;;) {
        if (tid == 0) {
            s_anchor = (long long)atomicAdd(B.counter, 1ull);
            s_nJ = 0;
            s_nK = 0;
            s_unit = 0;
            unsigned stop = (J0.ctrl && ctrl_load(J0.ctrl)) ? PCF_GAVE_UP_ABORT : 0u;
            if (++taken > B.n_anchors + 1) stop |= PCF_GAVE_UP_CAP;
            if (stop && J0.status) ctrl_store(J0.status, stop);
            s_stop = stop;
        }
        __syncthreads();
        const long long g = s_anchor;
        if (g >= B.n_anchors || s_stop) break;
        // the job of anchor g (a CTA's anchors only move forward in the queue)
        if (cur < 0 || g >= B.job[cur].anchor_begin + B.job[cur].nX) {
            int j = cur < 0 ? 0 : cur;
            while (j + 1 < B.n_jobs && g >= B.job[j + 1].anchor_begin) ++j;
            if (cur >= 0 && in_smem && C.since) {
                flush_hist(C.U, nb3, B.job[cur].g_count);
                C.since = 0;
            }
            cur = j;
        }
        const TripArgs &A = B.job[cur];
        tri_anchor<MIXED, WEIGHTED>(A, (int)(g - A.anchor_begin), C);
        __syncthreads();
    }
    if (in_smem && cur >= 0) {
        for (int k = tid; k < nb3; k += kTThreads)
            if (C.U[k]) atomicAdd(B.job[cur].g_count + k, (unsigned long long)C.U[k]);
    }
    unsigned long long rr = C.n_rechk, nt = C.n_tri;
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(kFull, rr, off);
        nt += __shfl_down_sync(kFull, nt, off);
    }
    if (lane == 0) {
        if (rr) atomicAdd(J0.g_stats + 0, rr);
        if (nt) atomicAdd(J0.g_stats + 2, nt);
    }
}

// Anisotropic triplets (3ani_k.cuh:8,109; 3aniBPC_k.cuh:210,959): ordered
// triples anchored at point 1 = the anchor i; the lists hold every X (and
// for XXY every Y) neighbour with its exact side bin and angle bin, and all
// ordered (j, k), j != k, are counted into the bins^5 histogram
// [b(d12)][b(d31)][b(d23)][t12][t31] in global memory.
// GATES (periodic, PCF_REF_NODE_GATES): each ordered triangle counts as many
// times as the reference's node-gate blocks count it (node_gates.cuh), on the
// reference's node grid A.gate.  ISO3 (with GATES): the isotropic bins^3
// histogram [b(d12)][b(d23)][b(d31)] of the same ordered triangles
// (3isoBPC_k.cuh:191,940), from lists without angle bins.
template <bool MIXED, bool WEIGHTED, bool GATES = false, bool ISO3 = false>
__global__ void __launch_bounds__(kTThreads, 1) k_triplets_ani(const TripArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int bins = A.rXX.bins;
    float4 *sJ = reinterpret_cast<float4 *>(smem);
    float4 *sK = sJ + A.capJ;
    unsigned short *aJ = reinterpret_cast<unsigned short *>(sK + (MIXED ? A.capK : 0));
    unsigned short *aK = aJ + A.capJ;
    float *swJ = reinterpret_cast<float *>(aK + (MIXED ? A.capK : 0) + 8);
    float *swK = swJ + (WEIGHTED ? A.capJ : 0);
    // node / image words of the gated counts, 16-byte aligned past the weights
    unsigned *gJ = reinterpret_cast<unsigned *>(
        (reinterpret_cast<uintptr_t>(swK + (WEIGHTED && MIXED ? A.capK : 0)) + 15) & ~(uintptr_t)15);
    unsigned *gK = gJ + A.capJ;
    __shared__ int s_anchor, s_nJ, s_nK;
    __shared__ unsigned s_stop;
    __shared__ GateBlock s_gates[GATES ? 64 : 1];
    __shared__ signed char s_gate_by[GATES ? 64 : 1][2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (GATES) {
        for (int k = tid; k < 64; k += kTThreads) {
            s_gates[k] = kGateBlocks[k];
            s_gate_by[k][0] = kGateByImage[k][0];
            s_gate_by[k][1] = kGateByImage[k][1];
        }
    }
    unsigned n_rechk = 0;
    unsigned long long n_tri = 0;
    long long taken = 0;
    const long long B = bins, B2 = B * B, B3 = B2 * B, B4 = B3 * B;
    for (;;) {
        if (tid == 0) {
            s_anchor = (int)atomicAdd(A.counter, 1ull);
            s_nJ = 0;
            s_nK = 0;
            unsigned stop = (A.ctrl && ctrl_load(A.ctrl)) ? PCF_GAVE_UP_ABORT : 0u;
            if (++taken > (long long)A.nX + 1) stop |= PCF_GAVE_UP_CAP;
            if (stop && A.status) ctrl_store(A.status, stop);
            s_stop = stop;
        }
        __syncthreads();
        const int i = s_anchor;
        if (i >= A.nX || s_stop) break;
        const float hx = A.X.x[i], hy = A.X.y[i], hz = A.X.z[i];
        const float hw = WEIGHTED ? A.X.w[i] : 1.f;
        const int P = A.P;
        const int cix = min(max((int)__fdiv_rn(hx, A.cell), 0), P - 1);
        const int ciy = min(max((int)__fdiv_rn(hy, A.cell), 0), P - 1);
        const int ciz = min(max((int)__fdiv_rn(hz, A.cell), 0), P - 1);
        build_list<!ISO3>(A, A.X, hx, hy, hz, cix, ciy, ciz, -1, A.rXX, sJ, WEIGHTED ? swJ : nullptr,
                          A.capJ, &s_nJ, n_rechk, aJ, 1, GATES ? gJ : nullptr);
        if (MIXED)
            build_list<!ISO3>(A, A.Y, hx, hy, hz, cix, ciy, ciz, -1, A.rXY, sK,
                              WEIGHTED ? swK : nullptr, A.capK, &s_nK, n_rechk, aK, 1,
                              GATES ? gK : nullptr);
        GateNode n1{};
        if (GATES) n1 = gate_unpack(A.gate, gate_pack(A.gate, hx, hy, hz, 0u));
        __syncthreads();
        const int nJ = s_nJ, nK = MIXED ? s_nK : s_nJ;
        if (nJ > A.capJ || (MIXED && nK > A.capK)) {
            // lists beyond shared memory: flagged for the host, anchor skipped
            if (tid == 0) atomicAdd(A.g_stats + 3, 1ull);
            __syncthreads();
            continue;
        }
        const float4 *LK = MIXED ? sK : sJ;
        const unsigned short *AK = MIXED ? aK : aJ;
        const float *WK = MIXED ? swK : swJ;
        for (int jj = warp; jj < nJ; jj += kTWarps) {
            const float4 ej = sJ[jj];
            const int jidx = (int)((unsigned)__float_as_int(ej.w) >> 8);
            const unsigned short pj = ISO3 ? (unsigned short)(__float_as_int(ej.w) & 255) : aJ[jj];
            const long long base = ISO3 ? (long long)pj * B2 : (long long)(pj & 255) * B4 + (long long)(pj >> 8) * B;
            const double wij = WEIGHTED ? (double)hw * (double)swJ[jj] : 1.0;
            GateNode n2{};
            if (GATES) n2 = gate_unpack(A.gate, gJ[jj]);
            const unsigned *GK = MIXED ? gK : gJ;
            for (int kk = lane; kk < nK; kk += 32) {
                if (!MIXED && kk == jj) continue;
                const float4 ek = LK[kk];
                const float dx = ek.x - ej.x, dy = ek.y - ej.y, dz = ek.z - ej.z;
                const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                const PairRule &r3 = MIXED ? A.rXY : A.rXX;
                int c = fast_bin(d2, A.fc, bins);
                if (c == -1) {
                    ++n_rechk;
                    const int kidx = (int)((unsigned)__float_as_int(ek.w) >> 8);
                    const Cat &CK = MIXED ? A.Y : A.X;
                    c = exact_third(hx, hy, hz, A.X.x[jidx], A.X.y[jidx], A.X.z[jidx], CK.x[kidx],
                                    CK.y[kidx], CK.z[kidx], A.bpc, A.box, r3);
                }
                if (c >= 0) {
                    int mult = 1;
                    if (GATES) {
                        mult = gate_mult(A.gate, n1, n2, gate_unpack(A.gate, GK[kk]), s_gates, s_gate_by);
                        if (mult == 0) continue;
                    }
                    long long slot;
                    if (ISO3) {
                        slot = base + (long long)c * B + (__float_as_int(ek.w) & 255);
                    } else {
                        const unsigned short pk = AK[kk];
                        slot = base + (long long)(pk & 255) * B3 + (long long)c * B2 + (pk >> 8);
                    }
                    n_tri += (unsigned long long)mult;
                    if (WEIGHTED) atomicAdd(A.g_wsum + slot, wij * (double)WK[kk] * (double)mult);
                    else atomicAdd(A.g_count + slot, (unsigned long long)mult);
                }
            }
        }
        __syncthreads();
    }
    unsigned long long rr = n_rechk;
    for (int off = 16; off > 0; off >>= 1) {
        rr += __shfl_down_sync(kFull, rr, off);
        n_tri += __shfl_down_sync(kFull, n_tri, off);
    }
    if (lane == 0) {
        if (rr) atomicAdd(A.g_stats + 0, rr);
        if (n_tri) atomicAdd(A.g_stats + 2, n_tri);
    }
}

__global__ void k_to_double(const unsigned long long *__restrict__ c, const double *__restrict__ w,
                            int weighted, long long n, double *__restrict__ out) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = weighted ? w[t] : (double)c[t];
}

// Ordered-triple histogram from the oriented counts U[b_ij][b_jk][b_ki].
__global__ void k_trip_finalize(const unsigned long long *__restrict__ cnt,
                                const double *__restrict__ ws, int weighted, int mixed, int bins,
                                double *__restrict__ out) {
    const int n3 = bins * bins * bins;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const int a = t / (bins * bins), b = (t / bins) % bins, c = t % bins;
    auto U = [&](int x, int y, int z) -> double {
        const int s = (x * bins + y) * bins + z;
        return weighted ? ws[s] : (double)cnt[s];
    };
    double v;
    if (mixed) v = U(a, b, c) + U(a, c, b);
    else v = U(a, b, c) + U(b, c, a) + U(c, a, b) + U(a, c, b) + U(c, b, a) + U(b, a, c);
    out[t] = v;
}

}  // namespace

// Largest stencil population of any cell of g: bounds an anchor's lists
// (memoised per cell structure, dmax and periodicity: the rows are fixed by
// them and the structure's P).
static int64_t max_stencil_scan(const CellGrid &g, int P, const std::vector<RowDesc> &rows, bool bpc);
static int64_t max_stencil(const CellGrid &g, float dmax, const std::vector<RowDesc> &rows, bool bpc) {
    for (const auto &m : g.stencil_memo)
        if (m.first.first == dmax && m.first.second == bpc) return m.second;
    const int64_t v = max_stencil_scan(g, g.P, rows, bpc);
    g.stencil_memo.push_back({{dmax, bpc}, v});
    return v;
}
static int64_t max_stencil_scan(const CellGrid &g, int P, const std::vector<RowDesc> &rows, bool bpc) {
    const std::vector<int> &cs = g.h_start;
    int64_t best = 0;
    for (int ix = 0; ix < P; ++ix)
        for (int iy = 0; iy < P; ++iy)
            for (int iz = 0; iz < P; ++iz) {
                int64_t n = 0;
                for (const RowDesc &rw : rows) {
                    int nx = ix + rw.dx, ny = iy + rw.dy;
                    if (bpc) { nx = (nx + P) % P; ny = (ny + P) % P; }
                    else if (nx < 0 || nx >= P || ny < 0 || ny >= P) continue;
                    const int col = (nx * P + ny) * P;
                    const int zlo = iz - rw.kz, zhi = iz + rw.kz;
                    const int lo = std::max(zlo, 0), hi = std::min(zhi, P - 1);
                    if (lo <= hi) n += cs[col + hi + 1] - cs[col + lo];
                    if (bpc && zlo < 0) n += cs[col + P] - cs[col + zlo + P];
                    if (bpc && zhi >= P) n += cs[col + zhi - P + 1] - cs[col];
                }
                best = std::max(best, n);
            }
    return best;
}

// Arguments of one isotropic triplet histogram over the cell structures of
// x (and y for XXY) at P partitions: catalogs, side rules, FP32 windows and
// the shared-memory layout (smem: dynamic bytes).  The buffers (rows,
// counter, histograms, overflow lists) are the caller's.
static void trip_setup(pcf_ctx *ctx, const pcf_grid *X, const pcf_grid *Y, int P, int n_rows, int bins,
                       float dmax, uint32_t flags, bool weighted, TripArgs &A, size_t &smem) {
    const bool bpc = (flags & PCF_BPC) != 0, mixed = Y != nullptr;
    const CellGrid &gx = *X->cells;
    const CellGrid &gy = mixed ? *Y->cells : gx;
    // side rules: X-X sides need d > 0; X-Y sides only with periodic boxes
    // (3iso_k.cuh:158,160 vs 3isoBPC_k.cuh:165,170)
    PairRule rXX = make_pair_rule(bins, dmax, flags & ~PCF_DS_EXACT, false, bpc, false);
    PairRule rXY = rXX;
    rXY.flags = bpc ? PCF_RULE_EXCL : 0u;
    if (flags & PCF_RULE_CUSTOM) rXY.flags = rXX.flags;
    memset(&A, 0, sizeof(A));
    A.X = {gx.x(), gx.y(), gx.z(), gx.w(), gx.cell_start.as<int>()};
    A.Y = {gy.x(), gy.y(), gy.z(), gy.w(), gy.cell_start.as<int>()};
    A.nX = (int)X->n;
    A.n_rows = n_rows;
    A.P = P;
    A.cell = gx.cell;
    A.box = X->box;
    A.bpc = bpc ? 1 : 0;
    A.rXX = rXX;
    A.rXY = rXY;
    A.flush_budget = ctx->trip_flush_budget;
    A.ctrl = ctx->d_abort;
    A.status = ctx->d_status;
    A.mixed = mixed ? 1 : 0;
    {
        // windows: the FP32 side |v_k - v_j| carries up to three roundings of
        // coordinate differences (plus the image shift of the anchor when
        // periodic); the bounds below keep a >= 8x margin
        const double dd = rXX.dd;
        const double rmax = (double)dmax * rXX.ds + 1.0;
        const double Lx = bpc ? (double)X->box : (double)dmax;
        const double e_d2 = dd * std::ldexp(1.0, -17) + (double)dmax * Lx * std::ldexp(1.0, -18);
        const double wr = rmax * std::ldexp(1.0, -17) + rXX.ds * Lx * std::ldexp(1.0, -18);
        A.fc.dsf = (float)rXX.ds;
        A.fc.ds2 = A.fc.dsf * A.fc.dsf;
        A.fc.lo = (float)(dd - e_d2);
        A.fc.hi = (float)(dd + e_d2);
        A.fc.w = std::min(8000u, (unsigned)std::ceil((wr + std::ldexp(1.0, -16)) * 32768.0) + 1u);
    }
    const int n3 = bins * bins * bins;
    // histogram + 32 dummy slots (the adds of 0 of lanes without a triangle)
    const size_t u_bytes = ((size_t)(n3 + 32) * 4 + 15) & ~(size_t)15;
    const size_t smem_max = 227 * 1024 - 64;
    A.hist_in_smem = (!weighted && u_bytes <= 150 * 1024) ? 1 : 0;
    const size_t hist_b = A.hist_in_smem ? u_bytes : 0;
    const size_t ent = 16 + (weighted ? 4 : 0);
    const size_t room = smem_max - hist_b;
    if (mixed && !(A.hist_in_smem && !weighted)) {
        A.capJ = (int)(room / ent / 3);
        A.capK = (int)(room / ent) - A.capJ;
    } else {  // XXX, or XXY with one pooled buffer (J up, K down; see tri_anchor)
        A.capJ = (int)(room / ent);
        A.capK = 0;
    }
    smem = hist_b + (size_t)(A.capJ + A.capK) * ent;
}

// Per-CTA overflow lists for lists of up to gcap entries (J, K and weights).
static pcf_status trip_overflow(pcf_ctx *ctx, int64_t gmax, bool mixed, bool weighted, int grid,
                                TripArgs &A) {
    A.gcap = (int)std::min<int64_t>(gmax, 1 << 24);
    PCF_CU(ctx, ctx->scratch_c.ensure(sizeof(float4) * (size_t)A.gcap * grid * (mixed ? 2 : 1) +
                                      (weighted ? sizeof(float) * (size_t)A.gcap * grid * 2 : 0) + 256));
    char *sc = ctx->scratch_c.as<char>();
    A.gJ = reinterpret_cast<float4 *>(sc);
    A.gK = mixed ? A.gJ + (size_t)A.gcap * grid : nullptr;
    float *wbase = reinterpret_cast<float *>(sc + sizeof(float4) * (size_t)A.gcap * grid * (mixed ? 2 : 1));
    A.gwJ = weighted ? wbase : nullptr;
    A.gwK = weighted && mixed ? wbase + (size_t)A.gcap * grid : nullptr;
    return PCF_OK;
}

static pcf_status count_triplets_ordered(pcf_ctx *ctx, const pcf_grid *x_, const pcf_grid *y_, int bins,
                                         float dmax, uint32_t flags, double *hist, pcf_stats *stats,
                                         bool iso3);

extern "C" pcf_status pcf_count_triplets(pcf_ctx *ctx, int kind, const pcf_grid *x_,
                                         const pcf_grid *y_, int bins, float dmax, uint32_t flags,
                                         double *hist, pcf_stats *stats) {
    if (!ctx || !x_ || !hist || bins < 1 || !(dmax > 0.f)) return PCF_ERR_INVALID_ARG;
    if (kind == PCF_ANI) return pcf_count_triplets_ani(ctx, x_, y_, bins, dmax, flags, hist, stats);
    if (kind != PCF_ISO) return PCF_ERR_INVALID_ARG;
    if (flags & PCF_REF_NODE_GATES)
        return count_triplets_ordered(ctx, x_, y_, bins, dmax, flags, hist, stats, true);
    if (bins > 255 || (int64_t)bins * bins * bins > (1 << 26)) return PCF_ERR_UNSUPPORTED;
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, x_);
        if (s0 == PCF_OK && y_) s0 = grid_finish(ctx, y_);
        if (s0 != PCF_OK) return s0;
    }
    pcf_grid *X = const_cast<pcf_grid *>(x_);
    pcf_grid *Y = const_cast<pcf_grid *>(y_);
    const bool bpc = (flags & PCF_BPC) != 0, mixed = Y != nullptr;
    if (X->n >= (1 << 24) || (Y && Y->n >= (1 << 24))) return PCF_ERR_UNSUPPORTED;
    if (ctx_abort_requested(ctx) != PCF_OK) return PCF_ERR_TIMEOUT;
    int P = 0;
    pcf_status s = prepare_grids(ctx, X, Y, dmax, PCF_ISO, bpc, &P);
    if (s != PCF_OK) return s;
    const CellGrid &gx = *X->cells;
    const CellGrid &gy = mixed ? *Y->cells : gx;
    PairPlan plan;
    plan_pairs(gx, X->box, dmax, false, false, plan, ctx->sm_count * 24);
    const bool weighted = !(X->unit_weights && (!mixed || Y->unit_weights));
    TripArgs A;
    size_t smem = 0;
    trip_setup(ctx, X, Y, P, (int)plan.rows.size(), bins, dmax, flags, weighted, A, smem);
    const int n3 = bins * bins * bins;
    // overflow lists: bounded by the largest stencil population of any cell
    const int64_t gmax = std::max<int64_t>(max_stencil(gx, dmax, plan.rows, bpc),
                                           mixed ? max_stencil(gy, dmax, plan.rows, bpc) : 0) + 32;
    const int grid = ctx->sm_count;
    s = trip_overflow(ctx, gmax, mixed, weighted, grid, A);
    if (s != PCF_OK) return s;
    // rows + counter through the plan slot
    PlanSlot *sl = nullptr;
    s = stage_plan(ctx, plan, &sl);
    if (s != PCF_OK) return s;
    A.rows = sl->d_rows.as<RowDesc>();
    A.counter = sl->d_counter.as<unsigned long long>();
    // histogram scratch: [u64 n3][f64 n3][stats 8][f64 out n3]
    PCF_CU(ctx, ctx->d_hist.ensure((size_t)n3 * 24 + 64));
    char *hp = ctx->d_hist.as<char>();
    A.g_count = reinterpret_cast<unsigned long long *>(hp);
    A.g_wsum = reinterpret_cast<double *>(hp + (size_t)n3 * 8);
    A.g_stats = reinterpret_cast<unsigned long long *>(hp + (size_t)n3 * 16);
    double *d_out = reinterpret_cast<double *>(hp + (size_t)n3 * 16 + 64);
    PCF_CU(ctx, cudaMemsetAsync(hp, 0, (size_t)n3 * 16 + 64, ctx->stream));

    auto kfn = mixed ? (weighted ? k_triplets<true, true> : k_triplets<true, false>)
                     : (weighted ? k_triplets<false, true> : k_triplets<false, false>);
    PCF_CU(ctx, ensure_smem_limit(reinterpret_cast<const void *>(kfn), ctx->device, smem));
    cudaEvent_t pe0 = nullptr, pe1 = nullptr;
    if (ctx->profile) {
        s = profile_events(ctx, &pe0, &pe1);
        if (s != PCF_OK) return s;
        PCF_CU(ctx, cudaEventRecord(pe0, ctx->stream));
    }
    PCF_CU(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    kfn<<<grid, kTThreads, smem, ctx->stream>>>(A);
    PCF_CU(ctx, cudaGetLastError());
    PCF_CU(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if (pe1) PCF_CU(ctx, cudaEventRecord(pe1, ctx->stream));
    PCF_CU(ctx, cudaEventRecord(sl->done, ctx->stream));
    ++ctx->launches;
    const bool dev_out = (flags & PCF_DEVICE_OUT) != 0;
    k_trip_finalize<<<(n3 + 255) / 256, 256, 0, ctx->stream>>>(A.g_count, A.g_wsum, weighted ? 1 : 0,
                                                                mixed ? 1 : 0, bins,
                                                                dev_out ? hist : d_out);
    PCF_CU(ctx, cudaGetLastError());
    ++ctx->launches;
    if (stats || !dev_out) {  // through the context's page-locked buffer (see count_pairs_impl)
        const size_t hb = dev_out ? 0 : sizeof(double) * n3;
        s = pcf_ensure_pinned(ctx, hb + 64);
        if (s != PCF_OK) return s;
        char *hp = static_cast<char *>(ctx->h_pinned);
        if (hb) PCF_CU(ctx, cudaMemcpyAsync(hp, d_out, hb, cudaMemcpyDeviceToHost, ctx->stream));
        PCF_CU(ctx, cudaMemcpyAsync(hp + hb, A.g_stats, 32, cudaMemcpyDeviceToHost, ctx->stream));
        PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
        s = ctx_queue_status(ctx);
        if (s != PCF_OK) return s;
        if (hb) memcpy(hist, hp, hb);
        unsigned long long hs[4];
        memcpy(hs, hp + hb, sizeof(hs));
        if (stats) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            stats->pairs = (double)hs[2];  // unordered triangles (XXY: per unordered XX pair)
            stats->candidates = 0;
            stats->rechecks = (double)hs[0];
            stats->kernel_ms = ms;
            stats->partitions = P;
            stats->work_items = (int)X->n;
        }
    }
    return PCF_OK;
}

// One data catalog against n_rand random catalogs: DDD once, RRR_i, DDR_i
// and DRR_i per random catalog, as the jobs of two persistent launches
// (k_triplets_batch: the XXX jobs, then the XXY jobs).  All grids take one partition count (the one a call
// on the largest catalog would use; results do not depend on it).
extern "C" pcf_status pcf_batch_triplets(pcf_ctx *ctx, const pcf_grid *d_, const pcf_grid *const *r_,
                                         int n_rand, int bins, float dmax, uint32_t flags, double *ddd,
                                         double *rrr, double *ddr, double *drr, pcf_stats *stats) {
    if (!ctx || !d_ || bins < 1 || !(dmax > 0.f) || n_rand < 0 || (n_rand > 0 && !r_) ||
        (!ddd && !rrr && !ddr && !drr))
        return PCF_ERR_INVALID_ARG;
    if (bins > 255 || (int64_t)bins * bins * bins > (1 << 26)) return PCF_ERR_UNSUPPORTED;
    if (flags & PCF_REF_NODE_GATES) {
        ctx->last_error = "PCF_REF_NODE_GATES counts run per call (pcf_count_triplets)";
        return PCF_ERR_UNSUPPORTED;
    }
    if (ctx_abort_requested(ctx) != PCF_OK) return PCF_ERR_TIMEOUT;
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, d_);
        for (int i = 0; s0 == PCF_OK && i < n_rand; ++i)
            if (r_[i]) s0 = grid_finish(ctx, r_[i]);
        if (s0 != PCF_OK) return s0;
    }
    const bool bpc = (flags & PCF_BPC) != 0;
    pcf_grid *D = const_cast<pcf_grid *>(d_);
    std::vector<pcf_grid *> R((size_t)n_rand);
    pcf_grid *big = D;
    bool weighted = !D->unit_weights;
    for (int i = 0; i < n_rand; ++i) {
        R[i] = const_cast<pcf_grid *>(r_[i]);
        if (!R[i]) return PCF_ERR_INVALID_ARG;
        if (R[i]->box != D->box) return PCF_ERR_MISMATCH;
        if (R[i]->n >= (1 << 24)) return PCF_ERR_UNSUPPORTED;
        if (R[i]->n > big->n) big = R[i];
        weighted = weighted || !R[i]->unit_weights;
    }
    if (D->n >= (1 << 24)) return PCF_ERR_UNSUPPORTED;
    int P = 0;
    pcf_status s = prepare_grids(ctx, big, nullptr, dmax, PCF_ISO, bpc, &P);
    if (s != PCF_OK) return s;
    // every structure queued before the first is completed
    if ((s = grid_ensure_cells(ctx, D, P, true)) != PCF_OK) return s;
    for (pcf_grid *g : R)
        if ((s = grid_ensure_cells(ctx, g, P, true)) != PCF_OK) return s;
    if ((s = grid_finish(ctx, D)) != PCF_OK) return s;
    for (pcf_grid *g : R)
        if ((s = grid_finish(ctx, g)) != PCF_OK) return s;
    PairPlan plan;
    plan_pairs(*D->cells, D->box, dmax, false, false, plan, ctx->sm_count * 24);
    const int n3 = bins * bins * bins;

    // jobs: (X, Y) in output order
    struct Job { pcf_grid *x, *y; double *out; };
    std::vector<Job> jobs;
    if (ddd) jobs.push_back({D, nullptr, ddd});
    for (int i = 0; i < n_rand; ++i) {
        if (rrr) jobs.push_back({R[i], nullptr, rrr + (size_t)i * n3});
        if (ddr) jobs.push_back({D, R[i], ddr + (size_t)i * n3});
        if (drr) jobs.push_back({R[i], D, drr + (size_t)i * n3});
    }
    const int nj = (int)jobs.size();
    std::vector<TripArgs> args((size_t)nj);
    size_t smem = 0;
    long long anchors = 0;
    bool any_mixed = false;
    int64_t gmax = 0;
    std::map<const pcf_grid *, int64_t> stencil;  // per grid
    auto stencil_of = [&](const pcf_grid *g) {
        auto it = stencil.find(g);
        if (it != stencil.end()) return it->second;
        return stencil[g] = max_stencil(*g->cells, dmax, plan.rows, bpc);
    };
    for (int k = 0; k < nj; ++k) {
        size_t sm = 0;
        trip_setup(ctx, jobs[k].x, jobs[k].y, P, (int)plan.rows.size(), bins, dmax, flags, weighted,
                   args[k], sm);
        smem = std::max(smem, sm);
        args[k].anchor_begin = anchors;
        anchors += jobs[k].x->n;
        any_mixed = any_mixed || jobs[k].y;
        gmax = std::max<int64_t>(gmax, stencil_of(jobs[k].x));
        if (jobs[k].y) gmax = std::max<int64_t>(gmax, stencil_of(jobs[k].y));
    }
    const int grid = ctx->sm_count;
    TripArgs ov;
    s = trip_overflow(ctx, gmax + 32, any_mixed, weighted, grid, ov);
    if (s != PCF_OK) return s;

    // rows + counter through the plan slot; histograms per job
    PlanSlot *sl = nullptr;
    s = stage_plan(ctx, plan, &sl);
    if (s != PCF_OK) return s;
    const size_t nh = (size_t)nj * n3;
    PCF_CU(ctx, ctx->d_hist.ensure(nh * 24 + 64));
    char *hp = ctx->d_hist.as<char>();
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(hp);
    double *wsum = reinterpret_cast<double *>(hp + nh * 8);
    unsigned long long *gstats = reinterpret_cast<unsigned long long *>(hp + nh * 16);
    double *d_out = reinterpret_cast<double *>(hp + nh * 16 + 64);
    PCF_CU(ctx, cudaMemsetAsync(hp, 0, nh * 16 + 64, ctx->stream));
    for (int k = 0; k < nj; ++k) {
        TripArgs &A = args[k];
        A.gcap = ov.gcap;
        A.gJ = ov.gJ;
        A.gK = ov.gK;
        A.gwJ = ov.gwJ;
        A.gwK = ov.gwK;
        A.rows = sl->d_rows.as<RowDesc>();
        A.counter = sl->d_counter.as<unsigned long long>();
        A.g_count = cnt + (size_t)k * n3;
        A.g_wsum = wsum + (size_t)k * n3;
        A.g_stats = gstats;
    }
    // launches per kind (the XXX jobs, then the XXY jobs), each over one
    // anchor queue of up to kBatchJobs jobs with its own counter
    std::vector<std::vector<TripArgs>> groups;
    for (int m = 0; m < 2; ++m) {
        std::vector<TripArgs> cur;
        for (int k = 0; k < nj; ++k) {
            if ((jobs[k].y ? 1 : 0) != m) continue;
            cur.push_back(args[k]);
            if ((int)cur.size() == kBatchJobs) {
                groups.push_back(cur);
                cur.clear();
            }
        }
        if (!cur.empty()) groups.push_back(cur);
    }
    if (groups.size() > 8) return PCF_ERR_UNSUPPORTED;  // counters of the plan slot
    cudaEvent_t pe0 = nullptr, pe1 = nullptr;
    if (ctx->profile) {
        s = profile_events(ctx, &pe0, &pe1);
        if (s != PCF_OK) return s;
        PCF_CU(ctx, cudaEventRecord(pe0, ctx->stream));
    }
    PCF_CU(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    unsigned long long *ctr = sl->d_counter.as<unsigned long long>();
    std::unique_ptr<TripBatch> tb(new TripBatch);
    for (size_t q = 0; q < groups.size(); ++q) {
        memset(tb.get(), 0, sizeof(TripBatch));
        long long a0 = 0;
        for (size_t k = 0; k < groups[q].size(); ++k) {
            tb->job[k] = groups[q][k];
            tb->job[k].anchor_begin = a0;
            a0 += tb->job[k].nX;
        }
        tb->n_jobs = (int)groups[q].size();
        tb->n_anchors = a0;
        tb->counter = ctr + q;
        const bool m = groups[q][0].mixed != 0;
        auto kfn = m ? (weighted ? k_triplets_batch<true, true> : k_triplets_batch<true, false>)
                     : (weighted ? k_triplets_batch<false, true> : k_triplets_batch<false, false>);
        PCF_CU(ctx, ensure_smem_limit(reinterpret_cast<const void *>(kfn), ctx->device, smem));
        kfn<<<grid, kTThreads, smem, ctx->stream>>>(*tb);
        PCF_CU(ctx, cudaGetLastError());
        ++ctx->launches;
    }
    PCF_CU(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    if (pe1) PCF_CU(ctx, cudaEventRecord(pe1, ctx->stream));
    PCF_CU(ctx, cudaEventRecord(sl->done, ctx->stream));
    for (int k = 0; k < nj; ++k) {
        k_trip_finalize<<<(n3 + 255) / 256, 256, 0, ctx->stream>>>(
            cnt + (size_t)k * n3, wsum + (size_t)k * n3, weighted ? 1 : 0, jobs[k].y ? 1 : 0, bins,
            d_out + (size_t)k * n3);
        PCF_CU(ctx, cudaGetLastError());
        ++ctx->launches;
    }
    std::vector<double> host(nh);
    unsigned long long hs[4] = {0, 0, 0, 0};
    PCF_CU(ctx, cudaMemcpyAsync(host.data(), d_out, sizeof(double) * nh, cudaMemcpyDeviceToHost,
                                ctx->stream));
    PCF_CU(ctx, cudaMemcpyAsync(hs, gstats, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    s = ctx_queue_status(ctx);
    if (s != PCF_OK) return s;
    for (int k = 0; k < nj; ++k) memcpy(jobs[k].out, host.data() + (size_t)k * n3, sizeof(double) * n3);
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->pairs = (double)hs[2];
        stats->candidates = 0;
        stats->rechecks = (double)hs[0];
        stats->kernel_ms = ms;
        stats->partitions = P;
        stats->work_items = (int)std::min<long long>(anchors, INT32_MAX);
    }
    return PCF_OK;
}

// Anisotropic triplets (bins^5).  The histogram lives in global memory (u64
// counts or FP64 sums); lists stay in shared memory (an anchor whose lists
// do not fit makes the call fail with PCF_ERR_UNSUPPORTED).
// Ordered-triangle counts through k_triplets_ani: the bins^5 anisotropic
// histogram, or (iso3, with PCF_REF_NODE_GATES) the bins^3 isotropic one.
static pcf_status count_triplets_ordered(pcf_ctx *ctx, const pcf_grid *x_, const pcf_grid *y_, int bins,
                                         float dmax, uint32_t flags, double *hist, pcf_stats *stats,
                                         bool iso3) {
    const int64_t nh = iso3 ? (int64_t)bins * bins * bins : (int64_t)bins * bins * bins * bins * bins;
    if (bins > 255 || nh > ((int64_t)1 << 31)) return PCF_ERR_UNSUPPORTED;
    const bool gates = (flags & PCF_REF_NODE_GATES) != 0;
    if (gates) {
        if (!(flags & PCF_BPC)) {
            ctx->last_error = "PCF_REF_NODE_GATES applies to periodic counts (PCF_BPC)";
            return PCF_ERR_INVALID_ARG;
        }
        if (x_->user_P < 1 || x_->user_P > 512 ||
            (y_ && (y_->user_P != x_->user_P || y_->box != x_->box))) {
            ctx->last_error = "PCF_REF_NODE_GATES: the reference's node grid is the partitions given to "
                              "pcf_grid_build (1 to 512), the same for both grids";
            return PCF_ERR_INVALID_ARG;
        }
    }
    cudaSetDevice(ctx->device);
    {
        pcf_status s0 = grid_finish(ctx, x_);
        if (s0 == PCF_OK && y_) s0 = grid_finish(ctx, y_);
        if (s0 != PCF_OK) return s0;
    }
    pcf_grid *X = const_cast<pcf_grid *>(x_);
    pcf_grid *Y = const_cast<pcf_grid *>(y_);
    const bool bpc = (flags & PCF_BPC) != 0, mixed = Y != nullptr;
    if (X->n >= (1 << 24) || (Y && Y->n >= (1 << 24))) return PCF_ERR_UNSUPPORTED;
    if (ctx_abort_requested(ctx) != PCF_OK) return PCF_ERR_TIMEOUT;
    int P = 0;
    pcf_status s = prepare_grids(ctx, X, Y, dmax, PCF_ISO, bpc, &P);
    if (s != PCF_OK) return s;
    const CellGrid &gx = *X->cells;
    const CellGrid &gy = mixed ? *Y->cells : gx;
    PairPlan plan;
    plan_pairs(gx, X->box, dmax, false, false, plan, ctx->sm_count * 24);
    PairRule rXX = make_pair_rule(bins, dmax, flags & ~PCF_DS_EXACT, false, bpc, false);
    PairRule rXY = rXX;
    rXY.flags = bpc ? PCF_RULE_EXCL : 0u;
    if (flags & PCF_RULE_CUSTOM) rXY.flags = rXX.flags;
    TripArgs A;
    memset(&A, 0, sizeof(A));
    A.X = {gx.x(), gx.y(), gx.z(), gx.w(), gx.cell_start.as<int>()};
    A.Y = {gy.x(), gy.y(), gy.z(), gy.w(), gy.cell_start.as<int>()};
    A.nX = (int)X->n;
    A.n_rows = (int)plan.rows.size();
    A.P = P;
    A.cell = gx.cell;
    A.box = X->box;
    A.bpc = bpc ? 1 : 0;
    A.rXX = rXX;
    A.rXY = rXY;
    A.ctrl = ctx->d_abort;
    A.status = ctx->d_status;
    if (gates) A.gate = gate_geometry(X->box, dmax, X->user_P);
    {
        const double dd = rXX.dd;
        const double rmax = (double)dmax * rXX.ds + 1.0;
        const double Lx = bpc ? (double)X->box : (double)dmax;
        const double e_d2 = dd * std::ldexp(1.0, -17) + (double)dmax * Lx * std::ldexp(1.0, -18);
        const double wr = rmax * std::ldexp(1.0, -17) + rXX.ds * Lx * std::ldexp(1.0, -18);
        A.fc.dsf = (float)rXX.ds;
        A.fc.ds2 = A.fc.dsf * A.fc.dsf;
        A.fc.lo = (float)(dd - e_d2);
        A.fc.hi = (float)(dd + e_d2);
        A.fc.w = std::min(8000u, (unsigned)std::ceil((wr + std::ldexp(1.0, -16)) * 32768.0) + 1u);
    }
    const bool weighted = !(X->unit_weights && (!mixed || Y->unit_weights));
    const size_t ent = 16 + 2 + (weighted ? 4 : 0) + (gates ? 4 : 0);
    const size_t room = 227 * 1024 - 256 - (gates ? 64 * sizeof(GateBlock) + 128 + 64 : 0);
    if (mixed) {
        A.capJ = (int)(room / ent / 3);
        A.capK = (int)(room / ent) - A.capJ - 8;
    } else {
        A.capJ = (int)(room / ent) - 8;
        A.capK = 0;
    }
    const size_t smem = (size_t)(A.capJ + A.capK) * ent + 64;
    const int64_t n5 = nh;
    PlanSlot *sl = nullptr;
    s = stage_plan(ctx, plan, &sl);
    if (s != PCF_OK) return s;
    A.rows = sl->d_rows.as<RowDesc>();
    A.counter = sl->d_counter.as<unsigned long long>();
    PCF_CU(ctx, ctx->d_hist.ensure((size_t)n5 * 16 + 128));
    char *hp = ctx->d_hist.as<char>();
    A.g_count = reinterpret_cast<unsigned long long *>(hp);
    A.g_wsum = reinterpret_cast<double *>(hp);  // one of the two is used
    A.g_stats = reinterpret_cast<unsigned long long *>(hp + (size_t)n5 * 8);
    double *d_out = reinterpret_cast<double *>(hp + (size_t)n5 * 8 + 128);
    PCF_CU(ctx, cudaMemsetAsync(hp, 0, (size_t)n5 * 8 + 128, ctx->stream));
    void (*kfn)(const TripArgs);
    if (iso3)
        kfn = mixed ? (weighted ? k_triplets_ani<true, true, true, true> : k_triplets_ani<true, false, true, true>)
                    : (weighted ? k_triplets_ani<false, true, true, true> : k_triplets_ani<false, false, true, true>);
    else if (gates)
        kfn = mixed ? (weighted ? k_triplets_ani<true, true, true> : k_triplets_ani<true, false, true>)
                    : (weighted ? k_triplets_ani<false, true, true> : k_triplets_ani<false, false, true>);
    else
        kfn = mixed ? (weighted ? k_triplets_ani<true, true> : k_triplets_ani<true, false>)
                    : (weighted ? k_triplets_ani<false, true> : k_triplets_ani<false, false>);
    PCF_CU(ctx, ensure_smem_limit(reinterpret_cast<const void *>(kfn), ctx->device, smem));
    PCF_CU(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    kfn<<<ctx->sm_count, kTThreads, smem, ctx->stream>>>(A);
    PCF_CU(ctx, cudaGetLastError());
    PCF_CU(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    PCF_CU(ctx, cudaEventRecord(sl->done, ctx->stream));
    k_to_double<<<(unsigned)((n5 + 255) / 256), 256, 0, ctx->stream>>>(A.g_count, A.g_wsum,
                                                                       weighted ? 1 : 0, n5, d_out);
    PCF_CU(ctx, cudaGetLastError());
    ctx->launches += 2;
    const bool dev_out = (flags & PCF_DEVICE_OUT) != 0;
    unsigned long long hs[4] = {0, 0, 0, 0};
    PCF_CU(ctx, cudaMemcpyAsync(hs, A.g_stats, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
    PCF_CU(ctx, cudaMemcpyAsync(hist, d_out, sizeof(double) * n5,
                                dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
    PCF_CU(ctx, cudaStreamSynchronize(ctx->stream));
    s = ctx_queue_status(ctx);
    if (s != PCF_OK) return s;
    if (hs[3]) {
        ctx->last_error = "neighbour lists of the anisotropic triplet kernel exceed shared memory";
        return PCF_ERR_UNSUPPORTED;
    }
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        stats->pairs = (double)hs[2];
        stats->rechecks = (double)hs[0];
        stats->candidates = 0;
        stats->kernel_ms = ms;
        stats->partitions = P;
        stats->work_items = (int)X->n;
    }
    return PCF_OK;
}

pcf_status pcf_count_triplets_ani(pcf_ctx *ctx, const pcf_grid *x_, const pcf_grid *y_, int bins,
                                  float dmax, uint32_t flags, double *hist, pcf_stats *stats) {
    return count_triplets_ordered(ctx, x_, y_, bins, dmax, flags, hist, stats, false);
}

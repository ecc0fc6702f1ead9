/*
 * pcf_oracle.c -- CPU FP64 oracle for grid-node pair / triplet counting.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and only as the checker.
 *
 * It restates, with brute-force loops, the histogram rules of the reference
 * CUDA kernels (3PCFGPU, paths relative to the reference root):
 *   cuda/kernels/2iso_k.cuh:8-120        XX2iso / XY2iso
 *   cuda/kernels/2isoBPC_k.cuh:8-565     XX2iso_BPC / XY2iso_BPC / RR analytic
 *   cuda/kernels/2ani_k.cuh:7-135        XX2ani / XY2ani
 *   cuda/kernels/2aniBPC_k.cuh:8-682     XX2ani_BPC / XY2ani_BPC
 *   cuda/kernels/3iso_k.cuh:8-179        XXX3iso / XXY3iso
 *   cuda/kernels/3isoBPC_k.cuh:8-188     count123 / count123_mixed (image rule)
 *   cuda/kernels/3isoBPC_k.cuh:1694-2119 DD2iso_forBPC, make_ff_av(_ref),
 *                                        make_histo_analitic
 *   cuda/kernels/3ani_k.cuh:8-209        XXX3ani / XXY3ani
 *   cuda/kernels/3aniBPC_k.cuh:8-207     count123_ani / count123_animixed
 *                                        (XXX3ani_BPC / XXY3ani_BPC)
 *   cuda/pcf2isoBPC.cuh:199-202, cuda/pcf3isoBPC.cuh:233-247 (constants)
 *
 * Canonical (FP64) rule, shared with the CUDA library:
 *   separation  dx = (double)x2 - (double)x1   (exact); with periodic
 *               boundaries the minimum image (|dx| > L/2 -> dx -+ L, exact).
 *   d2          = (dx*dx + dy*dy) + dz*dz, each op rounded, no FMA.
 *   in range    d2 < (double)(float)(dmax*dmax)   [or <= for 2ani BPC],
 *               and d2 > 0 where the reference tests d > 0.
 *   bin         = (int)(sqrt(d2) * ds), dropped when >= bins,
 *               ds = floor(bins/dmax * 1e6)/1e6 (or bins/dmax, 2iso BPC).
 * The reference computes d2 in FP32; ORC_REF32_* precisions reproduce that
 * (with the FMA contraction pattern named) so that the reference's own
 * outputs can be matched bit for bit, which is how this oracle is pinned.
 *
 * Built with -ffp-contract=off (see Makefile) so no FMA is formed silently.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef struct { float x, y, z, w; } opt;

enum {
    ORC_FP64 = 0,          /* canonical FP64 rule                                */
    ORC_REF32_NOFMA = 1,   /* FP32 d2, ((dx*dx + dy*dy) + dz*dz), no contraction */
    ORC_REF32_FMA_A = 2,   /* FP32 d2 = fma(dz,dz, fma(dy,dy, dx*dx))            */
    ORC_REF32_FMA_B = 3,   /* FP32 d2 = fma(dz,dz, fma(dx,dx, dy*dy))            */
    ORC_REF32_FMA_C = 4,   /* FP32 d2 = fma(dx,dx, fma(dy,dy, dz*dz))            */
    ORC_REF32_CPU_BPC = 5  /* the reference's CPU periodic engines, see cpu_bpc_slot */
};
#define RULE_EXCL_ZERO 1u  /* require d2 > 0 (every component for 2ani)          */
#define RULE_INCLUSIVE 2u  /* d2 <= dd_max instead of d2 < dd_max                */

double orc_ds(int bins, float dmax, int exact)
{
    /* 2iso_k.cuh:37 (floored to 1e-6) and 2isoBPC_k.cuh:36 (exact). */
    double q = (double)bins / (double)dmax;
    return exact ? q : floor(q * 1000000.0) / 1000000.0;
}

static inline double sep64(float a, float b, int bpc, double L)
{
    double d = (double)b - (double)a;
    if (bpc) {
        if (d > 0.5 * L) d -= L;
        else if (d < -0.5 * L) d += L;
    }
    return d;
}

static inline float d2_ref32(float fx, float fy, float fz, int prec)
{
    switch (prec) {
    case ORC_REF32_FMA_A: return fmaf(fz, fz, fmaf(fy, fy, fx * fx));
    case ORC_REF32_FMA_B: return fmaf(fz, fz, fmaf(fx, fx, fy * fy));
    case ORC_REF32_FMA_C: return fmaf(fx, fx, fmaf(fy, fy, fz * fz));
    default: {
        float a = fx * fx;
        float b = fy * fy;
        float c = fz * fz;
        float s = a + b;
        return s + c;
    }
    }
}

/* Squared separation components of a pair: returns the three per-axis
 * squares folded the way the rule needs (iso: total; ani: z and perp). */
static inline void pair_d2(const opt *p, const opt *q, int bpc, double L, int prec,
                           double *d2_iso, double *d2_z, double *d2_perp)
{
    if (prec == ORC_FP64 || bpc) {
        double dx = sep64(p->x, q->x, bpc, L);
        double dy = sep64(p->y, q->y, bpc, L);
        double dz = sep64(p->z, q->z, bpc, L);
        double xx = dx * dx, yy = dy * dy, zz = dz * dz;
        double s = xx + yy;
        *d2_iso = s + zz;
        *d2_z = zz;
        *d2_perp = s;
    } else {
        float fx = q->x - p->x, fy = q->y - p->y, fz = q->z - p->z;
        *d2_iso = (double)d2_ref32(fx, fy, fz, prec);
        *d2_z = (double)(fz * fz);
        float a = fx * fx, b = fy * fy;
        *d2_perp = (double)(a + b);
    }
}

static inline int in_range(double d2, double ddmax, unsigned rule)
{
    if (rule & RULE_EXCL_ZERO) { if (!(d2 > 0.0)) return 0; }
    if (rule & RULE_INCLUSIVE) return d2 <= ddmax;
    return d2 < ddmax;
}

static inline int bin_of(double d2, double ds, int bins)
{
    int b = (int)(sqrt(d2) * ds);
    return (b >= 0 && b < bins) ? b : -1;
}

/* Histogram slot of one pair under the rule, or -1. */
static inline int pair_slot(const opt *p, const opt *q, int ani, int bpc, double L, int prec,
                            unsigned rule, double ddmax, double ds, int bins)
{
    double d2, dz2, dp2;
    pair_d2(p, q, bpc, L, prec, &d2, &dz2, &dp2);
    if (!ani) {
        if (!in_range(d2, ddmax, rule)) return -1;
        return bin_of(d2, ds, bins);
    }
    if (!in_range(dz2, ddmax, rule) || !in_range(dp2, ddmax, rule)) return -1;
    int bz = bin_of(dz2, ds, bins), bp = bin_of(dp2, ds, bins);
    if (bz < 0 || bp < 0) return -1;
    return bz * bins + bp;
}

/*
 * The reference's CPU periodic engines, restated for pinning
 * (cpp/2PCFisotropic/BPC/2PCF.h:151-335, :338-495, :498-700 and
 * cpp/2PCFanisotropic/BPC/2PCFani.h:152-700).  p is the point the engine's
 * outer loop holds (x = elements[i].x), q the inner one.  All in FP32:
 *   direct pass   d = p - q per axis; iso: dis = (dx*dx + dy*dy) + dz*dz,
 *                 counted when dis <= dd_max (2PCF.h:199,232,274,316) under
 *                 RULE_INCLUSIVE, else dis < dd_max (the fine DD of the
 *                 3-point engine, 3PCFiso.h:1760);
 *   image pass    a wrapped axis uses fabs(d) - L (2PCF.h:358), counted when
 *                 dis < dd_max (2PCF.h:362).  With dmax < L/2 a pair lands in
 *                 the pass that wraps exactly the axes with |d| > L/2.
 *   ani           dz2 = dz*dz, r2 = dx*dx + dy*dy, both < dd_max in every
 *                 pass (2PCFani.h:207,238,492);
 *   bin           (int)(sqrt((double)dis) * ds), ds floored to 1e-6 in both
 *                 engines (2PCF.h:74, 2PCFani.h:72); no d > 0 test and no
 *                 bin cap (a bin >= bins is dropped here; the engine would
 *                 write past its histogram);
 *   weight        the product is formed in FP32 before the FP64 sum:
 *                 2*w1*w2 for XX (2PCF.h:200), w1*w2 for XY.
 * Returns the slot or -1; *wprod receives the FP32 weight product.
 */
static inline int cpu_bpc_slot(const opt *p, const opt *q, int ani, int self, float L,
                               float ddf, double ds, int bins, unsigned rule, double *wprod)
{
    float d[3] = {p->x - q->x, p->y - q->y, p->z - q->z};
    int wrapped = 0;
    for (int k = 0; k < 3; ++k) {
        if (fabsf(d[k]) > 0.5f * L) { d[k] = fabsf(d[k]) - L; wrapped = 1; }
    }
    int slot;
    if (!ani) {
        float a = d[0] * d[0], b = d[1] * d[1], c = d[2] * d[2];
        float s = a + b;
        double dis = (double)(s + c);
        const int incl = !wrapped && (rule & RULE_INCLUSIVE);
        if (incl ? !(dis <= (double)ddf) : !(dis < (double)ddf)) return -1;
        int bn = (int)(sqrt(dis) * ds);
        if (bn < 0 || bn >= bins) return -1;
        slot = bn;
    } else {
        float z2 = d[2] * d[2];
        float a = d[0] * d[0], b = d[1] * d[1];
        float r2 = a + b;
        if (!(z2 < ddf && r2 < ddf)) return -1;
        int bz = (int)(sqrt((double)z2) * ds), bp = (int)(sqrt((double)r2) * ds);
        if (bz < 0 || bz >= bins || bp < 0 || bp >= bins) return -1;
        slot = bz * bins + bp;
    }
    float w = self ? (2.0f * p->w) * q->w : p->w * q->w;
    *wprod = (double)w;
    return slot;
}

/* Neumaier (compensated) summation: s + c carries the sum of every term with
 * an error of about one rounding of the total, so the order of the additions
 * (threads, cells) does not show in the result.  Every term added here (an
 * FP32 x FP32 product, times 2) is exact in FP64. */
static inline void nsum_add(double *s, double *c, double x)
{
    double t = *s + x;
    if (fabs(*s) >= fabs(x)) *c += (*s - t) + x;
    else *c += (x - t) + *s;
    *s = t;
}

/* Cells of side >= dmax * 1.001 over the box: every pair within reach of the
 * rule (|d| per axis < dmax, or <= for the inclusive rule, after the minimum
 * image) lies in the same or an adjacent cell.  Returns the cells per side,
 * 0 when the box holds fewer than 3 (no pruning possible). */
static int prune_cells(float L, float dmax)
{
    double c = (double)L / ((double)dmax * 1.001);
    int P = (int)c;
    if (P > 256) P = 256;
    return P >= 3 ? P : 0;
}

static inline int cell_of(float x, int P, float L)
{
    int c = (int)((double)x * (double)P / (double)L);
    return c < 0 ? 0 : (c >= P ? P - 1 : c);
}

/*
 * Pair histogram.  self != 0: XX over catalog A, ordered pairs i != j
 * (each unordered pair adds 2*w_i*w_j, as the reference launches both
 * orders); self == 0: XY, every A x B pair once.
 * ds <= 0 selects orc_ds(bins, dmax, ds_exact); ds > 0 is used as given.
 * out has bins (iso) or bins*bins (ani) doubles and is overwritten.
 * method: 0 automatic, 1 every pair (brute force), 2 cell-pruned (only pairs
 * of the same or adjacent cells of side >= dmax are tested; falls back to
 * brute force when the box holds fewer than 3 such cells).  Both visit every
 * pair the rule can accept, so they give the same histogram.
 */
int orc_pairs_m(int ani, int bpc, int self, unsigned rule, int ds_exact, double ds_in, int prec,
                const opt *A, long nA, const opt *B, long nB, float L, int bins, float dmax,
                double *out, int method)
{
    const int nb = ani ? bins * bins : bins;
    const double ds = ds_in > 0 ? ds_in : orc_ds(bins, dmax, ds_exact);
    const float ddf = dmax * dmax;
    const double ddmax = (double)ddf;
    const double Ld = (double)L;
    const int cpu = prec == ORC_REF32_CPU_BPC;
    if (self) { B = A; nB = nA; }
    memset(out, 0, sizeof(double) * (size_t)nb);
    int P = 0;
    if (method == 2 || (method == 0 && (double)nA * (double)nB > 2e8)) P = prune_cells(L, dmax);
    int nt = omp_get_max_threads();
    double *priv = (double *)calloc((size_t)nt * nb * 2, sizeof(double));
    if (!priv) return -1;
    /* cell-ordered index of B (pruned method) */
    long *bstart = NULL, *border = NULL;
    if (P) {
        long ncell = (long)P * P * P;
        bstart = (long *)calloc((size_t)ncell + 1, sizeof(long));
        border = (long *)malloc(sizeof(long) * (size_t)(nB > 0 ? nB : 1));
        long *fill = (long *)calloc((size_t)ncell, sizeof(long));
        if (!bstart || !border || !fill) return -1;
        for (long j = 0; j < nB; ++j) {
            long c = ((long)cell_of(B[j].x, P, L) * P + cell_of(B[j].y, P, L)) * P +
                     cell_of(B[j].z, P, L);
            ++bstart[c + 1];
        }
        for (long c = 0; c < ncell; ++c) bstart[c + 1] += bstart[c];
        for (long j = 0; j < nB; ++j) {
            long c = ((long)cell_of(B[j].x, P, L) * P + cell_of(B[j].y, P, L)) * P +
                     cell_of(B[j].z, P, L);
            border[bstart[c] + fill[c]++] = j;
        }
        free(fill);
    }
#pragma omp parallel
    {
        double *h = priv + (size_t)omp_get_thread_num() * nb * 2;
        double *hc = h + nb;
        /* one pair (i, j): adds its weight to its slot */
#define ORC_PAIR(pi, pj, wmul)                                                              \
        do {                                                                                \
            double wq = 0.0;                                                                \
            int s_;                                                                         \
            if (cpu) s_ = cpu_bpc_slot(pi, pj, ani, self, L, ddf, ds, bins, rule, &wq);           \
            else {                                                                          \
                s_ = pair_slot(pi, pj, ani, bpc, Ld, prec, rule, ddmax, ds, bins);          \
                wq = (wmul) * ((double)(pi)->w * (double)(pj)->w);                          \
            }                                                                               \
            if (s_ >= 0) nsum_add(&h[s_], &hc[s_], wq);                                     \
        } while (0)
        if (!P) {
#pragma omp for schedule(dynamic, 16)
            for (long i = 0; i < nA; ++i) {
                const opt *p = &A[i];
                long j0 = self ? i + 1 : 0;
                for (long j = j0; j < nB; ++j) ORC_PAIR(p, &B[j], self ? 2.0 : 1.0);
            }
        } else {
            /* XX: each unordered pair once, from its lower index, adding
             * 2*w_i*w_j as the brute-force loop does (the rule is symmetric
             * in the two points; the emulated CPU rule forms 2*w1*w2 itself) */
#pragma omp for schedule(dynamic, 64)
            for (long i = 0; i < nA; ++i) {
                const opt *p = &A[i];
                int cx = cell_of(p->x, P, L), cy = cell_of(p->y, P, L), cz = cell_of(p->z, P, L);
                for (int ox = -1; ox <= 1; ++ox) {
                    int nx = cx + ox;
                    if (nx < 0 || nx >= P) { if (!bpc) continue; nx = (nx + P) % P; }
                    for (int oy = -1; oy <= 1; ++oy) {
                        int ny = cy + oy;
                        if (ny < 0 || ny >= P) { if (!bpc) continue; ny = (ny + P) % P; }
                        for (int oz = -1; oz <= 1; ++oz) {
                            int nz = cz + oz;
                            if (nz < 0 || nz >= P) { if (!bpc) continue; nz = (nz + P) % P; }
                            long c = ((long)nx * P + ny) * P + nz;
                            for (long t = bstart[c]; t < bstart[c + 1]; ++t) {
                                long j = border[t];
                                if (self && j <= i) continue;
                                ORC_PAIR(p, &B[j], self ? 2.0 : 1.0);
                            }
                        }
                    }
                }
            }
        }
#undef ORC_PAIR
    }
    for (int k = 0; k < nb; ++k) {
        double s = 0.0, c = 0.0;
        for (int t = 0; t < nt; ++t) {
            nsum_add(&s, &c, priv[(size_t)t * nb * 2 + k]);
            nsum_add(&s, &c, priv[(size_t)t * nb * 2 + nb + k]);
        }
        out[k] = s + c;
    }
    free(priv);
    free(bstart);
    free(border);
    return 0;
}

int orc_pairs(int ani, int bpc, int self, unsigned rule, int ds_exact, double ds_in, int prec,
              const opt *A, long nA, const opt *B, long nB, float L, int bins, float dmax,
              double *out)
{
    return orc_pairs_m(ani, bpc, self, rule, ds_exact, ds_in, prec, A, nA, B, nB, L, bins, dmax,
                       out, 0);
}

/* ----------------------------------------------------------------------- */
/* Triplets (isotropic): ordered triples, bin = b(d12)*bins^2 + b(d23)*bins */
/* + b(d31) (3iso_k.cuh:71-77), weight w1*w2*w3.  With periodic boundaries  */
/* the consistent embedding of count123 (3isoBPC_k.cuh:56-75): points 2, 3  */
/* take their minimum image relative to point 1 and d23 = |img3 - img2|.    */
/* ----------------------------------------------------------------------- */

typedef struct { int idx; int bin; double v[3]; } nbr_t;

/* FP32 side as the plain reference kernels compute it (3iso_k.cuh:57,66,69),
 * with the contraction pattern selected by prec. */
static int side_bin32(const opt *p, const opt *q, int prec, double ddmax, unsigned rule,
                      double ds, int bins)
{
    float fx = q->x - p->x, fy = q->y - p->y, fz = q->z - p->z;
    double d2 = (double)d2_ref32(fx, fy, fz, prec);
    if (!in_range(d2, ddmax, rule)) return -1;
    return bin_of(d2, ds, bins);
}

static int side_bin(const double v[3], double ddmax, unsigned rule, double ds, int bins)
{
    double xx = v[0] * v[0], yy = v[1] * v[1], zz = v[2] * v[2];
    double d2 = (xx + yy) + zz;
    if (!in_range(d2, ddmax, rule)) return -1;
    return bin_of(d2, ds, bins);
}

/* Neighbours of point p among Q[j0..nQ) with a valid side bin. */
static nbr_t *neighbours(const opt *p, const opt *Q, long j0, long nQ, int bpc, double L,
                         unsigned rule, double ddmax, double ds, int bins, int prec, long *cnt)
{
    long cap = 64, n = 0;
    nbr_t *a = (nbr_t *)malloc(sizeof(nbr_t) * cap);
    for (long j = j0; j < nQ; ++j) {
        double v[3] = {sep64(p->x, Q[j].x, bpc, L), sep64(p->y, Q[j].y, bpc, L),
                       sep64(p->z, Q[j].z, bpc, L)};
        int b = prec ? side_bin32(p, &Q[j], prec, ddmax, rule, ds, bins)
                     : side_bin(v, ddmax, rule, ds, bins);
        if (b < 0) continue;
        if (n == cap) { cap *= 2; a = (nbr_t *)realloc(a, sizeof(nbr_t) * cap); }
        a[n].idx = (int)j; a[n].bin = b;
        a[n].v[0] = v[0]; a[n].v[1] = v[1]; a[n].v[2] = v[2];
        ++n;
    }
    *cnt = n;
    return a;
}

/* ----------------------------------------------------------------------- */
/* The reference's periodic 3-point node gates (3aniBPC_k.cuh:210-957        */
/* XXX3ani_BPC, :959-1708 XXY3ani_BPC; 3isoBPC_k.cuh:191-939, 940-1693 hold   */
/* the same 64 blocks).  Each thread takes one ordered node triple           */
/* (n1, n2, n3) of the reference's grid (size s = box / partitions, node     */
/* corner = (float)(int)(x / s) * s, create_grid.cuh:120-135) and runs the   */
/* point loop once per block whose gate passes, with that block's image      */
/* flags F2 (node 2 seen through its x/y/z image) and F3.  A triangle in     */
/* range through the images (S2, S3) of its sides 12 and 31 is therefore     */
/* counted once per passing block with (F2, F3) == (S2, S3).  A gate needs   */
/* the edge flags A2 / A3 (fa_k: nodes 1 and k within dmax + s of opposite   */
/* faces along a) and up to three node-distance tests, pair p in {12, 23,    */
/* 31}:  dd_p + k*L^2 - 2*(sum of dn_p over the listed axes)*L <= M,         */
/* M = (dmax + s*sqrt(3))^2, k = 0 with no axes meaning dd_p <= M.           */
/* The table is the reference's blocks in source order, as written there:    */
/* four same-image blocks (xy, xz, yz, xyz) test 23 through the image where  */
/* 31 is meant, block (F2 = x, A2 = y, F3 = xyz) is gated for node 2's y     */
/* image but counts with its x image (no block counts S2 = y, S3 = xyz),     */
/* block (xy, z) sums dz23 twice, block (xyz, xz) adds 3L^2 for one axis.    */
/* Gates evaluate in FP32 with the multiply-adds fused, the reference's      */
/* kernels being built with contraction on; exact whenever the node corners  */
/* and their sums are exact (e.g. integer lattices).                          */
/* ----------------------------------------------------------------------- */
typedef struct { signed char pair, k, ax[3]; } gate_test;
typedef struct { unsigned char f2, f3, a2, a3; gate_test t[3]; } gate_block;
static const gate_block kGates[64] = {
    {0, 0, 0, 0, {{0, 0, {-1, -1, -1}}, {1, 0, {-1, -1, -1}}, {2, 0, {-1, -1, -1}}}},
    {0, 1, 0, 1, {{0, 0, {-1, -1, -1}}, {1, 1, {0, -1, -1}}, {2, 1, {0, -1, -1}}}},
    {0, 2, 0, 2, {{0, 0, {-1, -1, -1}}, {1, 1, {1, -1, -1}}, {2, 1, {1, -1, -1}}}},
    {0, 4, 0, 4, {{0, 0, {-1, -1, -1}}, {1, 1, {2, -1, -1}}, {2, 1, {2, -1, -1}}}},
    {0, 3, 0, 3, {{0, 0, {-1, -1, -1}}, {1, 2, {0, 1, -1}}, {2, 2, {0, 1, -1}}}},
    {0, 5, 0, 5, {{0, 0, {-1, -1, -1}}, {1, 2, {0, 2, -1}}, {2, 2, {0, 2, -1}}}},
    {0, 6, 0, 6, {{0, 0, {-1, -1, -1}}, {1, 2, {1, 2, -1}}, {2, 2, {1, 2, -1}}}},
    {0, 7, 0, 7, {{0, 0, {-1, -1, -1}}, {1, 3, {0, 1, 2}}, {2, 3, {0, 1, 2}}}},
    {1, 0, 1, 0, {{2, 0, {-1, -1, -1}}, {1, 1, {0, -1, -1}}, {0, 1, {0, -1, -1}}}},
    {2, 0, 2, 0, {{2, 0, {-1, -1, -1}}, {1, 1, {1, -1, -1}}, {0, 1, {1, -1, -1}}}},
    {4, 0, 4, 0, {{2, 0, {-1, -1, -1}}, {1, 1, {2, -1, -1}}, {0, 1, {2, -1, -1}}}},
    {3, 0, 3, 0, {{2, 0, {-1, -1, -1}}, {1, 2, {0, 1, -1}}, {0, 2, {0, 1, -1}}}},
    {5, 0, 5, 0, {{2, 0, {-1, -1, -1}}, {1, 2, {0, 2, -1}}, {0, 2, {0, 2, -1}}}},
    {6, 0, 6, 0, {{2, 0, {-1, -1, -1}}, {1, 2, {1, 2, -1}}, {0, 2, {1, 2, -1}}}},
    {7, 0, 7, 0, {{2, 0, {-1, -1, -1}}, {1, 3, {0, 1, 2}}, {0, 3, {0, 1, 2}}}},
    {1, 1, 1, 1, {{1, 0, {-1, -1, -1}}, {2, 1, {0, -1, -1}}, {0, 1, {0, -1, -1}}}},
    {2, 2, 2, 2, {{1, 0, {-1, -1, -1}}, {2, 1, {1, -1, -1}}, {0, 1, {1, -1, -1}}}},
    {4, 4, 4, 4, {{1, 0, {-1, -1, -1}}, {2, 1, {2, -1, -1}}, {0, 1, {2, -1, -1}}}},
    {3, 3, 3, 3, {{1, 0, {-1, -1, -1}}, {1, 2, {0, 1, -1}}, {0, 2, {0, 1, -1}}}},
    {5, 5, 5, 5, {{1, 0, {-1, -1, -1}}, {1, 2, {0, 2, -1}}, {0, 2, {0, 2, -1}}}},
    {6, 6, 6, 6, {{1, 0, {-1, -1, -1}}, {1, 2, {1, 2, -1}}, {0, 2, {1, 2, -1}}}},
    {7, 7, 7, 7, {{1, 0, {-1, -1, -1}}, {1, 3, {0, 1, 2}}, {0, 3, {0, 1, 2}}}},
    {1, 2, 1, 2, {{0, 1, {0, -1, -1}}, {2, 1, {1, -1, -1}}, {1, 2, {0, 1, -1}}}},
    {1, 4, 1, 4, {{0, 1, {0, -1, -1}}, {2, 1, {2, -1, -1}}, {1, 2, {0, 2, -1}}}},
    {1, 3, 1, 3, {{0, 1, {0, -1, -1}}, {2, 2, {0, 1, -1}}, {1, 1, {1, -1, -1}}}},
    {1, 5, 1, 5, {{0, 1, {0, -1, -1}}, {2, 2, {0, 2, -1}}, {1, 1, {2, -1, -1}}}},
    {1, 6, 1, 6, {{0, 1, {0, -1, -1}}, {2, 2, {1, 2, -1}}, {1, 3, {0, 1, 2}}}},
    {1, 7, 1, 7, {{0, 1, {0, -1, -1}}, {2, 3, {0, 1, 2}}, {1, 2, {1, 2, -1}}}},
    {2, 1, 2, 1, {{0, 1, {1, -1, -1}}, {2, 1, {0, -1, -1}}, {1, 2, {0, 1, -1}}}},
    {2, 4, 2, 4, {{0, 1, {1, -1, -1}}, {2, 1, {2, -1, -1}}, {1, 2, {1, 2, -1}}}},
    {2, 3, 2, 3, {{0, 1, {1, -1, -1}}, {2, 2, {0, 1, -1}}, {1, 1, {0, -1, -1}}}},
    {2, 5, 2, 5, {{0, 1, {1, -1, -1}}, {2, 2, {0, 2, -1}}, {1, 3, {0, 1, 2}}}},
    {2, 6, 2, 6, {{0, 1, {1, -1, -1}}, {2, 2, {1, 2, -1}}, {1, 1, {2, -1, -1}}}},
    {1, 7, 2, 7, {{0, 1, {1, -1, -1}}, {2, 3, {0, 1, 2}}, {1, 2, {0, 2, -1}}}},
    {4, 1, 4, 1, {{0, 1, {2, -1, -1}}, {2, 1, {0, -1, -1}}, {1, 2, {0, 2, -1}}}},
    {4, 2, 4, 2, {{0, 1, {2, -1, -1}}, {2, 1, {1, -1, -1}}, {1, 2, {1, 2, -1}}}},
    {4, 3, 4, 3, {{0, 1, {2, -1, -1}}, {2, 2, {0, 1, -1}}, {1, 3, {0, 1, 2}}}},
    {4, 5, 4, 5, {{0, 1, {2, -1, -1}}, {2, 2, {0, 2, -1}}, {1, 1, {0, -1, -1}}}},
    {4, 6, 4, 6, {{0, 1, {2, -1, -1}}, {2, 2, {1, 2, -1}}, {1, 1, {1, -1, -1}}}},
    {4, 7, 4, 7, {{0, 1, {2, -1, -1}}, {2, 3, {0, 1, 2}}, {1, 2, {0, 1, -1}}}},
    {3, 1, 3, 1, {{0, 2, {0, 1, -1}}, {2, 1, {0, -1, -1}}, {1, 1, {1, -1, -1}}}},
    {3, 2, 3, 2, {{0, 2, {0, 1, -1}}, {2, 1, {1, -1, -1}}, {1, 1, {0, -1, -1}}}},
    {3, 4, 3, 4, {{0, 2, {0, 1, -1}}, {2, 1, {2, -1, -1}}, {1, 3, {2, 1, 2}}}},
    {3, 5, 3, 5, {{0, 2, {0, 1, -1}}, {2, 2, {0, 2, -1}}, {1, 2, {1, 2, -1}}}},
    {3, 6, 3, 6, {{0, 2, {0, 1, -1}}, {2, 2, {1, 2, -1}}, {1, 2, {0, 2, -1}}}},
    {3, 7, 3, 7, {{0, 2, {0, 1, -1}}, {2, 3, {0, 1, 2}}, {1, 1, {2, -1, -1}}}},
    {5, 1, 5, 1, {{0, 2, {0, 2, -1}}, {2, 1, {0, -1, -1}}, {1, 1, {2, -1, -1}}}},
    {5, 2, 5, 2, {{0, 2, {0, 2, -1}}, {2, 1, {1, -1, -1}}, {1, 3, {0, 1, 2}}}},
    {5, 4, 5, 4, {{0, 2, {0, 2, -1}}, {2, 1, {2, -1, -1}}, {1, 1, {0, -1, -1}}}},
    {5, 3, 5, 3, {{0, 2, {0, 2, -1}}, {2, 2, {0, 1, -1}}, {1, 2, {1, 2, -1}}}},
    {5, 6, 5, 6, {{0, 2, {0, 2, -1}}, {2, 2, {1, 2, -1}}, {1, 2, {0, 1, -1}}}},
    {5, 7, 5, 7, {{0, 2, {0, 2, -1}}, {2, 3, {0, 1, 2}}, {1, 1, {1, -1, -1}}}},
    {6, 1, 6, 1, {{0, 2, {2, 1, -1}}, {2, 1, {0, -1, -1}}, {1, 3, {0, 1, 2}}}},
    {6, 2, 6, 2, {{0, 2, {2, 1, -1}}, {2, 1, {1, -1, -1}}, {1, 1, {2, -1, -1}}}},
    {6, 4, 6, 4, {{0, 2, {2, 1, -1}}, {2, 1, {2, -1, -1}}, {1, 1, {1, -1, -1}}}},
    {6, 3, 6, 3, {{0, 2, {2, 1, -1}}, {2, 2, {0, 1, -1}}, {1, 2, {0, 2, -1}}}},
    {6, 5, 6, 5, {{0, 2, {2, 1, -1}}, {2, 2, {0, 2, -1}}, {1, 2, {0, 1, -1}}}},
    {6, 7, 6, 7, {{0, 2, {2, 1, -1}}, {2, 3, {0, 1, 2}}, {1, 1, {0, -1, -1}}}},
    {7, 1, 7, 1, {{0, 3, {0, 1, 2}}, {2, 1, {0, -1, -1}}, {1, 2, {1, 2, -1}}}},
    {7, 2, 7, 2, {{0, 3, {0, 1, 2}}, {2, 1, {1, -1, -1}}, {1, 2, {0, 2, -1}}}},
    {7, 4, 7, 4, {{0, 3, {0, 1, 2}}, {2, 1, {2, -1, -1}}, {1, 2, {0, 1, -1}}}},
    {7, 3, 7, 3, {{0, 3, {0, 1, 2}}, {2, 2, {0, 1, -1}}, {1, 1, {2, -1, -1}}}},
    {7, 5, 7, 5, {{0, 3, {0, 1, 2}}, {2, 2, {0, 2, -1}}, {1, 3, {1, -1, -1}}}},
    {7, 6, 7, 6, {{0, 3, {0, 1, 2}}, {2, 2, {1, 2, -1}}, {1, 1, {0, -1, -1}}}},
};

typedef struct {
    float s, L, L2, M, fd, fdn;
    int P;
} gate_geom;

static gate_geom gate_setup(float L, float dmax, int P)
{
    gate_geom g;
    g.P = P;
    g.s = L / (float)P;                                 /* main.cu:216 */
    g.L = L;
    g.L2 = L * L;
    float dmn = (float)((double)dmax + (double)g.s * sqrt(3.0)); /* pcf3aniBPC.cuh:59-60 */
    g.M = dmn * dmn;
    g.fd = dmax + g.s;
    g.fdn = L - g.fd;
    return g;
}

static inline void gate_corner(const gate_geom *g, const opt *p, float n[3])
{
    const float c[3] = {p->x, p->y, p->z};
    for (int a = 0; a < 3; ++a) {
        int r = (int)(c[a] / g->s);
        if (r > g->P - 1) r = g->P - 1;
        if (r < 0) r = 0;
        n[a] = (float)r * g->s;
    }
}

static inline unsigned wrap_bits(const opt *p, const opt *q, double L)
{
    const double d[3] = {(double)q->x - (double)p->x, (double)q->y - (double)p->y,
                         (double)q->z - (double)p->z};
    unsigned b = 0;
    for (int a = 0; a < 3; ++a)
        if (d[a] > 0.5 * L || d[a] < -0.5 * L) b |= 1u << a;
    return b;
}

/* Number of reference blocks that count the ordered triangle (1, 2, 3) with
 * node corners n1, n2, n3 whose sides 12 and 31 are in range through the
 * images s2, s3. */
static int gate_mult(const gate_geom *g, const float n1[3], const float n2[3], const float n3[3],
                     unsigned s2, unsigned s3)
{
    float dn[3][3], dd[3];
    for (int a = 0; a < 3; ++a) {
        dn[0][a] = fabsf(n2[a] - n1[a]);
        dn[1][a] = fabsf(n3[a] - n2[a]);
        dn[2][a] = fabsf(n1[a] - n3[a]);
    }
    for (int q = 0; q < 3; ++q)
        dd[q] = fmaf(dn[q][2], dn[q][2], fmaf(dn[q][1], dn[q][1], dn[q][0] * dn[q][0]));
    unsigned f2 = 0, f3 = 0;
    for (int a = 0; a < 3; ++a) {
        if ((n1[a] <= g->fd && n2[a] >= g->fdn) || (n2[a] <= g->fd && n1[a] >= g->fdn)) f2 |= 1u << a;
        if ((n1[a] <= g->fd && n3[a] >= g->fdn) || (n3[a] <= g->fd && n1[a] >= g->fdn)) f3 |= 1u << a;
    }
    int m = 0;
    for (int b = 0; b < 64; ++b) {
        const gate_block *B = &kGates[b];
        if (B->f2 != s2 || B->f3 != s3) continue;
        if ((f2 & B->a2) != B->a2 || (f3 & B->a3) != B->a3) continue;
        int ok = 1;
        for (int t = 0; t < 3 && ok; ++t) {
            const gate_test *T = &B->t[t];
            float v = dd[T->pair];
            if (T->ax[0] >= 0) {
                float sm = dn[T->pair][T->ax[0]];
                if (T->ax[1] >= 0) sm = sm + dn[T->pair][T->ax[1]];
                if (T->ax[2] >= 0) sm = sm + dn[T->pair][T->ax[2]];
                v = fmaf((float)T->k, g->L2, v);
                v = fmaf(-(2.0f * sm), g->L, v);
            }
            ok = v <= g->M;
        }
        m += ok;
    }
    return m;
}

/*
 * mixed == 0: XXX over X (all three sides: 0 < d2 < dd_max).
 * mixed != 0: XXY with points 1,2 from X and point 3 from Y; side 12 needs
 *   0 < d2, sides 23 and 31 need 0 < d2 only with periodic boundaries
 *   (3iso_k.cuh:158,160 vs 3isoBPC_k.cuh:165,170).
 * out: bins^3 doubles, overwritten.
 */
int orc_triplets_iso(int bpc, int mixed, int prec, const opt *X, long nX, const opt *Y, long nY,
                     float L, int bins, float dmax, int gate_P, double *out)
{
    if (bpc) prec = ORC_FP64; /* FP32 emulation covers the plain kernels only */
    const int gated = bpc && gate_P > 0;
    gate_geom gg = gate_setup(L, dmax, gated ? gate_P : 1);
    const long nb = (long)bins * bins * bins;
    const double ds = orc_ds(bins, dmax, 0);
    const float ddf = dmax * dmax;
    const double ddmax = (double)ddf;
    const double Ld = (double)L;
    const unsigned rXX = RULE_EXCL_ZERO;
    const unsigned rXY = bpc ? RULE_EXCL_ZERO : 0u;
    const long b2 = (long)bins * bins;
    memset(out, 0, sizeof(double) * (size_t)nb);
    int nt = omp_get_max_threads();
    double *priv = (double *)calloc((size_t)nt * nb, sizeof(double));
    if (!priv) return -1;
#pragma omp parallel
    {
        double *h = priv + (size_t)omp_get_thread_num() * nb;
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < nX; ++i) {
            const opt *p = &X[i];
            long n2, n3;
            nbr_t *N2 = neighbours(p, X, i + 1, nX, bpc, Ld, rXX, ddmax, ds, bins, prec, &n2);
            if (!mixed) {
                for (long a = 0; a < n2; ++a) {
                    const nbr_t *q = &N2[a];
                    double wij = (double)p->w * (double)X[q->idx].w;
                    for (long b = a + 1; b < n2; ++b) {
                        const nbr_t *r = &N2[b];
                        double v[3] = {r->v[0] - q->v[0], r->v[1] - q->v[1], r->v[2] - q->v[2]};
                        int bjk = prec ? side_bin32(&X[q->idx], &X[r->idx], prec, ddmax, rXX, ds, bins)
                                       : side_bin(v, ddmax, rXX, ds, bins);
                        if (bjk < 0) continue;
                        double w = wij * (double)X[r->idx].w;
                        long A = q->bin, Bb = bjk, C = r->bin; /* (ij, jk, ki) */
                        /* orderings (1,2,3): (i,q,r) (q,r,i) (r,i,q) (i,r,q) (r,q,i) (q,i,r) */
                        double m[6] = {1, 1, 1, 1, 1, 1};
                        if (gated) {
                            const opt *P3[3] = {p, &X[q->idx], &X[r->idx]};
                            float nc[3][3];
                            for (int u = 0; u < 3; ++u) gate_corner(&gg, P3[u], nc[u]);
                            static const int ord[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1},
                                                          {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
                            for (int o = 0; o < 6; ++o) {
                                const int u = ord[o][0], t2 = ord[o][1], t3 = ord[o][2];
                                m[o] = gate_mult(&gg, nc[u], nc[t2], nc[t3], wrap_bits(P3[u], P3[t2], Ld),
                                                 wrap_bits(P3[u], P3[t3], Ld));
                            }
                        }
                        h[A * b2 + Bb * bins + C] += w * m[0];
                        h[Bb * b2 + C * bins + A] += w * m[1];
                        h[C * b2 + A * bins + Bb] += w * m[2];
                        h[C * b2 + Bb * bins + A] += w * m[3];
                        h[Bb * b2 + A * bins + C] += w * m[4];
                        h[A * b2 + C * bins + Bb] += w * m[5];
                    }
                }
            } else {
                nbr_t *N3 = neighbours(p, Y, 0, nY, bpc, Ld, rXY, ddmax, ds, bins, prec, &n3);
                for (long a = 0; a < n2; ++a) {
                    const nbr_t *q = &N2[a];
                    double wij = (double)p->w * (double)X[q->idx].w;
                    for (long b = 0; b < n3; ++b) {
                        const nbr_t *r = &N3[b];
                        double v[3] = {r->v[0] - q->v[0], r->v[1] - q->v[1], r->v[2] - q->v[2]};
                        int bjk = prec ? side_bin32(&X[q->idx], &Y[r->idx], prec, ddmax, rXY, ds, bins)
                                       : side_bin(v, ddmax, rXY, ds, bins);
                        if (bjk < 0) continue;
                        double w = wij * (double)Y[r->idx].w;
                        long A = q->bin, Bb = bjk, C = r->bin;
                        /* orderings (1,2,3): (i,q,r) and (q,i,r), point 3 from Y */
                        double m0 = 1, m1 = 1;
                        if (gated) {
                            float c1[3], c2[3], c3[3];
                            gate_corner(&gg, p, c1);
                            gate_corner(&gg, &X[q->idx], c2);
                            gate_corner(&gg, &Y[r->idx], c3);
                            m0 = gate_mult(&gg, c1, c2, c3, wrap_bits(p, &X[q->idx], Ld),
                                           wrap_bits(p, &Y[r->idx], Ld));
                            m1 = gate_mult(&gg, c2, c1, c3, wrap_bits(&X[q->idx], p, Ld),
                                           wrap_bits(&X[q->idx], &Y[r->idx], Ld));
                        }
                        h[A * b2 + Bb * bins + C] += w * m0;
                        h[A * b2 + C * bins + Bb] += w * m1;
                    }
                }
                free(N3);
            }
            free(N2);
        }
    }
    for (int t = 0; t < nt; ++t)
        for (long k = 0; k < nb; ++k) out[k] += priv[(size_t)t * nb + k];
    free(priv);
    return 0;
}

/* ----------------------------------------------------------------------- */
/* Triplets (anisotropic, bins^5): a=b(d12), b=b(d31), c=b(d23),            */
/* With periodic boundaries the reference folds the sign of dz:             */
/* dz = |z2 - z1| - L*f (3aniBPC_k.cuh:57,73), f = 1 when the pair uses its */
/* z image, i.e. +|dz| without a z wrap and -|dz_min| with one.             */
/* t=(int)((1+dz12/d12)*bins/2), p=(int)((1+dz31/d31)*bins/2)               */
/* (3ani_k.cuh:75-91), each dropped when >= bins.  Ordered triples are      */
/* enumerated directly (no symmetry: the angles are anchored at point 1).   */
/* ----------------------------------------------------------------------- */
static inline double bpc_dz(float z1, float z2, double L)
{
    double d = fabs((double)z2 - (double)z1);
    return d > 0.5 * L ? d - L : d;
}

static inline int ani_angle_bin(double dz, double d, int bins)
{
    double c = 1.0 + dz / d;
    double th = (double)((float)bins / 2.0f);
    int t = (int)(c * th);
    return (t >= 0 && t < bins) ? t : -1;
}

int orc_triplets_ani(int bpc, int mixed, const opt *X, long nX, const opt *Y, long nY, float L,
                     int bins, float dmax, int gate_P, double *out)
{
    const long B = bins;
    const long nb = B * B * B * B * B;
    const double ds = orc_ds(bins, dmax, 0);
    const float ddf = dmax * dmax;
    const double ddmax = (double)ddf;
    const double Ld = (double)L;
    const unsigned rXX = RULE_EXCL_ZERO;
    const unsigned rXY = bpc ? RULE_EXCL_ZERO : 0u;
    if (!mixed) { Y = X; nY = nX; }
    const int gated = bpc && gate_P > 0;
    gate_geom gg = gate_setup(L, dmax, gated ? gate_P : 1);
    memset(out, 0, sizeof(double) * (size_t)nb);
    int nt = omp_get_max_threads();
    double *priv = (double *)calloc((size_t)nt * nb, sizeof(double));
    if (!priv) return -1;
#pragma omp parallel
    {
        double *h = priv + (size_t)omp_get_thread_num() * nb;
#pragma omp for schedule(dynamic, 1)
        for (long i = 0; i < nX; ++i) {
            const opt *p = &X[i];
            long n2, n3;
            float n1c[3], n2c[3], n3c[3];
            if (gated) gate_corner(&gg, p, n1c);
            nbr_t *N2 = neighbours(p, X, 0, nX, bpc, Ld, rXX, ddmax, ds, bins, 0, &n2);
            nbr_t *N3 = neighbours(p, Y, 0, nY, bpc, Ld, mixed ? rXY : rXX, ddmax, ds, bins, 0, &n3);
            for (long a = 0; a < n2; ++a) {
                const nbr_t *q = &N2[a];
                if (q->idx == i) continue;
                double d12 = sqrt((q->v[0] * q->v[0] + q->v[1] * q->v[1]) + q->v[2] * q->v[2]);
                int t = ani_angle_bin(bpc ? bpc_dz(p->z, X[q->idx].z, Ld) : q->v[2], d12, bins);
                if (t < 0) continue;
                double wij = (double)p->w * (double)X[q->idx].w;
                unsigned s2 = 0;
                if (gated) {
                    gate_corner(&gg, &X[q->idx], n2c);
                    s2 = wrap_bits(p, &X[q->idx], Ld);
                }
                for (long b = 0; b < n3; ++b) {
                    const nbr_t *r = &N3[b];
                    if (!mixed && (r->idx == i || r->idx == q->idx)) continue;
                    double v[3] = {r->v[0] - q->v[0], r->v[1] - q->v[1], r->v[2] - q->v[2]};
                    int c = side_bin(v, ddmax, mixed ? rXY : rXX, ds, bins);
                    if (c < 0) continue;
                    double d31 = sqrt((r->v[0] * r->v[0] + r->v[1] * r->v[1]) + r->v[2] * r->v[2]);
                    int pp = ani_angle_bin(bpc ? bpc_dz(p->z, Y[r->idx].z, Ld) : r->v[2], d31, bins);
                    if (pp < 0) continue;
                    double w = wij * (double)Y[r->idx].w;
                    if (gated) {
                        gate_corner(&gg, &Y[r->idx], n3c);
                        int m = gate_mult(&gg, n1c, n2c, n3c, s2, wrap_bits(p, &Y[r->idx], Ld));
                        if (m == 0) continue;
                        w *= (double)m;
                    }
                    long slot = (((q->bin * B + r->bin) * B + c) * B + t) * B + pp;
                    h[slot] += w;
                }
            }
            free(N2);
            free(N3);
        }
    }
    for (int t = 0; t < nt; ++t)
        for (long k = 0; k < nb; ++k) out[k] += priv[(size_t)t * nb + k];
    free(priv);
    return 0;
}

/* ----------------------------------------------------------------------- */
/* Analytic periodic-box histograms.                                         */
/* ----------------------------------------------------------------------- */

/* Coefficient 3k^2+3k+1 as the reference computes it in 32-bit int
 * (2isoBPC_k.cuh:564), i.e. wrapping modulo 2^32 once k exceeds 26754;
 * wrap == 0 evaluates it in 64-bit instead. */
static inline double shell_coef(long k, int wrap)
{
    if (wrap) {
        uint32_t u = 3u * (uint32_t)k * (uint32_t)k + 3u * (uint32_t)k + 1u;
        return (double)(int32_t)u;
    }
    return (double)(3 * k * k + 3 * k + 1);
}

/* alpha of RR2iso_BPC_analytic (pcf2isoBPC.cuh:199-202):
 * dr = dmax/bins in FP32, beta = (np*np)/L^3 in FP32, alpha = 8 dr^3 acos(0) beta / 3. */
static double rr_alpha(long np, float L, float dmax, long bins)
{
    float drf = dmax / (float)bins;
    double dr = (double)drf;
    float L3 = L * L * L;
    float betaf = (float)(np * np) / L3;
    double beta = (double)betaf;
    return 8 * dr * dr * dr * acos(0.0) * beta / 3;
}

void orc_analytic_rr(int bins, long np, float L, float dmax, int wrap, double *out)
{
    double alpha = rr_alpha(np, L, dmax, bins);
    for (long k = 0; k < bins; ++k) out[k] = alpha * shell_coef(k, wrap);
}

/* Does every corner of the cube [r1, r1+h]x[r2, r2+h]x[r3, r3+h] satisfy the
 * triangle inequality (3isoBPC_k.cuh:2040-2052 / 2078-2090)? */
static int all_corners(double ri, double rj, double rk, double h)
{
    int v = 0;
    for (int a = 0; a < 2; ++a) {
        double r1 = ri + (double)a * h;
        for (int b = 0; b < 2; ++b) {
            double r2 = rj + (double)b * h;
            for (int c = 0; c < 2; ++c) {
                double r3 = rk + (double)c * h;
                if (r1 + r2 >= r3 && r1 + r3 >= r2 && r2 + r3 >= r1) ++v;
            }
        }
    }
    return v;
}

/*
 * Analytic 3iso with periodic boundaries (pcf3isoBPC.cuh:177-347 with the
 * kernels of 3isoBPC_k.cuh:1694-2119).  D: the data catalog (n points),
 * ptt / bn_ref: the reference's sub-binning (100 / 200 in the reference).
 * Produces DDR (written twice by the reference, as DDR and DRR) and RRR,
 * bins^3 each.  Uses the canonical FP64 pair rule for the fine DD.
 * wrap: reproduce the reference's 32-bit coefficient overflow.
 * fine_dd / fine_dd_ref (optional, may be NULL): receive the fine DD histograms.
 */
/* make_ff_av_ref (3isoBPC_k.cuh:2001; the same average as the CPU engine's
 * cpp/3PCFisotropic/BPC/3PCFiso.h:1584-1604): per coarse bin i and
 * sub-bin j, the mean over the ptt fine bins k of
 * (r_i + r_j + r_k) * (DD/RR - 1).  ff_ref: bn_ref * bins, added to. */
void orc_ff_average_ref(const double *dd_ref, const double *rr_ref, int bins, float dmax, int ptt,
                        int bn_ref, double *ff_ref)
{
    for (int i = 0; i < bins; ++i) {
        for (int j = 0; j < bn_ref; ++j) {
            for (int k = 0; k < ptt; ++k) {
                double drr = dmax / (double)bins;
                double drr_ref = drr / bn_ref;
                double dr_ptt_ref = dmax / (double)((long)ptt * bn_ref * bins);
                double ri = i * drr, rj = j * drr_ref, rk = (k + 0.5) * dr_ptt_ref;
                long i_ = (long)i * bn_ref, j_ = (long)j * ptt;
                long s = i_ * ptt + j_ + k;
                double f = (ri + rj + rk) * ((dd_ref[s] / rr_ref[s]) - 1) / (double)ptt;
                ff_ref[i_ + j] += f;
            }
        }
    }
}

static int analytic_3iso_impl(const opt *D, long n, float L, int bins, float dmax, int ptt,
                              int bn_ref, int wrap, double *DDR, double *RRR, double *ff_av_out,
                              double *ff_ref_out, int refine)
{
    const long bn_ff = (long)ptt * bins;
    const long bn_ff_ref = (long)ptt * bn_ref * bins;
    double *dd_ff = (double *)calloc(bn_ff, sizeof(double));
    double *dd_ref = (double *)calloc(bn_ff_ref, sizeof(double));
    double *rr_ff = (double *)calloc(bn_ff, sizeof(double));
    double *rr_ref = (double *)calloc(bn_ff_ref, sizeof(double));
    double *ff_av = (double *)calloc(bins, sizeof(double));
    double *ff_ref = (double *)calloc((long)bn_ref * bins, sizeof(double));
    if (!dd_ff || !dd_ref || !rr_ff || !rr_ref || !ff_av || !ff_ref) return -1;

    /* constants, pcf3isoBPC.cuh:233-247 */
    float L3 = L * L * L;
    float betaf = (float)(n * n) / L3;
    double beta = (double)betaf;
    float dr_ff_f = dmax / (float)bn_ff;
    double dr_ff = (double)dr_ff_f;
    double alpha_ff = 8 * dr_ff * dr_ff * dr_ff * acos(0.0) * beta / 3;
    float dr_ffr_f = dmax / (float)bn_ff_ref;
    double dr_ffr = (double)dr_ffr_f;
    double alpha_ffr = 8 * dr_ffr * dr_ffr * dr_ffr * acos(0.0) * beta / 3;
    double dr = dmax / (double)bins;
    double dr_ref = dr / bn_ref;
    float Vf = L * L;
    double V = (double)Vf;
    double beta_3D = n / V;
    double gama = 8 * (4 * acos(0.0) * acos(0.0)) * (n * beta_3D * beta_3D);
    gama /= V;
    double alpha_ref = gama * dr_ref * dr_ref * dr_ref;
    double alpha = gama * dr * dr * dr;

    /* fine DD (DD2iso_forBPC): ordered pairs, periodic, 0 < d2 < dd_max, ds in FP32 */
    float dsf_ref = (float)bn_ff_ref / dmax;
    float dsf = (float)bn_ff / dmax;
    orc_pairs(0, 1, 1, RULE_EXCL_ZERO, 0, (double)dsf_ref, ORC_FP64, D, n, 0, 0, L, (int)bn_ff_ref,
              dmax, dd_ref);
    orc_pairs(0, 1, 1, RULE_EXCL_ZERO, 0, (double)dsf, ORC_FP64, D, n, 0, 0, L, (int)bn_ff, dmax,
              dd_ff);
    for (long k = 0; k < bn_ff; ++k) rr_ff[k] = alpha_ff * shell_coef(k, wrap);
    for (long k = 0; k < bn_ff_ref; ++k) rr_ref[k] = alpha_ffr * shell_coef(k, wrap);

    /* make_ff_av (3isoBPC_k.cuh:1984) */
    for (int i = 0; i < bins; ++i) {
        for (int j = 0; j < ptt; ++j) {
            long i_ = (long)i * ptt;
            float idm = (float)i * dmax;
            double ri = idm / (double)bins;
            double rj = (j + 0.5) * dmax / (double)bn_ff;
            double v = (ri + rj) * ((dd_ff[i_ + j] / rr_ff[i_ + j]) - 1) / (double)ptt;
            ff_av[i] += v;
        }
    }
    orc_ff_average_ref(dd_ref, rr_ref, bins, dmax, ptt, bn_ref, ff_ref);
    if (refine < 0) {  /* caller wants ff, ff_ref and alpha_ref only */
        if (ff_av_out) memcpy(ff_av_out, ff_av, sizeof(double) * bins);
        if (ff_ref_out) memcpy(ff_ref_out, ff_ref, sizeof(double) * bn_ref * bins);
        if (DDR) DDR[0] = alpha_ref;
        free(dd_ff); free(dd_ref); free(rr_ff); free(rr_ref); free(ff_av); free(ff_ref);
        return 0;
    }
    /* make_histo_analitic (3isoBPC_k.cuh:2021) */
    const long b2 = (long)bins * bins;
    memset(DDR, 0, sizeof(double) * b2 * bins);
    memset(RRR, 0, sizeof(double) * b2 * bins);
#pragma omp parallel for collapse(3) schedule(dynamic, 1)
    for (int i = 0; i < bins; ++i)
        for (int j = 0; j < bins; ++j)
            for (int k = 0; k < bins; ++k) {
                double dr2 = dr * 0.5;
                double ri = (double)i * dr, rj = (double)j * dr, rk = (double)k * dr;
                long i_ = (long)i * bn_ref, j_ = (long)j * bn_ref, k_ = (long)k * bn_ref;
                int v_in = all_corners(ri, rj, rk, dr);
                long slot = i * b2 + (long)j * bins + k;
                if (v_in == 8) {
                    double s = alpha * (ri + dr2) * (rj + dr2) * (rk + dr2);
                    RRR[slot] = s;
                    double f = 1;
                    f += ff_av[i] / (3 * (ri + dr2));
                    f += ff_av[j] / (3 * (rj + dr2));
                    f += ff_av[k] / (3 * (rk + dr2));
                    f *= s;
                    DDR[slot] += f;
                } else if (v_in > 0) {
                    int con = 0;
                    double h = dr_ref, h2 = dr_ref * 0.5;
                    double S_av = 0.0, f_av = 0.0;
                    for (int u = 0; u < bn_ref; ++u) {
                        double ru = ri + ((double)u * h);
                        for (int v = 0; v < bn_ref; ++v) {
                            double rv = rj + ((double)v * h);
                            for (int w = 0; w < bn_ref; ++w) {
                                double rw = rk + ((double)w * h);
                                if (all_corners(ru, rv, rw, h) != 8) continue;
                                double c = (ru + h2) * (rv + h2) * (rw + h2);
                                S_av += c;
                                double f = 1;
                                f += ff_ref[i_ + u] / (3 * (ru + h2));
                                f += ff_ref[j_ + v] / (3 * (rv + h2));
                                f += ff_ref[k_ + w] / (3 * (rw + h2));
                                f *= c;
                                f_av += f;
                                con = 1;
                            }
                        }
                    }
                    if (con) {
                        RRR[slot] += S_av * alpha_ref;
                        DDR[slot] += f_av * alpha_ref;
                    }
                }
            }
    if (ff_av_out) memcpy(ff_av_out, ff_av, sizeof(double) * bins);
    if (ff_ref_out) memcpy(ff_ref_out, ff_ref, sizeof(double) * bn_ref * bins);
    free(dd_ff); free(dd_ref); free(rr_ff); free(rr_ref); free(ff_av); free(ff_ref);
    return 0;
}

int orc_analytic_3iso(const opt *D, long n, float L, int bins, float dmax, int ptt, int bn_ref,
                      int wrap, double *DDR, double *RRR, double *ff_av_out, double *ff_ref_out)
{
    return analytic_3iso_impl(D, n, L, bins, dmax, ptt, bn_ref, wrap, DDR, RRR, ff_av_out,
                              ff_ref_out, 1);
}

/* ff_av, ff_av_ref and alpha_ref only (no sub-grid refinement). */
int orc_analytic_ff(const opt *D, long n, float L, int bins, float dmax, int ptt, int bn_ref,
                    int wrap, double *ff_av_out, double *ff_ref_out, double *alpha_ref_out)
{
    return analytic_3iso_impl(D, n, L, bins, dmax, ptt, bn_ref, wrap, alpha_ref_out, NULL,
                              ff_av_out, ff_ref_out, -1);
}

/* One partially covered coarse bin of make_histo_analitic, evaluated alone
 * (lets tests check single bins at the reference's full 200^3 sub-grid). */
int orc_analytic_bin(int i, int j, int k, int bins, float dmax, int bn_ref, double alpha_ref,
                     const double *ff_ref, double *rrr, double *ddr)
{
    double dr = dmax / (double)bins;
    double dr_ref = dr / bn_ref, h2 = dr_ref * 0.5;
    double ri = (double)i * dr, rj = (double)j * dr, rk = (double)k * dr;
    long i_ = (long)i * bn_ref, j_ = (long)j * bn_ref, k_ = (long)k * bn_ref;
    double S_av = 0, f_av = 0;
    int con = 0;
    for (int u = 0; u < bn_ref; ++u) {
        double ru = ri + ((double)u * dr_ref);
        for (int v = 0; v < bn_ref; ++v) {
            double rv = rj + ((double)v * dr_ref);
            for (int w = 0; w < bn_ref; ++w) {
                double rw = rk + ((double)w * dr_ref);
                if (all_corners(ru, rv, rw, dr_ref) != 8) continue;
                double c = (ru + h2) * (rv + h2) * (rw + h2);
                S_av += c;
                double f = 1;
                f += ff_ref[i_ + u] / (3 * (ru + h2));
                f += ff_ref[j_ + v] / (3 * (rv + h2));
                f += ff_ref[k_ + w] / (3 * (rw + h2));
                f *= c;
                f_av += f;
                con = 1;
            }
        }
    }
    *rrr = con ? S_av * alpha_ref : 0.0;
    *ddr = con ? f_av * alpha_ref : 0.0;
    return all_corners(ri, rj, rk, dr);
}

int orc_version(void) { return 1; }

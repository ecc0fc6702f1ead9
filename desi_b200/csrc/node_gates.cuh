// Node gates of the reference's periodic 3-point CUDA kernels, for the
// PCF_REF_NODE_GATES mode of the periodic triplet counts.
//
// XXX3iso_BPC / XXY3iso_BPC (cuda/kernels/3isoBPC_k.cuh:191,940) and
// XXX3ani_BPC / XXY3ani_BPC (cuda/kernels/3aniBPC_k.cuh:210,959) give one
// thread an ordered node triple (n1, n2, n3) of the reference's grid (node
// size s = box / partitions, node corner = (float)(int)(x / s) * s,
// main.cu:216, create_grid.cuh:120-135) and run their point loop once per
// "image block" whose gate passes, with that block's flags F2 (node 2 taken
// through its x / y / z image) and F3 (node 3).  All four kernels hold the
// same 64 blocks.  A triangle in range through the images S2 of its side 12
// and S3 of its side 31 is counted once per passing block with (F2, F3) ==
// (S2, S3); with dmax < box/2 the images are the nearest ones.  A gate needs
// edge flags (fa_k: nodes 1 and k within dmax + s of opposite faces along
// axis a) and up to three node-distance tests on pair p in {12, 23, 31}:
//   dd_p + k*L^2 - 2*(sum of |dn_p| over the listed axes)*L <= M,
//   M = (dmax + s*sqrt(3))^2, and k = 0 with no axes meaning dd_p <= M.
// kGateBlocks lists the reference's blocks in source order, as written
// there.  Five of them differ from the nearest-image geometry:
//   * blocks 18-21 (node 2 and node 3 through the same xy / xz / yz / xyz
//     images) test pair 23 through that image where pair 31 is meant, so
//     they pass only on coarse node grids;
//   * block 33 is gated for node 2's y image and node 3's xyz image but
//     counts with node 2's x image: no block counts (S2, S3) = (y, xyz), and
//     (x, xyz) triangles can be counted twice;
//   * block 42 (xy, z) sums |dz23| twice instead of |dx23| + |dz23|;
//   * block 62 (xyz, xz) adds 3 L^2 for a single projected axis.
// Gates evaluate in FP32 with the multiply-adds fused (the reference's
// kernels are built with contraction on).
#pragma once

struct GateTest {
    signed char pair, k, ax[3];
};
struct GateBlock {
    unsigned char f2, f3, a2, a3;  // image flags (bit 0 x, 1 y, 2 z); edge flags required
    GateTest t[3];
};
struct GateGeom {
    float s, L, L2, M, fd, fdn;  // node size, box, box^2, M, dmax + s, box - (dmax + s)
    int P;
};

__constant__ GateBlock kGateBlocks[64] = {
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
// blocks whose flags are (F2, F3), indexed by F2 | F3 << 3; -1: none
__constant__ signed char kGateByImage[64][2] = {
{0, -1}, {8, -1}, {9, -1}, {11, -1}, {10, -1}, {12, -1}, {13, -1}, {14, -1},
{1, -1}, {15, -1}, {28, -1}, {40, -1}, {34, -1}, {46, -1}, {52, -1}, {58, -1},
{2, -1}, {22, -1}, {16, -1}, {41, -1}, {35, -1}, {47, -1}, {53, -1}, {59, -1},
{4, -1}, {24, -1}, {30, -1}, {18, -1}, {36, -1}, {49, -1}, {55, -1}, {61, -1},
{3, -1}, {23, -1}, {29, -1}, {42, -1}, {17, -1}, {48, -1}, {54, -1}, {60, -1},
{5, -1}, {25, -1}, {31, -1}, {43, -1}, {37, -1}, {19, -1}, {56, -1}, {62, -1},
{6, -1}, {26, -1}, {32, -1}, {44, -1}, {38, -1}, {50, -1}, {20, -1}, {63, -1},
{7, -1}, {27, 33}, {-1, -1}, {45, -1}, {39, -1}, {51, -1}, {57, -1}, {21, -1}
};

// The reference's node geometry for box L, dmax and P nodes per side
// (pcf3isoBPC.cuh / pcf3aniBPC.cuh:59-60 for M, main.cu:216 for s).
inline GateGeom gate_geometry(float L, float dmax, int P) {
    GateGeom g;
    g.P = P;
    g.s = L / (float)P;
    g.L = L;
    g.L2 = L * L;
    const float dmn = (float)((double)dmax + (double)g.s * 1.7320508075688772);
    g.M = dmn * dmn;
    g.fd = dmax + g.s;
    g.fdn = L - g.fd;
    return g;
}

// One list entry's node and image: node indices of the reference's grid (9
// bits per axis, partitions <= 512) and the axes along which the entry is
// joined to the anchor through its periodic image (bits 27-29).
__device__ __forceinline__ unsigned gate_pack(const GateGeom &g, float x, float y, float z, unsigned wrap) {
    const int rx = min(max((int)__fdiv_rn(x, g.s), 0), g.P - 1);
    const int ry = min(max((int)__fdiv_rn(y, g.s), 0), g.P - 1);
    const int rz = min(max((int)__fdiv_rn(z, g.s), 0), g.P - 1);
    return (unsigned)rx | ((unsigned)ry << 9) | ((unsigned)rz << 18) | (wrap << 27);
}

struct GateNode {
    float x, y, z;  // node corner
    unsigned wrap;  // image axes relative to the anchor
};

__device__ __forceinline__ GateNode gate_unpack(const GateGeom &g, unsigned v) {
    GateNode n;
    n.x = __fmul_rn((float)(v & 511u), g.s);
    n.y = __fmul_rn((float)((v >> 9) & 511u), g.s);
    n.z = __fmul_rn((float)((v >> 18) & 511u), g.s);
    n.wrap = (v >> 27) & 7u;
    return n;
}

__device__ __forceinline__ float gate_pick(int i, float a, float b, float c) {
    return i == 0 ? a : (i == 1 ? b : c);
}

// Times the reference's blocks count the ordered triangle (1, 2, 3) with node
// corners n1, n2, n3, its sides 12 and 31 in range through the images
// n2.wrap and n3.wrap: 0, 1 or 2.  blocks / by_image: kGateBlocks and
// kGateByImage (copied to shared memory by the caller).
__device__ __forceinline__ int gate_mult(const GateGeom &g, const GateNode &n1, const GateNode &n2,
                                         const GateNode &n3, const GateBlock *blocks,
                                         const signed char (*by_image)[2]) {
    const signed char *blk = by_image[n2.wrap | (n3.wrap << 3)];
    if (blk[0] < 0) return 0;
    // |dn| per pair (12, 23, 31) and axis, and the squared node distances
    const float x12 = fabsf(__fsub_rn(n2.x, n1.x)), y12 = fabsf(__fsub_rn(n2.y, n1.y)),
                z12 = fabsf(__fsub_rn(n2.z, n1.z));
    const float x23 = fabsf(__fsub_rn(n3.x, n2.x)), y23 = fabsf(__fsub_rn(n3.y, n2.y)),
                z23 = fabsf(__fsub_rn(n3.z, n2.z));
    const float x31 = fabsf(__fsub_rn(n1.x, n3.x)), y31 = fabsf(__fsub_rn(n1.y, n3.y)),
                z31 = fabsf(__fsub_rn(n1.z, n3.z));
    const float d12 = __fmaf_rn(z12, z12, __fmaf_rn(y12, y12, __fmul_rn(x12, x12)));
    const float d23 = __fmaf_rn(z23, z23, __fmaf_rn(y23, y23, __fmul_rn(x23, x23)));
    const float d31 = __fmaf_rn(z31, z31, __fmaf_rn(y31, y31, __fmul_rn(x31, x31)));
    unsigned f2 = 0, f3 = 0;
    f2 |= ((n1.x <= g.fd && n2.x >= g.fdn) || (n2.x <= g.fd && n1.x >= g.fdn)) ? 1u : 0u;
    f2 |= ((n1.y <= g.fd && n2.y >= g.fdn) || (n2.y <= g.fd && n1.y >= g.fdn)) ? 2u : 0u;
    f2 |= ((n1.z <= g.fd && n2.z >= g.fdn) || (n2.z <= g.fd && n1.z >= g.fdn)) ? 4u : 0u;
    f3 |= ((n1.x <= g.fd && n3.x >= g.fdn) || (n3.x <= g.fd && n1.x >= g.fdn)) ? 1u : 0u;
    f3 |= ((n1.y <= g.fd && n3.y >= g.fdn) || (n3.y <= g.fd && n1.y >= g.fdn)) ? 2u : 0u;
    f3 |= ((n1.z <= g.fd && n3.z >= g.fdn) || (n3.z <= g.fd && n1.z >= g.fdn)) ? 4u : 0u;
    int m = 0;
    for (int e = 0; e < 2; ++e) {
        const int b = blk[e];
        if (b < 0) break;
        const GateBlock &B = blocks[b];
        if ((f2 & B.a2) != B.a2 || (f3 & B.a3) != B.a3) continue;
        bool ok = true;
        for (int t = 0; t < 3 && ok; ++t) {
            const GateTest &T = B.t[t];
            const int p = T.pair;
            float v = gate_pick(p, d12, d23, d31);
            if (T.ax[0] >= 0) {
                const float dx = gate_pick(p, x12, x23, x31), dy = gate_pick(p, y12, y23, y31),
                            dz = gate_pick(p, z12, z23, z31);
                float sm = gate_pick(T.ax[0], dx, dy, dz);
                if (T.ax[1] >= 0) sm = __fadd_rn(sm, gate_pick(T.ax[1], dx, dy, dz));
                if (T.ax[2] >= 0) sm = __fadd_rn(sm, gate_pick(T.ax[2], dx, dy, dz));
                v = __fmaf_rn((float)T.k, g.L2, v);
                v = __fmaf_rn(-__fmul_rn(2.0f, sm), g.L, v);
            }
            ok = v <= g.M;
        }
        m += ok ? 1 : 0;
    }
    return m;
}

// legacy.cu -- the reference's C++ entry points (include/pcf_legacy.h) on
// top of the C ABI: grid each catalog straight from the caller's device
// arrays, count, and write the reference's files.
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

#include "../../include/pcf_legacy.h"
#include "pcf_internal.cuh"
#include "pcf_io.hpp"

namespace {

// The points of nodes [node_off, node_off + nnodes) of a device DNode array
// form one contiguous range [lo, hi) of the device point array (the nodes'
// start / end index it, cuda/main.cu:300-317).  Only the node table is read
// back; the points stay on the device.
bool node_range(const DNode *dnode, int node_off, int nnodes, int &lo, int &hi) {
    lo = hi = 0;
    if (nnodes <= 0) return true;
    std::vector<DNode> h((size_t)nnodes);
    if (cudaMemcpy(h.data(), dnode + node_off, sizeof(DNode) * nnodes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    lo = h[0].start;
    hi = h[0].end;
    for (const DNode &n : h) {
        lo = std::min(lo, n.start);
        hi = std::max(hi, n.end);
    }
    return true;
}

// Largest coordinate of n device points (all >= 0, so their float bits
// order like unsigned integers).
__global__ void k_max_coord(const PointW3D *__restrict__ p, int n, unsigned *out) {
    unsigned m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, max(__float_as_uint(fmaxf(p[i].x, 0.f)),
                       max(__float_as_uint(fmaxf(p[i].y, 0.f)), __float_as_uint(fmaxf(p[i].z, 0.f)))));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// A device catalog: the point range of its nodes.
struct DevCat {
    const PointW3D *p = nullptr;
    int n = 0;
};

bool device_catalog(const DNode *dnode, const PointW3D *pts, int node_off, int nnodes, DevCat &c) {
    int lo, hi;
    if (!node_range(dnode, node_off, nnodes, lo, hi)) return false;
    c.p = pts + lo;
    c.n = hi - lo;
    return true;
}

// Box of the non-periodic entry points, which receive none: ceil(max + 1)
// over every catalog, as the reference sizes it from its files
// (cuda/create_grid.cuh:75).
bool auto_box(const DevCat &a, const std::vector<DevCat> &r, float &box) {
    unsigned *d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned)) != cudaSuccess) return false;
    cudaMemset(d, 0, sizeof(unsigned));
    auto scan = [&](const DevCat &c) {
        if (c.n > 0) k_max_coord<<<std::min(1024, (c.n + 255) / 256), 256>>>(c.p, c.n, d);
    };
    scan(a);
    for (const DevCat &c : r) scan(c);
    unsigned h = 0;
    const bool ok = cudaMemcpy(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(d);
    float mx;
    memcpy(&mx, &h, sizeof(mx));
    box = (float)std::ceil((double)mx + 1.0);
    return ok;
}

struct Session {
    pcf_ctx *ctx = nullptr;
    bool ok = true;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    Session() {
        int dev = 0;  // the caller's current device, which holds its arrays
        if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
        check(pcf_ctx_create(dev, &ctx), "pcf_ctx_create");
    }
    ~Session() {
        if (ctx) pcf_ctx_destroy(ctx);
        if (ok)
            std::cout << "Spent "
                      << std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count()
                      << " miliseconds to compute and save all the histograms." << std::endl;
    }
    bool check(pcf_status s, const char *what) {
        if (s != PCF_OK && ok) {
            std::cout << what << ": " << pcf_status_string(s) << std::endl;
            ok = false;
        }
        return ok;
    }
};

// 2-point family: DD, and RR / DR per random file.
void two_point(std::string *names, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
               int *nR, int *accR, int nrand, int bn, float box, float dmax, bool ani, bool bpc) {
    Session S;
    DevCat D;
    std::vector<DevCat> R((size_t)std::max(nrand, 0));
    if (!device_catalog(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "node table"); return; }
    for (int i = 0; i < nrand; ++i)
        if (!device_catalog(dR, pR, accR[i], nR[i], R[i])) { S.check(PCF_ERR_CUDA, "node table"); return; }
    if (!bpc && !auto_box(D, R, box)) { S.check(PCF_ERR_CUDA, "box"); return; }
    const int kind = ani ? PCF_ANI : PCF_ISO;
    const uint32_t f = bpc ? (PCF_BPC | (ani ? 0u : (uint32_t)PCF_DS_EXACT)) : 0u;
    const std::string tag = std::string(ani ? "ani_" : "iso_") + (bpc ? "BPC_" : "");
    std::vector<double> h(ani ? (size_t)bn * bn : (size_t)bn);
    auto save = [&](const std::string &n) { ani ? pcfio::save2d(n, bn, h.data()) : pcfio::save1d(n, bn, h.data()); };
    pcf_grid *gD = nullptr;
    auto pts = [](const DevCat &c) { return reinterpret_cast<const pcf_point *>(c.p); };
    if (!S.check(pcf_grid_build(S.ctx, pts(D), D.n, box, 0, &gD), "grid")) return;
    if (S.check(pcf_count_pairs(S.ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr), "DD"))
        save("DD" + tag + names[0]);
    for (int i = 0; i < nrand && S.ok; ++i) {
        pcf_grid *gR = nullptr;
        if (!S.check(pcf_grid_build(S.ctx, pts(R[i]), R[i].n, box, 0, &gR), "grid")) break;
        if (S.check(pcf_count_pairs(S.ctx, kind, gR, nullptr, bn, dmax, f, h.data(), nullptr), "RR"))
            save("RR" + tag + names[i + 1]);
        if (S.check(pcf_count_pairs(S.ctx, kind, gD, gR, bn, dmax, f, h.data(), nullptr), "DR"))
            save("DR" + tag + names[i + 1]);
        pcf_grid_free(S.ctx, gR);
    }
    pcf_grid_free(S.ctx, gD);
}

// 3-point family: DDD, and RRR / DDR / DRR per random file.  Periodic:
// counted as the reference's kernels count on the caller's node grid
// (PCF_REF_NODE_GATES, partitions = box / size_node).
void three_point(std::string *names, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *accR, int nrand, int bn, float size_node, float box, float dmax, bool ani,
                 bool bpc) {
    Session S;
    DevCat D;
    std::vector<DevCat> R((size_t)std::max(nrand, 0));
    if (!device_catalog(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "node table"); return; }
    for (int i = 0; i < nrand; ++i)
        if (!device_catalog(dR, pR, accR[i], nR[i], R[i])) { S.check(PCF_ERR_CUDA, "node table"); return; }
    if (!bpc && !auto_box(D, R, box)) { S.check(PCF_ERR_CUDA, "box"); return; }
    const int kind = ani ? PCF_ANI : PCF_ISO;
    const int parts = bpc && size_node > 0.f ? (int)std::lround(box / size_node) : 0;
    const uint32_t f = bpc ? (PCF_BPC | (parts > 0 ? (uint32_t)PCF_REF_NODE_GATES : 0u)) : 0u;
    const std::string tag = std::string(ani ? "ani_" : "iso_") + (bpc ? "BPC_" : "");
    const size_t nb = ani ? (size_t)bn * bn * bn * bn * bn : (size_t)bn * bn * bn;
    std::vector<double> h(nb);
    auto save = [&](const std::string &n) { ani ? pcfio::save5d(n, bn, h.data()) : pcfio::save3d(n, bn, h.data()); };
    pcf_grid *gD = nullptr;
    auto pts = [](const DevCat &c) { return reinterpret_cast<const pcf_point *>(c.p); };
    if (!S.check(pcf_grid_build(S.ctx, pts(D), D.n, box, parts, &gD), "grid")) return;
    if (S.check(pcf_count_triplets(S.ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr), "DDD"))
        save("DDD" + tag + names[0]);
    for (int i = 0; i < nrand && S.ok; ++i) {
        pcf_grid *gR = nullptr;
        if (!S.check(pcf_grid_build(S.ctx, pts(R[i]), R[i].n, box, parts, &gR), "grid")) break;
        if (S.check(pcf_count_triplets(S.ctx, kind, gR, nullptr, bn, dmax, f, h.data(), nullptr), "RRR"))
            save("RRR" + tag + names[i + 1]);
        if (S.check(pcf_count_triplets(S.ctx, kind, gD, gR, bn, dmax, f, h.data(), nullptr), "DDR"))
            save("DDR" + tag + names[i + 1]);
        if (S.check(pcf_count_triplets(S.ctx, kind, gR, gD, bn, dmax, f, h.data(), nullptr), "DRR"))
            save("DRR" + tag + names[i + 1]);
        pcf_grid_free(S.ctx, gR);
    }
    pcf_grid_free(S.ctx, gD);
}

}  // namespace

void pcf_2iso(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR, int *nR,
              int *aR, int nr, int bn, float, float dmax) {
    two_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, dmax, false, false);
}
void pcf_2ani(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR, int *nR,
              int *aR, int nr, int bn, float, float dmax) {
    two_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, dmax, true, false);
}
void pcf_2iso_BPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                  int *nR, int *aR, int nr, int bn, float, float box, float dmax) {
    two_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, box, dmax, false, true);
}
void pcf_2aniBPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *aR, int nr, int bn, float, float box, float dmax) {
    two_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, box, dmax, true, true);
}
void pcf_3iso(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR, int *nR,
              int *aR, int nr, int bn, float, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, 0.f, dmax, false, false);
}
void pcf_3isoBPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *aR, int nr, int bn, float size_node, float box, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, size_node, box, dmax, false, true);
}
void pcf_3ani(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR, int *nR,
              int *aR, int nr, int bn, float, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, 0.f, dmax, true, false);
}
void pcf_3aniBPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *aR, int nr, int bn, float size_node, float box, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, size_node, box, dmax, true, true);
}

void pcf_2iso_BPCanalytic(std::string name, DNode *dD, PointW3D *pD, int nD, int bn, int np, float,
                          float box, float dmax) {
    Session S;
    DevCat D;
    if (!device_catalog(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "node table"); return; }
    pcf_grid *g = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, reinterpret_cast<const pcf_point *>(D.p), D.n, box, 0, &g),
                 "grid"))
        return;
    std::vector<double> h((size_t)bn);
    if (S.check(pcf_count_pairs(S.ctx, PCF_ISO, g, nullptr, bn, dmax, PCF_BPC | PCF_DS_EXACT, h.data(), nullptr), "DD"))
        pcfio::save1d("DDiso_BPCanalytic_" + name, bn, h.data());
    if (S.check(pcf_analytic_rr(S.ctx, bn, np, box, dmax, 1, h.data()), "RR")) {
        pcfio::save1d("RRiso_BPCanalytic_" + name, bn, h.data());
        pcfio::save1d("DRiso_BPCanalytic_" + name, bn, h.data());
    }
    pcf_grid_free(S.ctx, g);
}

void pcf_3isoBPC_analytic(std::string name, DNode *dD, PointW3D *pD, int nD, int bn, int, float,
                          float box, float dmax) {
    Session S;
    DevCat D;
    if (!device_catalog(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "node table"); return; }
    pcf_grid *g = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, reinterpret_cast<const pcf_point *>(D.p), D.n, box, 0, &g),
                 "grid"))
        return;
    const size_t n3 = (size_t)bn * bn * bn;
    std::vector<double> ddd(n3), ddr(n3), rrr(n3);
    if (S.check(pcf_analytic_3iso(S.ctx, g, bn, dmax, 0, 0, 1, ddd.data(), ddr.data(), rrr.data(), nullptr),
                "analytic")) {
        pcfio::save3d("DDDiso_BPCanalytic_" + name, bn, ddd.data());
        pcfio::save3d("DDRiso_BPCanalytic_" + name, bn, ddr.data());
        pcfio::save3d("DRRiso_BPCanalytic_" + name, bn, ddr.data());
        pcfio::save3d("RRRiso_BPCanalytic_" + name, bn, rrr.data());
    }
    pcf_grid_free(S.ctx, g);
}

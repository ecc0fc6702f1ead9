// legacy.cu -- the reference's C++ entry points (include/pcf_legacy.h) on
// top of the C ABI: gather each catalog from the caller's device arrays,
// grid it, count, and write the reference's files.
#include <chrono>
#include <iostream>
#include <vector>

#include "../../include/pcf_legacy.h"
#include "pcf_internal.cuh"
#include "pcf_io.hpp"

namespace {

// Points of the nodes [node_off, node_off + nnodes) of a device DNode array
// (their start/end index the device point array), copied to the host.
bool gather(const DNode *dnode, const PointW3D *pts, int node_off, int nnodes,
            std::vector<pcf_point> &out) {
    out.clear();
    if (nnodes <= 0) return true;
    std::vector<DNode> h((size_t)nnodes);
    if (cudaMemcpy(h.data(), dnode + node_off, sizeof(DNode) * nnodes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    int lo = h[0].start, hi = h[0].end;
    for (const DNode &n : h) {
        lo = std::min(lo, n.start);
        hi = std::max(hi, n.end);
    }
    out.resize((size_t)(hi - lo));
    return cudaMemcpy(out.data(), pts + lo, sizeof(PointW3D) * (hi - lo), cudaMemcpyDeviceToHost) ==
           cudaSuccess;
}

float auto_box(const std::vector<pcf_point> &a, const std::vector<std::vector<pcf_point>> &r) {
    double mx = 0;
    auto scan = [&](const std::vector<pcf_point> &v) {
        for (const pcf_point &p : v) mx = std::max(mx, (double)std::max(p.x, std::max(p.y, p.z)));
    };
    scan(a);
    for (auto &v : r) scan(v);
    return (float)std::ceil(mx + 1);
}

struct Session {
    pcf_ctx *ctx = nullptr;
    bool ok = true;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    Session() { check(pcf_ctx_create(0, &ctx), "pcf_ctx_create"); }
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
    std::vector<pcf_point> D;
    std::vector<std::vector<pcf_point>> R((size_t)std::max(nrand, 0));
    if (!gather(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "gather"); return; }
    for (int i = 0; i < nrand; ++i)
        if (!gather(dR, pR, accR[i], nR[i], R[i])) { S.check(PCF_ERR_CUDA, "gather"); return; }
    if (!bpc) box = auto_box(D, R);
    const int kind = ani ? PCF_ANI : PCF_ISO;
    const uint32_t f = bpc ? (PCF_BPC | (ani ? 0u : (uint32_t)PCF_DS_EXACT)) : 0u;
    const std::string tag = std::string(ani ? "ani_" : "iso_") + (bpc ? "BPC_" : "");
    std::vector<double> h(ani ? (size_t)bn * bn : (size_t)bn);
    auto save = [&](const std::string &n) { ani ? pcfio::save2d(n, bn, h.data()) : pcfio::save1d(n, bn, h.data()); };
    pcf_grid *gD = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, D.data(), (int64_t)D.size(), box, 0, &gD), "grid")) return;
    if (S.check(pcf_count_pairs(S.ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr), "DD"))
        save("DD" + tag + names[0]);
    for (int i = 0; i < nrand && S.ok; ++i) {
        pcf_grid *gR = nullptr;
        if (!S.check(pcf_grid_build(S.ctx, R[i].data(), (int64_t)R[i].size(), box, 0, &gR), "grid")) break;
        if (S.check(pcf_count_pairs(S.ctx, kind, gR, nullptr, bn, dmax, f, h.data(), nullptr), "RR"))
            save("RR" + tag + names[i + 1]);
        if (S.check(pcf_count_pairs(S.ctx, kind, gD, gR, bn, dmax, f, h.data(), nullptr), "DR"))
            save("DR" + tag + names[i + 1]);
        pcf_grid_free(S.ctx, gR);
    }
    pcf_grid_free(S.ctx, gD);
}

// 3-point family: DDD, and RRR / DDR / DRR per random file.
void three_point(std::string *names, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *accR, int nrand, int bn, float box, float dmax, bool ani, bool bpc) {
    Session S;
    std::vector<pcf_point> D;
    std::vector<std::vector<pcf_point>> R((size_t)std::max(nrand, 0));
    if (!gather(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "gather"); return; }
    for (int i = 0; i < nrand; ++i)
        if (!gather(dR, pR, accR[i], nR[i], R[i])) { S.check(PCF_ERR_CUDA, "gather"); return; }
    if (!bpc) box = auto_box(D, R);
    const int kind = ani ? PCF_ANI : PCF_ISO;
    const uint32_t f = bpc ? PCF_BPC : 0u;
    const std::string tag = std::string(ani ? "ani_" : "iso_") + (bpc ? "BPC_" : "");
    const size_t nb = ani ? (size_t)bn * bn * bn * bn * bn : (size_t)bn * bn * bn;
    std::vector<double> h(nb);
    auto save = [&](const std::string &n) { ani ? pcfio::save5d(n, bn, h.data()) : pcfio::save3d(n, bn, h.data()); };
    pcf_grid *gD = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, D.data(), (int64_t)D.size(), box, 0, &gD), "grid")) return;
    if (S.check(pcf_count_triplets(S.ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr), "DDD"))
        save("DDD" + tag + names[0]);
    for (int i = 0; i < nrand && S.ok; ++i) {
        pcf_grid *gR = nullptr;
        if (!S.check(pcf_grid_build(S.ctx, R[i].data(), (int64_t)R[i].size(), box, 0, &gR), "grid")) break;
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
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, dmax, false, false);
}
void pcf_3isoBPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *aR, int nr, int bn, float, float box, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, box, dmax, false, true);
}
void pcf_3ani(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR, int *nR,
              int *aR, int nr, int bn, float, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, 0.f, dmax, true, false);
}
void pcf_3aniBPC(std::string *n, DNode *dD, PointW3D *pD, int nD, DNode *dR, PointW3D *pR,
                 int *nR, int *aR, int nr, int bn, float, float box, float dmax) {
    three_point(n, dD, pD, nD, dR, pR, nR, aR, nr, bn, box, dmax, true, true);
}

void pcf_2iso_BPCanalytic(std::string name, DNode *dD, PointW3D *pD, int nD, int bn, int np, float,
                          float box, float dmax) {
    Session S;
    std::vector<pcf_point> D;
    if (!gather(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "gather"); return; }
    pcf_grid *g = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, D.data(), (int64_t)D.size(), box, 0, &g), "grid")) return;
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
    std::vector<pcf_point> D;
    if (!gather(dD, pD, 0, nD, D)) { S.check(PCF_ERR_CUDA, "gather"); return; }
    pcf_grid *g = nullptr;
    if (!S.check(pcf_grid_build(S.ctx, D.data(), (int64_t)D.size(), box, 0, &g), "grid")) return;
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

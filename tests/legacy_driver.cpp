// Test driver: calls the reference-signature entry points of libpcf.so the
// way the reference's main.cu does (device DNode + cell-ordered PointW3D
// arrays), one node per catalog.  Usage: legacy_driver <kind> <data> <rand> n bins dmax box
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "pcf_legacy.h"

static std::vector<PointW3D> read(const char *path, int n) {
    std::ifstream f(path);
    std::vector<PointW3D> v((size_t)n);
    for (auto &p : v) f >> p.x >> p.y >> p.z >> p.w;
    return v;
}

int main(int argc, char **argv) {
    if (argc < 8) return 2;
    std::string kind = argv[1];
    int n = atoi(argv[4]), bn = atoi(argv[5]);
    float dmax = (float)atof(argv[6]), box = (float)atof(argv[7]);
    auto D = read(argv[2], n);
    auto R = read(argv[3], n);
    DNode hD{{0, 0, 0}, n, 0, n}, hR{{0, 0, 0}, n, 0, n};
    DNode *dD, *dR;
    PointW3D *pD, *pR;
    cudaMalloc(&dD, sizeof(DNode));
    cudaMalloc(&dR, sizeof(DNode));
    cudaMalloc(&pD, sizeof(PointW3D) * n);
    cudaMalloc(&pR, sizeof(PointW3D) * n);
    cudaMemcpy(dD, &hD, sizeof(DNode), cudaMemcpyHostToDevice);
    cudaMemcpy(dR, &hR, sizeof(DNode), cudaMemcpyHostToDevice);
    cudaMemcpy(pD, D.data(), sizeof(PointW3D) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(pR, R.data(), sizeof(PointW3D) * n, cudaMemcpyHostToDevice);
    std::string names[2] = {"data", "rand"};
    int nR = 1, acc = 0;
    float sn = box / 10;
    if (kind == "2iso") pcf_2iso(names, dD, pD, 1, dR, pR, &nR, &acc, 1, bn, sn, dmax);
    else if (kind == "2aniBPC") pcf_2aniBPC(names, dD, pD, 1, dR, pR, &nR, &acc, 1, bn, sn, box, dmax);
    else if (kind == "3iso") pcf_3iso(names, dD, pD, 1, dR, pR, &nR, &acc, 1, bn, sn, dmax);
    else if (kind == "3isoBPC") pcf_3isoBPC(names, dD, pD, 1, dR, pR, &nR, &acc, 1, bn, sn, box, dmax);
    else if (kind == "2isoBPCa") pcf_2iso_BPCanalytic("data", dD, pD, 1, bn, n, sn, box, dmax);
    else return 3;
    return 0;
}

// ref_harness.cpp -- drives the reference's own CPU/OpenMP engines in place.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY (the shipped library never loads it).
// This file is ours; it #includes one reference engine header, chosen at
// compile time, straight from the reference tree (see oracle/Makefile):
//   -DREF_ENGINE_2ISO  cpp/2PCFisotropic/normal/2PCF.h      NODE2P (1-D)
//   -DREF_ENGINE_2ISO_BPC cpp/2PCFisotropic/BPC/2PCF.h      NODE2P (1-D)
//   -DREF_ENGINE_2ANI  cpp/2PCFanisotropic/normal/2PCFani.h NODE2P (2-D)
//   -DREF_ENGINE_2ANI_BPC cpp/2PCFanisotropic/BPC/2PCFani.h NODE2P (2-D)
// The engines hard-code `#pragma omp parallel num_threads(2)`
// (e.g. cpp/2PCFisotropic/normal/2PCF.h:163); OpenMP directives are
// macro-expanded, so the function-like macro below routes that clause to a
// thread count the caller sets (2 reproduces the engines as shipped).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <omp.h>

static int g_ref_threads = 2;
#define num_threads(x) num_threads(g_ref_threads)

#if defined(REF_ENGINE_2ISO) || defined(REF_ENGINE_2ISO_BPC)
#include "2PCF.h"
#define REF_2D 0
#elif defined(REF_ENGINE_2ANI) || defined(REF_ENGINE_2ANI_BPC)
#include "2PCFani.h"
#define REF_2D 1
#else
#error "select an engine"
#endif

namespace {

// Node grids sized the way the engines index them:
// partitions = (int)((size_box/size_node)+1)  (2PCF.h:109).
struct Grid {
    int parts;
    Node ***n;
    explicit Grid(int p) : parts(p) {
        n = new Node **[p];
        for (int i = 0; i < p; ++i) {
            n[i] = new Node *[p];
            for (int j = 0; j < p; ++j) n[i][j] = new Node[p];
        }
    }
    ~Grid() {
        for (int i = 0; i < parts; ++i) {
            for (int j = 0; j < parts; ++j) {
                for (int k = 0; k < parts; ++k) delete[] n[i][j][k].elements;
                delete[] n[i][j];
            }
            delete[] n[i];
        }
        delete[] n;
    }
};

PointW3D *copy_pts(const float *p, int n) {
    PointW3D *a = new PointW3D[n];
    std::memcpy(a, p, sizeof(PointW3D) * (size_t)n);
    return a;
}

int run(const float *D, const float *R, int n, float L, float size_node, float dmax, int bins,
        double *out, bool cross) {
    int parts = (int)((L / size_node) + 1);
    Grid gD(parts), gR(parts);
    PointW3D *dD = copy_pts(D, n);
    PointW3D *dR = copy_pts(R ? R : D, n);
    std::streambuf *old = std::cout.rdbuf(nullptr);  // engines print progress
    NODE2P eng(bins, n, L, size_node, dmax, dD, gD.n, dR, gR.n);
#if REF_2D
    double **h = new double *[bins];
    for (int i = 0; i < bins; ++i) {
        h[i] = new double[bins];
        for (int j = 0; j < bins; ++j) h[i][j] = 0.0;
    }
    if (cross) eng.make_histoXY(h, eng.meshData(), eng.meshRand());
    else eng.make_histoXX(h, eng.meshData());
    for (int i = 0; i < bins; ++i) {
        for (int j = 0; j < bins; ++j) out[i * bins + j] = h[i][j];
        delete[] h[i];
    }
    delete[] h;
#else
    for (int i = 0; i < bins; ++i) out[i] = 0.0;
    if (cross) eng.make_histoXY(out, eng.meshData(), eng.meshRand());
    else eng.make_histoXX(out, eng.meshData());
#endif
    std::cout.rdbuf(old);
    delete[] dD;
    delete[] dR;
    return 0;
}

}  // namespace

extern "C" {

void ref_set_threads(int t) { g_ref_threads = t > 0 ? t : 1; }
int ref_get_threads(void) { return g_ref_threads; }
int ref_is_2d(void) { return REF_2D; }

// XX over one catalog of n points (DD or RR).
int ref_xx(const float *pts, int n, float L, float size_node, float dmax, int bins, double *out) {
    return run(pts, nullptr, n, L, size_node, dmax, bins, out, false);
}

// XY between two catalogs of n points each (DR).
int ref_xy(const float *D, const float *R, int n, float L, float size_node, float dmax, int bins,
           double *out) {
    return run(D, R, n, L, size_node, dmax, bins, out, true);
}
}

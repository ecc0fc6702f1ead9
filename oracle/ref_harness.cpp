// ref_harness.cpp -- drives the reference's own CPU/OpenMP engines in place.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY (the shipped library never loads it).
// This file is ours; it #includes one reference engine header, chosen at
// compile time, straight from the reference tree (see oracle/Makefile):
//   -DREF_ENGINE_2ISO  cpp/2PCFisotropic/normal/2PCF.h      NODE2P (1-D)
//   -DREF_ENGINE_2ISO_BPC cpp/2PCFisotropic/BPC/2PCF.h      NODE2P (1-D)
//   -DREF_ENGINE_2ANI  cpp/2PCFanisotropic/normal/2PCFani.h NODE2P (2-D)
//   -DREF_ENGINE_2ANI_BPC cpp/2PCFanisotropic/BPC/2PCFani.h NODE2P (2-D)
//   -DREF_ENGINE_2ISO_ANALYTIC cpp/2PCFisotropic/BPC_analitic/2PCF.h
//                      NODE2P: periodic DD plus the analytic RR (2PCF.h:329-360)
//   -DREF_ENGINE_3ISO_BPC cpp/3PCFisotropic/BPC/3PCFiso.h   NODE3P: periodic
//                      DDD (make_histoXXX, :218) and the analytic path's
//                      averaged correction factors (make_histo_analitic, :1484)
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
#include <new>
#include <string>
#include <vector>
#include <omp.h>
#include <unistd.h>

static int g_ref_threads = 2;
#define num_threads(x) num_threads(g_ref_threads)

#if defined(REF_ENGINE_2ISO) || defined(REF_ENGINE_2ISO_BPC) || defined(REF_ENGINE_2ISO_ANALYTIC)
#include "2PCF.h"
#define REF_2D 0
#elif defined(REF_ENGINE_2ANI) || defined(REF_ENGINE_2ANI_BPC)
#include "2PCFani.h"
#define REF_2D 1
#elif defined(REF_ENGINE_3ISO_BPC)
#include "3PCFiso.h"
#define REF_3P 1
#else
#error "select an engine"
#endif

namespace {

// Node grids sized the way the engines index them: partitions =
// (int)((size_box/size_node)+1) for the 2-point engines (2PCF.h:109),
// ceil(size_box/size_node) for NODE3P (3PCFiso.h:83).
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

struct Quiet {  // the engines print progress on stdout
    std::streambuf *old;
    Quiet() : old(std::cout.rdbuf(nullptr)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

#ifndef REF_3P
PointW3D *copy_pts(const float *p, int n) {
    PointW3D *a = new PointW3D[n];
    for (int i = 0; i < n; ++i) {
        a[i].x = p[4 * i];
        a[i].y = p[4 * i + 1];
        a[i].z = p[4 * i + 2];
        a[i].w = p[4 * i + 3];
    }
    return a;
}
#endif

#if !defined(REF_3P) && !defined(REF_ENGINE_2ISO_ANALYTIC)
int run(const float *D, const float *R, int n, float L, float size_node, float dmax, int bins,
        double *out, bool cross) {
    int parts = (int)((L / size_node) + 1);
    Grid gD(parts), gR(parts);
    PointW3D *dD = copy_pts(D, n);
    PointW3D *dR = copy_pts(R ? R : D, n);
    {
        Quiet q;
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
    }
    delete[] dD;
    delete[] dR;
    return 0;
}
#endif

#ifdef REF_3P
// Points as the engine's main() prepares them: border tags fx/fy/fz of
// cpp/3PCFisotropic/BPC/main.cpp:162-176 (+1 within d_max of the low face,
// -1 beyond L - d_max, else 0).
PointW3D *tagged_pts(const float *p, int n, float L, float dmax) {
    PointW3D *a = new PointW3D[n];
    const float front = L - dmax;
    auto tag = [&](float v) -> short { return v < dmax ? 1 : (v > front ? -1 : 0); };
    for (int i = 0; i < n; ++i) {
        a[i].x = p[4 * i];
        a[i].y = p[4 * i + 1];
        a[i].z = p[4 * i + 2];
        a[i].w = p[4 * i + 3];
        a[i].fx = tag(a[i].x);
        a[i].fy = tag(a[i].y);
        a[i].fz = tag(a[i].z);
    }
    return a;
}

double ***new3(int b) {
    double ***h = new double **[b];
    for (int i = 0; i < b; ++i) {
        h[i] = new double *[b];
        for (int j = 0; j < b; ++j) {
            h[i][j] = new double[b];
            for (int k = 0; k < b; ++k) h[i][j][k] = 0.0;
        }
    }
    return h;
}

void free3(double ***h, int b) {
    for (int i = 0; i < b; ++i) {
        for (int j = 0; j < b; ++j) delete[] h[i][j];
        delete[] h[i];
    }
    delete[] h;
}

int read_column(const std::string &path, double *out, int n) {
    std::ifstream f(path.c_str());
    if (!f) return -1;
    for (int i = 0; i < n; ++i)
        if (!(f >> out[i])) return -1;
    return 0;
}
#endif

}  // namespace

extern "C" {

void ref_set_threads(int t) { g_ref_threads = t > 0 ? t : 1; }
int ref_get_threads(void) { return g_ref_threads; }

#if !defined(REF_3P) && !defined(REF_ENGINE_2ISO_ANALYTIC)
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
#endif

#ifdef REF_ENGINE_2ISO_ANALYTIC
int ref_is_2d(void) { return 0; }

// Periodic DD (out_dd) and the analytic RR (out_rr) of one catalog.
int ref_dd_rr_analytic(const float *pts, int n, float L, float size_node, float dmax, int bins,
                       double *out_dd, double *out_rr) {
    int parts = (int)((L / size_node) + 1);
    Grid g(parts);
    PointW3D *d = copy_pts(pts, n);
    for (int i = 0; i < bins; ++i) out_dd[i] = out_rr[i] = 0.0;
    {
        Quiet q;
        NODE2P eng(bins, n, L, size_node, dmax, d, g.n);
        eng.make_histoXX(out_dd, out_rr, eng.meshData());
    }
    delete[] d;
    return 0;
}
#endif

#ifdef REF_3P
// Periodic DDD (bins^3, [i][j][k] flattened) of one catalog.
int ref3_xxx(const float *pts, int n, float L, float size_node, float dmax, int bins, double *out) {
    const int parts = (int)std::ceil(L / size_node);
    Grid g(parts);
    PointW3D *d = tagged_pts(pts, n, L, dmax);
    double ***h = new3(bins);
    {
        Quiet q;
        NODE3P eng(bins, n, L, size_node, dmax, d, g.n);
        eng.make_histoXXX(h, eng.meshData());
    }
    for (int i = 0; i < bins; ++i)
        for (int j = 0; j < bins; ++j)
            for (int k = 0; k < bins; ++k) out[((size_t)i * bins + j) * bins + k] = h[i][j][k];
    free3(h, bins);
    delete[] d;
    return 0;
}

// The analytic path's averaged correction factors: ff_av (bins) and
// ff_av_ref (200 * bins), and the fine DD behind ff_av_ref (100 * 200 * bins
// bins; dd_ref may be NULL).  The engine writes them as text into the
// working directory, so the call runs inside `workdir`.
int ref3_analytic_ff(const float *pts, int n, float L, float size_node, float dmax, int bins,
                     const char *workdir, double *ff_av, double *ff_av_ref, double *dd_ref) {
    char old[4096];
    if (!getcwd(old, sizeof(old))) return -1;
    if (chdir(workdir) != 0) return -1;
    const int parts = (int)std::ceil(L / size_node);
    int rc = 0;
    {
        Grid g(parts);
        PointW3D *d = tagged_pts(pts, n, L, dmax);
        double ***xxx = new3(bins), ***xxy = new3(bins);
        {
            Quiet q;
            // NODE3P never sets its member ll (size_box^2, 3PCFiso.h:52), which
            // the fine DD's image passes read to prune node pairs
            // (3PCFiso.h:1925-2039): built on the stack it holds whatever the
            // stack held, and the fine DD changes from call to call.  Built in
            // zero-filled storage, ll = 0 and the prune keeps every node pair,
            // so each pair is decided by its own distance test.
            alignas(NODE3P) unsigned char buf[sizeof(NODE3P)];
            memset(buf, 0, sizeof(buf));
            NODE3P *eng = new (buf) NODE3P(bins, n, L, size_node, dmax, d, g.n);
            eng->make_histo_analitic(xxy, xxx, eng->meshData());
            eng->~NODE3P();
        }
        free3(xxx, bins);
        free3(xxy, bins);
        delete[] d;
        rc = read_column("ff_av.dat", ff_av, bins);
        if (rc == 0) rc = read_column("ff_av_ref.dat", ff_av_ref, 200 * bins);
        if (rc == 0 && dd_ref) rc = read_column("DD.dat", dd_ref, 100 * 200 * bins);
    }
    if (chdir(old) != 0) return -1;
    return rc;
}
#endif
}

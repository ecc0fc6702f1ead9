// Host build of the reference's pair and triplet CUDA kernels -- test
// infrastructure only (the checker; nothing in the library links it).
//
// The kernel headers cuda/kernels/2iso_k.cuh, 2isoBPC_k.cuh, 2ani_k.cuh,
// 2aniBPC_k.cuh, 3iso_k.cuh, 3isoBPC_k.cuh, 3ani_k.cuh and 3aniBPC_k.cuh are
// included unmodified from the reference tree (-I<ref>/cuda) and compiled by
// the host compiler: __global__ / __device__ expand to nothing, blockIdx is a
// thread-local that the loops below set, and the double atomicAdd becomes an
// OpenMP atomic add.  Each kernel body then runs once per node pair / triple
// with blockDim 1, the same ones the reference's launches cover
// (pcf2iso.cuh:95-103, pcf2isoBPC.cuh:100-108, pcf2ani.cuh:89-97,
// pcf2aniBPC.cuh:89-97, pcf3iso.cuh:102-114, pcf3isoBPC.cuh:102-114,
// pcf3ani.cuh:102-114, pcf3aniBPC.cuh:102-114; one random file, node and bin
// offsets 0).  Nodes are built as main.cu:216-329 builds them: size_node =
// box / partitions, make_nodos (create_grid.cuh:104-139), then the non-empty
// nodes in (row, col, mom) order with their points contiguous.
//
// Two cross kernels are not run: XY2ani (2ani_k.cuh:70) reads the weight of
// its R point from the D array (2ani_k.cuh:128), past its end whenever R is
// the longer catalog, and XY2ani_BPC (2aniBPC_k.cuh:345) multiplies pairs
// that need no periodic image by w1 before any assignment (declared :372,
// read :410, first set :429), so its DR is undefined.  Their slots of the
// output are NaN.
//
// The arithmetic is the host's FP32 / FP64 without FMA contraction (the
// Makefile passes -ffp-contract=off); the device build fuses some
// multiply-adds, so the two agree bit for bit wherever the FP32 sums are
// exact (integer lattices), which is how the fixtures that pin this build to
// the B200 run of the same kernels are made.  Threads add in any order:
// sums are exact with unit weights (the 3-point kernels multiply every third
// point's weight into a running product, so only unit weights are meaningful
// there).
//
//   int ref2_hist(int ani, int bpc, const float *D, int nD, const float *R,
//                 int nR, int bins, float dmax, int partitions, float box,
//                 double *out)
//     out: DD, RR, DR, each bins (iso) or bins^2 (ani) doubles.
//   int ref3_hist(...same arguments...)
//     out: DDD, RRR, DDR, DRR, each bins^3 (iso) or bins^5 (ani) doubles;
//     with nR == 0 only DDD.
//   D, R: float32 x y z w rows; outputs are overwritten.
#include <math.h>
#include <string.h>

#include <vector>

#define __global__
#define __device__
namespace {
struct Dim3H {
    unsigned x, y, z;
};
thread_local Dim3H blockIdx, threadIdx, blockDim;
inline double atomicAdd(double *a, double v) {
#pragma omp atomic
    *a += v;
    return 0.0;
}
}  // namespace

#include "create_grid.cuh"
#include "kernels/2aniBPC_k.cuh"
#include "kernels/2ani_k.cuh"
#include "kernels/2isoBPC_k.cuh"
#include "kernels/2iso_k.cuh"
#include "kernels/3aniBPC_k.cuh"
#include "kernels/3ani_k.cuh"
#include "kernels/3isoBPC_k.cuh"
#include "kernels/3iso_k.cuh"

namespace {

struct Flat {
    std::vector<DNode> nodes;
    std::vector<PointW3D> pts;
};

Flat flatten(const float *xyzw, int np, int partitions, float size_node) {
    std::vector<PointW3D> dat((size_t)np);
    memcpy(dat.data(), xyzw, sizeof(PointW3D) * (size_t)np);
    Node ***nod = new Node **[partitions];
    for (int i = 0; i < partitions; ++i) {
        nod[i] = new Node *[partitions];
        for (int j = 0; j < partitions; ++j) nod[i][j] = new Node[partitions];
    }
    make_nodos(nod, dat.data(), partitions, size_node, np);
    Flat f;
    for (int r = 0; r < partitions; ++r)
        for (int c = 0; c < partitions; ++c)
            for (int m = 0; m < partitions; ++m) {
                const Node &nd = nod[r][c][m];
                if (nd.len <= 0) continue;
                DNode d;
                d.nodepos = nd.nodepos;
                d.len = nd.len;
                d.start = (int)f.pts.size();
                for (int k = 0; k < nd.len; ++k) f.pts.push_back(nd.elements[k]);
                d.end = (int)f.pts.size();
                f.nodes.push_back(d);
            }
    for (int i = 0; i < partitions; ++i) {
        for (int j = 0; j < partitions; ++j) {
            for (int k = 0; k < partitions; ++k) delete[] nod[i][j][k].elements;
            delete[] nod[i][j];
        }
        delete[] nod[i];
    }
    delete[] nod;
    return f;
}

// Runs body() once per node pair (a, b), a < na, b < nb.
template <class F>
void each_pair(int na, int nb, F body) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int a = 0; a < na; ++a) {
        blockDim = {1, 1, 1};
        threadIdx = {0, 0, 0};
        for (int b = 0; b < nb; ++b) {
            blockIdx = {(unsigned)a, (unsigned)b, 0u};
            body();
        }
    }
}

// -2 when a coordinate lies outside the node array (make_nodos does not
// clamp), else 0.
int check_nodes(const float *P, int n, int partitions, float size_node) {
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            if (!(P[4 * i + a] >= 0.f) || (int)(P[4 * i + a] / size_node) >= partitions) return -2;
    return 0;
}

// Runs body() once per node triple (a, b, c), a < na, b < nb, c < nc.
template <class F>
void each_triple(int na, int nb, int nc, F body) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int a = 0; a < na; ++a) {
        blockDim = {1, 1, 1};
        threadIdx = {0, 0, 0};
        for (int b = 0; b < nb; ++b)
            for (int c = 0; c < nc; ++c) {
                blockIdx = {(unsigned)a, (unsigned)b, (unsigned)c};
                body();
            }
    }
}

}  // namespace

extern "C" int ref3_hist(int ani, int bpc, const float *D, int nD, const float *R, int nR, int bins,
                         float dmax, int partitions, float box, double *out) {
    if (!D || nD < 1 || nR < 0 || (nR > 0 && !R) || bins < 1 || partitions < 1 || !out) return -1;
    const float size_node = box / (float)partitions;
    if (check_nodes(D, nD, partitions, size_node) || check_nodes(R, nR, partitions, size_node)) return -2;
    Flat fd = flatten(D, nD, partitions, size_node);
    Flat fr = nR > 0 ? flatten(R, nR, partitions, size_node) : Flat();
    const int mD = (int)fd.nodes.size(), mR = (int)fr.nodes.size();
    float d_max_node = dmax + size_node * sqrt(3.0);
    d_max_node *= d_max_node;
    const size_t nb = ani ? (size_t)bins * bins * bins * bins * bins : (size_t)bins * bins * bins;
    memset(out, 0, sizeof(double) * nb * (nR > 0 ? 4 : 1));
    PointW3D *pD = fd.pts.data(), *pR = fr.pts.data();
    DNode *nDn = fd.nodes.data(), *nRn = fr.nodes.data();
    double *hDDD = out, *hRRR = out + nb, *hDDR = out + 2 * nb, *hDRR = out + 3 * nb;

    if (ani && bpc) {
        each_triple(mD, mD, mD, [&] { XXX3ani_BPC(hDDD, pD, nDn, mD, bins, dmax, d_max_node, box, size_node); });
        if (nR == 0) return 0;
        each_triple(mR, mR, mR, [&] { XXX3ani_BPC(hRRR, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0); });
        each_triple(mD, mD, mR, [&] {
            XXY3ani_BPC(hDDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0, true);
        });
        each_triple(mR, mR, mD, [&] {
            XXY3ani_BPC(hDRR, pR, nRn, mR, pD, nDn, mD, bins, dmax, d_max_node, box, size_node, 0, 0, false);
        });
    } else if (ani) {
        each_triple(mD, mD, mD, [&] { XXX3ani(hDDD, pD, nDn, mD, bins, dmax, d_max_node); });
        if (nR == 0) return 0;
        each_triple(mR, mR, mR, [&] { XXX3ani(hRRR, pR, nRn, mR, bins, dmax, d_max_node, 0, 0); });
        each_triple(mD, mD, mR, [&] { XXY3ani(hDDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, 0, 0, true); });
        each_triple(mR, mR, mD, [&] { XXY3ani(hDRR, pR, nRn, mR, pD, nDn, mD, bins, dmax, d_max_node, 0, 0, false); });
    } else if (bpc) {
        each_triple(mD, mD, mD, [&] { XXX3iso_BPC(hDDD, pD, nDn, mD, bins, dmax, d_max_node, box, size_node); });
        if (nR == 0) return 0;
        each_triple(mR, mR, mR, [&] { XXX3iso_BPC(hRRR, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0); });
        each_triple(mD, mD, mR, [&] {
            XXY3iso_BPC(hDDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0, true);
        });
        each_triple(mR, mR, mD, [&] {
            XXY3iso_BPC(hDRR, pR, nRn, mR, pD, nDn, mD, bins, dmax, d_max_node, box, size_node, 0, 0, false);
        });
    } else {
        each_triple(mD, mD, mD, [&] { XXX3iso(hDDD, pD, nDn, mD, bins, dmax, d_max_node); });
        if (nR == 0) return 0;
        each_triple(mR, mR, mR, [&] { XXX3iso(hRRR, pR, nRn, mR, bins, dmax, d_max_node, 0, 0); });
        each_triple(mD, mD, mR, [&] { XXY3iso(hDDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, 0, 0, true); });
        each_triple(mR, mR, mD, [&] { XXY3iso(hDRR, pR, nRn, mR, pD, nDn, mD, bins, dmax, d_max_node, 0, 0, false); });
    }
    return 0;
}

extern "C" int ref2_hist(int ani, int bpc, const float *D, int nD, const float *R, int nR, int bins,
                         float dmax, int partitions, float box, double *out) {
    if (!D || nD < 1 || !R || nR < 1 || bins < 1 || partitions < 1 || !out) return -1;
    const float size_node = box / (float)partitions;
    if (check_nodes(D, nD, partitions, size_node) || check_nodes(R, nR, partitions, size_node)) return -2;
    Flat fd = flatten(D, nD, partitions, size_node), fr = flatten(R, nR, partitions, size_node);
    const int mD = (int)fd.nodes.size(), mR = (int)fr.nodes.size();
    float d_max_node = dmax + size_node * sqrt(3.0);
    d_max_node *= d_max_node;
    const size_t nb = ani ? (size_t)bins * bins : (size_t)bins;
    memset(out, 0, sizeof(double) * nb * 3);
    PointW3D *pD = fd.pts.data(), *pR = fr.pts.data();
    DNode *nDn = fd.nodes.data(), *nRn = fr.nodes.data();
    double *hDD = out, *hRR = out + nb, *hDR = out + 2 * nb;
    if (ani) {
        if (bpc) {
            each_pair(mD, mD, [&] { XX2ani_BPC(hDD, pD, nDn, mD, bins, dmax, d_max_node, box, size_node); });
            each_pair(mR, mR, [&] { XX2ani_BPC(hRR, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0); });
        } else {
            each_pair(mD, mD, [&] { XX2ani(hDD, pD, nDn, mD, bins, dmax, d_max_node); });
            each_pair(mR, mR, [&] { XX2ani(hRR, pR, nRn, mR, bins, dmax, d_max_node, 0, 0); });
        }
        for (size_t k = 0; k < nb; ++k) hDR[k] = NAN;
    } else if (bpc) {
        each_pair(mD, mD, [&] { XX2iso_BPC(hDD, pD, nDn, mD, bins, dmax, d_max_node, box, size_node); });
        each_pair(mR, mR, [&] { XX2iso_BPC(hRR, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0); });
        each_pair(mD, mR, [&] {
            XY2iso_BPC(hDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, box, size_node, 0, 0);
        });
    } else {
        each_pair(mD, mD, [&] { XX2iso(hDD, pD, nDn, mD, bins, dmax, d_max_node); });
        each_pair(mR, mR, [&] { XX2iso(hRR, pR, nRn, mR, bins, dmax, d_max_node, 0, 0); });
        each_pair(mD, mR, [&] { XY2iso(hDR, pD, nDn, mD, pR, nRn, mR, bins, dmax, d_max_node, 0, 0); });
    }
    return 0;
}

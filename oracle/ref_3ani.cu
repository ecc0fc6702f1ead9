// Harness over the reference's anisotropic 3-point kernels -- fixture
// generation only.  Plain: XXX3ani, XXY3ani (cuda/kernels/3ani_k.cuh:8,109),
// launched as pcf_3ani does (pcf3ani.cuh:77-112).  Periodic: XXX3ani_BPC,
// XXY3ani_BPC (cuda/kernels/3aniBPC_k.cuh:210,959), launched as pcf_3aniBPC
// does (pcf3aniBPC.cuh:87-115).  Both: 8x8x8 threads per block, one thread
// per ordered node triple, d_max_node = (dmax + size_node*sqrt(3))^2, one
// random file (node and bin offsets 0).  The reference's own writer keeps
// only bn^3 of the bn^5 histogram (pcf3ani.cuh:123, pcf3aniBPC.cuh:123);
// this harness copies every bin back.  Nodes are built as main.cu:219-329 builds them (make_nodos, then the
// non-empty nodes in (row, col, mom) order with their points contiguous).
// The headers are included unmodified from the reference tree (-I<ref>/cuda).
//
//   ref_3ani.out D.f4 R.f4 N BINS DMAX PARTITIONS BOX BPC OUT.bin
//     D.f4, R.f4: N points each, float32 x y z w; BPC: 0 plain, 1 periodic;
//     OUT.bin: DDD, RRR, DDR, DRR, bins^5 doubles each.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "create_grid.cuh"
#include "kernels/3ani_k.cuh"
#include "kernels/3aniBPC_k.cuh"

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            fprintf(stderr, "%s: %s\n", #call, cudaGetErrorString(e_));          \
            exit(2);                                                               \
        }                                                                          \
    } while (0)

struct Flat {
    std::vector<DNode> nodes;
    std::vector<PointW3D> pts;
};

static Flat flatten(PointW3D *dat, int np, int partitions, float size_node) {
    Node ***nod = new Node **[partitions];
    for (int i = 0; i < partitions; ++i) {
        nod[i] = new Node *[partitions];
        for (int j = 0; j < partitions; ++j) nod[i][j] = new Node[partitions];
    }
    make_nodos(nod, dat, partitions, size_node, np);
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

static std::vector<PointW3D> read_f4(const char *path, int n) {
    std::vector<PointW3D> v((size_t)n);
    FILE *fp = fopen(path, "rb");
    if (!fp || fread(v.data(), sizeof(PointW3D), (size_t)n, fp) != (size_t)n) {
        fprintf(stderr, "cannot read %d points from %s\n", n, path);
        exit(1);
    }
    fclose(fp);
    return v;
}

int main(int argc, char **argv) {
    if (argc != 10) {
        fprintf(stderr, "usage: %s D.f4 R.f4 N BINS DMAX PARTITIONS BOX BPC OUT.bin\n", argv[0]);
        return 1;
    }
    const int np = atoi(argv[3]), bn = atoi(argv[4]), partitions = atoi(argv[6]);
    const bool bpc = atoi(argv[8]) != 0;
    const float dmax = (float)atof(argv[5]), box = (float)atof(argv[7]);
    std::vector<PointW3D> D = read_f4(argv[1], np), R = read_f4(argv[2], np);
    const float size_node = box / (float)partitions;
    Flat fd = flatten(D.data(), np, partitions, size_node);
    Flat fr = flatten(R.data(), np, partitions, size_node);
    const int nD = (int)fd.nodes.size(), nR = (int)fr.nodes.size();
    float d_max_node = dmax + size_node * sqrt(3.0);
    d_max_node *= d_max_node;

    DNode *dnD, *dnR;
    PointW3D *dpD, *dpR;
    CK(cudaMalloc(&dnD, sizeof(DNode) * nD));
    CK(cudaMalloc(&dnR, sizeof(DNode) * nR));
    CK(cudaMalloc(&dpD, sizeof(PointW3D) * np));
    CK(cudaMalloc(&dpR, sizeof(PointW3D) * np));
    CK(cudaMemcpy(dnD, fd.nodes.data(), sizeof(DNode) * nD, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dnR, fr.nodes.data(), sizeof(DNode) * nR, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dpD, fd.pts.data(), sizeof(PointW3D) * np, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dpR, fr.pts.data(), sizeof(PointW3D) * np, cudaMemcpyHostToDevice));

    const size_t nb5 = (size_t)bn * bn * bn * bn * bn;
    double *h[4];
    for (int k = 0; k < 4; ++k) {
        CK(cudaMalloc(&h[k], sizeof(double) * nb5));
        CK(cudaMemset(h[k], 0, sizeof(double) * nb5));
    }
    const int t = 8;
    const int bD = (nD + t - 1) / t, bR = (nR + t - 1) / t;
    const dim3 thr(t, t, t);
    if (bpc) {
        XXX3ani_BPC<<<dim3(bD, bD, bD), thr>>>(h[0], dpD, dnD, nD, bn, dmax, d_max_node, box, size_node);
        XXX3ani_BPC<<<dim3(bR, bR, bR), thr>>>(h[1], dpR, dnR, nR, bn, dmax, d_max_node, box, size_node, 0, 0);
        XXY3ani_BPC<<<dim3(bD, bD, bR), thr>>>(h[2], dpD, dnD, nD, dpR, dnR, nR, bn, dmax, d_max_node, box,
                                               size_node, 0, 0, true);
        XXY3ani_BPC<<<dim3(bR, bR, bD), thr>>>(h[3], dpR, dnR, nR, dpD, dnD, nD, bn, dmax, d_max_node, box,
                                               size_node, 0, 0, false);
    } else {
        XXX3ani<<<dim3(bD, bD, bD), thr>>>(h[0], dpD, dnD, nD, bn, dmax, d_max_node);
        XXX3ani<<<dim3(bR, bR, bR), thr>>>(h[1], dpR, dnR, nR, bn, dmax, d_max_node, 0, 0);
        XXY3ani<<<dim3(bD, bD, bR), thr>>>(h[2], dpD, dnD, nD, dpR, dnR, nR, bn, dmax, d_max_node, 0, 0, true);
        XXY3ani<<<dim3(bR, bR, bD), thr>>>(h[3], dpR, dnR, nR, dpD, dnD, nD, bn, dmax, d_max_node, 0, 0, false);
    }
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());

    std::vector<double> out(nb5);
    FILE *fo = fopen(argv[9], "wb");
    if (!fo) return 1;
    for (int k = 0; k < 4; ++k) {
        CK(cudaMemcpy(out.data(), h[k], sizeof(double) * nb5, cudaMemcpyDeviceToHost));
        fwrite(out.data(), sizeof(double), nb5, fo);
        cudaFree(h[k]);
    }
    fclose(fo);
    cudaFree(dnD);
    cudaFree(dnR);
    cudaFree(dpD);
    cudaFree(dpR);
    return 0;
}

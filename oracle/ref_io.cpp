// Harness over the reference's catalog reader (open_files,
// cuda/create_grid.cuh:35-78) -- test and baseline infrastructure only.
// The header is included unmodified from the reference tree (-I<ref>/cuda).
// open_files reads "../data/<name>" relative to the working directory, so
// the caller sets that up; it exits the process on a missing file, so the
// caller passes only files that exist.
#include <math.h>  // the header calls ceil, which main.cu's other includes provide
#include <cstring>
#include <string>
#include <vector>

#include "create_grid.cuh"

extern "C" int ref_open_files(const char *name, int n, float *out, float *box) {
    PointW3D *pts = new PointW3D[n];
    float size_box = *box;  // <= 0: the reader's automatic box
    open_files(std::string(name), n, pts, size_box);
    std::memcpy(out, pts, sizeof(PointW3D) * (size_t)n);
    delete[] pts;
    *box = size_box;
    return 0;
}

// The reference's histogram writers (create_grid.cuh:141-229): dims 1, 2 or 3
// of a bn^dims histogram, written to "../results/<name>" from the working
// directory the caller sets up.
extern "C" int ref_save_histogram(int dims, const char *name, int bn, const double *h) {
    size_t count = (size_t)bn;
    for (int d = 1; d < dims; ++d) count *= (size_t)bn;
    std::vector<double> v(h, h + count);
    if (dims == 1) save_histogram1D(std::string(name), bn, v.data());
    else if (dims == 2) save_histogram2D(std::string(name), bn, v.data());
    else if (dims == 3) save_histogram3D(std::string(name), bn, v.data());
    else return -1;
    return 0;
}

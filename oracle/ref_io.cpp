// Harness over the reference's catalog reader (open_files,
// cuda/create_grid.cuh:35-78) -- test and baseline infrastructure only.
// The header is included unmodified from the reference tree (-I<ref>/cuda).
// open_files reads "../data/<name>" relative to the working directory, so
// the caller sets that up; it exits the process on a missing file, so the
// caller passes only files that exist.
#include <math.h>  // the header calls ceil, which main.cu's other includes provide
#include <cstring>
#include <string>

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

// Test helper: this library's histogram writers (desi_b200/csrc/pcf_io.hpp,
// the ones PCF.out uses) on a raw double file.
//   io_writer DIMS BN IN_RAW OUT_NAME   (writes ../results/OUT_NAME)
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pcf_io.hpp"

int main(int argc, char **argv) {
    if (argc != 5) return 2;
    const int dims = std::atoi(argv[1]), bn = std::atoi(argv[2]);
    size_t count = (size_t)bn;
    for (int d = 1; d < dims; ++d) count *= (size_t)bn;
    std::vector<double> h(count);
    FILE *f = std::fopen(argv[3], "rb");
    if (!f || std::fread(h.data(), sizeof(double), count, f) != count) return 3;
    std::fclose(f);
    const bool ok = dims == 1 ? pcfio::save1d(argv[4], bn, h.data())
                  : dims == 2 ? pcfio::save2d(argv[4], bn, h.data())
                              : pcfio::save3d(argv[4], bn, h.data());
    return ok ? 0 : 1;
}

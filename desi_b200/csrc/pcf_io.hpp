// pcf_io.hpp -- catalog reader and histogram writers of the PCF.out drop-in,
// byte-compatible with the reference's (cuda/create_grid.cuh:35-78 and
// :141-266): catalogs are read from "../data/<name>" as whitespace-separated
// x y z w rows, histograms are written to "../results/<name>" as text with
// setprecision(12).
#pragma once

#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/pcf.h"
#include "../../include/pcf_ingest.h"

namespace pcfio {

// Reads the first n rows of ../data/<name>; returns false on a missing file
// or short read.  box_candidate receives ceil(max component + 1), the
// reference's automatic box (create_grid.cuh:75).
inline bool open_catalog(const std::string &name, long n, std::vector<pcf_point> &out,
                         float &box_candidate, std::string *err = nullptr) {
    const std::string path = "../data/" + name;
    {
        std::ifstream probe(path.c_str(), std::ios::in | std::ios::binary);
        if (probe.fail()) {
            if (err) *err = "Failed to load the file in " + path;
            return false;
        }
    }
    out.resize((size_t)n);
    int64_t got = 0;
    if (pcf_read_catalog(path.c_str(), n, out.data(), &got, &box_candidate) != PCF_OK) {
        if (err) *err = path + ": fewer than " + std::to_string(n) + " readable rows";
        return false;
    }
    return true;
}

inline bool open_out(const std::string &name, std::ofstream &f) {
    const std::string path = "../results/" + name;
    f.open(path.c_str(), std::ios::out | std::ios::binary);
    if (f.fail()) {
        std::cout << "Failed to save the the histogram in " << path << std::endl;
        return false;
    }
    return true;
}

// save_histogram1D (create_grid.cuh:141)
inline bool save1d(const std::string &name, int bn, const double *h) {
    std::ofstream f;
    if (!open_out(name, f)) return false;
    for (int i = 0; i < bn; ++i) f << std::setprecision(12) << h[i] << std::endl;
    return true;
}

// save_histogram2D (create_grid.cuh:166)
inline bool save2d(const std::string &name, int bn, const double *h) {
    std::ofstream f;
    if (!open_out(name, f)) return false;
    for (int i = 0; i < bn; ++i) {
        for (int j = 0; j < bn; ++j) f << std::setprecision(12) << h[i * bn + j] << ' ';
        f << "\n";
    }
    return true;
}

// save_histogram3D (create_grid.cuh:197)
inline bool save3d(const std::string &name, int bn, const double *h) {
    std::ofstream f;
    if (!open_out(name, f)) return false;
    for (int i = 0; i < bn; ++i) {
        for (int j = 0; j < bn; ++j) {
            for (int k = 0; k < bn; ++k) f << std::setprecision(12) << h[((size_t)i * bn + j) * bn + k] << ' ';
            f << "\n";
        }
        f << "\n" << std::endl;
    }
    return true;
}

// save_histogram5D (create_grid.cuh:230): the full bn^5 histogram (the
// reference's 3-point anisotropic paths call the 3-D writer on it and keep
// only its first bn^3 values, pcf3ani.cuh:123).
inline bool save5d(const std::string &name, int bn, const double *h) {
    std::ofstream f;
    if (!open_out(name, f)) return false;
    size_t idx = 0;
    for (int i = 0; i < bn; ++i) {
        for (int j = 0; j < bn; ++j) {
            for (int k = 0; k < bn; ++k) {
                for (int l = 0; l < bn; ++l) {
                    for (int m = 0; m < bn; ++m) f << std::setprecision(12) << h[idx++] << ' ';
                    f << "\n";
                }
                f << "\n";
            }
            f << "\n";
        }
        f << "\n" << std::endl;
    }
    return true;
}

}  // namespace pcfio

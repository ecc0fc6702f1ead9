// pcf_main.cpp -- PCF.out, the drop-in for the reference's command line
// (cuda/main.cu:45-429, help text cuda/PCF_help.cuh:3-47):
//
//   PCF.out <2iso|2ani|3iso|3ani> -n N -f DATA (-r RAND | -rd DIR/) -b BINS -d DMAX
//           [-bpc [-a]] [-p PARTS] [-s BOX]
//
// Same flags, defaults, paths (../data/<name> in, ../results/<name> out),
// file names and text formats as the reference; the histograms come from
// libpcf.so (include/pcf.h).  Differences: library errors print a message
// and exit(1) instead of crashing; 3-point names are not accumulated across
// random files (pcf3iso.cuh:127); the 3ani histograms are written in full
// (bins^5, save_histogram5D) rather than their first bins^3 values; -p sets
// the cells per box side, which the library uses when a periodic stencil
// fits them (2*ceil(dmax/cell) + 2 <= P) and otherwise replaces with its own
// choice (pair results do not depend on it); -rd counts RR and DR (3iso:
// DDD, RRR, DDR, DRR) of every random catalog of the directory in one
// persistent launch (pcf_batch_pairs, pcf_batch_triplets).  Periodic
// triplets (3iso / 3ani -bpc) count as the reference's CUDA kernels count on
// their node grid of -p nodes per side (PCF_REF_NODE_GATES, whose gates miss
// some triangles near the box edges), so the files match the reference's;
// the added switch -exact counts every triangle in range once instead (the
// reference's CPU engines' count).
#include <dirent.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/pcf.h"
#include "pcf_io.hpp"

using std::cout;
using std::endl;
using std::string;

static void show_help() {
    cout << "Use: ./PCF <calc_type> -n number_of_points -f datafile -b bins -d maximum_distance" << endl;
    cout << "-r randomfile || -rd randoms_directory" << endl;
    cout << "[-bpc [-a]][-p box_partitions] [-s size_box]" << endl;
    cout << "Computes the pair (2iso, 2ani) or triplet (3iso, 3ani) histograms of a data catalog\n"
            "and its random catalogs, with or without periodic boundaries (-bpc), on the GPU.\n"
            "Catalog files (in ../data/) hold four columns x y z w; -n rows are read.\n"
            "  -rd DIR/  uses every file of ../data/DIR/ as a random catalog\n"
            "  -bpc -a   isotropic only: RR / DDR / RRR from the analytic periodic formulas\n"
            "  -s BOX    box side (default: ceil(max coordinate + 1) over the files)\n"
            "  -exact    3iso / 3ani -bpc: count every triangle in range once, not through\n"
            "            the reference kernels' node gates on the -p grid\n"
            "Histograms are written to ../results/." << endl;
}

static void die(const char *what, pcf_status s, pcf_ctx *ctx) {
    cout << what << ": " << pcf_status_string(s);
    if (ctx && pcf_last_error(ctx)[0]) cout << " (" << pcf_last_error(ctx) << ")";
    cout << endl;
    exit(1);
}

#define CHECK(call)                               \
    do {                                          \
        pcf_status _s = (call);                   \
        if (_s != PCF_OK) die(#call, _s, ctx);    \
    } while (0)

int main(int argc, char **argv) {
    if (argc == 2 && (strcmp(argv[1], "--help") == 0 || strcmp(argv[1], "-h") == 0)) {
        show_help();
        return 0;
    }
    if (!(argc >= 8 && (strcmp(argv[1], "3iso") == 0 || strcmp(argv[1], "3ani") == 0 ||
                        strcmp(argv[1], "2iso") == 0 || strcmp(argv[1], "2ani") == 0))) {
        cout << "Invalid <calc_type> option or not enough parameters. \nSee --help for more information." << endl;
        exit(1);
    }
    const string type = argv[1];
    int np = 0, bn = 0, partitions = 35;
    bool bpc = false, analytic = false, rand_dir = false, size_box_provided = false, rand_required = false;
    bool exact = false;
    float size_box = 0, dmax = 0;
    string data_name, rand_name = "";
    for (int i = 2; i < argc; i++) {
        const bool has = i + 1 < argc;
        if (strcmp(argv[i], "-n") == 0 && has) { np = std::stoi(argv[++i]); }
        else if (strcmp(argv[i], "-f") == 0 && has) { data_name = argv[++i]; }
        else if ((strcmp(argv[i], "-r") == 0 || strcmp(argv[i], "-rd") == 0) && has) {
            rand_dir = strcmp(argv[i], "-rd") == 0;
            rand_name = argv[++i];
        } else if (strcmp(argv[i], "-b") == 0 && has) { bn = std::stoi(argv[++i]); }
        else if (strcmp(argv[i], "-d") == 0 && has) { dmax = std::stof(argv[++i]); }
        else if (strcmp(argv[i], "-bpc") == 0) { bpc = true; }
        else if (strcmp(argv[i], "-a") == 0) { analytic = true; }
        else if (strcmp(argv[i], "-exact") == 0) { exact = true; }
        else if (strcmp(argv[i], "-p") == 0 && has) { partitions = (int)std::stof(argv[++i]); }
        else if (strcmp(argv[i], "-s") == 0 && has) { size_box = std::stof(argv[++i]); size_box_provided = true; }
    }
    if (np == 0) { cout << "Missing number of points argument." << endl; exit(1); }
    if (bn == 0) { cout << "Missing number of bins argument." << endl; exit(1); }
    if (dmax == 0) { cout << "Missing maximum distance argument." << endl; exit(1); }
    if (!(bpc && analytic && (type == "3iso" || type == "2iso"))) {
        rand_required = true;
        if (rand_name == "") { cout << "Missing random file(s) location." << endl; exit(1); }
    }

    auto t0 = std::chrono::steady_clock::now();
    // catalogs (main.cu:136-211)
    std::vector<pcf_point> D;
    float boxD = 0;
    string err;
    if (!pcfio::open_catalog(data_name, np, D, boxD, &err)) { cout << err << endl; exit(1); }
    std::vector<string> rand_files, rand_labels;
    if (rand_required) {
        if (rand_dir) {
            string dir = "../data/" + rand_name;
            DIR *folder = opendir(dir.c_str());
            if (!folder) { cout << "Failed to open the directory " << dir << endl; exit(1); }
            while (dirent *e = readdir(folder)) {
                string nm = e->d_name;
                if (nm == "." || nm == "..") continue;
                rand_labels.push_back(nm);
                rand_files.push_back(rand_name + nm);
            }
            closedir(folder);
        } else {
            rand_files.push_back(rand_name);
            rand_labels.push_back(rand_name);
        }
    }
    std::vector<std::vector<pcf_point>> R(rand_files.size());
    float boxR = 0;
    for (size_t i = 0; i < rand_files.size(); ++i) {
        float b = 0;
        if (!pcfio::open_catalog(rand_files[i], np, R[i], b, &err)) { cout << err << endl; exit(1); }
        if (i == 0) boxR = b;  // the reference sizes the box from the first random file
    }
    if (!size_box_provided) size_box = boxR > boxD ? boxR : boxD;

    pcf_ctx *ctx = nullptr;
    CHECK(pcf_ctx_create(0, &ctx));
    pcf_grid *gD = nullptr;
    CHECK(pcf_grid_build(ctx, D.data(), np, size_box, partitions, &gD));
    std::vector<pcf_grid *> gR(R.size(), nullptr);
    for (size_t i = 0; i < R.size(); ++i) CHECK(pcf_grid_build(ctx, R[i].data(), np, size_box, partitions, &gR[i]));
    auto t1 = std::chrono::steady_clock::now();
    cout << "Succesfully readed the data. All set to compute the histograms in "
         << std::chrono::duration<double, std::milli>(t1 - t0).count() << " miliseconds" << endl;

    const string tag = bpc ? (analytic ? "BPCanalytic_" : "BPC_") : "";
    const size_t b1 = (size_t)bn, b2 = b1 * bn, b3 = b2 * bn, b5 = b3 * b2;
    if (type == "2iso" || type == "2ani") {
        const bool ani = type == "2ani";
        const int kind = ani ? PCF_ANI : PCF_ISO;
        // 2iso BPC bins with the unfloored bins/dmax (2isoBPC_k.cuh:36)
        const uint32_t f = bpc ? (PCF_BPC | (ani ? 0u : (uint32_t)PCF_DS_EXACT)) : 0u;
        const string sfx = ani ? "ani_" : "iso_";
        std::vector<double> h(ani ? b2 : b1);
        auto save = [&](const string &n) { ani ? pcfio::save2d(n, bn, h.data()) : pcfio::save1d(n, bn, h.data()); };
        CHECK(pcf_count_pairs(ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr));
        save("DD" + sfx + tag + data_name);
        if (analytic && !ani) {
            CHECK(pcf_analytic_rr(ctx, bn, np, size_box, dmax, 1, h.data()));
            save("RR" + sfx + tag + data_name);
            save("DR" + sfx + tag + data_name);  // the reference writes RR as DR (pcf2isoBPC.cuh:265)
        } else if (gR.size() > 1) {
            // -rd: every random catalog of the directory in one persistent
            // launch (the reference launches two kernels per file,
            // cuda/pcf2iso.cuh:96-104)
            const size_t nb = h.size(), nr = gR.size();
            std::vector<double> rr(nb * nr), dr(nb * nr);
            CHECK(pcf_batch_pairs(ctx, kind, gD, gR.data(), (int)nr, bn, dmax, f, nullptr, rr.data(),
                                  dr.data(), nullptr));
            for (size_t i = 0; i < nr; ++i) {
                std::copy(rr.begin() + i * nb, rr.begin() + (i + 1) * nb, h.begin());
                save("RR" + sfx + tag + rand_labels[i]);
                std::copy(dr.begin() + i * nb, dr.begin() + (i + 1) * nb, h.begin());
                save("DR" + sfx + tag + rand_labels[i]);
            }
        } else {
            for (size_t i = 0; i < gR.size(); ++i) {
                CHECK(pcf_count_pairs(ctx, kind, gR[i], nullptr, bn, dmax, f, h.data(), nullptr));
                save("RR" + sfx + tag + rand_labels[i]);
                CHECK(pcf_count_pairs(ctx, kind, gD, gR[i], bn, dmax, f, h.data(), nullptr));
                save("DR" + sfx + tag + rand_labels[i]);
            }
        }
    } else {
        const bool ani = type == "3ani";
        const int kind = ani ? PCF_ANI : PCF_ISO;
        const bool gated = bpc && !exact;
        const uint32_t f = bpc ? (PCF_BPC | (gated ? (uint32_t)PCF_REF_NODE_GATES : 0u)) : 0u;
        const string sfx = ani ? "ani_" : "iso_";
        std::vector<double> h(ani ? b5 : b3);
        auto save = [&](const string &n) { ani ? pcfio::save5d(n, bn, h.data()) : pcfio::save3d(n, bn, h.data()); };
        if (analytic && !ani) {
            std::vector<double> ddr(b3), rrr(b3);
            CHECK(pcf_analytic_3iso(ctx, gD, bn, dmax, 0, 0, 1, h.data(), ddr.data(), rrr.data(), nullptr));
            save("DDD" + sfx + tag + data_name);
            pcfio::save3d("DDR" + sfx + tag + data_name, bn, ddr.data());
            pcfio::save3d("DRR" + sfx + tag + data_name, bn, ddr.data());  // pcf3isoBPC.cuh:340
            pcfio::save3d("RRR" + sfx + tag + data_name, bn, rrr.data());
        } else if (!ani && gR.size() > 1 && !gated) {
            // -rd: DDD, and RRR / DDR / DRR of every random catalog, in one
            // persistent launch (the reference launches per file,
            // cuda/pcf3iso.cuh:101-112)
            const size_t nr = gR.size();
            std::vector<double> rrr(b3 * nr), ddr(b3 * nr), drr(b3 * nr);
            CHECK(pcf_batch_triplets(ctx, gD, gR.data(), (int)nr, bn, dmax, f, h.data(), rrr.data(),
                                     ddr.data(), drr.data(), nullptr));
            save("DDD" + sfx + tag + data_name);
            for (size_t i = 0; i < nr; ++i) {
                pcfio::save3d("RRR" + sfx + tag + rand_labels[i], bn, rrr.data() + i * b3);
                pcfio::save3d("DDR" + sfx + tag + rand_labels[i], bn, ddr.data() + i * b3);
                pcfio::save3d("DRR" + sfx + tag + rand_labels[i], bn, drr.data() + i * b3);
            }
        } else {
            CHECK(pcf_count_triplets(ctx, kind, gD, nullptr, bn, dmax, f, h.data(), nullptr));
            save("DDD" + sfx + tag + data_name);
            for (size_t i = 0; i < gR.size(); ++i) {
                CHECK(pcf_count_triplets(ctx, kind, gR[i], nullptr, bn, dmax, f, h.data(), nullptr));
                save("RRR" + sfx + tag + rand_labels[i]);
                CHECK(pcf_count_triplets(ctx, kind, gD, gR[i], bn, dmax, f, h.data(), nullptr));
                save("DDR" + sfx + tag + rand_labels[i]);
                CHECK(pcf_count_triplets(ctx, kind, gR[i], gD, bn, dmax, f, h.data(), nullptr));
                save("DRR" + sfx + tag + rand_labels[i]);
            }
        }
    }
    auto t2 = std::chrono::steady_clock::now();
    cout << "Spent " << std::chrono::duration<double, std::milli>(t2 - t1).count()
         << " miliseconds to compute and save all the histograms." << endl;
    for (auto g : gR) pcf_grid_free(ctx, g);
    pcf_grid_free(ctx, gD);
    pcf_ctx_destroy(ctx);
    cout << "Program terminated..." << endl;
    return 0;
}

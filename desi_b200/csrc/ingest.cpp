// ingest.cpp -- catalog ingestion: the reference reads catalogs with one
// ifstream >> per value on one thread (cuda/create_grid.cuh:35-78).  Here the
// text file is read whole and parsed by all host threads (std::from_chars,
// correctly rounded like strtof / operator>>), and a binary form -- raw
// little-endian float32 x, y, z, w per point, extension ".f4" -- loads with
// one read.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pcf_ingest.h"

namespace {

bool ends_with(const std::string &s, const char *suf) {
    const size_t n = strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

inline const char *skip_ws(const char *p, const char *e) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    return p;
}

}  // namespace

extern "C" pcf_status pcf_read_catalog(const char *path, int64_t n, pcf_point *out, int64_t *n_read,
                                       float *box_candidate) {
    if (!path || !out || n < 0) return PCF_ERR_INVALID_ARG;
    const std::string p = path;
    std::ifstream f(p, std::ios::binary | std::ios::ate);
    if (!f) return PCF_ERR_IO;
    const std::streamoff size = f.tellg();
    f.seekg(0);
    int64_t got = 0;
    if (ends_with(p, ".f4")) {
        const int64_t avail = (int64_t)(size / 16);
        got = std::min(avail, n);
        if (!f.read(reinterpret_cast<char *>(out), got * 16)) return PCF_ERR_IO;
    } else {
        std::vector<char> buf((size_t)size);
        if (size > 0 && !f.read(buf.data(), size)) return PCF_ERR_IO;
        // split into line-aligned chunks, count rows per chunk, then parse in place
        const int nt = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
        std::vector<size_t> cut((size_t)nt + 1, 0);
        cut[nt] = buf.size();
        for (int t = 1; t < nt; ++t) {
            size_t c = buf.size() * (size_t)t / nt;
            while (c < buf.size() && buf[c] != '\n') ++c;
            cut[t] = std::min(buf.size(), c + 1);
            if (cut[t] < cut[t - 1]) cut[t] = cut[t - 1];
        }
        std::vector<int64_t> rows((size_t)nt, 0);
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                int64_t r = 0;
                bool any = false;
                for (size_t i = cut[t]; i < cut[t + 1]; ++i) {
                    const char ch = buf[i];
                    if (ch == '\n') { if (any) ++r; any = false; }
                    else if (ch != ' ' && ch != '\t' && ch != '\r') any = true;
                }
                if (any) ++r;
                rows[t] = r;
            });
        for (auto &x : th) x.join();
        th.clear();
        std::vector<int64_t> first((size_t)nt + 1, 0);
        for (int t = 0; t < nt; ++t) first[t + 1] = first[t] + rows[t];
        std::vector<int> bad((size_t)nt, 0);
        for (int t = 0; t < nt; ++t)
            th.emplace_back([&, t] {
                const char *q = buf.data() + cut[t], *e = buf.data() + cut[t + 1];
                int64_t r = first[t];
                while (r < n && r < first[t + 1]) {
                    float v[4];
                    for (int k = 0; k < 4; ++k) {
                        q = skip_ws(q, e);
                        auto res = std::from_chars(q, e, v[k]);
                        if (res.ec != std::errc()) { bad[t] = 1; return; }
                        q = res.ptr;
                    }
                    out[r] = pcf_point{v[0], v[1], v[2], v[3]};
                    ++r;
                }
            });
        for (auto &x : th) x.join();
        for (int b : bad)
            if (b) return PCF_ERR_IO;
        got = std::min(n, first[nt]);
    }
    if (n_read) *n_read = got;
    if (box_candidate) {
        double mx = 0;
        for (int64_t i = 0; i < got; ++i) {
            const pcf_point &q = out[i];
            const float m = q.x > q.y ? (q.x > q.z ? q.x : q.z) : (q.y > q.z ? q.y : q.z);
            if (m > mx) mx = m;
        }
        *box_candidate = (float)std::ceil(mx + 1);  // create_grid.cuh:75
    }
    return got < n ? PCF_ERR_IO : PCF_OK;
}

extern "C" pcf_status pcf_write_catalog_f4(const char *path, const pcf_point *pts, int64_t n) {
    if (!path || (!pts && n > 0) || n < 0) return PCF_ERR_INVALID_ARG;
    std::ofstream f(path, std::ios::binary);
    if (!f) return PCF_ERR_IO;
    f.write(reinterpret_cast<const char *>(pts), n * 16);
    return f ? PCF_OK : PCF_ERR_IO;
}

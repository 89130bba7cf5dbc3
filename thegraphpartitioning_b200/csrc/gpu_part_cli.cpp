// gpu_part_cli.cpp -- drop-in replacement of the reference `gpu_part` executable.
//
// Accepts both command lines the reference has:
//   gpu_part <directory> <nvtxs> <nedges> <num_partitions>      (src/gpu_part.cu:880-888)
//       reads <directory>/row.txt (nvtxs+1 ints), column.txt and weight.txt
//       (nedges ints each), as readFile does (src/gpu_part.cu:786-800, 905-908)
//   gpu_part <row.txt> <column.txt> <num_partitions>              (README.md:130-138)
//       n = ints in row.txt - 1, nedges = last row pointer; unit edge weights
//       unless a weight.txt sits beside column.txt
// plus optional flags: --imbalance F (default 0.03), --seed N (default 0),
// --out FILE (default ./finalpartition.txt), --part-list FILE (one part id per
// line, the layout of gpmetis' .part.<k> file).
// Writes ./finalpartition.txt as "Partition q: v,v,..." lines
// (src/gpu_part.cu:1296-1322) and prints the reference's report sections
// (src/gpu_part.cu:1330-1381).  Exit codes: 1 bad arguments (as
// src/gpu_part.cu:891-894), 2 unreadable input file, 3 partitioner error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <string>
#include <vector>
#include <chrono>
#include <algorithm>
#include <sys/stat.h>
#include <thread>
#include <charconv>

#include <cuda_runtime.h>

#include "../../include/gp_partition.h"

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool file_exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

inline bool is_space(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

// Number of tokens in buf[b, e) (b and e on token boundaries).
size_t count_tokens(const char* buf, size_t b, size_t e) {
    size_t c = 0;
    bool in = false;
    for (size_t i = b; i < e; ++i) {
        const bool sp = is_space(buf[i]);
        c += (!sp && !in) ? 1 : 0;
        in = !sp;
    }
    return c;
}

// Integers of buf[b, e) written to out[first ..] (entries at or past `keep`
// are dropped); on a malformed token, *bad = its index within the range.
void parse_range(const char* buf, size_t b, size_t e, int64_t* out, size_t first, size_t keep, int64_t* bad) {
    const char* p = buf + b;
    const char* end = buf + e;
    size_t i = 0;
    *bad = -1;
    while (p < end) {
        while (p < end && is_space(*p)) ++p;
        if (p >= end) break;
        bool neg = false;
        if (*p == '-') { neg = true; ++p; }
        if (p >= end || *p < '0' || *p > '9') { *bad = (int64_t)i; return; }
        int64_t v = 0;
        while (p < end && *p >= '0' && *p <= '9') v = v * 10 + (*p++ - '0');
        if (p < end && !is_space(*p)) { *bad = (int64_t)i; return; }
        if (first + i < keep) out[first + i] = neg ? -v : v;
        ++i;
    }
}

// Whitespace-separated integers of a text file, parsed by all host threads:
// the file is cut into chunks at whitespace, a first pass counts each
// chunk's integers, a second parses them straight into their final places.
// max_count < 0: read all; otherwise the first max_count integers, and fewer
// is an error (as readFile, src/gpu_part.cu:786-800).
bool read_ints(const std::string& path, int64_t max_count, std::vector<int64_t>& out, std::string& err) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path; return false; }
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)sz + 1);
    size_t got = fread(buf.data(), 1, (size_t)sz, f);
    fclose(f);
    buf[got] = 0;
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    if (got < ((size_t)1 << 20)) nt = 1;
    nt = std::min<unsigned>(nt, 64);
    std::vector<size_t> cut(nt + 1), cnt(nt), first(nt + 1);
    cut[0] = 0;
    cut[nt] = got;
    for (unsigned t = 1; t < nt; ++t) {
        size_t b = got * t / nt;
        if (b < cut[t - 1]) b = cut[t - 1];
        while (b < got && !is_space(buf[b])) ++b;   // move to the end of the token
        cut[t] = b;
    }
    auto run = [&](auto&& fn) {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) th.emplace_back([&, t] { fn(t); });
        for (auto& x : th) x.join();
    };
    run([&](unsigned t) { cnt[t] = count_tokens(buf.data(), cut[t], cut[t + 1]); });
    first[0] = 0;
    for (unsigned t = 0; t < nt; ++t) first[t + 1] = first[t] + cnt[t];
    const size_t total = first[nt];
    const size_t keep = max_count < 0 ? total : std::min<size_t>(total, (size_t)max_count);
    out.resize(keep);
    std::vector<int64_t> bad(nt, -1);
    run([&](unsigned t) {
        if (first[t] < keep) parse_range(buf.data(), cut[t], cut[t + 1], out.data(), first[t], keep, &bad[t]);
    });
    for (unsigned t = 0; t < nt; ++t)
        if (bad[t] >= 0 && first[t] + (size_t)bad[t] < keep) {
            err = path + ": not an integer at element " + std::to_string(first[t] + (size_t)bad[t]);
            return false;
        }
    if (max_count > 0 && (int64_t)out.size() < max_count) {
        err = "Error reading file " + path + " at element " + std::to_string(out.size());
        return false;
    }
    return true;
}

void usage(const char* a0) {
    fprintf(stderr,
            "Usage: %s <directory> <nvtxs> <nedges> <num_partitions> [options]\n"
            "   or: %s <row.txt> <column.txt> <num_partitions> [options]\n"
            "options: --imbalance F  --seed N  --out FILE  --part-list FILE  --parse-only\n", a0, a0);
}

}  // namespace

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    float imbalance = 0.03f;
    uint64_t seed = 0;
    std::string out_path = "./finalpartition.txt", part_list;
    bool parse_only = false;   // read and check the input files only (no device work)
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto need = [&](const char* name) -> const char* {
            if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", name); exit(1); }
            return argv[++i];
        };
        if (a == "--imbalance") imbalance = (float)atof(need("--imbalance"));
        else if (a == "--seed") seed = strtoull(need("--seed"), nullptr, 10);
        else if (a == "--out") out_path = need("--out");
        else if (a == "--part-list") part_list = need("--part-list");
        else if (a == "--parse-only") parse_only = true;
        else if (a == "-h" || a == "--help") { usage(argv[0]); return 0; }
        else pos.push_back(a);
    }
    std::string row, col, wgt;
    int64_t nv = -1, ne = -1, k = 0;
    if (pos.size() == 4) {
        row = pos[0] + "/row.txt"; col = pos[0] + "/column.txt"; wgt = pos[0] + "/weight.txt";
        nv = atoll(pos[1].c_str()); ne = atoll(pos[2].c_str()); k = atoll(pos[3].c_str());
        if (nv <= 0 || ne <= 0 || k <= 0) {
            fprintf(stderr, "Invalid input: nvtxs, nedges, and numPartitions must be positive.\n");
            return 1;
        }
    } else if (pos.size() == 3) {
        row = pos[0]; col = pos[1];
        k = atoll(pos[2].c_str());
        size_t slash = col.find_last_of('/');
        std::string dir = slash == std::string::npos ? "." : col.substr(0, slash);
        if (file_exists(dir + "/weight.txt")) wgt = dir + "/weight.txt";
        if (k <= 0) { fprintf(stderr, "Invalid input: num_partitions must be positive.\n"); return 1; }
    } else {
        usage(argv[0]);
        return 1;
    }
    double t0 = now();
    std::vector<int64_t> rp, ci64, ew64;
    std::string err;
    if (!read_ints(row, nv >= 0 ? nv + 1 : -1, rp, err)) { fprintf(stderr, "%s\n", err.c_str()); return 2; }
    if (rp.size() < 2) { fprintf(stderr, "%s: need at least two row pointers\n", row.c_str()); return 2; }
    const int64_t n = (int64_t)rp.size() - 1;
    if (ne < 0) ne = rp.back();
    if (!read_ints(col, ne, ci64, err)) { fprintf(stderr, "%s\n", err.c_str()); return 2; }
    bool have_w = !wgt.empty();
    if (have_w && !read_ints(wgt, ne, ew64, err)) { fprintf(stderr, "%s\n", err.c_str()); return 2; }
    if (rp.back() != ne) {
        fprintf(stderr, "row pointers end at %lld but %lld column entries were given\n",
                (long long)rp.back(), (long long)ne);
        return 1;
    }
    std::vector<int32_t> ci(ci64.begin(), ci64.end()), ew;
    if (have_w) ew.assign(ew64.begin(), ew64.end());
    const double t_read = now() - t0;
    if (parse_only) {
        uint64_t h = 1469598103934665603ull;   // FNV-1a over the parsed integers
        auto mixin = [&](int64_t x) { h = (h ^ (uint64_t)x) * 1099511628211ull; };
        for (int64_t x : rp) mixin(x);
        for (int32_t x : ci) mixin(x);
        for (int32_t x : ew) mixin(x);
        printf("parsed n=%lld m=%lld weights=%d checksum=%016llx seconds=%.6f\n", (long long)n, (long long)ne,
               have_w ? 1 : 0, (unsigned long long)h, t_read);
        return 0;
    }

    std::vector<int32_t> part((size_t)n);
    gp_stats st;
    memset(&st, 0, sizeof st);
    const double t1 = now();
    int rc = gp_partition_ex(n, rp.data(), ci.data(), nullptr, have_w ? ew.data() : nullptr, (int32_t)k, imbalance,
                             seed, part.data(), nullptr, &st, nullptr, nullptr);
    const double t_part = now() - t1;
    if (rc != GP_OK) {
        fprintf(stderr, "partitioning failed (%d): %s\n", rc, gp_last_error());
        return rc == GP_EINVAL ? 1 : 3;
    }
    const double t2 = now();
    std::vector<std::vector<int64_t>> by_part((size_t)k);
    for (int64_t v = 0; v < n; ++v) by_part[part[v]].push_back(v);
    // formatted into one buffer (std::to_chars) and written at once
    std::vector<char> obuf;
    obuf.reserve((size_t)n * 9 + (size_t)k * 24);
    auto put_int = [&](int64_t x) {
        char tmp[24];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, x);
        obuf.insert(obuf.end(), tmp, r.ptr);
    };
    auto put_str = [&](const char* z) { obuf.insert(obuf.end(), z, z + strlen(z)); };
    for (int64_t q = 0; q < k; ++q) {
        put_str("Partition ");
        put_int(q);
        put_str(": ");
        const auto& vs = by_part[q];
        for (size_t i = 0; i < vs.size(); ++i) {
            put_int(vs[i]);
            if (i + 1 < vs.size()) obuf.push_back(',');
        }
        obuf.push_back('\n');
    }
    FILE* fo = fopen(out_path.c_str(), "wb");
    if (!fo) { fprintf(stderr, "Error: Cannot open %s for writing\n", out_path.c_str()); return 2; }
    fwrite(obuf.data(), 1, obuf.size(), fo);
    fclose(fo);
    if (!part_list.empty()) {
        obuf.clear();
        for (int64_t v = 0; v < n; ++v) { put_int(part[v]); obuf.push_back('\n'); }
        FILE* fp = fopen(part_list.c_str(), "wb");
        if (!fp) { fprintf(stderr, "Error: Cannot open %s for writing\n", part_list.c_str()); return 2; }
        fwrite(obuf.data(), 1, obuf.size(), fp);
        fclose(fp);
    }
    const double t_write = now() - t2;
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);

    printf("Graph Detail ******************************************************\n");
    printf("%-35s%10lld\n", "Number of Vertices:", (long long)n);
    printf("%-35s%10lld\n", "Number of Edges:", (long long)ne);
    printf("%-35s%10lld\n\n", "Number of Partitions:", (long long)k);
    printf("K-way GPU with Deterministic Refinement Details *******************\n");
    printf("%-35s%10lld\n", "Edge Cut:", (long long)st.cut);
    printf("Partition Sizes:\n");
    for (int64_t q = 0; q < k; ++q) printf("  Partition %lld:%10zu vertices\n", (long long)q, by_part[q].size());
    printf("%-35s%9.1f%%\n", "Balance Constraint:", imbalance * 100.0f);
    printf("%-35s%10.4f\n", "Imbalance (max part / average - 1):", st.imbalance);
    printf("%-35s%10d vertices\n", "Coarsest Graph:", st.coarsest_n);
    printf("%-35s%10d\n", "Levels:", st.levels);
    printf("%-35s%10s\n\n", "Output File:", out_path.c_str());
    printf("Timing Breakdown **************************************************\n");
    printf("%-35s%10.6fs\n", "  - File Reading Time:", t_read);
    printf("%-35s%10.6fs\n", "  - Host to Device Transfer:", st.ms_h2d / 1e3);
    printf("%-35s%10.6fs\n", "  - Coarsening Kernel Time:", st.ms_coarsen / 1e3);
    printf("%-35s%10.6fs\n", "  - Initial Partition Time:", st.ms_initial / 1e3);
    printf("%-35s%10.6fs\n", "  - Refinement + Projection Time:", st.ms_refine / 1e3);
    printf("%-35s%10.6fs\n", "  - Device to Host Transfer:", st.ms_d2h / 1e3);
    printf("%-35s%10.6fs\n", "Total Partition Time (device):", st.ms_total / 1e3);
    printf("%-35s%10.6fs\n", "Library Call Wall Time:", t_part);
    printf("%-35s%10.6fs\n\n", "  - Partition File Write Time:", t_write);
    printf("Memory Information ************************************************\n");
    printf("%-35s%10.2f MB\n\n", "Device Memory In Use:", (double)(totalb - freeb) / (1024.0 * 1024.0));
    return 0;
}

// gconvert -- SNAP edge list (.txt or .txt.gz) -> binary CSR (.bin), with the
// reference's command line and output (src/graph/convert.cpp:11-45):
//
//   gconvert <in.txt.gz> <out.bin> --directed|--undirected [--csv results/convert_stats.csv]
//
// The conversion runs on the GPU (gb_convert_snap_gpu: parsing, relabelling
// and compaction on the device; identical .bin).  Exit codes: 0 ok, 1 on a
// conversion error (message on stderr), 2 on a usage error.  The CSV gets one
// row per output file (keyed by its stem), replacing an older row.
#include <sys/resource.h>

#include <cstdio>
#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "graph_b200.h"

namespace {

// "--k v", "--k=v", bare "--flag", positionals (src/util/args.hpp:11-47).
struct Args {
    std::map<std::string, std::string> kv;
    std::vector<std::string> pos;
    Args(int argc, char** argv) {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a.rfind("--", 0) != 0) {
                pos.push_back(a);
                continue;
            }
            a = a.substr(2);
            const size_t eq = a.find('=');
            if (eq != std::string::npos) kv[a.substr(0, eq)] = a.substr(eq + 1);
            else if (i + 1 < argc && std::string(argv[i + 1]).rfind("--", 0) != 0) kv[a] = argv[++i];
            else kv[a] = "";
        }
    }
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    std::string get(const std::string& k, const std::string& d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
};

// "data/web-Google.bin" -> "web-Google" (src/util/csv.hpp:11-16)
std::string stem(const std::string& path) {
    const size_t s = path.find_last_of('/');
    const std::string base = s == std::string::npos ? path : path.substr(s + 1);
    const size_t d = base.find('.');
    return d == std::string::npos ? base : base.substr(0, d);
}

// Keep the header and every row whose first field is not key, then append row
// (src/util/csv.hpp:18-37).
void csvUpsert(const std::string& path, const std::string& header, const std::string& key, const std::string& row) {
    std::vector<std::string> keep;
    {
        std::ifstream in(path);
        std::string line;
        bool first = true;
        while (std::getline(in, line)) {
            if (first) {
                first = false;
                continue;
            }
            if (!line.empty() && line.substr(0, line.find(',')) != key) keep.push_back(line);
        }
    }
    std::ofstream out(path, std::ios::trunc);
    out << header << '\n';
    for (auto& l : keep) out << l << '\n';
    out << row << '\n';
}

}  // namespace

int main(int argc, char** argv) {
    Args args(argc, argv);
    if (args.pos.size() != 2 || args.has("directed") == args.has("undirected")) {
        std::fprintf(stderr, "usage: gconvert <in.txt.gz> <out.bin> --directed|--undirected [--csv path]\n");
        return 2;
    }
    const bool directed = args.has("directed");
    gb_convert_stats st{};
    if (gb_convert_snap_gpu(args.pos[0].c_str(), args.pos[1].c_str(), directed ? 1 : 0, &st) != GB_OK) {
        std::fprintf(stderr, "gconvert: %s\n", gb_last_error());
        return 1;
    }
    struct rusage ru;
    getrusage(RUSAGE_SELF, &ru);
    const double rssMb = ru.ru_maxrss / 1024.0;  // Linux reports KiB
    std::printf("%s -> %s (%s)\n", args.pos[0].c_str(), args.pos[1].c_str(), directed ? "directed" : "undirected");
    std::printf("  lines %llu, raw max id %llu, n %llu\n", (unsigned long long)st.lines,
                (unsigned long long)st.raw_max_id, (unsigned long long)st.n);
    std::printf("  entries %llu before dedup/self-loops, %llu after\n", (unsigned long long)st.m_before,
                (unsigned long long)st.m);
    std::printf("  %.2f s, peak RSS %.1f MB\n", st.seconds, rssMb);
    const std::string csv = args.get("csv", "results/convert_stats.csv");
    if (!csv.empty()) {
        const std::string name = stem(args.pos[1]);
        char row[512];
        std::snprintf(row, sizeof row, "%s,%d,%llu,%llu,%llu,%llu,%.2f,%.1f", name.c_str(), directed ? 1 : 0,
                      (unsigned long long)st.lines, (unsigned long long)st.n, (unsigned long long)st.m_before,
                      (unsigned long long)st.m, st.seconds, rssMb);
        csvUpsert(csv, "dataset,directed,lines,n,m_before,m,seconds,peak_rss_mb", name, row);
    }
    return 0;
}

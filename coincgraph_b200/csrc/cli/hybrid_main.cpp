// hybrid_main.cpp - drop-in hybrid_bfs / hybrid_sssp / hybrid_cc / hybrid_pr.
//
// Built four times (-DCIG_TOOL_BFS/SSSP/CC/PR=1) against libcig (include/cig.h).
// Keeps the reference tools' command line (gflags syntax, every flag of
// include/utils/app_skeleton.h:42-90 and the per-sample flags), their input
// files (graph.txt `u v [w]` per line, updates.txt `a|d u v w`, batches.txt
// `adds dels`), their per-batch flow (deletion phase, optional delete-stage
// check, insertion phase, cache service, batch check: samples/hybrid_sssp/
// hybrid_sssp.cu:417-558) and their log lines ([TIMER], [*-CHECK],
// "Overall: Test ...").  The --check work restates the reference's checks
// (samples/hybrid_sssp/hybrid_sssp.cu:211-330, samples/hybrid_cc/
// hybrid_cc_host.cu:8-32, samples/hybrid_pr/hybrid_pr_host.cu:9-56) and runs
// outside the batch timer, as in the reference.
//
// Deliberate differences: every failure, including a failed BFS/SSSP check,
// gives a non-zero exit status (the reference's BFS/SSSP return 0:
// app_skeleton.h:154-155); blank lines in input files are skipped; an
// update whose destination is out of range is rejected as invalid instead of
// being stored.
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>

#include <sys/stat.h>
#include <vector>

#include "cig.h"

#if defined(CIG_TOOL_BFS)
static const char *kName = "bfs", *kUpper = "BFS";
static const int kAlgo = CIG_BFS;
#elif defined(CIG_TOOL_SSSP)
static const char *kName = "sssp", *kUpper = "SSSP";
static const int kAlgo = CIG_SSSP;
#elif defined(CIG_TOOL_CC)
static const char *kName = "cc", *kUpper = "CC";
static const int kAlgo = CIG_CC;
#elif defined(CIG_TOOL_PR)
static const char *kName = "pr", *kUpper = "PR";
static const int kAlgo = CIG_PR;
#else
#error "define one of CIG_TOOL_BFS/SSSP/CC/PR"
#endif

static const uint32_t kInf = 0xFFFFFFFFu;

// ------------------------------------------------------------------ logging

#define LOG(...) log_line(__LINE__, __VA_ARGS__)

static void log_line(int line, const char *fmt, ...) {
    std::printf("hybrid_main.cpp:%d HOST: ", line);
    va_list ap;
    va_start(ap, fmt);
    std::vprintf(fmt, ap);
    va_end(ap);
    std::fflush(stdout);
}

struct Stopwatch {
    std::chrono::steady_clock::time_point t0;
    double acc = 0;
    bool running = false;
    explicit Stopwatch(bool start = false) {
        if (start) this->start();
    }
    void start() {
        t0 = std::chrono::steady_clock::now();
        running = true;
    }
    void stop() {
        if (running) acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        running = false;
    }
    double ms() const { return acc; }
};

// ------------------------------------------------------------------ flags

struct Flag {
    std::string value;
    char type;  // 's' string, 'i' int, 'd' double, 'b' bool
    std::string help;
};

static std::map<std::string, Flag> g_flags;

static void def(const char *name, char type, const char *value, const char *help) {
    g_flags[name] = Flag{value, type, help};
}

static void define_flags() {
    // include/utils/app_skeleton.h:42-90
    def("interactive", 'b', "false", "Run an interactive session (not supported)");
    def("cmdfile", 's', "", "A file with commands to execute (not supported)");
    def("prio_delta", 'i', "0", "The soft priority delta (accepted, no effect)");
    def("edge_factor", 'd', "1.0", "Unvisited edges = edge_factor * nedges (accepted, no effect)");
    def("alpha", 'd', "0.8", "DO heuristic parameter (accepted, no effect)");
    def("beta", 'd', "0.4", "DO heuristic parameter (accepted, no effect)");
    def("output", 's', "", "File to store output to");
    def("check", 'b', "true", "Check results");
    def("verbose", 'b', "true", "Verbose prints");
    def("lb_push", 's', "", "load-balancing policy for push (accepted, no effect)");
    def("lb_pull", 's', "", "load-balancing policy for pull (accepted, no effect)");
    def("graphfile", 's', "", "A file with a graph (market_big: `u v [w]` per line)");
    def("format", 's', "gr", "graph format (market_big; others are read the same way)");
    def("json", 's', "", "output running data as json format (accepted, no effect)");
    def("stats", 'b', "false", "Print graph statistics");
    def("gen_graph", 'b', "false", "Generate a random graph (not supported)");
    def("gen_nnodes", 'i', "100000", "(accepted, no effect)");
    def("gen_factor", 'i', "10", "(accepted, no effect)");
    def("gen_weights", 'b', "false", "(accepted, no effect)");
    def("gen_weight_range", 'i', "100", "(accepted, no effect)");
    def("block_size", 'i', "512", "Block size for traversal kernels (accepted, no effect)");
    def("wl_alloc_factor", 'd', "0.2", "Worklist allocation factor (accepted, no effect)");
    def("n_stream", 'i', "3", "the number of stream (accepted, no effect)");
    def("SEGMENT", 'i', "1", "the number of segment (1..512, validated, no effect)");
    def("priority_a", 'i', "1", "priority (accepted, no effect)");
    def("hybrid", 'i', "0", "0:zerocopy 1:explicit 2:hybrid (accepted, no effect)");
    def("weight_num", 'i', "0", "1: weights synthesised from ids (weights never reach the kernels)");
    def("weight", 'b', "true", "update records carry a weight column");
    def("updatefile", 's', "", "A file with the update records");
    def("update_size", 's', "", "A file with the per-batch `adds dels` sizes");
    def("cache", 'd', "4", "HBM edge-cache budget in GiB of 4-byte slots");
    def("cache_compat", 'b', "false", "map --cache through the reference's slot table (graph_datum.cuh:158-170)");
    def("index_budget", 'd', "0", "device GiB for the two position-index tables (0: a quarter of free memory each)");
    def("top_ranks", 'i', "10", "(accepted, no effect)");
    def("print_ranks", 'b', "false", "(accepted, no effect)");
    def("device", 'i', "0", "CUDA device ordinal");
    def("write_cigb", 'b', "false", "after parsing graphfile, write the binary sidecar graphfile.cigb");
    def("autotune", 'b', "false", "choose the closures' launch shape on the loaded graph (cig_autotune)");
#if defined(CIG_TOOL_PR)
    // samples/hybrid_pr/hybrid_pr.cu:21-24
    def("pr_max_batches", 'i', "10", "Maximum PR update batches (0 for static PR)");
    def("pr_max_rounds", 'i', "100", "Maximum PR rounds per initialization/batch (1..100)");
    def("error", 'd', "0.000001", "Absolute signed PR residual threshold");
    def("sparse", 'b', "false", "Compatibility flag; PR always uses sparse residual frontiers");
    def("pr_fp64", 'b', "false", "FP64 ranks and residuals (default FP32 ranks with Kahan sums)");
#else
    // samples/hybrid_{bfs,sssp,cc}/*.cu:20-27
    def("source_node", 'i', "0", "The source node (clamped to [0, nnodes-1]; CC ignores it)");
    def("weight_u255", 'b', "false", "SSSP: edge weights uniform in [1, 255] (extension; default (u+v)%128+1)");
    def("sparse", 'b', "false", "use async/push/dd + fusion for high-diameter (accepted, no effect)");
    def((std::string(kName) + "_max_batches").c_str(), 'i', "10", "Maximum number of update batches");
    def((std::string(kName) + "_print_checksum").c_str(), 'b', "false", "Print final checksums");
#endif
}

static bool parse_bool(const std::string &s, bool &out) {
    if (s == "true" || s == "1" || s == "yes" || s == "t" || s == "y") return out = true, true;
    if (s == "false" || s == "0" || s == "no" || s == "f" || s == "n") return out = false, true;
    return false;
}

static void usage_and_exit(const char *argv0, int code) {
    std::printf("%s: drop-in hybrid_%s on libcig (%s)\n\nFlags:\n", argv0, kName, cig_version());
    for (const auto &f : g_flags)
        std::printf("  --%s (%s) default: \"%s\"\n", f.first.c_str(), f.second.help.c_str(), f.second.value.c_str());
    std::exit(code);
}

static void parse_args(int argc, char **argv) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a.size() < 2 || a[0] != '-') {
            std::fprintf(stderr, "ERROR: unexpected argument '%s'\n", a.c_str());
            std::exit(1);
        }
        a = a.substr(a[1] == '-' ? 2 : 1);
        if (a == "help" || a == "helpfull") usage_and_exit(argv[0], 0);
        std::string name = a, value;
        bool has_value = false;
        const size_t eq = a.find('=');
        if (eq != std::string::npos) {
            name = a.substr(0, eq);
            value = a.substr(eq + 1);
            has_value = true;
        }
        auto it = g_flags.find(name);
        if (it == g_flags.end() && !has_value && name.rfind("no", 0) == 0) {
            auto jt = g_flags.find(name.substr(2));
            if (jt != g_flags.end() && jt->second.type == 'b') {
                jt->second.value = "false";
                continue;
            }
        }
        if (it == g_flags.end()) {
            std::fprintf(stderr, "ERROR: unknown command line flag '%s'\n", name.c_str());
            std::exit(1);
        }
        Flag &f = it->second;
        if (!has_value) {
            if (f.type == 'b') {
                value = "true";
            } else if (i + 1 < argc) {
                value = argv[++i];
            } else {
                std::fprintf(stderr, "ERROR: flag '%s' is missing its argument\n", name.c_str());
                std::exit(1);
            }
        }
        bool b;
        char *end = nullptr;
        errno = 0;
        if ((f.type == 'b' && !parse_bool(value, b)) ||
            (f.type == 'i' && (std::strtol(value.c_str(), &end, 10), end == value.c_str() || *end || errno)) ||
            (f.type == 'd' && (std::strtod(value.c_str(), &end), end == value.c_str() || *end || errno))) {
            std::fprintf(stderr, "ERROR: illegal value '%s' specified for flag '%s'\n", value.c_str(), name.c_str());
            std::exit(1);
        }
        f.value = value;
    }
}

static std::string S(const char *n) { return g_flags.at(n).value; }
static long long I(const char *n) { return std::strtoll(g_flags.at(n).value.c_str(), nullptr, 10); }
static double D(const char *n) { return std::strtod(g_flags.at(n).value.c_str(), nullptr); }
static bool B(const char *n) {
    bool b = false;
    parse_bool(g_flags.at(n).value, b);
    return b;
}
static std::string app_flag(const char *suffix) { return std::string(kName) + suffix; }

// ------------------------------------------------------------------ input

struct Fail : std::runtime_error {
    using std::runtime_error::runtime_error;
};

static std::vector<char> read_file(const std::string &path) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw Fail("cannot open " + path);
    std::vector<char> buf;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(static_cast<size_t>(std::max(0L, size)) + 1);
    const size_t got = size > 0 ? std::fread(buf.data(), 1, static_cast<size_t>(size), f) : 0;
    std::fclose(f);
    buf.resize(got);
    buf.push_back('\n');
    return buf;
}

static inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Parse an unsigned decimal; returns false if none.
static inline bool parse_u64(const char *&p, const char *end, uint64_t &out) {
    while (p < end && is_space(*p)) ++p;
    if (p >= end || *p < '0' || *p > '9') return false;
    uint64_t v = 0;
    while (p < end && *p >= '0' && *p <= '9') v = v * 10 + static_cast<uint64_t>(*p++ - '0');
    out = v;
    return true;
}

// graph.txt: one edge `u v [w]` per line, rows keep file order
// (ReadGraphMarket_bigdata, src/utils/parser.cpp:292-402).  Parsed in
// parallel over line-aligned chunks.
struct EdgeList {
    uint32_t n = 0;
    std::vector<uint32_t> src, dst;
};

// Binary sidecar `graphfile.cigb`: "CIGB0001", n (u32), m (u64), then the
// m sources and m destinations (u32) in file order.  Read instead of the
// text when it is at least as new as the text file; written by --write_cigb.
static const char kCigbMagic[8] = {'C', 'I', 'G', 'B', '0', '0', '0', '1'};

static bool read_cigb(const std::string &text_path, EdgeList &el) {
    const std::string path = text_path + ".cigb";
    struct stat st_t {}, st_b {};
    if (::stat(path.c_str(), &st_b) != 0) return false;
    if (::stat(text_path.c_str(), &st_t) == 0 && st_b.st_mtime < st_t.st_mtime) return false;
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char magic[8];
    uint32_t n = 0;
    uint64_t m = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCigbMagic, 8) == 0 &&
              std::fread(&n, sizeof(n), 1, f) == 1 && std::fread(&m, sizeof(m), 1, f) == 1;
    if (ok) {
        el.n = n;
        el.src.resize(m);
        el.dst.resize(m);
        ok = std::fread(el.src.data(), sizeof(uint32_t), m, f) == m && std::fread(el.dst.data(), sizeof(uint32_t), m, f) == m;
    }
    std::fclose(f);
    if (!ok) throw Fail("corrupt binary graph " + path);
    for (uint64_t i = 0; i < m; ++i)
        if (el.src[i] >= n || el.dst[i] >= n) throw Fail("binary graph " + path + " has an id >= n");
    return true;
}

static void write_cigb(const std::string &text_path, const EdgeList &el) {
    const std::string path = text_path + ".cigb";
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw Fail("cannot write " + path);
    const uint64_t m = el.src.size();
    bool ok = std::fwrite(kCigbMagic, 1, 8, f) == 8 && std::fwrite(&el.n, sizeof(el.n), 1, f) == 1 &&
              std::fwrite(&m, sizeof(m), 1, f) == 1 && std::fwrite(el.src.data(), sizeof(uint32_t), m, f) == m &&
              std::fwrite(el.dst.data(), sizeof(uint32_t), m, f) == m;
    ok = std::fclose(f) == 0 && ok;
    if (!ok) throw Fail("cannot write " + path);
}

static EdgeList read_graph(const std::string &path) {
    {
        EdgeList el;
        if (read_cigb(path, el)) return el;
    }
    const std::vector<char> buf = read_file(path);
    const char *base = buf.data();
    const size_t size = buf.size();
    const unsigned T = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<size_t> cut(T + 1, size);
    cut[0] = 0;
    for (unsigned t = 1; t < T; ++t) {
        size_t c = size * t / T;
        while (c < size && base[c - 1] != '\n') ++c;
        cut[t] = std::max(c, cut[t - 1]);
    }
    std::vector<std::vector<uint32_t>> ps(T), pd(T);
    std::vector<uint64_t> pmax(T, 0);
    std::vector<std::string> perr(T);
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t) {
        pool.emplace_back([&, t] {
            const char *p = base + cut[t], *end = base + cut[t + 1];
            while (p < end) {
                const char *eol = static_cast<const char *>(std::memchr(p, '\n', end - p));
                if (!eol) eol = end;
                const char *q = p;
                while (q < eol && is_space(*q)) ++q;
                if (q < eol && *q != '#' && *q != '%') {
                    uint64_t u, v;
                    if (!parse_u64(q, eol, u) || !parse_u64(q, eol, v)) {
                        perr[t] = "malformed graph line: " + std::string(p, eol);
                        return;
                    }
                    if (u >= kInf || v >= kInf) {
                        perr[t] = "vertex id exceeds 2^32-2";
                        return;
                    }
                    ps[t].push_back(static_cast<uint32_t>(u));
                    pd[t].push_back(static_cast<uint32_t>(v));
                    pmax[t] = std::max(pmax[t], std::max(u, v));
                }
                p = eol + 1;
            }
        });
    }
    for (auto &th : pool) th.join();
    EdgeList el;
    uint64_t m = 0, maxid = 0;
    bool any = false;
    for (unsigned t = 0; t < T; ++t) {
        if (!perr[t].empty()) throw Fail(perr[t]);
        m += ps[t].size();
        if (!ps[t].empty()) any = true;
        maxid = std::max(maxid, pmax[t]);
    }
    el.n = any ? static_cast<uint32_t>(maxid + 1) : 0;
    el.src.reserve(m);
    el.dst.reserve(m);
    for (unsigned t = 0; t < T; ++t) {
        el.src.insert(el.src.end(), ps[t].begin(), ps[t].end());
        el.dst.insert(el.dst.end(), pd[t].begin(), pd[t].end());
    }
    return el;
}

// batches.txt `adds dels` and updates.txt `a|d u v [w]` (include/framework/
// Loader.h:28-97): batch i takes the next `dels` 'd' records and the next
// `adds` 'a' records in file order.
struct Updates {
    std::vector<std::pair<uint64_t, uint64_t>> sizes;  // (adds, dels)
    std::vector<uint32_t> du, dv, au, av;
};

static Updates read_updates(const std::string &update_path, const std::string &size_path) {
    Updates up;
    {
        const std::vector<char> buf = read_file(size_path);
        const char *p = buf.data(), *end = p + buf.size();
        while (p < end) {
            const char *eol = static_cast<const char *>(std::memchr(p, '\n', end - p));
            if (!eol) eol = end;
            const char *q = p;
            uint64_t a, d;
            if (parse_u64(q, eol, a)) {
                if (!parse_u64(q, eol, d)) throw Fail("malformed batch-size line: " + std::string(p, eol));
                up.sizes.push_back({a, d});
            }
            p = eol + 1;
        }
    }
    const std::vector<char> buf = read_file(update_path);
    const char *p = buf.data(), *end = p + buf.size();
    while (p < end) {
        const char *eol = static_cast<const char *>(std::memchr(p, '\n', end - p));
        if (!eol) eol = end;
        const char *q = p;
        while (q < eol && is_space(*q)) ++q;
        if (q < eol) {
            const char type = *q++;
            uint64_t u, v;
            if ((type != 'a' && type != 'd') || !parse_u64(q, eol, u) || !parse_u64(q, eol, v) || u >= kInf ||
                v >= kInf)
                throw Fail("malformed update line: " + std::string(p, eol));
            (type == 'a' ? up.au : up.du).push_back(static_cast<uint32_t>(u));
            (type == 'a' ? up.av : up.dv).push_back(static_cast<uint32_t>(v));
        }
        p = eol + 1;
    }
    uint64_t ta = 0, td = 0;
    for (const auto &s : up.sizes) ta += s.first, td += s.second;
    if (ta > up.au.size() || td > up.dv.size())
        throw Fail("batch sizes ask for more records than the update file holds");
    return up;
}

// ------------------------------------------------------------------ engine

static cig_handle *g_h = nullptr;

static void ck(int rc, const char *what) {
    if (rc != CIG_OK) throw Fail(std::string(what) + " failed: " + cig_last_error(g_h));
}

struct Csr {
    std::vector<uint64_t> xadj;
    std::vector<uint32_t> adj;
};

static Csr export_graph(uint32_t n) {
    Csr g;
    g.xadj.resize(static_cast<size_t>(n) + 1);
    ck(cig_export_csr(g_h, g.xadj.data(), nullptr), "cig_export_csr");
    g.adj.resize(std::max<uint64_t>(g.xadj[n], 1));
    ck(cig_export_csr(g_h, g.xadj.data(), g.adj.data()), "cig_export_csr");
    return g;
}

static bool g_weight_u255 = false;  // --weight_u255 (hybrid_sssp)

static uint64_t weight(uint32_t u, uint32_t v) {
#if defined(CIG_TOOL_SSSP)
    if (g_weight_u255) {  // the library's CIG_FLAG_WEIGHT_U255 function (lowbias32, C. Wellons)
        uint32_t x = u * 0x9E3779B1u + v * 0x85EBCA77u;
        x ^= x >> 16;
        x *= 0x7FEB352Du;
        x ^= x >> 15;
        x *= 0x846CA68Bu;
        x ^= x >> 16;
        return 1u + x % 255u;
    }
    return (static_cast<uint64_t>(u) + v) % 128 + 1;
#else
    (void)u;
    (void)v;
    return 1;
#endif
}

// ------------------------------------------------------------------ checks

struct Bellman {
    uint64_t relaxable = 0, missing = 0;
    uint32_t first_src = kInf, first_dst = kInf, first_missing = kInf;
};

static Bellman check_bellman(const Csr &g, const std::vector<uint32_t> &dist, uint32_t source) {
    Bellman r;
    const uint32_t n = static_cast<uint32_t>(dist.size());
    std::vector<uint8_t> tight(n, 0);
    if (source < n) tight[source] = 1;
    for (uint32_t s = 0; s < n; ++s) {
        if (dist[s] == kInf) continue;
        for (uint64_t e = g.xadj[s]; e < g.xadj[s + 1]; ++e) {
            const uint32_t d = g.adj[e];
            if (d >= n) continue;
            const uint64_t cand = static_cast<uint64_t>(dist[s]) + weight(s, d);
            if (dist[d] != kInf && cand == dist[d]) tight[d] = 1;
            if (cand < dist[d]) {
                if (!r.relaxable) r.first_src = s, r.first_dst = d;
                ++r.relaxable;
            }
        }
    }
    for (uint32_t v = 0; v < n; ++v)
        if (dist[v] != kInf && !tight[v]) {
            if (!r.missing) r.first_missing = v;
            ++r.missing;
        }
    return r;
}

struct Witness {
    uint64_t invalid = 0, missing_edges = 0, wrong = 0;
    uint32_t first_vertex = kInf, first_parent = kInf;
};

static Witness check_parents(const Csr &g, const std::vector<uint32_t> &dist, const std::vector<uint32_t> &par,
                             uint32_t source) {
    Witness r;
    const uint32_t n = static_cast<uint32_t>(dist.size());
    for (uint32_t v = 0; v < n; ++v) {
        if (v == source || dist[v] == kInf) continue;
        const uint32_t p = par[v];
        bool valid = p < n && dist[p] != kInf;
        if (valid) {
            bool exists = false;
            for (uint64_t e = g.xadj[p]; e < g.xadj[p + 1] && !exists; ++e) exists = g.adj[e] == v;
            const bool matches = static_cast<uint64_t>(dist[p]) + weight(p, v) == dist[v];
            if (!exists)
                ++r.missing_edges;
            else if (!matches)
                ++r.wrong;
            valid = exists && matches;
        }
        if (!valid) {
            if (!r.invalid) r.first_vertex = v, r.first_parent = p;
            ++r.invalid;
        }
    }
    return r;
}

static uint64_t checksum(const std::vector<uint32_t> &vals) {
    uint64_t h = 1469598103934665603ull;
    for (uint32_t v = 0; v < vals.size(); ++v) {
        if (vals[v] == kInf) continue;
        h ^= static_cast<uint64_t>(v) + 0x9e3779b97f4a7c15ull + (static_cast<uint64_t>(vals[v]) << 6) +
             (static_cast<uint64_t>(vals[v]) >> 2);
        h *= 1099511628211ull;
    }
    return h;
}

static uint64_t cc_errors(const Csr &g, const std::vector<uint32_t> &labels) {
    const uint32_t n = static_cast<uint32_t>(labels.size());
    std::vector<uint32_t> expect(n, kInf), stack;
    for (uint32_t seed = 0; seed < n; ++seed) {
        if (expect[seed] != kInf) continue;
        expect[seed] = seed;
        stack.push_back(seed);
        while (!stack.empty()) {
            const uint32_t u = stack.back();
            stack.pop_back();
            for (uint64_t e = g.xadj[u]; e < g.xadj[u + 1]; ++e) {
                const uint32_t v = g.adj[e];
                if (expect[v] != kInf) continue;
                expect[v] = seed;
                stack.push_back(v);
            }
        }
    }
    uint64_t err = 0;
    for (uint32_t v = 0; v < n; ++v) err += labels[v] != expect[v];
    return err;
}

static bool pr_check(const Csr &g, const std::vector<float> &rank, const std::vector<float> &res, double eps,
                     const char *stage, int batch) {
    const size_t n = rank.size();
    auto multiply = [&](const std::vector<double> &x, std::vector<double> &next) {
        std::fill(next.begin(), next.end(), 0.15);
        for (size_t s = 0; s < n; ++s) {
            const uint64_t d = g.xadj[s + 1] - g.xadj[s];
            if (!d) continue;
            const double c = 0.85 * x[s] / static_cast<double>(d);
            for (uint64_t e = g.xadj[s]; e < g.xadj[s + 1]; ++e) next[g.adj[e]] += c;
        }
    };
    std::vector<double> ref(n, 0), next(n), actual(rank.begin(), rank.end());
    bool converged = false;
    for (unsigned round = 0; round < 10000; ++round) {
        multiply(ref, next);
        double delta = 0;
        for (size_t v = 0; v < n; ++v) delta += std::abs(next[v] - ref[v]);
        ref.swap(next);
        if (delta <= 1e-12 * std::max<size_t>(1, n)) {
            converged = true;
            break;
        }
    }
    multiply(actual, next);
    double l1 = 0, defect = 0, max_res = 0, max_err = 0, mass = 0;
    bool finite = true;
    for (size_t v = 0; v < n; ++v) {
        finite &= std::isfinite(rank[v]) && std::isfinite(res[v]) && rank[v] >= -eps;
        const double err = std::abs(rank[v] - ref[v]);
        l1 += err;
        max_err = std::max(max_err, err);
        defect += std::abs(next[v] - rank[v] - res[v]);
        max_res = std::max(max_res, static_cast<double>(std::abs(res[v])));
        mass += std::abs(ref[v]);
    }
    const double roundoff = 64 * std::numeric_limits<float>::epsilon() * std::max(1.0, mass);
    const double bound = (n * eps + roundoff) / 0.15;
    const bool ok = finite && converged && l1 <= bound && defect <= roundoff && max_res <= static_cast<float>(eps);
    std::printf("[PR-CHECK] stage=%s batch=%d %s l1_error=%.9g bound=%.9g max_error=%.9g invariant_l1=%.9g "
                "max_residual=%.9g\n",
                stage, batch, ok ? "passed" : "failed", l1, bound, max_err, defect, max_res);
    return ok;
}

// ------------------------------------------------------------------ main

static std::vector<uint32_t> values(uint32_t n) {
    std::vector<uint32_t> v(n);
    ck(cig_get_values(g_h, v.data()), "cig_get_values");
    return v;
}

static std::vector<uint32_t> parents(uint32_t n) {
    std::vector<uint32_t> v(n);
    ck(cig_get_parents(g_h, v.data()), "cig_get_parents");
    return v;
}

static bool run() {
    const std::string graphfile = S("graphfile");
    if (graphfile.empty()) throw Fail("A Graph File must be provided");
    if (I("SEGMENT") <= 0 || I("SEGMENT") > 512) throw Fail("SEGMENT must be in [1, 512]");
#if defined(CIG_TOOL_PR)
    const double eps = D("error");
    const long long max_rounds = I("pr_max_rounds");
    const long long max_batches_flag = I("pr_max_batches");
    if (!std::isfinite(eps) || eps <= 0 || !std::isfinite(static_cast<float>(eps)) ||
        static_cast<float>(eps) == 0 || max_batches_flag < 0 || max_rounds <= 0 || max_rounds > 100)
        throw Fail("PR requires finite error > 0, pr_max_batches >= 0 and 1 <= pr_max_rounds <= 100");
#else
    const long long max_batches_flag = I(app_flag("_max_batches").c_str());
    if (max_batches_flag < 0) throw Fail(std::string(kName) + "_max_batches must be nonnegative");
#endif
    const bool have_updates = !S("updatefile").empty();
    if (have_updates != !S("update_size").empty())
        throw Fail("Provide both updatefile and update_size, or neither");
#if defined(CIG_TOOL_BFS) || defined(CIG_TOOL_SSSP)
    if (!have_updates) throw Fail("Update File must be provided");
#endif
    const bool check = B("check");

    std::printf("\nLoading graph %s (%s)\n", graphfile.c_str(), S("format").c_str());
    Stopwatch sw_load(true);
    EdgeList el = read_graph(graphfile);
    if (el.n == 0) throw Fail(std::string(kUpper) + " requires a nonempty graph");
    if (B("write_cigb")) write_cigb(graphfile, el);
    Updates up;
    if (have_updates && max_batches_flag > 0) up = read_updates(S("updatefile"), S("update_size"));

    cig_options o;
    cig_options_default(&o);
    o.algo = kAlgo;
    o.device = static_cast<int32_t>(I("device"));
    o.cache_gib = D("cache");
    o.cache_compat = B("cache_compat") ? 1 : 0;
    o.index_budget_gib = D("index_budget");
#if defined(CIG_TOOL_PR)
    o.pr_epsilon = eps;
    o.pr_max_rounds = static_cast<int32_t>(max_rounds);
    if (B("pr_fp64")) o.flags |= CIG_FLAG_PR_FP64;
#else
#if defined(CIG_TOOL_SSSP)
    g_weight_u255 = B("weight_u255");
    if (g_weight_u255) o.flags |= CIG_FLAG_WEIGHT_U255;
#endif
    const long long src_flag = I("source_node");
    o.source = static_cast<uint32_t>(std::min<long long>(std::max<long long>(0, src_flag), el.n - 1));
#endif
    uint64_t max_phase = 0;
    for (const auto &s : up.sizes) max_phase = std::max(max_phase, std::max(s.first, s.second));
    o.max_batch = static_cast<uint32_t>(std::min<uint64_t>(max_phase, 0x7FFFFFFF));
    if (cig_create(&o, &g_h) != CIG_OK) throw Fail(std::string("cig_create failed: ") + cig_last_error(nullptr));
    ck(cig_load_edges(g_h, el.n, el.src.data(), el.dst.data(), el.src.size()), "cig_load_edges");
    const uint32_t n = el.n;
    const uint64_t m = el.src.size();
    std::vector<uint32_t>().swap(el.src);
    std::vector<uint32_t>().swap(el.dst);
    sw_load.stop();
    cig_graph_info info;
    ck(cig_graph_info_get(g_h, &info), "cig_graph_info_get");
    LOG("[CHUNK-LOAD] edges=%llu capacity_edges=%llu segments=%llu resident_segments=%llu pinned_bytes=%llu\n",
        static_cast<unsigned long long>(m), static_cast<unsigned long long>(info.arena_capacity_edges),
        static_cast<unsigned long long>(info.segments_total), static_cast<unsigned long long>(info.segments_resident),
        static_cast<unsigned long long>(info.pinned_bytes));
    LOG("Load graph time: %f ms (excluded)\n", sw_load.ms());

    Stopwatch sw_init(true);
    ck(cig_init(g_h), "cig_init");
    sw_init.stop();
#if !defined(CIG_TOOL_PR)
    if (B("autotune")) {
        cig_tune_result tr;
        ck(cig_autotune(g_h, &tr), "cig_autotune");
        LOG("[AUTOTUNE] blocks_per_sm=%u split_degree=%u pull_divisor=%u solve_ms=%.3f candidates=%u\n",
            tr.blocks_per_sm, tr.split_degree, tr.pull_divisor, tr.best_ms, tr.candidates);
    }
#endif
    bool success = true;
#if defined(CIG_TOOL_PR)
    LOG("[PR-INITIAL] compute_ms=%.3f alpha=0.85 base=0.15 dangling=drop\n", sw_init.ms());
    auto pr_values = [&](std::vector<float> &r, std::vector<float> &s) {
        r.resize(n);
        s.resize(n);
        ck(cig_get_pr(g_h, r.data(), s.data()), "cig_get_pr");
    };
    std::vector<float> rank, res;
    if (check) {
        pr_values(rank, res);
        if (!pr_check(export_graph(n), rank, res, eps, "initial", -1)) return false;
    }
#else
    LOG("Initial computation: %f ms (excluded)\n", sw_init.ms());
    const uint32_t source = o.source;
#endif
    const uint64_t available = up.sizes.size();
    const uint64_t batches = std::min<uint64_t>(static_cast<uint64_t>(max_batches_flag), available);
#if !defined(CIG_TOOL_PR)
    if (static_cast<uint64_t>(max_batches_flag) > available && have_updates)
        std::cout << "[" << kUpper << "] clamp " << kName << "_max_batches from " << max_batches_flag
                  << " to available update batches " << available << std::endl;
#endif
    uint64_t doff = 0, aoff = 0;
    for (uint64_t b = 0; b < batches; ++b) {
        const uint64_t na = up.sizes[b].first, nd = up.sizes[b].second;
        const uint32_t *du = up.du.data() + doff, *dv = up.dv.data() + doff;
        const uint32_t *au = up.au.data() + aoff, *av = up.av.data() + aoff;
        doff += nd;
        aoff += na;
#if defined(CIG_TOOL_PR)
        Stopwatch timer(true);
        cig_batch_stats st;
        ck(cig_apply_batch(g_h, du, dv, nd, au, av, na, &st), "cig_apply_batch");
        timer.stop();
        LOG("[PR-BATCH] batch=%llu touched_edges=%llu rounds=%llu residual_l1=%.6g missing_deletes=%llu\n",
            static_cast<unsigned long long>(b), static_cast<unsigned long long>(nd + na),
            static_cast<unsigned long long>(st.pr_rounds), st.pr_residual_l1,
            static_cast<unsigned long long>(st.missing_deletes));
        LOG("[TIMER][PR][batch %u] paper_algorithm_ms=%.3f\n", static_cast<unsigned>(b), timer.ms());
        if (check) {
            pr_values(rank, res);
            if (!pr_check(export_graph(n), rank, res, eps, "batch", static_cast<int>(b))) return false;
        }
#else
        std::cout << "batch number " << b << std::endl;
        Stopwatch sw_batch(true), sw_del(true);
        cig_batch_stats sd, si;
        ck(cig_delete_phase(g_h, du, dv, nd, &sd), "cig_delete_phase");
        sw_del.stop();
        sw_batch.stop();
        if (check) {
            const Csr g = export_graph(n);
            const std::vector<uint32_t> vals = values(n);
#if defined(CIG_TOOL_CC)
            const uint64_t errors = cc_errors(g, vals);
            success = success && errors == 0;
            LOG("[CC-DELETE-STAGE-CHECK][batch %u] %s errors=%llu label_checksum=%llu\n", static_cast<unsigned>(b),
                errors == 0 ? "passed" : "failed", static_cast<unsigned long long>(errors),
                static_cast<unsigned long long>(checksum(vals)));
#else
            const std::vector<uint32_t> pars = parents(n);
            const Bellman bc = check_bellman(g, vals, source);
            const Witness pw = check_parents(g, vals, pars, source);
            const bool src_ok = vals[source] == 0;
            const bool ok = src_ok && bc.relaxable == 0 && bc.missing == 0 && pw.invalid == 0;
            success = success && ok;
            LOG("[%s-DELETE-STAGE-CHECK][batch %u] %s source_ok=%d relaxable_edges=%llu missing_tight_witnesses=%llu "
                "invalid_parent_witness=%llu missing_parent_edges=%llu wrong_parent_distances=%llu first_src=%u "
                "first_dst=%u first_missing_witness=%u first_bad_vertex=%u first_bad_parent=%u distance_checksum=%llu\n",
                kUpper, static_cast<unsigned>(b), ok ? "passed" : "failed", src_ok ? 1 : 0,
                static_cast<unsigned long long>(bc.relaxable), static_cast<unsigned long long>(bc.missing),
                static_cast<unsigned long long>(pw.invalid), static_cast<unsigned long long>(pw.missing_edges),
                static_cast<unsigned long long>(pw.wrong), bc.first_src, bc.first_dst, bc.first_missing,
                pw.first_vertex, pw.first_parent, static_cast<unsigned long long>(checksum(vals)));
#endif
        }
        sw_batch.start();
        Stopwatch sw_add(true);
        ck(cig_insert_phase(g_h, au, av, na, &si), "cig_insert_phase");
        sw_add.stop();
        sw_batch.stop();
        LOG("[ATTR][%s][batch %u] deletion=%.3f add=%.3f device_delete=%.3f device_insert=%.3f device_cache=%.3f "
            "affected=%llu missing_deletes=%llu invalid_additions=%llu total=%.3f\n",
            kUpper, static_cast<unsigned>(b), sw_del.ms(), sw_add.ms(), sd.ms_delete, si.ms_insert, si.ms_cache,
            static_cast<unsigned long long>(sd.affected), static_cast<unsigned long long>(sd.missing_deletes),
            static_cast<unsigned long long>(si.invalid_additions), sw_batch.ms());
        LOG("[TIMER][%s][batch %u] total_batch: %.3f ms\n", kUpper, static_cast<unsigned>(b), sw_batch.ms());
        if (check) {
            const Csr g = export_graph(n);
            const std::vector<uint32_t> vals = values(n);
#if defined(CIG_TOOL_CC)
            const uint64_t errors = cc_errors(g, vals);
            success = success && errors == 0;
            LOG("[CC-BATCH-CHECK][batch %u] %s errors=%llu label_checksum=%llu\n", static_cast<unsigned>(b),
                errors == 0 ? "passed" : "failed", static_cast<unsigned long long>(errors),
                static_cast<unsigned long long>(checksum(vals)));
#else
            const std::vector<uint32_t> pars = parents(n);
            const Bellman bc = check_bellman(g, vals, source);
            const Witness pw = check_parents(g, vals, pars, source);
            const bool src_ok = vals[source] == 0;
            const bool ok = src_ok && bc.relaxable == 0 && bc.missing == 0 && pw.invalid == 0;
            success = success && ok;
            LOG("[%s-BATCH-CHECK][batch %u] %s source_ok=%d relaxable_edges=%llu missing_tight_witnesses=%llu "
                "invalid_parent_witness=%llu missing_parent_edges=%llu wrong_parent_distances=%llu "
                "distance_checksum=%llu\n",
                kUpper, static_cast<unsigned>(b), ok ? "passed" : "failed", src_ok ? 1 : 0,
                static_cast<unsigned long long>(bc.relaxable), static_cast<unsigned long long>(bc.missing),
                static_cast<unsigned long long>(pw.invalid), static_cast<unsigned long long>(pw.missing_edges),
                static_cast<unsigned long long>(pw.wrong), static_cast<unsigned long long>(checksum(vals)));
#endif
        }
#endif
    }

#if defined(CIG_TOOL_PR)
    pr_values(rank, res);
    if (check && !pr_check(export_graph(n), rank, res, eps, "final", static_cast<int>(batches))) return false;
    if (!S("output").empty()) {
        std::ofstream out(S("output"));
        if (!out) throw Fail("Cannot write PR output: " + S("output"));
        out << std::setprecision(std::numeric_limits<float>::max_digits10);
        for (uint32_t v = 0; v < n; ++v) out << v << ' ' << rank[v] << ' ' << res[v] << '\n';
        if (!out) throw Fail("Cannot write PR output: " + S("output"));
    }
    LOG("[PR-FINAL] vertices=%u batches=%u\n", n, static_cast<unsigned>(batches));
#else
    const std::vector<uint32_t> vals = values(n);
    uint64_t reachable = 0;
    for (uint32_t v : vals) reachable += v != kInf;
#if defined(CIG_TOOL_CC)
    if (check) {
        const uint64_t errors = cc_errors(export_graph(n), vals);
        success = success && errors == 0;
        LOG("[CC-FINAL-CHECK] %s errors=%llu\n", errors == 0 ? "passed" : "failed",
            static_cast<unsigned long long>(errors));
    }
    if (B(app_flag("_print_checksum").c_str()))
        LOG("[CC-FINAL-CHECK] label_checksum=%llu\n", static_cast<unsigned long long>(checksum(vals)));
    if (!S("output").empty()) {
        std::ofstream out(S("output"));
        for (uint32_t v = 0; v < n; ++v) out << v << ' ' << vals[v] << '\n';
        if (!out) throw Fail("cannot write " + S("output"));
    }
#else
    const std::vector<uint32_t> pars = parents(n);
    if (check) {
        const Csr g = export_graph(n);
        const Bellman bc = check_bellman(g, vals, source);
        const Witness pw = check_parents(g, vals, pars, source);
        const bool src_ok = vals[source] == 0;
        if (src_ok && bc.relaxable == 0 && bc.missing == 0 && pw.invalid == 0) {
            LOG("[%s-BELLMAN-CHECK] passed reachable=%llu relaxable_edges=0 missing_tight_witnesses=0\n", kUpper,
                static_cast<unsigned long long>(reachable));
        } else {
            success = false;
            LOG("[%s-BELLMAN-CHECK] failed source_ok=%d relaxable_edges=%llu missing_tight_witnesses=%llu "
                "invalid_parent_witness=%llu first_missing_witness=%u first_src=%u first_dst=%u\n",
                kUpper, src_ok ? 1 : 0, static_cast<unsigned long long>(bc.relaxable),
                static_cast<unsigned long long>(bc.missing), static_cast<unsigned long long>(pw.invalid),
                bc.first_missing, bc.first_src, bc.first_dst);
        }
    }
    const bool print_checksum = B(app_flag("_print_checksum").c_str());
    LOG("[%s-FINAL-CHECK] final_reachable=%llu checksum=%s\n", kUpper, static_cast<unsigned long long>(reachable),
        print_checksum ? "enabled" : "disabled");
    if (print_checksum) {
        uint64_t pc = 1099511628211ull;
        for (uint32_t v = 0; v < n; ++v) {
            if (vals[v] == kInf) continue;
            pc ^= static_cast<uint64_t>(v) + 0x517cc1b727220a95ull + (static_cast<uint64_t>(pars[v]) << 7) +
                  (static_cast<uint64_t>(pars[v]) >> 3);
            pc *= 1469598103934665603ull;
        }
        LOG("[%s-FINAL-CHECK] distance_checksum=%llu parent_checksum=%llu\n", kUpper,
            static_cast<unsigned long long>(checksum(vals)), static_cast<unsigned long long>(pc));
    }
    if (!S("output").empty()) {
        std::ofstream out(S("output"));
        for (uint32_t v = 0; v < n; ++v) out << v << ' ' << vals[v] << ' ' << pars[v] << ' ' << vals[v] << '\n';
        if (!out) throw Fail("cannot write " + S("output"));
    }
#endif
#endif
    return success;
}

int main(int argc, char **argv) {
    define_flags();
    parse_args(argc, argv);
    if (B("interactive") || !S("cmdfile").empty()) {
        std::fprintf(stderr, "%s: interactive and command-file sessions are not supported\n", kUpper);
        return 1;
    }
    std::printf("\nTesting single GPU %s\n", kUpper);
    std::printf("--------------------\n\n");
    bool ok = false;
    try {
        ok = run();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s: %s\n", kUpper, e.what());
        ok = false;
    }
    if (g_h) cig_destroy(g_h);
    std::printf("Overall: Test %s\n", ok ? "passed" : "FAILED");
    return ok ? 0 : 1;
}

// Seeded R-MAT graphs and update streams (declared in include/cig_gen.h).
//
// The reference has no compiled generator (include/framework/generator.h:80-111
// is never included).  This file follows the published R-MAT recursion
// (Chakrabarti, Zhan, Faloutsos 2004): each edge descends `scale` levels and
// picks a quadrant with probabilities a/b/c/d.  Randomness is counter based
// (SplitMix64 keyed by the edge index), so every thread count yields the same
// graph.  Rows are built by a counting pass plus a per-row sort and dedup.
#include "../../include/cig_gen.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <new>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <omp.h>

namespace {

inline uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

inline uint64_t mix64(uint64_t x) {
    uint64_t s = x;
    return splitmix64(s);
}

// Uniform integer in [0, bound) by 128-bit multiply (Lemire's method,
// without the rejection step: the bias is below 2^-32 for bound < 2^32).
inline uint32_t uniform_below(uint64_t &state, uint32_t bound) {
    const uint64_t r = splitmix64(state);
    return static_cast<uint32_t>((static_cast<unsigned __int128>(r) * bound) >> 64);
}

// Keyed bijection on [0, 2^bits): rounds of odd multiply, add and xorshift,
// each invertible modulo 2^bits.
struct Permutation {
    uint32_t bits;
    uint64_t mask;
    uint64_t mul[3], add[3];
    uint32_t zero_image;  // F(0); the preimage of 0 is sent here so that 0 stays fixed

    Permutation(uint32_t b, uint64_t seed) : bits(b), mask(b >= 64 ? ~0ULL : ((1ULL << b) - 1)) {
        uint64_t s = seed ^ 0x5851F42D4C957F2DULL;
        for (int r = 0; r < 3; ++r) {
            mul[r] = (splitmix64(s) | 1ULL) & mask;
            if (mul[r] == 0) mul[r] = 1;
            add[r] = splitmix64(s) & mask;
        }
        zero_image = static_cast<uint32_t>(raw(0));
    }
    uint64_t raw(uint64_t x) const {
        if (bits == 0) return 0;
        const uint32_t shift = bits / 2 + 1;
        for (int r = 0; r < 3; ++r) {
            x = (x * mul[r] + add[r]) & mask;
            if (shift < bits) x ^= x >> shift;
        }
        return x & mask;
    }
    uint32_t operator()(uint32_t x) const {
        if (x == 0) return 0;
        const uint64_t y = raw(x);
        return y == 0 ? zero_image : static_cast<uint32_t>(y);
    }
};

}  // namespace

struct cig_gen_graph {
    uint32_t n = 0;
    std::vector<uint64_t> xadj;
    std::vector<uint32_t> adj;
};

extern "C" int cig_gen_threads(void) { return omp_get_max_threads(); }

extern "C" int cig_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                            uint64_t seed, int symmetric, int permute, cig_gen_graph **out) {
    if (!out || scale > 31 || a < 0 || b < 0 || c < 0 || a + b + c >= 1.0) return -1;
    *out = nullptr;
    cig_gen_graph *g = new (std::nothrow) cig_gen_graph();
    if (!g) return -2;
    try {
        const uint32_t n = 1u << scale;
        const uint64_t samples = static_cast<uint64_t>(edge_factor) << scale;
        const uint64_t ta = static_cast<uint64_t>(a * 4294967296.0);
        const uint64_t tab = static_cast<uint64_t>((a + b) * 4294967296.0);
        const uint64_t tabc = static_cast<uint64_t>((a + b + c) * 4294967296.0);
        const Permutation perm(scale, seed);
        const uint64_t stored = symmetric ? 2 * samples : samples;
        std::vector<uint32_t> src(stored), dst(stored);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < static_cast<int64_t>(samples); ++i) {
            uint64_t state = mix64(seed * 0x9E3779B97F4A7C15ULL + static_cast<uint64_t>(i));
            uint32_t u = 0, v = 0;
            uint64_t bitsbuf = 0;
            for (uint32_t level = 0; level < scale; ++level) {
                if ((level & 1) == 0) bitsbuf = splitmix64(state);
                const uint64_t r = (level & 1) ? (bitsbuf >> 32) : (bitsbuf & 0xFFFFFFFFULL);
                u <<= 1;
                v <<= 1;
                if (r < ta) {
                } else if (r < tab) {
                    v |= 1;
                } else if (r < tabc) {
                    u |= 1;
                } else {
                    u |= 1;
                    v |= 1;
                }
            }
            if (permute) {
                u = perm(u);
                v = perm(v);
            }
            src[i] = u;
            dst[i] = v;
            if (symmetric) {
                src[samples + i] = v;
                dst[samples + i] = u;
            }
        }
        // Counting pass by source (self-loops dropped here).
        std::vector<std::atomic<uint32_t>> degree(n);
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < static_cast<int64_t>(n); ++v) degree[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < static_cast<int64_t>(stored); ++i)
            if (src[i] != dst[i]) degree[src[i]].fetch_add(1, std::memory_order_relaxed);
        std::vector<uint64_t> start(static_cast<size_t>(n) + 1, 0);
        for (uint32_t v = 0; v < n; ++v) start[v + 1] = start[v] + degree[v].load(std::memory_order_relaxed);
        std::vector<uint32_t> rows(start[n]);
        std::vector<std::atomic<uint64_t>> cursor(n);
#pragma omp parallel for schedule(static)
        for (int64_t v = 0; v < static_cast<int64_t>(n); ++v) cursor[v].store(start[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < static_cast<int64_t>(stored); ++i)
            if (src[i] != dst[i]) rows[cursor[src[i]].fetch_add(1, std::memory_order_relaxed)] = dst[i];
        std::vector<uint32_t>().swap(src);
        std::vector<uint32_t>().swap(dst);
        // Sort and dedup each row; rows end up ordered by destination.
        std::vector<uint32_t> kept(n);
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < static_cast<int64_t>(n); ++v) {
            uint32_t *b0 = rows.data() + start[v];
            uint32_t *e0 = rows.data() + start[v + 1];
            std::sort(b0, e0);
            kept[v] = static_cast<uint32_t>(std::unique(b0, e0) - b0);
        }
        g->n = n;
        g->xadj.assign(static_cast<size_t>(n) + 1, 0);
        for (uint32_t v = 0; v < n; ++v) g->xadj[v + 1] = g->xadj[v] + kept[v];
        g->adj.resize(g->xadj[n]);
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < static_cast<int64_t>(n); ++v)
            std::memcpy(g->adj.data() + g->xadj[v], rows.data() + start[v], sizeof(uint32_t) * kept[v]);
    } catch (...) {
        delete g;
        return -2;
    }
    *out = g;
    return 0;
}

extern "C" int cig_gen_sizes(const cig_gen_graph *g, uint32_t *n, uint64_t *m) {
    if (!g) return -1;
    if (n) *n = g->n;
    if (m) *m = g->adj.size();
    return 0;
}

extern "C" int cig_gen_copy_csr(const cig_gen_graph *g, uint64_t *xadj, uint32_t *adj) {
    if (!g || !xadj || (!adj && !g->adj.empty())) return -1;
    std::memcpy(xadj, g->xadj.data(), sizeof(uint64_t) * g->xadj.size());
    if (!g->adj.empty()) std::memcpy(adj, g->adj.data(), sizeof(uint32_t) * g->adj.size());
    return 0;
}

extern "C" int cig_gen_borrow_csr(const cig_gen_graph *g, const uint64_t **xadj, const uint32_t **adj) {
    if (!g || !xadj || !adj) return -1;
    *xadj = g->xadj.data();
    *adj = g->adj.data();
    return 0;
}

extern "C" void cig_gen_free(cig_gen_graph *g) { delete g; }

namespace {

inline uint64_t key_of(uint32_t u, uint32_t v) { return (static_cast<uint64_t>(u) << 32) | v; }

// The evolving edge set: the base CSR (sorted rows, no duplicates) minus the
// deleted base edges plus the alive insertions.  Insertions live in a dense
// vector with swap-remove so that deletion sampling stays uniform.
class EdgeSet {
public:
    explicit EdgeSet(const cig_gen_graph &g) : g_(g) {}

    uint64_t base_edges() const { return g_.adj.size(); }

    bool in_base(uint32_t u, uint32_t v) const {
        if (u >= g_.n) return false;
        const uint32_t *b = g_.adj.data() + g_.xadj[u];
        const uint32_t *e = g_.adj.data() + g_.xadj[u + 1];
        return std::binary_search(b, e, v);
    }

    bool contains(uint32_t u, uint32_t v) const {
        const uint64_t k = key_of(u, v);
        if (in_base(u, v)) return deleted_base_.find(k) == deleted_base_.end();
        return added_index_.find(k) != added_index_.end();
    }

    // Uniform draw of an alive edge; returns false if the set is empty.
    bool sample(uint64_t &state, uint32_t &u, uint32_t &v) const {
        const uint64_t total = base_edges() + added_.size();
        if (total == 0 || base_edges() - deleted_base_.size() + added_.size() == 0) return false;
        for (uint64_t attempt = 0; attempt < (1ULL << 40); ++attempt) {
            const uint64_t r = splitmix64(state);
            const uint64_t j = static_cast<uint64_t>((static_cast<unsigned __int128>(r) * total) >> 64);
            if (j < base_edges()) {
                const auto it = std::upper_bound(g_.xadj.begin(), g_.xadj.end(), j);
                const uint32_t su = static_cast<uint32_t>((it - g_.xadj.begin()) - 1);
                const uint32_t sv = g_.adj[j];
                if (deleted_base_.count(key_of(su, sv))) continue;
                u = su;
                v = sv;
                return true;
            }
            const uint64_t k = added_[j - base_edges()];
            u = static_cast<uint32_t>(k >> 32);
            v = static_cast<uint32_t>(k & 0xFFFFFFFFULL);
            return true;
        }
        return false;
    }

    void erase(uint32_t u, uint32_t v) {
        const uint64_t k = key_of(u, v);
        if (in_base(u, v)) {
            deleted_base_.insert(k);
            return;
        }
        const auto it = added_index_.find(k);
        if (it == added_index_.end()) return;
        const size_t pos = it->second;
        const uint64_t last = added_.back();
        added_[pos] = last;
        added_index_[last] = pos;
        added_.pop_back();
        added_index_.erase(k);
    }

    void insert(uint32_t u, uint32_t v) {
        const uint64_t k = key_of(u, v);
        if (in_base(u, v)) {
            deleted_base_.erase(k);
            return;
        }
        added_index_.emplace(k, added_.size());
        added_.push_back(k);
    }

private:
    const cig_gen_graph &g_;
    std::unordered_set<uint64_t> deleted_base_;
    std::vector<uint64_t> added_;
    std::unordered_map<uint64_t, size_t> added_index_;
};

}  // namespace

extern "C" int cig_gen_updates(const cig_gen_graph *g, uint32_t nbatches, const uint64_t *del_sizes,
                               const uint64_t *add_sizes, uint64_t seed, int symmetric,
                               uint32_t *del_u, uint32_t *del_v, uint32_t *add_u, uint32_t *add_v) {
    if (!g || (nbatches && (!del_sizes || !add_sizes))) return -1;
    if (g->n < 2) return -1;
    try {
        EdgeSet set(*g);
        uint64_t state = mix64(seed ^ 0xD1B54A32D192ED03ULL);
        uint64_t dpos = 0, apos = 0;
        for (uint32_t batch = 0; batch < nbatches; ++batch) {
            const uint64_t nd = del_sizes[batch], na = add_sizes[batch];
            if (symmetric && ((nd & 1) || (na & 1))) return -1;
            const uint64_t step = symmetric ? 2 : 1;
            for (uint64_t i = 0; i < nd; i += step) {
                uint32_t u, v;
                if (!set.sample(state, u, v)) return -3;
                set.erase(u, v);
                del_u[dpos] = u;
                del_v[dpos] = v;
                ++dpos;
                if (symmetric) {
                    set.erase(v, u);
                    del_u[dpos] = v;
                    del_v[dpos] = u;
                    ++dpos;
                }
            }
            for (uint64_t i = 0; i < na; i += step) {
                uint32_t u = 0, v = 0;
                bool found = false;
                for (uint64_t attempt = 0; attempt < (1ULL << 24) && !found; ++attempt) {
                    u = uniform_below(state, g->n);
                    v = uniform_below(state, g->n);
                    found = u != v && !set.contains(u, v);
                }
                if (!found) return -3;
                set.insert(u, v);
                add_u[apos] = u;
                add_v[apos] = v;
                ++apos;
                if (symmetric) {
                    set.insert(v, u);
                    add_u[apos] = v;
                    add_v[apos] = u;
                    ++apos;
                }
            }
        }
    } catch (...) {
        return -2;
    }
    return 0;
}

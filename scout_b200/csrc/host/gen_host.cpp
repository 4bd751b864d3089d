// gen_host.cpp -- seeded synthetic workloads and initial states.
//
// R-MAT graphs stand in for the reference's datasets; the update-stream samplers follow the
// sampling rules of the reference's tools/generate_*_batches.py, and the initial states
// follow tools/compute_initial_mis.py, tools/greedy_color.cpp, tools/bfs_ground_truth.cu and
// the min-id labels of tools/excc_src/excc_v1.cu. Every random draw comes from a
// counter-based mixer, so a seed gives the same output on any machine and thread count.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <omp.h>

namespace scout {

static inline uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser (Steele, Lea, Flood: "Fast splittable pseudorandom number
    // generators", OOPSLA 2014).
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(mix64(seed ^ 0x5C07ULL)) {}
    uint64_t next() { s += 0x9E3779B97F4A7C15ULL; return mix64(s); }
    uint64_t below(uint64_t k) { return k ? next() % k : 0; }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Parallel LSD radix sort of 64-bit keys on the low `bits` bits (11-bit digits).
static void radix_sort_u64(std::vector<uint64_t>& a, int bits) {
    const int D = 11, B = 1 << D;
    std::vector<uint64_t> tmp(a.size());
    const size_t n = a.size();
    int nt = omp_get_max_threads();
    std::vector<size_t> hist((size_t)nt * B);
    for (int shift = 0; shift < bits; shift += D) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
        {
            int t = omp_get_thread_num();
            size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t* h = &hist[(size_t)t * B];
            for (size_t i = lo; i < hi; i++) h[(a[i] >> shift) & (B - 1)]++;
        }
        size_t run = 0;
        for (int d = 0; d < B; d++)
            for (int t = 0; t < nt; t++) {
                size_t c = hist[(size_t)t * B + d];
                hist[(size_t)t * B + d] = run;
                run += c;
            }
#pragma omp parallel num_threads(nt)
        {
            int t = omp_get_thread_num();
            size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t* h = &hist[(size_t)t * B];
            for (size_t i = lo; i < hi; i++) tmp[h[(a[i] >> shift) & (B - 1)]++] = a[i];
        }
        a.swap(tmp);
    }
}

int gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, Csr& out) {
    if (scale < 1 || scale > 30 || edge_factor < 1) return host_fail(SCOUT_E_INVALID, "bad R-MAT size");
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return host_fail(SCOUT_E_INVALID, "bad R-MAT probabilities");
    const int64_t n = (int64_t)1 << scale;
    const int64_t m = n * (int64_t)edge_factor;
    const uint64_t ta = (uint64_t)(a * 4294967296.0);
    const uint64_t tab = (uint64_t)((a + b) * 4294967296.0);
    const uint64_t tabc = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t sh = mix64(seed * 0x2545F4914F6CDD1DULL + 0xA0761D6478BD642FULL);

    std::vector<uint64_t> keys((size_t)(2 * m));
    std::vector<char> keep((size_t)m);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; i++) {
        uint64_t u = 0, v = 0;
        uint64_t r = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0) r = mix64(sh ^ ((uint64_t)i * 64 + (uint64_t)l));
            uint64_t x = (l & 1) ? (r >> 32) : (r & 0xFFFFFFFFULL);
            uint64_t bu, bv;
            if (x < ta) { bu = 0; bv = 0; }
            else if (x < tab) { bu = 0; bv = 1; }
            else if (x < tabc) { bu = 1; bv = 0; }
            else { bu = 1; bv = 1; }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        keys[2 * i] = (u << scale) | v;
        keys[2 * i + 1] = (v << scale) | u;
        keep[i] = (u != v);
    }
    // Drop self-loops, then sort and deduplicate (symmetrised, both directions kept).
    size_t w = 0;
    for (int64_t i = 0; i < m; i++)
        if (keep[i]) { keys[w++] = keys[2 * i]; keys[w++] = keys[2 * i + 1]; }
    keys.resize(w);
    std::vector<char>().swap(keep);
    radix_sort_u64(keys, 2 * scale);
    size_t u_end = keys.empty() ? 0 : 1;
    for (size_t i = 1; i < keys.size(); i++)
        if (keys[i] != keys[u_end - 1]) keys[u_end++] = keys[i];
    keys.resize(u_end);

    out.n = n;
    out.off.assign((size_t)n + 1, 0);
    out.adj.resize(keys.size());
    for (size_t i = 0; i < keys.size(); i++) out.off[(keys[i] >> scale) + 1]++;
    for (int64_t v = 0; v < n; v++) out.off[v + 1] += out.off[v];
    const uint64_t low = (uint64_t)n - 1;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < keys.size(); i++) out.adj[i] = (int32_t)(keys[i] & low);
    return SCOUT_OK;
}

// Open-addressing set of undirected pair keys (min << 32 | max).
class PairSet {
public:
    explicit PairSet(size_t expect) {
        size_t cap = 16;
        while (cap < expect * 2 + 16) cap <<= 1;
        slots_.assign(cap, EMPTY);
        mask_ = cap - 1;
    }
    bool insert(uint64_t k) {
        size_t h = (size_t)mix64(k) & mask_;
        while (true) {
            if (slots_[h] == EMPTY) { slots_[h] = k; return true; }
            if (slots_[h] == k) return false;
            h = (h + 1) & mask_;
        }
    }
    bool contains(uint64_t k) const {
        size_t h = (size_t)mix64(k) & mask_;
        while (true) {
            if (slots_[h] == EMPTY) return false;
            if (slots_[h] == k) return true;
            h = (h + 1) & mask_;
        }
    }
private:
    static constexpr uint64_t EMPTY = ~0ULL;
    std::vector<uint64_t> slots_;
    size_t mask_ = 0;
};

static inline uint64_t pair_key(int64_t u, int64_t v) {
    uint64_t a = (uint64_t)std::min(u, v), b = (uint64_t)std::max(u, v);
    return (a << 32) | b;
}

static inline int64_t row_of(const Csr& g, int64_t pos) {
    // searchsorted(nindex, pos, side="right") - 1 (generate_mixed_batches.py:89)
    auto it = std::upper_bound(g.off.begin(), g.off.end(), pos);
    return (int64_t)(it - g.off.begin()) - 1;
}

static bool csr_adjacent(const Csr& g, bool sorted, int64_t u, int64_t v) {
    const int32_t* b = g.adj.data() + g.off[u];
    const int32_t* e = g.adj.data() + g.off[u + 1];
    if (sorted) return std::binary_search(b, e, (int32_t)v);
    return std::find(b, e, (int32_t)v) != e;
}

static bool csr_rows_sorted(const Csr& g) {
    for (int64_t v = 0; v < g.n; v++)
        for (int64_t i = g.off[v] + 1; i < g.off[v + 1]; i++)
            if (g.adj[i - 1] > g.adj[i]) return false;
    return true;
}

int gen_stream(const Csr& g, int kind, int64_t batch_size, int64_t nbatches, double insert_ratio,
               double lowdeg_frac, uint64_t seed, scout_edge* out) {
    if (batch_size < 0 || nbatches < 0 || insert_ratio < 0 || insert_ratio > 1)
        return host_fail(SCOUT_E_INVALID, "bad stream parameters");
    const int64_t total = batch_size * nbatches;
    if (total == 0) return SCOUT_OK;
    const int64_t n_ins = (int64_t)std::llround((double)total * insert_ratio);
    const int64_t n_del = total - n_ins;
    const int64_t nnz = g.nnz();
    if (n_del > 0 && nnz == 0) return host_fail(SCOUT_E_INVALID, "graph has no edge to delete");
    if (2 * n_del > nnz) return host_fail(SCOUT_E_INVALID, "stream asks for more deletions than the graph has edges");
    const bool sorted = csr_rows_sorted(g);
    Rng rng(seed);
    PairSet used((size_t)total);
    std::vector<scout_edge> pool;
    pool.reserve((size_t)total);

    // 1/degree weights for the low-degree sampler (generate_low_degree_batches.py:56-66).
    std::vector<double> cum;
    if (kind == SCOUT_STREAM_LOWDEG) {
        cum.resize((size_t)g.n);
        double run = 0;
        for (int64_t v = 0; v < g.n; v++) {
            int64_t d = g.off[v + 1] - g.off[v];
            run += d > 0 ? 1.0 / (double)d : 0.0;
            cum[v] = run;
        }
    }
    const int64_t limit = 64 * total + 1000000;   // bounded retries instead of an endless loop
    int64_t tries = 0;
    while ((int64_t)pool.size() < n_del) {
        if (++tries > limit) return host_fail(SCOUT_E_INVALID, "could not sample enough distinct existing edges");
        int64_t u, v;
        if (kind == SCOUT_STREAM_LOWDEG && rng.unit() < lowdeg_frac) {
            double x = rng.unit() * cum.back();
            u = (int64_t)(std::upper_bound(cum.begin(), cum.end(), x) - cum.begin());
            if (u >= g.n) u = g.n - 1;
            int64_t d = g.off[u + 1] - g.off[u];
            if (d == 0) continue;
            v = g.adj[g.off[u] + (int64_t)rng.below((uint64_t)d)];
        } else {
            // First endpoint proportional to degree, second a uniform neighbour: the same
            // distribution as a uniform draw over the directed entries.
            int64_t pos = (int64_t)rng.below((uint64_t)nnz);
            u = row_of(g, pos);
            v = g.adj[pos];
        }
        if (u == v) continue;
        if (!used.insert(pair_key(u, v))) continue;
        pool.push_back(scout_edge{(int32_t)std::min(u, v), (int32_t)std::max(u, v)});
    }
    tries = 0;
    while ((int64_t)pool.size() < total) {
        if (++tries > limit) return host_fail(SCOUT_E_INVALID, "could not sample enough distinct non-edges");
        int64_t u, v;
        if (kind == SCOUT_STREAM_PREFERENTIAL) {
            u = row_of(g, (int64_t)rng.below((uint64_t)nnz));
            v = row_of(g, (int64_t)rng.below((uint64_t)nnz));
        } else {
            u = (int64_t)rng.below((uint64_t)g.n);
            v = (int64_t)rng.below((uint64_t)g.n);
        }
        if (u == v) continue;
        uint64_t k = pair_key(u, v);
        if (used.contains(k)) continue;
        if (csr_adjacent(g, sorted, u, v)) continue;
        used.insert(k);
        pool.push_back(scout_edge{(int32_t)std::min(u, v), (int32_t)std::max(u, v)});
    }
    // Fisher-Yates shuffle of the pooled deletions and insertions.
    for (int64_t i = total - 1; i > 0; i--) {
        int64_t j = (int64_t)rng.below((uint64_t)(i + 1));
        std::swap(pool[i], pool[j]);
    }
    std::memcpy(out, pool.data(), sizeof(scout_edge) * (size_t)total);
    return SCOUT_OK;
}

int init_state(const Csr& g, int problem, int32_t source, int32_t* out) {
    const int64_t n = g.n;
    switch (problem) {
    case SCOUT_MIS: {   // compute_initial_mis.py:32-43
        std::vector<char> blocked((size_t)n, 0);
        for (int64_t v = 0; v < n; v++) {
            out[v] = 0;
            if (blocked[v]) continue;
            out[v] = 1;
            for (int64_t i = g.off[v]; i < g.off[v + 1]; i++) blocked[g.adj[i]] = 1;
        }
        return SCOUT_OK;
    }
    case SCOUT_COLORING: {   // greedy_color.cpp:37-52
        std::vector<int64_t> mark;
        for (int64_t v = 0; v < n; v++) out[v] = -1;
        for (int64_t v = 0; v < n; v++) {
            for (int64_t i = g.off[v]; i < g.off[v + 1]; i++) {
                int32_t c = out[g.adj[i]];
                if (c >= 0) {
                    if (c >= (int32_t)mark.size()) mark.resize((size_t)c + 1, -1);
                    mark[c] = v;
                }
            }
            int32_t c = 0;
            while (c < (int32_t)mark.size() && mark[c] == v) c++;
            out[v] = c;
        }
        return SCOUT_OK;
    }
    case SCOUT_BFS: {   // levels from `source`, -1 unreached
        if (source < 0 || source >= n) return host_fail(SCOUT_E_INVALID, "source out of range");
        for (int64_t v = 0; v < n; v++) out[v] = -1;
        std::vector<int32_t> q;
        q.reserve((size_t)n);
        out[source] = 0;
        q.push_back(source);
        for (size_t h = 0; h < q.size(); h++) {
            int32_t x = q[h];
            for (int64_t i = g.off[x]; i < g.off[x + 1]; i++) {
                int32_t y = g.adj[i];
                if (out[y] < 0) { out[y] = out[x] + 1; q.push_back(y); }
            }
        }
        return SCOUT_OK;
    }
    case SCOUT_CC: {   // min-vertex-id labels: union-find where the lower root wins
        std::vector<int32_t> p((size_t)n);
        std::iota(p.begin(), p.end(), 0);
        auto find = [&](int32_t x) {
            while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
            return x;
        };
        for (int64_t v = 0; v < n; v++)
            for (int64_t i = g.off[v]; i < g.off[v + 1]; i++) {
                int32_t a = find((int32_t)v), b = find(g.adj[i]);
                if (a != b) { if (a < b) p[b] = a; else p[a] = b; }
            }
        for (int64_t v = 0; v < n; v++) out[v] = find((int32_t)v);
        return SCOUT_OK;
    }
    default:
        return host_fail(SCOUT_E_INVALID, "unknown problem");
    }
}

}  // namespace scout

using namespace scout;

extern "C" {

int scout_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, scout_csr** out) {
    if (!out) return host_fail(SCOUT_E_INVALID, "null argument");
    auto* h = new scout_csr();
    int rc = gen_rmat(scale, edge_factor, a, b, c, seed, h->g);
    if (rc != SCOUT_OK) { delete h; return rc; }
    *out = h;
    return SCOUT_OK;
}

int scout_csr_from_arrays(int64_t n, const int64_t* off, const int32_t* adj, scout_csr** out) {
    if (!out || !off || n < 1 || n > INT32_MAX) return host_fail(SCOUT_E_INVALID, "bad argument");
    if (off[0] != 0) return host_fail(SCOUT_E_INVALID, "offsets must start at 0");
    for (int64_t v = 0; v < n; v++)
        if (off[v + 1] < off[v]) return host_fail(SCOUT_E_INVALID, "offsets must be monotone");
    int64_t nnz = off[n];
    for (int64_t i = 0; i < nnz; i++)
        if (adj[i] < 0 || adj[i] >= n) return host_fail(SCOUT_E_INVALID, "neighbour id out of range");
    auto* h = new scout_csr();
    h->g.n = n;
    h->g.off.assign(off, off + n + 1);
    h->g.adj.assign(adj, adj + nnz);
    *out = h;
    return SCOUT_OK;
}
int scout_csr_free(scout_csr* g) { delete g; return SCOUT_OK; }
int64_t scout_csr_nodes(const scout_csr* g) { return g ? g->g.n : SCOUT_E_INVALID; }
int64_t scout_csr_nnz(const scout_csr* g) { return g ? g->g.nnz() : SCOUT_E_INVALID; }
const int64_t* scout_csr_offsets(const scout_csr* g) { return g ? g->g.off.data() : nullptr; }
const int32_t* scout_csr_adj(const scout_csr* g) { return g ? g->g.adj.data() : nullptr; }

int scout_gen_stream(const scout_csr* g, int kind, int64_t batch_size, int64_t nbatches, double insert_ratio,
                     double lowdeg_frac, uint64_t seed, scout_edge* out) {
    if (!g || (!out && batch_size * nbatches > 0)) return host_fail(SCOUT_E_INVALID, "null argument");
    if (kind < SCOUT_STREAM_MIXED || kind > SCOUT_STREAM_LOWDEG) return host_fail(SCOUT_E_INVALID, "unknown stream kind");
    return gen_stream(g->g, kind, batch_size, nbatches, insert_ratio, lowdeg_frac, seed, out);
}

int scout_init_state(const scout_csr* g, int problem, int32_t source, int32_t* out) {
    if (!g || !out) return host_fail(SCOUT_E_INVALID, "null argument");
    return init_state(g->g, problem, source, out);
}

}  // extern "C"

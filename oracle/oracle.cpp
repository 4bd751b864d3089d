// ORACLE -- test infrastructure, not product code.
//
// A single-threaded CPU restatement of the reference engines (anonymous-artifacts/SCOUT),
// used only by tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py to check
// the CUDA engine. Nothing in the scout_b200 package links or calls it. It is independent of
// the package's own host code (no shared sources).
//
// What it restates, rule by rule (path:line inside the reference project):
//   OGraph      FlashGraph + DeltaOverlay + HybridGraph row semantics   core/FlashGraph.h:200-388
//   classify    toggle classification at parse time                     core/cli_setup.h:87-103
//   OBfs        processBatch, gpu_relax_round, gpu_deletion_round,
//               gpu_full_bfs, cascade bound 200, deferral, 200000 caps   src/bfs/scout_bfs.cu:46-515, 593-602
//   OCc         CCLabels, bidirectional_reachability_check, bound rule,
//               deferred recompute                                       src/cc/scout_cc.cu:280-441, 469, 516-527
//   OColoring   propose / detect / apply rounds, 200000 / 20M caps       src/coloring/scout_coloring.cu:46-100, 172-277
//   OMisRef     2-hop packed rows + per-edge repair rule                 src/mis/scout_mis.cu:173-215, 290-362, 500-627, 738-749, 835-842
//   OMisId      the engine's deterministic vertex-id-priority variant of the same 2-hop rule
//   gt_*        from-scratch BFS, min-id CC, greedy colour, greedy MIS  tools/bfs_ground_truth.cu, excc_v1.cu:520-531,
//                                                                        greedy_color.cpp:37-52, compute_initial_mis.py:32-43
// Parallel kernels are executed in one fixed sequential order. Where the reference's outcome
// depends on thread interleaving (atomic push order under the 200000-entry caps, MIS cluster
// races) the restatement picks that order and raises the `truncated` statistic instead of
// claiming the reference's exact result.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

constexpr int UNREACHED = -1;
constexpr int64_t MAX_ROUND = 200000;          // MAX_ROUND_FRONTIER / MAX_ROUND_VERTS
constexpr int64_t MAX_ROUND_ELEMS = 20000000;  // MAX_ROUND_CSR_ELEMS (coloring)

// ------------------------------------------------------------------------------------------
// OGraph: base CSR + DeltaOverlay (FlashGraph.h:200-311) + HybridGraph (331-388)
// ------------------------------------------------------------------------------------------
struct OGraph {
    int n = 0;
    std::vector<int64_t> off;
    std::vector<int32_t> adj;
    std::unordered_map<int, std::vector<int>> added;
    std::unordered_map<int, std::unordered_set<int>> removed;

    bool base_adjacent(int u, int v) const {
        for (int64_t i = off[u]; i < off[u + 1]; i++)
            if (adj[i] == v) return true;
        return false;
    }
    // isAdjacentDelta then the linear base-row scan (FlashGraph.h:209-225, 356-366)
    bool is_adjacent(int u, int v) const {
        auto a = added.find(u);
        if (a != added.end() && std::find(a->second.begin(), a->second.end(), v) != a->second.end()) return true;
        auto r = removed.find(u);
        if (r != removed.end() && r->second.count(v)) return false;
        return base_adjacent(u, v);
    }
    void insert_edge(int u, int v) {   // FlashGraph.h:227-234, 284-291
        auto ru = removed.find(u);
        if (ru != removed.end() && ru->second.count(v)) {
            ru->second.erase(v);
            auto rv = removed.find(v);
            if (rv != removed.end()) rv->second.erase(u);
            return;
        }
        added[u].push_back(v);
        added[v].push_back(u);
    }
    void remove_edge(int u, int v) {   // FlashGraph.h:236-243, 295-310
        auto au = added.find(u);
        if (au != added.end()) {
            auto it = std::find(au->second.begin(), au->second.end(), v);
            if (it != au->second.end()) {
                au->second.erase(it);
                auto av = added.find(v);
                if (av != added.end()) {
                    auto jt = std::find(av->second.begin(), av->second.end(), u);
                    if (jt != av->second.end()) av->second.erase(jt);
                }
                return;
            }
        }
        removed[u].insert(v);
        removed[v].insert(u);
    }
    void neighbors_into(int v, std::vector<int>& out) const {   // FlashGraph.h:246-265
        out.clear();
        auto r = removed.find(v);
        if (r == removed.end() || r->second.empty()) {
            out.insert(out.end(), adj.begin() + off[v], adj.begin() + off[v + 1]);
        } else {
            for (int64_t i = off[v]; i < off[v + 1]; i++)
                if (!r->second.count(adj[i])) out.push_back(adj[i]);
        }
        auto a = added.find(v);
        if (a != added.end()) out.insert(out.end(), a->second.begin(), a->second.end());
    }
    int64_t degree(int v) const {   // FlashGraph.h:267-274
        int64_t d = off[v + 1] - off[v];
        auto r = removed.find(v);
        if (r != removed.end()) d -= (int64_t)r->second.size();
        auto a = added.find(v);
        if (a != added.end()) d += (int64_t)a->second.size();
        return d;
    }
};

struct Edit { int u, v; bool ins; };

// parse_batch_file filter + classification against the current graph (cli_setup.h:95-99).
std::vector<Edit> classify(const OGraph& g, const int32_t* uv, int64_t m, bool against_base) {
    std::vector<Edit> out;
    out.reserve((size_t)m);
    for (int64_t i = 0; i < m; i++) {
        int u = uv[2 * i], v = uv[2 * i + 1];
        if (u < 0 || u >= g.n || v < 0 || v >= g.n || u == v) continue;
        bool adj = against_base ? g.base_adjacent(u, v) : g.is_adjacent(u, v);
        out.push_back({u, v, !adj});
    }
    return out;
}

// Statistics slots shared by all engines (int64[32]).
enum Stat {
    S_INS = 0, S_DEL, S_INS_NOOP, S_DEL_NOOP, S_CONFLICT, S_DEFERRED, S_FALLBACK, S_TRUNCATED,
    S_ROUNDS, S_STILL_CONNECTED, S_SPLIT, S_INCONCLUSIVE, S_TOUCHED, S_INS_REPAIRED, S_DEL_LOCAL,
    S_MERGED, S_MAX_ROUNDS, S_CHANGED, S_NSTATS = 32
};

struct Engine {
    int problem = 0;
    OGraph g;
    int64_t st[S_NSTATS] = {0};
    virtual ~Engine() = default;
    virtual void batch(const int32_t* uv, int64_t m) = 0;
    virtual void finish() {}
    virtual void solution(int32_t* out) = 0;
};

// bound_by_cumulative_degree (chunking.h:20-32)
int64_t bound_by_cumulative_degree(const OGraph& g, const std::vector<int>& cand, int64_t cap) {
    int64_t n = 0, probe = 0;
    for (int v : cand) {
        if (n >= cap) break;
        int64_t d = g.degree(v);
        if (probe + d > cap) break;
        probe += d;
        n++;
    }
    return n;
}

// ------------------------------------------------------------------------------------------
// BFS (scout_bfs.cu). hl = host mirror `level`, dl = device array `d_level`.
// ------------------------------------------------------------------------------------------
struct OBfs : Engine {
    std::vector<int> hl, dl;
    int source = 0;
    int64_t bound = 200;
    bool defer = true;

    // gpu_relax (scout_bfs.cu:46-54)
    static bool relax(int& slot, int cand) {
        if (slot == UNREACHED || slot > cand) { slot = cand; return true; }
        return false;
    }

    // gpu_relax_round (scout_bfs.cu:177-272) executed in frontier order.
    std::vector<int> relax_round(std::vector<int>& frontier, int64_t& raw_next_out) {
        raw_next_out = 0;
        if (frontier.empty()) return {};
        int64_t num_f = bound_by_cumulative_degree(g, frontier, MAX_ROUND);
        if (num_f < (int64_t)frontier.size()) st[S_TRUNCATED]++;   // the remainder is dropped
        if (num_f == 0) return {};
        std::vector<int> aux((size_t)num_f);
        for (int64_t i = 0; i < num_f; i++) aux[i] = hl[frontier[i]];
        std::vector<int> next_ids;
        int64_t next_count = 0;
        std::vector<int> row;
        for (int64_t i = 0; i < num_f; i++) {
            g.neighbors_into(frontier[i], row);
            int lv = aux[i];
            for (int u : row)
                if (relax(dl[u], lv + 1)) {
                    int64_t pos = next_count++;
                    if (pos < MAX_ROUND) next_ids.push_back(u);
                }
        }
        raw_next_out = next_count;
        if (next_count > MAX_ROUND) st[S_TRUNCATED]++;
        for (int id : next_ids) hl[id] = dl[id];   // gather_levels + mirror (244-262)
        return next_ids;
    }

    // gpu_deletion_round (scout_bfs.cu:325-415): compute on a snapshot, then apply.
    std::vector<int> deletion_round(std::vector<int>& work) {
        if (work.empty()) return {};
        int64_t num_w = bound_by_cumulative_degree(g, work, MAX_ROUND);
        if (num_w < (int64_t)work.size()) st[S_TRUNCATED]++;
        if (num_w == 0) return {};
        std::vector<int> newl((size_t)num_w);
        std::vector<int> next_ids;
        int64_t next_count = 0;
        std::vector<int> row;
        for (int64_t i = 0; i < num_w; i++) {
            int w = work[i];
            int old_level = hl[w];
            g.neighbors_into(w, row);
            int best = UNREACHED;
            for (int x : row) {
                int ln = dl[x];
                if (ln != UNREACHED && (best == UNREACHED || ln < best)) best = ln;
            }
            int nl = best == UNREACHED ? UNREACHED : best + 1;
            newl[i] = nl;
            if (nl != old_level)
                for (int x : row) {
                    int ln = dl[x];
                    if (ln != UNREACHED && old_level != UNREACHED && ln == old_level + 1) {
                        int64_t pos = next_count++;
                        if (pos < MAX_ROUND) next_ids.push_back(x);
                    }
                }
        }
        for (int64_t i = 0; i < num_w; i++) dl[work[i]] = newl[i];
        for (int64_t i = 0; i < num_w; i++) hl[work[i]] = newl[i];
        if (next_count > MAX_ROUND) st[S_TRUNCATED]++;
        return next_ids;
    }

    // gpu_full_bfs (scout_bfs.cu:274-323): chunks bounded by cumulative degree; a vertex
    // whose own degree exceeds the cap is never expanded (bound_by_cumulative_degree admits 0).
    void full_bfs() {
        std::fill(hl.begin(), hl.end(), UNREACHED);
        std::fill(dl.begin(), dl.end(), UNREACHED);
        hl[source] = 0;
        dl[source] = 0;
        std::vector<int> frontier = {source};
        while (!frontier.empty()) {
            std::vector<int> next;
            size_t i = 0;
            while (i < frontier.size()) {
                std::vector<int> chunk;
                int64_t sum = 0;
                while (i < frontier.size()) {
                    int64_t d = g.degree(frontier[i]);
                    if (!chunk.empty() && (sum + d > MAX_ROUND || (int64_t)chunk.size() >= MAX_ROUND)) break;
                    chunk.push_back(frontier[i]);
                    sum += d;
                    i++;
                }
                int64_t raw = 0;
                std::vector<int> cn = relax_round(chunk, raw);
                next.insert(next.end(), cn.begin(), cn.end());
            }
            frontier.swap(next);
        }
    }

    void batch(const int32_t* uv, int64_t m) override {   // processBatch (436-515)
        std::vector<Edit> edits = classify(g, uv, m, false);
        for (const Edit& e : edits) {
            int u = e.u, v = e.v;
            if (e.ins) {
                g.insert_edge(u, v);
                st[S_INS]++;
                bool iv = hl[u] != UNREACHED && (hl[v] == UNREACHED || hl[u] + 1 < hl[v]);
                bool iu = hl[v] != UNREACHED && (hl[u] == UNREACHED || hl[v] + 1 < hl[u]);
                if (!iu && !iv) { st[S_INS_NOOP]++; continue; }
                std::vector<int> frontier;
                if (iv) { hl[v] = hl[u] + 1; dl[v] = hl[v]; frontier.push_back(v); }
                if (iu) { hl[u] = hl[v] + 1; dl[u] = hl[u]; frontier.push_back(u); }
                int64_t raw;
                while (!frontier.empty()) {
                    frontier = relax_round(frontier, raw);
                    st[S_ROUNDS]++;
                }
                st[S_INS_REPAIRED]++;
            } else {
                g.remove_edge(u, v);
                st[S_DEL]++;
                bool tree = (hl[u] != UNREACHED && hl[v] == hl[u] + 1) || (hl[v] != UNREACHED && hl[u] == hl[v] + 1);
                if (!tree) { st[S_DEL_NOOP]++; continue; }
                int child = hl[u] > hl[v] ? u : v;
                std::vector<int> work = {child};
                int64_t touched = 0;
                bool fb = false;
                while (!work.empty()) {
                    touched += (int64_t)work.size();
                    if (touched > bound) {
                        if (defer) st[S_DEFERRED]++;
                        else full_bfs();
                        fb = true;
                        break;
                    }
                    work = deletion_round(work);
                    st[S_ROUNDS]++;
                }
                if (fb) st[S_FALLBACK]++;
                else st[S_DEL_LOCAL]++;
            }
        }
    }
    void finish() override {   // deferred catch-up (scout_bfs.cu:593-602)
        if (defer && st[S_DEFERRED] > 0) full_bfs();
    }
    void solution(int32_t* out) override { std::copy(hl.begin(), hl.end(), out); }
};

// ------------------------------------------------------------------------------------------
// CC (scout_cc.cu)
// ------------------------------------------------------------------------------------------
int find_root(std::vector<int>& parent, int v) {   // scout_cc.cu:280-289
    int root = v;
    while (parent[root] != root) root = parent[root];
    while (parent[v] != root) { int nx = parent[v]; parent[v] = root; v = nx; }
    return root;
}

void gt_cc_graph(const OGraph& g, std::vector<int>& lab);

struct OCc : Engine {
    std::vector<int> label, lp;
    int64_t bound = 5000;
    bool defer = true;

    int find(int v) { return find_root(lp, label[v]); }
    bool unite_v(int u, int v) {   // scout_cc.cu:365-370
        int ru = find(u), rv = find(v);
        if (ru == rv) return false;
        if (ru < rv) lp[rv] = ru; else lp[ru] = rv;
        return true;
    }
    void split(const std::vector<int>& side) {   // scout_cc.cu:371-375
        int fresh = (int)lp.size();
        lp.push_back(fresh);
        for (int w : side) label[w] = fresh;
    }
    void reset_from_roots(const std::vector<int>& root) {   // scout_cc.cu:376-380
        label = root;
        lp.resize(label.size());
        for (size_t i = 0; i < lp.size(); i++) lp[i] = (int)i;
    }

    enum Reach { STILL_CONNECTED, SPLIT, INCONCLUSIVE };
    // bidirectional_reachability_check (scout_cc.cu:300-342)
    Reach search(int u, int v, std::vector<int>& side) {
        side.clear();
        if (u == v) return STILL_CONNECTED;
        std::unordered_set<int> vu, vv;
        vu.insert(u);
        vv.insert(v);
        std::vector<int> fu = {u}, fv = {v}, row;
        int64_t touched = 2;
        while (!fu.empty() && !fv.empty()) {
            bool eu = fu.size() <= fv.size();
            std::vector<int>& fr = eu ? fu : fv;
            auto& vt = eu ? vu : vv;
            auto& vo = eu ? vv : vu;
            std::vector<int> next;
            for (int cur : fr) {
                g.neighbors_into(cur, row);
                for (int x : row) {
                    if (vo.count(x)) return STILL_CONNECTED;
                    if (vt.count(x)) continue;
                    vt.insert(x);
                    next.push_back(x);
                    touched++;
                    if (touched > bound) return INCONCLUSIVE;
                }
            }
            if (eu) fu = next; else fv = next;
        }
        if (fu.empty()) side.assign(vu.begin(), vu.end());
        else side.assign(vv.begin(), vv.end());
        return SPLIT;
    }
    void recompute() {
        std::vector<int> roots;
        gt_cc_graph(g, roots);
        reset_from_roots(roots);
    }
    void batch(const int32_t* uv, int64_t m) override {   // processBatch (392-441)
        std::vector<Edit> edits = classify(g, uv, m, false);
        std::vector<int> side;
        for (const Edit& e : edits) {
            if (e.ins) {
                g.insert_edge(e.u, e.v);
                st[S_INS]++;
                if (unite_v(e.u, e.v)) st[S_MERGED]++; else st[S_INS_NOOP]++;
            } else {
                g.remove_edge(e.u, e.v);
                st[S_DEL]++;
                if (find(e.u) != find(e.v)) { st[S_DEL_NOOP]++; continue; }
                Reach r = search(e.u, e.v, side);
                if (r == STILL_CONNECTED) st[S_STILL_CONNECTED]++;
                else if (r == SPLIT) { st[S_SPLIT]++; split(side); }
                else {
                    st[S_INCONCLUSIVE]++;
                    if (defer) st[S_DEFERRED]++;
                    else { recompute(); st[S_FALLBACK]++; }
                }
            }
        }
    }
    void finish() override {
        if (defer && st[S_DEFERRED] > 0) recompute();
    }
    void solution(int32_t* out) override {   // canonical: min vertex id of each class
        std::unordered_map<int, int> mn;
        for (int v = 0; v < g.n; v++) {
            int r = find(v);
            auto it = mn.find(r);
            if (it == mn.end()) mn.emplace(r, v);
        }
        for (int v = 0; v < g.n; v++) out[v] = mn[find(v)];
    }
};

// ------------------------------------------------------------------------------------------
// Coloring (scout_coloring.cu)
// ------------------------------------------------------------------------------------------
struct OColoring : Engine {
    std::vector<int> color, marker;

    // gpu_color_round (scout_coloring.cu:172-241)
    std::vector<int> round(const std::vector<int>& rv) {
        std::vector<int> ids;
        std::vector<std::vector<int>> rows;
        int64_t elems = 0;
        std::vector<int> scratch;
        for (int v : rv) {
            if ((int64_t)ids.size() >= MAX_ROUND) break;
            g.neighbors_into(v, scratch);
            if (elems + (int64_t)scratch.size() > MAX_ROUND_ELEMS) break;
            ids.push_back(v);
            rows.push_back(scratch);
            elems += (int64_t)scratch.size();
        }
        if (ids.size() < rv.size()) st[S_TRUNCATED]++;   // not carried to the next round
        if (ids.empty()) return {};
        std::vector<int> prop(ids.size());
        for (size_t t = 0; t < ids.size(); t++) {   // propose_color_kernel (46-64)
            int c = 0;
            bool found = false;
            while (!found) {
                found = true;
                for (int x : rows[t]) if (color[x] == c) { found = false; break; }
                if (!found) c++;
            }
            prop[t] = c;
        }
        for (size_t t = 0; t < ids.size(); t++) marker[ids[t]] = prop[t];
        std::vector<int> retry;   // detect_conflict_kernel (69-87)
        for (size_t t = 0; t < ids.size(); t++) {
            bool lose = false;
            for (int x : rows[t]) if (x < ids[t] && marker[x] == prop[t]) { lose = true; break; }
            if (lose && (int64_t)retry.size() < MAX_ROUND) retry.push_back(ids[t]);
        }
        for (size_t t = 0; t < ids.size(); t++) color[ids[t]] = prop[t];   // apply (89-93)
        for (int id : ids) marker[id] = -2;   // clear_marker (97-100)
        return retry;
    }
    void batch(const int32_t* uv, int64_t m) override {   // processBatch (243-277)
        std::vector<Edit> edits = classify(g, uv, m, false);
        std::vector<int> need;
        std::unordered_set<int> seen;
        for (const Edit& e : edits) {
            if (e.ins) {
                g.insert_edge(e.u, e.v);
                st[S_INS]++;
                if (color[e.u] != color[e.v]) { st[S_INS_NOOP]++; continue; }
                st[S_CONFLICT]++;
                int loser = e.u > e.v ? e.u : e.v;
                if (seen.insert(loser).second) need.push_back(loser);
            } else {
                g.remove_edge(e.u, e.v);
                st[S_DEL]++;
            }
        }
        // The reference iterates an unordered_set; the order only matters under the
        // truncation caps, which raise S_TRUNCATED.
        std::sort(need.begin(), need.end());
        int64_t rounds = 0;
        while (!need.empty()) {
            rounds++;
            need = round(need);
        }
        st[S_ROUNDS] += rounds;
        st[S_MAX_ROUNDS] = std::max(st[S_MAX_ROUNDS], rounds);
    }
    void solution(int32_t* out) override { std::copy(color.begin(), color.end(), out); }
};

// ------------------------------------------------------------------------------------------
// MIS, reference rule (scout_mis.cu)
// ------------------------------------------------------------------------------------------
// get_h_hop_neighborhood (173-215): BFS order, start vertex first; records hop-1 rows.
std::vector<int> two_hop_ball(const OGraph& g, int s, std::vector<char>& vis,
                              std::unordered_map<int, std::vector<int>>& hop1) {
    std::vector<int> ball = {s}, cur = {s}, nxt, tracker = {s}, row;
    vis[s] = 1;
    for (int hop = 0; hop < 2; hop++) {
        if (cur.empty()) break;
        for (int c : cur) {
            g.neighbors_into(c, row);
            if (hop == 1 && !hop1.count(c)) hop1[c] = row;
            for (int x : row)
                if (!vis[x]) { vis[x] = 1; tracker.push_back(x); nxt.push_back(x); ball.push_back(x); }
        }
        cur.swap(nxt);
        nxt.clear();
    }
    for (int t : tracker) vis[t] = 0;
    return ball;
}

// Conditional application of pre-classified edits (launchBatchGPU, scout_mis.cu:743-749).
void apply_conditional(OGraph& g, const std::vector<Edit>& edits) {
    for (const Edit& e : edits) {
        if (e.ins && !g.is_adjacent(e.u, e.v)) g.insert_edge(e.u, e.v);
        else if (!e.ins && g.is_adjacent(e.u, e.v)) g.remove_edge(e.u, e.v);
    }
}

struct OMisRef : Engine {
    std::vector<char> mis;
    void batch(const int32_t* uv, int64_t m) override {
        // Every batch is classified against the base graph (scout_mis.cu:835-842).
        std::vector<Edit> edits = classify(g, uv, m, true);
        for (const Edit& e : edits) st[e.ins ? S_INS : S_DEL]++;
        apply_conditional(g, edits);
        // Packed rows (launchBatch 544-626): endpoint -> 2-hop ball, hop-1 vertex -> row.
        std::vector<int> uniq;
        std::unordered_set<int> us;
        for (const Edit& e : edits) {
            if (us.insert(e.u).second) uniq.push_back(e.u);
            if (us.insert(e.v).second) uniq.push_back(e.v);
        }
        std::vector<char> vis((size_t)g.n, 0);
        std::unordered_map<int, std::vector<int>> hop1, packed;
        for (int x : uniq) packed[x] = two_hop_ball(g, x, vis, hop1);
        for (auto& kv : hop1)
            if (!us.count(kv.first)) packed.emplace(kv.first, kv.second);
        auto row_of = [&](int x) -> const std::vector<int>* {
            auto it = packed.find(x);
            return it == packed.end() ? nullptr : &it->second;
        };
        // process_clusters_csr_kernel (290-362), edges in batch order.
        for (const Edit& e : edits) {
            int u = e.u, v = e.v;
            bool ui = mis[u], vi = mis[v];
            if (e.ins) {
                if (ui && vi) {
                    st[S_CONFLICT]++;
                    int rem = u > v ? u : v;
                    mis[rem] = 0;
                    const std::vector<int>* r = row_of(rem);
                    if (r)
                        for (int nb : *r) {
                            if (mis[nb]) continue;
                            const std::vector<int>* nr = row_of(nb);
                            if (!nr) continue;
                            bool ok = true;
                            for (int x : *nr) if (mis[x]) { ok = false; break; }
                            if (ok) { mis[nb] = 1; break; }
                        }
                }
            } else {
                int a = -1, partner = -1;
                if (ui && !vi) { a = v; partner = u; }
                else if (!ui && vi) { a = u; partner = v; }
                if (a >= 0) {
                    bool ok = true;
                    const std::vector<int>* r = row_of(a);
                    if (r) for (int x : *r) if (x != partner && mis[x]) { ok = false; break; }
                    if (ok) mis[a] = 1;
                }
            }
        }
    }
    void solution(int32_t* out) override { for (int v = 0; v < g.n; v++) out[v] = mis[v]; }
};

// ------------------------------------------------------------------------------------------
// MIS, deterministic vertex-id-priority rule of the CUDA engine. Same trigger as the
// reference (an inserted edge inside the set drops max(u,v); a deleted edge frees its
// non-member endpoint) and the same 2-hop region, but every vertex that may have lost its
// last set neighbour is re-admitted in ascending id order, which keeps the set maximal.
// ------------------------------------------------------------------------------------------
struct OMisId : Engine {
    std::vector<char> mis;
    bool against_base = false;   // 1: reference MIS CLI classification + conditional apply
    void batch(const int32_t* uv, int64_t m) override {
        std::vector<Edit> edits = classify(g, uv, m, against_base);
        for (const Edit& e : edits) st[e.ins ? S_INS : S_DEL]++;
        if (against_base) apply_conditional(g, edits);
        else
            for (const Edit& e : edits) { if (e.ins) g.insert_edge(e.u, e.v); else g.remove_edge(e.u, e.v); }
        std::vector<int> removed, cand;
        for (const Edit& e : edits)
            if (e.ins && mis[e.u] && mis[e.v]) { st[S_CONFLICT]++; removed.push_back(std::max(e.u, e.v)); }
        for (int r : removed) mis[r] = 0;
        std::vector<int> row;
        for (int r : removed) {
            cand.push_back(r);
            g.neighbors_into(r, row);
            cand.insert(cand.end(), row.begin(), row.end());
        }
        for (const Edit& e : edits)
            if (!e.ins) { cand.push_back(e.u); cand.push_back(e.v); }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        for (int c : cand) {
            if (mis[c]) continue;
            g.neighbors_into(c, row);
            bool ok = true;
            for (int x : row) if (mis[x]) { ok = false; break; }
            if (ok) { mis[c] = 1; st[S_CHANGED]++; }
        }
        st[S_TOUCHED] += (int64_t)cand.size();
    }
    void solution(int32_t* out) override { for (int v = 0; v < g.n; v++) out[v] = mis[v]; }
};

// ------------------------------------------------------------------------------------------
// Ground truth
// ------------------------------------------------------------------------------------------
void gt_cc_graph(const OGraph& g, std::vector<int>& lab) {
    std::vector<int> p(g.n);
    std::iota(p.begin(), p.end(), 0);
    std::vector<int> row;
    for (int v = 0; v < g.n; v++) {
        g.neighbors_into(v, row);
        for (int x : row) {
            int a = find_root(p, v), b = find_root(p, x);
            if (a != b) { if (a < b) p[b] = a; else p[a] = b; }
        }
    }
    lab.resize(g.n);
    for (int v = 0; v < g.n; v++) lab[v] = find_root(p, v);
}

OGraph make_graph(int64_t n, const int64_t* off, const int32_t* adj) {
    OGraph g;
    g.n = (int)n;
    g.off.assign(off, off + n + 1);
    g.adj.assign(adj, adj + off[n]);
    return g;
}

}  // namespace

extern "C" {

// ---- graph --------------------------------------------------------------------------------
void* orc_graph_new(int64_t n, const int64_t* off, const int32_t* adj) {
    return new OGraph(make_graph(n, off, adj));
}
void orc_graph_free(void* g) { delete (OGraph*)g; }
int orc_graph_is_adjacent(void* g, int u, int v) { return ((OGraph*)g)->is_adjacent(u, v) ? 1 : 0; }
void orc_graph_insert(void* g, int u, int v) { ((OGraph*)g)->insert_edge(u, v); }
void orc_graph_remove(void* g, int u, int v) { ((OGraph*)g)->remove_edge(u, v); }
int64_t orc_graph_degree(void* g, int v) { return ((OGraph*)g)->degree(v); }
int64_t orc_graph_row(void* g, int v, int32_t* out, int64_t cap) {
    std::vector<int> row;
    ((OGraph*)g)->neighbors_into(v, row);
    for (int64_t i = 0; i < (int64_t)row.size() && i < cap; i++) out[i] = row[i];
    return (int64_t)row.size();
}
// One batch of toggles (u, v pairs): each pair is classified against the graph as it stood
// before the batch (cli_setup.h:87-103), then applied; self-loops and out-of-range ids skipped.
void orc_graph_toggle_batch(void* gp, const int32_t* uv, int64_t m) {
    OGraph* g = (OGraph*)gp;
    std::vector<char> ins((size_t)m, 0);
    for (int64_t i = 0; i < m; i++) {
        const int u = uv[2 * i], v = uv[2 * i + 1];
        if (u == v || u < 0 || v < 0 || u >= g->n || v >= g->n) { ins[i] = 2; continue; }
        ins[i] = g->is_adjacent(u, v) ? 0 : 1;
    }
    for (int64_t i = 0; i < m; i++) {
        if (ins[i] == 2) continue;
        if (ins[i]) g->insert_edge(uv[2 * i], uv[2 * i + 1]);
        else g->remove_edge(uv[2 * i], uv[2 * i + 1]);
    }
}
int64_t orc_graph_nnz(void* gp) {
    OGraph* g = (OGraph*)gp;
    int64_t s = 0;
    for (int v = 0; v < g->n; v++) s += g->degree(v);
    return s;
}
void orc_graph_export(void* gp, int64_t* off, int32_t* adj) {
    OGraph* g = (OGraph*)gp;
    std::vector<int> row;
    off[0] = 0;
    for (int v = 0; v < g->n; v++) {
        g->neighbors_into(v, row);
        std::copy(row.begin(), row.end(), adj + off[v]);
        off[v + 1] = off[v] + (int64_t)row.size();
    }
}

// ---- engines ------------------------------------------------------------------------------
// problem: 0 MIS (reference rule), 1 coloring, 2 BFS, 3 CC, 4 MIS (vertex-id priority).
// init: MIS 0/1 flags, coloring colours, BFS levels (-1 unreached), CC root ids (resolved).
// bound: BFS cascade bound / CC search bound; < 0 selects the reference default
// (BFS 200; CC 5000, or n when the average degree is below 10).
// flags: bit 0 = defer (the reference default); bit 1 = MIS-id classifies against the base.
void* orc_engine_new(int problem, int64_t n, const int64_t* off, const int32_t* adj, const int32_t* init,
                     int64_t bound, int flags) {
    Engine* e = nullptr;
    bool defer = flags & 1;
    switch (problem) {
    case 0: {
        auto* x = new OMisRef();
        x->mis.assign(init, init + n);
        e = x;
        break;
    }
    case 1: {
        auto* x = new OColoring();
        x->color.assign(init, init + n);
        x->marker.assign((size_t)n, -2);
        e = x;
        break;
    }
    case 2: {
        auto* x = new OBfs();
        x->hl.assign(init, init + n);
        x->dl = x->hl;
        x->bound = bound < 0 ? 200 : bound;
        x->defer = defer;
        e = x;
        break;
    }
    case 3: {
        auto* x = new OCc();
        std::vector<int> roots(init, init + n);
        x->reset_from_roots(roots);
        double avg = (double)off[n] / (double)n;   // directed entries / nodes (scout_cc.cu:466-469)
        x->bound = bound >= 0 ? bound : (avg < 10.0 ? n : 5000);
        x->defer = defer;
        e = x;
        break;
    }
    case 4: {
        auto* x = new OMisId();
        x->mis.assign(init, init + n);
        x->against_base = (flags & 2) != 0;
        e = x;
        break;
    }
    default:
        return nullptr;
    }
    e->problem = problem;
    e->g = make_graph(n, off, adj);
    return e;
}
void orc_engine_free(void* e) { delete (Engine*)e; }
void orc_engine_batch(void* e, const int32_t* uv, int64_t m) { ((Engine*)e)->batch(uv, m); }
void orc_engine_finish(void* e) { ((Engine*)e)->finish(); }
void orc_engine_solution(void* e, int32_t* out) { ((Engine*)e)->solution(out); }
void orc_engine_stats(void* e, int64_t* out) { std::memcpy(out, ((Engine*)e)->st, sizeof(int64_t) * S_NSTATS); }
void* orc_engine_graph(void* e) { return &((Engine*)e)->g; }

// ---- ground truth -------------------------------------------------------------------------
void orc_gt_bfs(int64_t n, const int64_t* off, const int32_t* adj, int source, int32_t* out) {
    for (int64_t v = 0; v < n; v++) out[v] = UNREACHED;
    std::vector<int> q = {source};
    out[source] = 0;
    for (size_t h = 0; h < q.size(); h++) {
        int x = q[h];
        for (int64_t i = off[x]; i < off[x + 1]; i++)
            if (out[adj[i]] == UNREACHED) { out[adj[i]] = out[x] + 1; q.push_back(adj[i]); }
    }
}
void orc_gt_cc(int64_t n, const int64_t* off, const int32_t* adj, int32_t* out) {
    OGraph g = make_graph(n, off, adj);
    std::vector<int> lab;
    gt_cc_graph(g, lab);
    std::copy(lab.begin(), lab.end(), out);
}
void orc_gt_greedy_color(int64_t n, const int64_t* off, const int32_t* adj, int32_t* out) {
    for (int64_t v = 0; v < n; v++) out[v] = -1;
    std::vector<int64_t> mark;
    for (int64_t v = 0; v < n; v++) {
        for (int64_t i = off[v]; i < off[v + 1]; i++) {
            int c = out[adj[i]];
            if (c >= 0) { if (c >= (int)mark.size()) mark.resize(c + 1, -1); mark[c] = v; }
        }
        int c = 0;
        while (c < (int)mark.size() && mark[c] == v) c++;
        out[v] = c;
    }
}
void orc_gt_greedy_mis(int64_t n, const int64_t* off, const int32_t* adj, int32_t* out) {
    std::vector<char> blocked((size_t)n, 0);
    for (int64_t v = 0; v < n; v++) {
        out[v] = 0;
        if (blocked[v]) continue;
        out[v] = 1;
        for (int64_t i = off[v]; i < off[v + 1]; i++) blocked[adj[i]] = 1;
    }
}
// Returns the number of edges with both ends in the set (independence violations) and
// stores in *undominated the number of non-members without a member neighbour.
int64_t orc_check_mis(int64_t n, const int64_t* off, const int32_t* adj, const int32_t* flags, int64_t* undominated) {
    int64_t bad = 0, und = 0;
    for (int64_t v = 0; v < n; v++) {
        bool dom = false;
        for (int64_t i = off[v]; i < off[v + 1]; i++) {
            if (flags[v] && flags[adj[i]]) bad++;
            if (flags[adj[i]]) dom = true;
        }
        if (!flags[v] && !dom) und++;
    }
    if (undominated) *undominated = und;
    return bad / 2;
}
// Number of directed entries whose endpoints share a colour (2x the monochromatic edges).
int64_t orc_check_coloring(int64_t n, const int64_t* off, const int32_t* adj, const int32_t* color) {
    int64_t bad = 0;
    for (int64_t v = 0; v < n; v++)
        for (int64_t i = off[v]; i < off[v + 1]; i++)
            if (color[v] == color[adj[i]]) bad++;
    return bad;
}

}  // extern "C"

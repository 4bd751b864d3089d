// multi.cu -- the batched multi-stream engine.
//
// The reference runs one update stream per process (one graph, one problem, batches in
// order: scout_bfs.cu:517-629, scout_cc.cu:443-554, scout_coloring.cu:279-371,
// scout_mis.cu:769-1013). Many small independent streams would each pay the whole per-batch
// fixed cost (about fifty kernel launches and two host synchronisations here). The batched
// engine keeps K streams of one problem as a disjoint union in one HBM graph store: stream k
// owns vertex ids [base_k, base_k + n_k). A round takes at most one pending batch of each
// stream, offsets its ids into the stream's range and runs the union of the round's batches
// as ONE batch through the engine: one merge pass, one persistent repair kernel whose device
// work queues hold the work items of every stream in the round, one commit. Streams share
// no vertex, and every repair rule is local to a connected component (BFS levels with one
// level-0 root per stream, min-vertex-id component labels, lower-id-wins colour rounds,
// vertex-id-priority MIS), so each stream's solution is exactly what it would be alone:
// ids are offset, never reordered, inside a stream.
#include "ctx.cuh"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

extern "C" int scout_graph_reserve(scout_ctx*, int64_t, int64_t);

namespace scout {
int host_fail(int code, const std::string& msg);
}

struct scout_multi {
    scout_ctx* ctx = nullptr;
    int problem = 0;
    struct Stream {
        int64_t n = 0, base = 0;
        std::vector<int64_t> off;
        std::vector<int32_t> adj;
        std::vector<int32_t> init;
        int32_t source = 0;
    };
    std::vector<Stream> streams;
    std::vector<int64_t> bases;   // stream bases, ascending
    int64_t total_n = 0;
    bool sealed = false;
    bool staged = false;          // a round is assembled in pin for scout_multi_run_all
    int64_t staged_total = 0;
    bool staged_ops = false;
    scout_edge* pin = nullptr;    // page-locked union batch
    uint8_t* pin_ops = nullptr;
    int64_t pin_cap = 0;
    int64_t last_round_edits = 0;
};

using namespace scout;

namespace {

int mfail(scout_multi* m, int code, const std::string& msg) {
    if (m && m->ctx) m->ctx->err = msg;
    return host_fail(code, msg);
}

int multi_seal(scout_multi* m) {
    if (m->sealed) return SCOUT_OK;
    if (m->streams.empty()) return mfail(m, SCOUT_E_STATE, "no stream added");
    scout_ctx* c = m->ctx;
    int64_t nnz = 0;
    for (auto& s : m->streams) nnz += s.off.back();
    SCOUT_RC(scout_graph_reserve(c, m->total_n, nnz));
    int slot = 0;
    for (auto& s : m->streams) {
        std::vector<int32_t> ids(s.n), elems(s.adj.size());
        for (int64_t v = 0; v < s.n; v++) ids[v] = (int32_t)(s.base + v);
        for (size_t i = 0; i < s.adj.size(); i++) elems[i] = (int32_t)(s.adj[i] + s.base);
        SCOUT_RC(scout_stage_rows(c, slot, ids.data(), s.off.data(), elems.data(), s.n, (int64_t)elems.size()));
        slot ^= 1;
    }
    SCOUT_RC(scout_graph_seal(c));
    // the union's initial solution: labels are vertex ids and move with the stream's base
    std::vector<int32_t> init(m->total_n);
    for (auto& s : m->streams)
        for (int64_t v = 0; v < s.n; v++)
            init[s.base + v] = (m->problem == SCOUT_CC) ? (int32_t)(s.init[v] + s.base) : s.init[v];
    SCOUT_RC(scout_state_upload(c, m->problem, init.data(), m->total_n));
    if (m->problem == SCOUT_BFS) {
        std::vector<int32_t> src;
        for (auto& s : m->streams) src.push_back((int32_t)(s.base + s.source));
        SCOUT_RC(dev_alloc(c, (void**)&c->d_sources, src.size() * 4, "BFS roots"));
        SCOUT_CU(c, cudaMemcpy(c->d_sources, src.data(), src.size() * 4, cudaMemcpyHostToDevice));
        c->nsrc = (int)src.size();
        c->source = src[0];
    }
    for (auto& s : m->streams) {   // the device holds the graphs now
        std::vector<int64_t>().swap(s.off);
        std::vector<int32_t>().swap(s.adj);
        std::vector<int32_t>().swap(s.init);
    }
    m->sealed = true;
    return SCOUT_OK;
}

int stream_of(const scout_multi* m, int64_t id) {
    auto it = std::upper_bound(m->bases.begin(), m->bases.end(), id);
    return (int)(it - m->bases.begin()) - 1;
}

}  // namespace

extern "C" {

int scout_multi_create(int device, int problem, uint64_t hbm_budget_bytes, scout_multi** out) {
    if (!out) return host_fail(SCOUT_E_INVALID, "scout_multi_create: null output");
    *out = nullptr;
    if (problem < SCOUT_MIS || problem > SCOUT_CC) return host_fail(SCOUT_E_INVALID, "unknown problem");
    scout_ctx* c = nullptr;
    SCOUT_RC(scout_ctx_create(device, hbm_budget_bytes, &c));
    scout_multi* m = new scout_multi();
    m->ctx = c;
    m->problem = problem;
    *out = m;
    return SCOUT_OK;
}

int scout_multi_destroy(scout_multi* m) {
    if (!m) return SCOUT_OK;
    if (m->pin) cudaFreeHost(m->pin);
    if (m->pin_ops) cudaFreeHost(m->pin_ops);
    scout_ctx_destroy(m->ctx);
    delete m;
    return SCOUT_OK;
}

scout_ctx* scout_multi_context(scout_multi* m) { return m ? m->ctx : nullptr; }

int scout_multi_add_stream(scout_multi* m, int64_t n, const int64_t* off, const int32_t* adj, const int32_t* init,
                           int32_t source, int32_t* stream_id) {
    if (!m || n < 1 || !off || !init || (off[n] > 0 && !adj)) return mfail(m, SCOUT_E_INVALID, "bad stream arguments");
    if (m->sealed) return mfail(m, SCOUT_E_STATE, "streams are added before the first round");
    if (m->total_n + n >= INT32_MAX) return mfail(m, SCOUT_E_CAPACITY, "the union of the streams exceeds 2^31 - 1 vertices");
    if (m->problem == SCOUT_BFS && (source < 0 || source >= n)) return mfail(m, SCOUT_E_INVALID, "source out of range");
    scout_multi::Stream s;
    s.n = n;
    s.base = m->total_n;
    s.off.assign(off, off + n + 1);
    if (s.off[0] != 0) return mfail(m, SCOUT_E_INVALID, "offsets must start at 0");
    for (int64_t v = 0; v < n; v++)
        if (s.off[v + 1] < s.off[v]) return mfail(m, SCOUT_E_INVALID, "offsets must be non-decreasing");
    s.adj.assign(adj, adj + off[n]);
    for (int32_t w : s.adj)
        if (w < 0 || w >= n) return mfail(m, SCOUT_E_INVALID, "neighbour id out of range");
    s.init.assign(init, init + n);
    if (m->problem == SCOUT_CC)
        for (int32_t l : s.init)
            if (l < 0 || l >= n) return mfail(m, SCOUT_E_INVALID, "component label out of range");
    s.source = source;
    m->bases.push_back(s.base);
    m->total_n += n;
    m->streams.push_back(std::move(s));
    if (stream_id) *stream_id = (int32_t)(m->streams.size() - 1);
    return SCOUT_OK;
}

int scout_multi_seal(scout_multi* m) {
    if (!m) return SCOUT_E_INVALID;
    return multi_seal(m);
}

}  // extern "C"

namespace {

// The union batch of a round in the engine's page-locked buffer: stream-local ids offset
// into the stream's range; an id outside the stream's graph becomes -1, which the engine
// skips like any out-of-range edit.
int assemble(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
             const int64_t* counts, const uint8_t* const* ops, int64_t* total_out, bool* any_ops_out) {
    if (!m || k < 0 || (k > 0 && (!stream_ids || !edits || !counts))) return mfail(m, SCOUT_E_INVALID, "bad round arguments");
    SCOUT_RC(multi_seal(m));
    const int S = (int)m->streams.size();
    std::vector<int64_t> start(k + 1, 0);
    std::vector<char> seen(S, 0);
    bool any_ops = false;
    for (int i = 0; i < k; i++) {
        const int sid = stream_ids[i];
        if (sid < 0 || sid >= S) return mfail(m, SCOUT_E_INVALID, "stream id out of range");
        if (seen[sid]) return mfail(m, SCOUT_E_INVALID, "a round holds at most one batch per stream");
        seen[sid] = 1;
        if (counts[i] < 0 || (counts[i] > 0 && !edits[i])) return mfail(m, SCOUT_E_INVALID, "bad batch");
        start[i + 1] = start[i] + counts[i];
        any_ops |= ops && ops[i];
    }
    const int64_t total = start[k];
    if (total > m->pin_cap) {
        if (m->pin) cudaFreeHost(m->pin);
        if (m->pin_ops) cudaFreeHost(m->pin_ops);
        m->pin = nullptr;
        m->pin_ops = nullptr;
        m->pin_cap = 0;
        const int64_t cap = total + total / 4 + 4096;
        SCOUT_CU(m->ctx, cudaHostAlloc((void**)&m->pin, (size_t)cap * sizeof(scout_edge), cudaHostAllocPortable));
        SCOUT_CU(m->ctx, cudaHostAlloc((void**)&m->pin_ops, (size_t)cap, cudaHostAllocPortable));
        m->pin_cap = cap;
    }
#pragma omp parallel for schedule(dynamic, 1) if (total > 65536)
    for (int i = 0; i < k; i++) {
        const scout_multi::Stream& s = m->streams[stream_ids[i]];
        const scout_edge* src = edits[i];
        scout_edge* dst = m->pin + start[i];
        const int32_t base = (int32_t)s.base, n = (int32_t)s.n;
        for (int64_t j = 0; j < counts[i]; j++) {
            const int32_t u = src[j].u, v = src[j].v;
            const bool ok = u >= 0 && u < n && v >= 0 && v < n;
            dst[j].u = ok ? u + base : -1;
            dst[j].v = ok ? v + base : -1;
        }
        if (any_ops) {
            if (ops[i]) std::memcpy(m->pin_ops + start[i], ops[i], (size_t)counts[i]);
            else std::memset(m->pin_ops + start[i], SCOUT_OP_TOGGLE, (size_t)counts[i]);
        }
    }
    m->last_round_edits = total;
    *total_out = total;
    *any_ops_out = any_ops;
    return SCOUT_OK;
}

}  // namespace

extern "C" {

int scout_multi_round(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops, const scout_sched* sched,
                      scout_batch_stats* stats) {
    int64_t total = 0;
    bool any_ops = false;
    SCOUT_RC(assemble(m, k, stream_ids, edits, counts, ops, &total, &any_ops));
    return scout_repair(m->ctx, m->problem, m->pin, any_ops ? m->pin_ops : nullptr, total, sched, stats);
}

int scout_multi_stage(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops) {
    int64_t total = 0;
    bool any_ops = false;
    if (m) m->staged = false;
    SCOUT_RC(assemble(m, k, stream_ids, edits, counts, ops, &total, &any_ops));
    m->staged = true;
    m->staged_total = total;
    m->staged_ops = any_ops;
    return SCOUT_OK;
}

int scout_multi_run_all(int32_t ne, scout_multi* const* ms, const scout_sched* sched, scout_batch_stats* stats) {
    if (ne < 1 || ne > 4 || !ms || !stats) return host_fail(SCOUT_E_INVALID, "bad round arguments");
    scout_ctx* cs[4];
    int problems[4];
    const scout_edge* edits[4];
    const uint8_t* ops[4];
    int64_t counts[4];
    for (int i = 0; i < ne; i++) {
        scout_multi* m = ms[i];
        if (!m || !m->staged) return mfail(m, SCOUT_E_STATE, "every engine of a fused round needs a staged round");
        cs[i] = m->ctx;
        problems[i] = m->problem;
        edits[i] = m->pin;
        ops[i] = m->staged_ops ? m->pin_ops : nullptr;
        counts[i] = m->staged_total;
        std::memset(&stats[i], 0, sizeof(scout_batch_stats));
    }
    const int rc = union_run(cs, problems, edits, ops, counts, ne, sched, stats);
    for (int i = 0; i < ne; i++) ms[i]->staged = false;
    return rc;
}

int scout_multi_probe(scout_multi* m, int32_t k, const int32_t* stream_ids, const scout_edge* const* edits,
                      const int64_t* counts, const uint8_t* const* ops, const scout_sched* sched, double* variant_ms,
                      float* features, scout_batch_stats* stats) {
    int64_t total = 0;
    bool any_ops = false;
    SCOUT_RC(assemble(m, k, stream_ids, edits, counts, ops, &total, &any_ops));
    return scout_repair_probe(m->ctx, m->problem, m->pin, any_ops ? m->pin_ops : nullptr, total, sched, variant_ms,
                              features, stats);
}

int scout_multi_commit(scout_multi* m, int32_t* const* mirrors, int64_t* changed) {
    if (!m || !mirrors) return mfail(m, SCOUT_E_INVALID, "bad commit arguments");
    if (!m->sealed) return mfail(m, SCOUT_E_STATE, "no round ran");
    scout_ctx* c = m->ctx;
    // the union's changed entries, then a scatter into each stream's mirror
    const int32_t* pairs = nullptr;
    int64_t cnt = 0;
    SCOUT_RC(commit_gather(c, m->problem, &pairs, &cnt));
    int64_t diff = 0;
    for (int64_t i = 0; i < cnt; i++) {
        const int64_t id = pairs[2 * i];
        int32_t x = pairs[2 * i + 1];
        if (id < 0 || id >= m->total_n) continue;
        const int k = stream_of(m, id);
        int32_t* mir = mirrors[k];
        if (!mir) continue;
        const scout_multi::Stream& s = m->streams[k];
        if (m->problem == SCOUT_CC) x -= (int32_t)s.base;
        const int64_t v = id - s.base;
        if (mir[v] != x) { mir[v] = x; diff++; }
    }
    if (changed) *changed = diff;
    return SCOUT_OK;
}

int scout_multi_download(scout_multi* m, int32_t stream, int32_t* out, int64_t n) {
    if (!m || !out) return mfail(m, SCOUT_E_INVALID, "bad download arguments");
    SCOUT_RC(multi_seal(m));
    if (stream < 0 || stream >= (int32_t)m->streams.size()) return mfail(m, SCOUT_E_INVALID, "stream id out of range");
    const scout_multi::Stream& s = m->streams[stream];
    if (n != s.n) return mfail(m, SCOUT_E_INVALID, "output size differs from the stream's vertex count");
    scout_ctx* c = m->ctx;
    int32_t* d = nullptr;
    switch (m->problem) {
    case SCOUT_MIS: d = c->mis; break;
    case SCOUT_COLORING: d = c->color; break;
    case SCOUT_BFS: d = c->level; break;
    default: d = c->label; break;
    }
    cudaSetDevice(c->device);
    SCOUT_CU(c, cudaMemcpyAsync(out, d + s.base, (size_t)s.n * 4, cudaMemcpyDeviceToHost, c->s_main));
    SCOUT_CU(c, cudaStreamSynchronize(c->s_main));
    if (m->problem == SCOUT_CC)
        for (int64_t v = 0; v < s.n; v++) out[v] -= (int32_t)s.base;
    return SCOUT_OK;
}

int scout_multi_reserve(scout_multi* m, int64_t max_round_edits) {
    if (!m) return SCOUT_E_INVALID;
    SCOUT_RC(multi_seal(m));
    if (max_round_edits > m->pin_cap) {
        if (m->pin) cudaFreeHost(m->pin);
        if (m->pin_ops) cudaFreeHost(m->pin_ops);
        m->pin = nullptr;
        m->pin_ops = nullptr;
        m->pin_cap = 0;
        SCOUT_CU(m->ctx, cudaHostAlloc((void**)&m->pin, (size_t)max_round_edits * sizeof(scout_edge), cudaHostAllocPortable));
        SCOUT_CU(m->ctx, cudaHostAlloc((void**)&m->pin_ops, (size_t)max_round_edits, cudaHostAllocPortable));
        m->pin_cap = max_round_edits;
    }
    return scout_reserve(m->ctx, max_round_edits);
}

int scout_multi_streams(scout_multi* m, int32_t* count, int64_t* total_vertices) {
    if (!m) return SCOUT_E_INVALID;
    if (count) *count = (int32_t)m->streams.size();
    if (total_vertices) *total_vertices = m->total_n;
    return SCOUT_OK;
}

}  // extern "C"

// graph_host.cpp -- .egr reader/writer, edge-update scratchpad, hybrid graph and compactor.
//
// Behaviour follows the reference's core/FlashGraph.h and core/flash_compactor.h; errors
// are returned as SCOUT_E* codes instead of exit(1).
#include "host.hpp"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace scout {

static thread_local std::string g_host_err;

int host_fail(int code, const std::string& msg) {
    g_host_err = msg;
    return code;
}
const char* host_last_error() { return g_host_err.c_str(); }

// ---------------------------------------------------------------------------------------
// EgrFile (FlashGraph::map_file / adopt, FlashGraph.h:106-117, 130-192)
// ---------------------------------------------------------------------------------------
int EgrFile::open(const std::string& path, bool madv_random) {
    close();
    int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) return host_fail(SCOUT_E_IO, "could not open " + path);
    struct stat st;
    if (fstat(fd, &st) != 0) { ::close(fd); return host_fail(SCOUT_E_IO, "fstat failed for " + path); }
    size_t sz = (size_t)st.st_size;
    if (sz < 8) { ::close(fd); return host_fail(SCOUT_E_FORMAT, "truncated .egr header in " + path); }
    void* m = mmap(nullptr, sz, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) { ::close(fd); return host_fail(SCOUT_E_IO, "mmap failed for " + path); }
    if (madv_random) madvise(m, sz, MADV_RANDOM);   // scattered row access: no readahead

    const char* p = (const char*)m;
    int32_t nodes, e32;
    std::memcpy(&nodes, p, 4);
    std::memcpy(&e32, p + 4, 4);
    size_t hdr = 8;
    uint64_t edges;
    bool wide;
    if (e32 == -1) {
        if (sz < 16) { munmap(m, sz); ::close(fd); return host_fail(SCOUT_E_FORMAT, "truncated wide header in " + path); }
        std::memcpy(&edges, p + 8, 8);
        hdr = 16;
        wide = true;
    } else {
        if (nodes < 1 || e32 < 0) {
            munmap(m, sz); ::close(fd);
            return host_fail(SCOUT_E_FORMAT, "invalid header in " + path);
        }
        edges = (uint64_t)e32;
        wide = false;
    }
    if (nodes < 1) { munmap(m, sz); ::close(fd); return host_fail(SCOUT_E_FORMAT, "invalid node count in " + path); }
    size_t stride = wide ? 8 : 4;
    size_t need = hdr + (size_t)(nodes + 1) * stride + (size_t)edges * 4;
    if (sz < need) {
        munmap(m, sz); ::close(fd);
        return host_fail(SCOUT_E_FORMAT, "file " + path + " is shorter than its header declares");
    }
    fd_ = fd;
    base_ = m;
    size_ = sz;
    n_ = nodes;
    e_ = edges;
    wide_ = wide;
    nindex_ = p + hdr;
    nlist_ = (const int32_t*)(p + hdr + (size_t)(nodes + 1) * stride);
    path_ = path;
    // The offsets must be monotone and end at the edge count, or row reads would leave
    // the mapping.
    if (off(0) != 0 || (uint64_t)off(n_) != e_) {
        close();
        return host_fail(SCOUT_E_FORMAT, "nindex of " + path + " does not span [0, edges]");
    }
    return SCOUT_OK;
}

void EgrFile::close() {
    if (base_ && base_ != MAP_FAILED) munmap(base_, size_);
    if (fd_ >= 0) ::close(fd_);
    base_ = nullptr;
    fd_ = -1;
    size_ = 0;
    n_ = 0;
    e_ = 0;
    nindex_ = nullptr;
    nlist_ = nullptr;
}

static bool fwrite_all(const void* p, size_t sz, size_t cnt, FILE* f) {
    return cnt == 0 || std::fwrite(p, sz, cnt, f) == cnt;
}

int write_egr(const std::string& path, int64_t n, const int64_t* off, const int32_t* adj, bool wide) {
    if (n < 1 || n > INT32_MAX) return host_fail(SCOUT_E_INVALID, "node count out of range");
    int64_t nnz = off[n];
    if (!wide && nnz > INT32_MAX) return host_fail(SCOUT_E_INVALID, "narrow .egr needs fewer than 2^31 entries");
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return host_fail(SCOUT_E_IO, "could not open " + path + " for writing");
    int32_t n32 = (int32_t)n;
    bool ok = fwrite_all(&n32, 4, 1, f);
    if (wide) {
        int32_t s = -1;
        uint64_t e = (uint64_t)nnz;
        ok = ok && fwrite_all(&s, 4, 1, f) && fwrite_all(&e, 8, 1, f);
        ok = ok && fwrite_all(off, 8, (size_t)n + 1, f);
    } else {
        int32_t e = (int32_t)nnz;
        ok = ok && fwrite_all(&e, 4, 1, f);
        std::vector<int32_t> o32((size_t)n + 1);
        for (int64_t i = 0; i <= n; i++) o32[i] = (int32_t)off[i];
        ok = ok && fwrite_all(o32.data(), 4, o32.size(), f);
    }
    ok = ok && fwrite_all(adj, 4, (size_t)nnz, f);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? SCOUT_OK : host_fail(SCOUT_E_IO, "short write to " + path);
}

// ---------------------------------------------------------------------------------------
// Scratchpad (DeltaOverlay, FlashGraph.h:200-311)
// ---------------------------------------------------------------------------------------
int Scratchpad::adjacency(int32_t u, int32_t v) const {
    auto it = rows.find(u);
    if (it == rows.end()) return -1;
    const DeltaRow& r = it->second;
    if (std::find(r.add.begin(), r.add.end(), v) != r.add.end()) return 1;
    if (r.tomb.count(v)) return 0;
    return -1;
}

void Scratchpad::insert_edge(int32_t u, int32_t v) {
    // un_tombstone (FlashGraph.h:284-291): a tombstoned base edge comes back in place.
    auto iu = rows.find(u);
    if (iu != rows.end() && iu->second.tomb.count(v)) {
        iu->second.tomb.erase(v);
        auto iv = rows.find(v);
        if (iv != rows.end()) iv->second.tomb.erase(u);
    } else {
        rows[u].add.push_back(v);
        rows[v].add.push_back(u);
    }
    edit_count++;
}

void Scratchpad::remove_edge(int32_t u, int32_t v) {
    // forget_delta_edge (FlashGraph.h:295-310): an added edge is forgotten (first copy).
    bool forgotten = false;
    auto iu = rows.find(u);
    if (iu != rows.end()) {
        auto& au = iu->second.add;
        auto pu = std::find(au.begin(), au.end(), v);
        if (pu != au.end()) {
            au.erase(pu);
            auto iv = rows.find(v);
            if (iv != rows.end()) {
                auto& av = iv->second.add;
                auto pv = std::find(av.begin(), av.end(), u);
                if (pv != av.end()) av.erase(pv);
            }
            forgotten = true;
        }
    }
    if (!forgotten) {
        rows[u].tomb.insert(v);
        rows[v].tomb.insert(u);
    }
    edit_count++;
}

// ---------------------------------------------------------------------------------------
// HGraph (HybridGraph, FlashGraph.h:331-388)
// ---------------------------------------------------------------------------------------
bool HGraph::is_adjacent(int32_t u, int32_t v) const {
    int d = delta.adjacency(u, v);
    if (d >= 0) return d == 1;
    const int32_t* b = base.row(u);
    const int32_t* e = b + base.degree(u);
    for (const int32_t* p = b; p != e; ++p)
        if (*p == v) return true;
    return false;
}

int64_t HGraph::degree(int32_t v) const {
    int64_t d = base.degree(v);
    const DeltaRow* r = delta.find(v);
    if (r) d += (int64_t)r->add.size() - (int64_t)r->tomb.size();
    return d;
}

int64_t HGraph::neighbors_write(int32_t v, int32_t* out) const {
    const int32_t* b = base.row(v);
    int64_t bd = base.degree(v);
    const DeltaRow* r = delta.find(v);
    int64_t k = 0;
    if (!r || r->tomb.empty()) {
        std::memcpy(out, b, (size_t)bd * 4);
        k = bd;
    } else {
        for (int64_t i = 0; i < bd; i++)
            if (!r->tomb.count(b[i])) out[k++] = b[i];
    }
    if (r) {
        for (int32_t a : r->add) out[k++] = a;
    }
    return k;
}

void HGraph::neighbors_into(int32_t v, std::vector<int32_t>& out) const {
    const DeltaRow* r = delta.find(v);
    int64_t cap = base.degree(v) + (r ? (int64_t)r->add.size() : 0);
    out.resize((size_t)cap);
    int64_t k = neighbors_write(v, out.data());
    out.resize((size_t)k);
}

// compact_flash_graph (flash_compactor.h:23-119) followed by remap + clear. The bytes are the
// reference's (header, offsets, then every merged row in vertex order); the merged degrees
// and rows are computed over the host threads (the scratchpad and the mapped base graph are
// only read), the rows in windows of about COMPACT_WINDOW entries, each gathered into one
// buffer at its final offsets and written with one call.
constexpr uint64_t COMPACT_WINDOW = 1ull << 25;   // 32 M entries, 128 MB

int HGraph::compact(const std::string& out_path) {
    const int64_t n = base.nodes();
    std::vector<uint64_t> nidx((size_t)n + 1);
    std::vector<int64_t> deg((size_t)n);
    int64_t bad = n;
#pragma omp parallel for schedule(static) reduction(min : bad)
    for (int64_t v = 0; v < n; v++) {
        deg[(size_t)v] = degree((int32_t)v);
        if (deg[(size_t)v] < 0) bad = std::min(bad, v);
    }
    if (bad < n) return host_fail(SCOUT_E_STATE, "negative merged degree at vertex " + std::to_string(bad));
    nidx[0] = 0;
    for (int64_t v = 0; v < n; v++) nidx[(size_t)v + 1] = nidx[(size_t)v] + (uint64_t)deg[(size_t)v];
    const std::string tmp = out_path + ".tmp." + std::to_string(getpid());
    FILE* out = std::fopen(tmp.c_str(), "wb");
    if (!out) return host_fail(SCOUT_E_IO, "could not open " + tmp + " for writing");
    int32_t n32 = (int32_t)n, sentinel = -1;
    uint64_t ne = nidx[(size_t)n];
    bool ok = fwrite_all(&n32, 4, 1, out) && fwrite_all(&sentinel, 4, 1, out) && fwrite_all(&ne, 8, 1, out) &&
              fwrite_all(nidx.data(), 8, nidx.size(), out);
    std::vector<int32_t> buf;
    for (int64_t v0 = 0; ok && v0 < n;) {
        // the window: vertices [v0, v1) whose rows hold at most COMPACT_WINDOW entries (one
        // vertex at least)
        auto it = std::upper_bound(nidx.begin() + v0 + 1, nidx.end(), nidx[(size_t)v0] + COMPACT_WINDOW);
        int64_t v1 = (int64_t)(it - nidx.begin()) - 1;
        if (v1 <= v0) v1 = v0 + 1;
        const uint64_t w0 = nidx[(size_t)v0];
        buf.resize((size_t)(nidx[(size_t)v1] - w0));
        int64_t mism = n;
#pragma omp parallel reduction(min : mism)
        {
            std::vector<int32_t> row;
#pragma omp for schedule(dynamic, 1024)
            for (int64_t v = v0; v < v1; v++) {
                neighbors_into((int32_t)v, row);
                if ((uint64_t)row.size() != nidx[(size_t)v + 1] - nidx[(size_t)v]) {
                    mism = std::min(mism, v);
                } else if (!row.empty()) {
                    std::memcpy(buf.data() + (nidx[(size_t)v] - w0), row.data(), row.size() * 4);
                }
            }
        }
        if (mism < n) {
            std::fclose(out);
            std::remove(tmp.c_str());
            return host_fail(SCOUT_E_STATE, "degree mismatch at vertex " + std::to_string(mism));
        }
        ok = fwrite_all(buf.data(), 4, buf.size(), out);
        v0 = v1;
    }
    ok = ok && std::fflush(out) == 0 && fsync(fileno(out)) == 0;
    std::fclose(out);
    if (!ok) { std::remove(tmp.c_str()); return host_fail(SCOUT_E_IO, "write to " + tmp + " failed"); }
    if (std::rename(tmp.c_str(), out_path.c_str()) != 0) {
        std::remove(tmp.c_str());
        return host_fail(SCOUT_E_IO, "rename " + tmp + " -> " + out_path + " failed");
    }
    std::string dir = ".";
    size_t slash = out_path.find_last_of('/');
    if (slash != std::string::npos) dir = out_path.substr(0, slash);
    int dfd = ::open(dir.c_str(), O_RDONLY);
    if (dfd >= 0) { fsync(dfd); ::close(dfd); }
    // remap (FlashGraph.h:56-66): the new mapping is built before the old one is dropped.
    EgrFile fresh;
    int rc = fresh.open(out_path, true);
    if (rc != SCOUT_OK) return rc;
    base.close();
    rc = base.open(out_path, true);
    delta.clear();
    return rc;
}

}  // namespace scout

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
using namespace scout;

extern "C" {

int scout_egr_open(const char* path, int madv_random, scout_egr** out) {
    if (!path || !out) return host_fail(SCOUT_E_INVALID, "null argument");
    auto* h = new scout_egr();
    int rc = h->f.open(path, madv_random != 0);
    if (rc != SCOUT_OK) { delete h; return rc; }
    *out = h;
    return SCOUT_OK;
}
int scout_egr_close(scout_egr* g) { delete g; return SCOUT_OK; }
int64_t scout_egr_nodes(const scout_egr* g) { return g ? g->f.nodes() : SCOUT_E_INVALID; }
int64_t scout_egr_edges(const scout_egr* g) { return g ? (int64_t)g->f.edges() : SCOUT_E_INVALID; }
int scout_egr_is_wide(const scout_egr* g) { return g ? (int)g->f.wide() : SCOUT_E_INVALID; }
int scout_egr_offsets(const scout_egr* g, int64_t* out) {
    if (!g || !out) return host_fail(SCOUT_E_INVALID, "null argument");
    for (int64_t v = 0; v <= g->f.nodes(); v++) out[v] = g->f.off(v);
    return SCOUT_OK;
}
const int32_t* scout_egr_nlist(const scout_egr* g) { return g ? g->f.nlist() : nullptr; }
int scout_egr_write(const char* path, int64_t n, const int64_t* off, const int32_t* adj, int wide) {
    if (!path || !off || (!adj && n > 0 && off[n] > 0)) return host_fail(SCOUT_E_INVALID, "null argument");
    return write_egr(path, n, off, adj, wide != 0);
}

int scout_hgraph_open(const char* path, int madv_random, scout_hgraph** out) {
    if (!path || !out) return host_fail(SCOUT_E_INVALID, "null argument");
    auto* h = new scout_hgraph();
    int rc = h->g.open(path, madv_random != 0);
    if (rc != SCOUT_OK) { delete h; return rc; }
    *out = h;
    return SCOUT_OK;
}
int scout_hgraph_close(scout_hgraph* h) { delete h; return SCOUT_OK; }
int64_t scout_hgraph_nodes(const scout_hgraph* h) { return h ? h->g.nodes() : SCOUT_E_INVALID; }

static bool in_range(const scout_hgraph* h, int32_t v) { return v >= 0 && v < h->g.nodes(); }

int scout_hgraph_is_adjacent(const scout_hgraph* h, int32_t u, int32_t v) {
    if (!h || !in_range(h, u) || !in_range(h, v)) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    return h->g.is_adjacent(u, v) ? 1 : 0;
}
int scout_hgraph_insert(scout_hgraph* h, int32_t u, int32_t v) {
    if (!h || !in_range(h, u) || !in_range(h, v)) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    h->g.insert_edge(u, v);
    return SCOUT_OK;
}
int scout_hgraph_remove(scout_hgraph* h, int32_t u, int32_t v) {
    if (!h || !in_range(h, u) || !in_range(h, v)) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    h->g.remove_edge(u, v);
    return SCOUT_OK;
}
int64_t scout_hgraph_degree(const scout_hgraph* h, int32_t v) {
    if (!h || !in_range(h, v)) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    return h->g.degree(v);
}
int64_t scout_hgraph_neighbors(const scout_hgraph* h, int32_t v, int32_t* out, int64_t cap) {
    if (!h || !in_range(h, v)) return host_fail(SCOUT_E_INVALID, "vertex out of range");
    std::vector<int32_t> row;
    h->g.neighbors_into(v, row);
    if (out) std::memcpy(out, row.data(), sizeof(int32_t) * (size_t)std::min<int64_t>(cap, (int64_t)row.size()));
    return (int64_t)row.size();
}
int64_t scout_hgraph_delta_edits(const scout_hgraph* h) { return h ? h->g.delta.edit_count : SCOUT_E_INVALID; }
int scout_hgraph_compact(scout_hgraph* h, const char* out_path) {
    if (!h || !out_path) return host_fail(SCOUT_E_INVALID, "null argument");
    return h->g.compact(out_path);
}

}  // extern "C"

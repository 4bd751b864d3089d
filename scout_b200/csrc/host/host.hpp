// host.hpp -- internal C++ types behind scout_host.h.
//
// EgrFile      storage-resident .egr reader (mmap), the role of FlashGraph
//              (core/FlashGraph.h:35-193 in the reference).
// Scratchpad   in-memory edge-update overlay with the reference's row semantics
//              (core/FlashGraph.h:200-311): a row is the base row minus tombstoned
//              neighbours, followed by the added neighbours in insertion order.
// HGraph       EgrFile + Scratchpad (core/FlashGraph.h:331-388).
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <unordered_map>
#include <unordered_set>

#include "../../../include/scout_host.h"

namespace scout {

// Sets the thread-local message returned by scout_last_error(NULL) for host calls.
int host_fail(int code, const std::string& msg);
const char* host_last_error();

class EgrFile {
public:
    EgrFile() = default;
    EgrFile(const EgrFile&) = delete;
    EgrFile& operator=(const EgrFile&) = delete;
    ~EgrFile() { close(); }

    // Maps the file read-only; returns SCOUT_OK or an error code (never exits).
    int open(const std::string& path, bool madv_random);
    void close();

    int64_t nodes() const { return n_; }
    uint64_t edges() const { return e_; }
    bool wide() const { return wide_; }
    const std::string& path() const { return path_; }

    inline int64_t off(int64_t v) const {
        return wide_ ? (int64_t)((const uint64_t*)nindex_)[v] : (int64_t)((const int32_t*)nindex_)[v];
    }
    inline int64_t degree(int64_t v) const { return off(v + 1) - off(v); }
    inline const int32_t* row(int64_t v) const { return nlist_ + off(v); }
    const int32_t* nlist() const { return nlist_; }

private:
    int fd_ = -1;
    void* base_ = nullptr;
    size_t size_ = 0;
    int64_t n_ = 0;
    uint64_t e_ = 0;
    bool wide_ = false;
    const char* nindex_ = nullptr;
    const int32_t* nlist_ = nullptr;
    std::string path_;
};

int write_egr(const std::string& path, int64_t n, const int64_t* off, const int32_t* adj, bool wide);

// Scratchpad entry of one vertex. `add` keeps insertion order (it is appended to the row);
// `tomb` is the set of tombstoned base neighbours (every occurrence in the base row is
// skipped, as in DeltaOverlay::neighbors_into).
struct DeltaRow {
    std::vector<int32_t> add;
    std::unordered_set<int32_t> tomb;
};

class Scratchpad {
public:
    std::unordered_map<int32_t, DeltaRow> rows;
    int64_t edit_count = 0;

    // isAdjacentDelta (FlashGraph.h:209-225): 1 adjacent, 0 not adjacent, -1 undecided.
    int adjacency(int32_t u, int32_t v) const;
    void insert_edge(int32_t u, int32_t v);   // FlashGraph.h:227-234
    void remove_edge(int32_t u, int32_t v);   // FlashGraph.h:236-243
    void clear() { rows.clear(); edit_count = 0; }
    const DeltaRow* find(int32_t v) const {
        auto it = rows.find(v);
        return it == rows.end() ? nullptr : &it->second;
    }
};

class HGraph {
public:
    EgrFile base;
    Scratchpad delta;

    int open(const std::string& path, bool madv_random) { return base.open(path, madv_random); }
    int64_t nodes() const { return base.nodes(); }
    bool is_adjacent(int32_t u, int32_t v) const;
    void insert_edge(int32_t u, int32_t v) { delta.insert_edge(u, v); }
    void remove_edge(int32_t u, int32_t v) { delta.remove_edge(u, v); }
    int64_t degree(int32_t v) const;
    void neighbors_into(int32_t v, std::vector<int32_t>& out) const;
    // Writes the merged row into out (capacity >= degree(v)); returns its length.
    int64_t neighbors_write(int32_t v, int32_t* out) const;
    int compact(const std::string& out_path);
};

// Text I/O helpers (core/cli_setup.h:64-131).
int list_batch_files_sorted(const std::string& dir, std::vector<std::string>& out);
int parse_batch_text(const char* data, size_t len, int64_t n, std::vector<scout_edge>& out);
int parse_batch_file(const std::string& path, int64_t n, std::vector<scout_edge>& out);
int read_ints_fast(const std::string& path, std::vector<int64_t>& out);
int decode_state(const std::vector<int64_t>& vals, int problem, int64_t n, int32_t* sol, int64_t* aux);

// Host CSR container used by the generators.
struct Csr {
    int64_t n = 0;
    std::vector<int64_t> off;
    std::vector<int32_t> adj;
    int64_t nnz() const { return (int64_t)adj.size(); }
};

int gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, Csr& out);
int gen_stream(const Csr& g, int kind, int64_t batch_size, int64_t nbatches, double insert_ratio,
               double lowdeg_frac, uint64_t seed, scout_edge* out);
int init_state(const Csr& g, int problem, int32_t source, int32_t* out);

}  // namespace scout

struct scout_egr { scout::EgrFile f; };
struct scout_hgraph { scout::HGraph g; };
struct scout_csr { scout::Csr g; };

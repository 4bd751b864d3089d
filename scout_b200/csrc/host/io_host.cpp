// io_host.cpp -- batch folders and initial-state files (core/cli_setup.h:64-131 and the
// initial-state blocks of each reference main()).
#ifdef _OPENMP
#include <omp.h>
#endif
#include "host.hpp"

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>

namespace scout {

namespace fs = std::filesystem;

// list_batch_files_sorted (cli_setup.h:64-74): every regular file of the folder, ordered by
// the integer value of its stem ("10.mtx" after "2.mtx"). A stem that does not start with an
// integer makes the reference throw; here it is an error code.
int list_batch_files_sorted(const std::string& dir, std::vector<std::string>& out) {
    out.clear();
    std::error_code ec;
    fs::directory_iterator it(dir, ec);
    if (ec) return host_fail(SCOUT_E_IO, "could not list batch folder " + dir);
    std::vector<std::pair<long long, std::string>> files;
    for (const auto& e : it) {
        if (!e.is_regular_file()) continue;
        std::string stem = e.path().stem().string();
        const char* s = stem.c_str();
        char* end = nullptr;
        errno = 0;
        long long k = std::strtoll(s, &end, 10);
        if (end == s || errno == ERANGE || k < INT_MIN || k > INT_MAX)
            return host_fail(SCOUT_E_FORMAT, "batch file name without a numeric stem: " + e.path().string());
        files.emplace_back(k, e.path().string());
    }
    std::stable_sort(files.begin(), files.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& f : files) out.push_back(f.second);
    return SCOUT_OK;
}

static inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// One formatted int extraction as std::istream >> int does it: skip whitespace, optional
// sign, at least one digit, stop at the first non-digit; out-of-range values fail.
static inline bool extract_int(const char*& p, const char* end, int64_t& out) {
    while (p < end && is_ws(*p)) ++p;
    const char* q = p;
    bool neg = false;
    if (q < end && (*q == '+' || *q == '-')) { neg = (*q == '-'); ++q; }
    if (q >= end || *q < '0' || *q > '9') return false;
    int64_t v = 0;
    bool overflow = false;
    while (q < end && *q >= '0' && *q <= '9') {
        if (!overflow) {
            v = v * 10 + (*q - '0');
            if (v > (int64_t)INT_MAX + 1) overflow = true;
        }
        ++q;
    }
    if (overflow) return false;
    if (neg) v = -v;
    if (v > INT_MAX || v < INT_MIN) return false;
    out = v;
    p = q;
    return true;
}

// parse_batch_file (cli_setup.h:87-103) minus classification: a line is kept if its first
// two whitespace-separated tokens parse as ints; ids become 0-indexed; out-of-range ids and
// self-loops are dropped. Large files are cut at line boundaries into one chunk per host
// thread, parsed in parallel and concatenated in file order.
static void parse_lines(const char* p, const char* end, int64_t n, std::vector<scout_edge>& out) {
    while (p < end) {
        const char* nl = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        const char* le = nl ? nl : end;
        const char* q = p;
        int64_t src, dst;
        if (extract_int(q, le, src) && extract_int(q, le, dst)) {
            src--;
            dst--;
            if (src >= 0 && src < n && dst >= 0 && dst < n && src != dst)
                out.push_back(scout_edge{(int32_t)src, (int32_t)dst});
        }
        p = nl ? nl + 1 : end;
    }
}

int parse_batch_text(const char* data, size_t len, int64_t n, std::vector<scout_edge>& out) {
    out.clear();
    const char* end = data + len;
    int T = 1;
#ifdef _OPENMP
    if (len >= ((size_t)1 << 20)) T = std::max(1, std::min(omp_get_max_threads(), (int)(len >> 18)));
#endif
    if (T == 1) {
        out.reserve(len / 12);
        parse_lines(data, end, n, out);
        return SCOUT_OK;
    }
    // chunk k starts after the first newline at or past k * len / T (chunk 0 at the start)
    std::vector<const char*> cut((size_t)T + 1);
    cut[0] = data;
    cut[T] = end;
    for (int k = 1; k < T; k++) {
        const char* q = data + len * (size_t)k / (size_t)T;
        const char* nl = (const char*)std::memchr(q, '\n', (size_t)(end - q));
        cut[k] = nl ? nl + 1 : end;
        if (cut[k] < cut[k - 1]) cut[k] = cut[k - 1];
    }
    std::vector<std::vector<scout_edge>> part((size_t)T);
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int k = 0; k < T; k++) {
        part[k].reserve((size_t)(cut[k + 1] - cut[k]) / 12);
        parse_lines(cut[k], cut[k + 1], n, part[k]);
    }
    size_t total = 0;
    for (auto& v : part) total += v.size();
    out.reserve(total);
    for (auto& v : part) out.insert(out.end(), v.begin(), v.end());
    return SCOUT_OK;
}

static int slurp(const std::string& path, std::string& buf) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return host_fail(SCOUT_E_IO, "could not open " + path);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) { std::fclose(f); return host_fail(SCOUT_E_IO, "could not size " + path); }
    buf.assign((size_t)sz, '\0');
    size_t got = sz ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    buf.resize(got);
    return SCOUT_OK;
}

int parse_batch_file(const std::string& path, int64_t n, std::vector<scout_edge>& out) {
    std::string buf;
    int rc = slurp(path, buf);
    if (rc != SCOUT_OK) return rc;
    return parse_batch_text(buf.data(), buf.size(), n, out);
}

// read_ints_fast (cli_setup.h:110-131): strtoll over the whole file, skipping one byte
// whenever no integer starts at the cursor. A missing file yields no values (the reference
// returns an empty vector); here that is SCOUT_E_IO so callers can tell.
int read_ints_fast(const std::string& path, std::vector<int64_t>& out) {
    out.clear();
    std::string buf;
    int rc = slurp(path, buf);
    if (rc != SCOUT_OK) return rc;
    out.reserve(buf.size() / 4);
    const char* p = buf.c_str();
    char* e;
    while (*p) {
        long long v = std::strtoll(p, &e, 10);
        if (e == p) { ++p; continue; }
        out.push_back(v);
        p = e;
    }
    return SCOUT_OK;
}

// find_root with path compression over a parent array (scout_cc.cu:280-289). Values outside
// [0, n) are treated as self-parents (the reference would index out of bounds) and a parent
// cycle is reported as a format error (the reference would loop forever).
static int find_roots(std::vector<int32_t>& parent, int64_t n, int32_t* roots) {
    for (int64_t v = 0; v < n; v++)
        if (parent[v] < 0 || parent[v] >= n) parent[v] = (int32_t)v;
    for (int64_t v = 0; v < n; v++) {
        int32_t r = (int32_t)v;
        int64_t steps = 0;
        while (parent[r] != r) {
            r = parent[r];
            if (++steps > n) return host_fail(SCOUT_E_FORMAT, "parent cycle in component file");
        }
        int32_t x = (int32_t)v;
        while (parent[x] != r) {
            int32_t nx = parent[x];
            parent[x] = r;
            x = nx;
        }
        roots[v] = r;
    }
    return SCOUT_OK;
}

int decode_state(const std::vector<int64_t>& vals, int problem, int64_t n, int32_t* sol, int64_t* aux) {
    int64_t a = 0;
    switch (problem) {
    case SCOUT_MIS:
        std::fill(sol, sol + n, 0);
        for (int64_t id : vals) {
            int64_t node = (int64_t)(int32_t)id - 1;
            if (node >= 0 && node < n) { sol[node] = 1; a++; }
        }
        break;
    case SCOUT_COLORING: {
        std::fill(sol, sol + n, 0);
        int64_t k = std::min<int64_t>(n, (int64_t)vals.size());
        int32_t mx = -1;
        for (int64_t i = 0; i < k; i++) sol[i] = (int32_t)vals[i];
        for (int64_t i = 0; i < n; i++) mx = std::max(mx, sol[i]);
        a = (int64_t)mx + 1;
        break;
    }
    case SCOUT_BFS:
        std::fill(sol, sol + n, -1);
        for (size_t k = 0; k + 1 < vals.size(); k += 2) {
            int64_t idx = (int64_t)(int32_t)vals[k] - 1;
            int32_t lv = (int32_t)vals[k + 1];
            if (idx >= 0 && idx < n) { sol[idx] = lv; if (lv >= 0) a++; }
        }
        break;
    case SCOUT_CC: {
        std::vector<int32_t> parent((size_t)n);
        for (int64_t v = 0; v < n; v++) parent[v] = (int32_t)v;
        int64_t k = std::min<int64_t>(n, (int64_t)vals.size());
        for (int64_t i = 0; i < k; i++) parent[i] = (int32_t)vals[i];
        int rc = find_roots(parent, n, sol);
        if (rc != SCOUT_OK) return rc;
        std::vector<char> seen((size_t)n, 0);
        for (int64_t v = 0; v < n; v++)
            if (!seen[sol[v]]) { seen[sol[v]] = 1; a++; }
        break;
    }
    default:
        return host_fail(SCOUT_E_INVALID, "unknown problem");
    }
    if (aux) *aux = a;
    return SCOUT_OK;
}

}  // namespace scout

using namespace scout;

extern "C" {

int scout_parse_batch_file(const char* path, int64_t n, scout_edge* out, int64_t cap, int64_t* m) {
    if (!path || !m) return host_fail(SCOUT_E_INVALID, "null argument");
    std::vector<scout_edge> e;
    int rc = parse_batch_file(path, n, e);
    if (rc != SCOUT_OK) return rc;
    *m = (int64_t)e.size();
    if (!out || cap < (int64_t)e.size()) return e.empty() ? SCOUT_OK : host_fail(SCOUT_E_CAPACITY, "output too small");
    std::memcpy(out, e.data(), e.size() * sizeof(scout_edge));
    return SCOUT_OK;
}

int scout_read_ints(const char* path, int64_t* out, int64_t cap, int64_t* count) {
    if (!path || !count) return host_fail(SCOUT_E_INVALID, "null argument");
    std::vector<int64_t> v;
    int rc = read_ints_fast(path, v);
    if (rc != SCOUT_OK) return rc;
    *count = (int64_t)v.size();
    if (!out || cap < (int64_t)v.size()) return v.empty() ? SCOUT_OK : host_fail(SCOUT_E_CAPACITY, "output too small");
    std::memcpy(out, v.data(), v.size() * sizeof(int64_t));
    return SCOUT_OK;
}

int scout_load_state(const char* path, int problem, int64_t n, int32_t* sol, int64_t* aux) {
    if (!path || !sol || n < 1) return host_fail(SCOUT_E_INVALID, "bad argument");
    std::vector<int64_t> v;
    int rc = read_ints_fast(path, v);
    if (rc != SCOUT_OK) return rc;
    return decode_state(v, problem, n, sol, aux);
}

int scout_write_state(const char* path, int problem, int64_t n, const int32_t* sol) {
    if (!path || !sol) return host_fail(SCOUT_E_INVALID, "null argument");
    FILE* f = std::fopen(path, "w");
    if (!f) return host_fail(SCOUT_E_IO, std::string("could not open ") + path);
    std::string buf;
    buf.reserve(1 << 20);
    char tmp[48];
    for (int64_t v = 0; v < n; v++) {
        int k = 0;
        switch (problem) {
        case SCOUT_MIS: if (sol[v]) k = std::snprintf(tmp, sizeof tmp, "%lld\n", (long long)v + 1); break;
        case SCOUT_COLORING: case SCOUT_CC: k = std::snprintf(tmp, sizeof tmp, "%d\n", sol[v]); break;
        case SCOUT_BFS: k = std::snprintf(tmp, sizeof tmp, "%lld %d\n", (long long)v + 1, sol[v]); break;
        default: std::fclose(f); return host_fail(SCOUT_E_INVALID, "unknown problem");
        }
        buf.append(tmp, (size_t)k);
        if (buf.size() > (1 << 20)) { std::fwrite(buf.data(), 1, buf.size(), f); buf.clear(); }
    }
    std::fwrite(buf.data(), 1, buf.size(), f);
    return std::fclose(f) == 0 ? SCOUT_OK : host_fail(SCOUT_E_IO, "write failed");
}

int scout_write_batch_folder(const char* dir, const scout_edge* pairs, int64_t batch_size, int64_t nbatches) {
    if (!dir || (!pairs && batch_size * nbatches > 0)) return host_fail(SCOUT_E_INVALID, "null argument");
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return host_fail(SCOUT_E_IO, std::string("could not create ") + dir);
    char tmp[48];
    for (int64_t k = 0; k < nbatches; k++) {
        std::string path = std::string(dir) + "/" + std::to_string(k + 1) + ".mtx";
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) return host_fail(SCOUT_E_IO, "could not open " + path);
        std::string buf;
        buf.reserve((size_t)batch_size * 16);
        for (int64_t i = 0; i < batch_size; i++) {
            const scout_edge& e = pairs[k * batch_size + i];
            int w = std::snprintf(tmp, sizeof tmp, "%d %d\n", e.u + 1, e.v + 1);
            buf.append(tmp, (size_t)w);
        }
        std::fwrite(buf.data(), 1, buf.size(), f);
        if (std::fclose(f) != 0) return host_fail(SCOUT_E_IO, "write failed: " + path);
    }
    return SCOUT_OK;
}

}  // extern "C"

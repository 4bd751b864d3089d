// ORACLE -- benchmark baseline, not product code.
//
// From-scratch recomputation of each problem's solution on all host cores (OpenMP): the CPU
// baseline that a batch-dynamic engine has to beat, timed per batch on the updated graph.
//   BFS       direction-optimizing level-synchronous traversal from the source: top-down steps
//             claim neighbours with compare-and-swap, bottom-up steps scan unreached vertices
//             for a parent on the current level (Beamer, Asanovic, Patterson, SC 2012;
//             switch thresholds 14 and 24);
//   CC        union-find over every edge with compare-and-swap hooking of the higher root under
//             the lower one, then a flattening pass: min-vertex-id labels. The reference's host
//             recompute (src/cc/scout_cc.cu:86-116) is this algorithm;
//   colouring greedy smallest free colour in vertex-id order, and
//   MIS       greedy in vertex-id order: both sequential by definition (one core), the rules of
//             tools/greedy_color.cpp:37-52 and tools/compute_initial_mis.py:32-43.
// Built into liboracle.so next to oracle.cpp; bench.py's cpu_recompute leg calls it.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

double bfs_all_cores(int64_t n, const int64_t* off, const int32_t* adj, int32_t source, int32_t* lv) {
    const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) lv[v] = -1;
    lv[source] = 0;
    std::vector<int32_t> front{source}, next;
    const int64_t nnz = off[n];
    int64_t explored = 0;
    bool bottom_up = false;
    for (int32_t d = 0; !front.empty(); d++) {
        int64_t mf = 0;
#pragma omp parallel for reduction(+ : mf) schedule(static)
        for (int64_t i = 0; i < (int64_t)front.size(); i++) mf += off[front[i] + 1] - off[front[i]];
        explored += mf;
        if (!bottom_up && mf > (nnz - explored) / 14) bottom_up = true;
        else if (bottom_up && (int64_t)front.size() * 24 < n) bottom_up = false;
        next.clear();
        if (bottom_up) {
#pragma omp parallel
            {
                std::vector<int32_t> local;
#pragma omp for schedule(dynamic, 4096) nowait
                for (int64_t v = 0; v < n; v++) {
                    if (lv[v] >= 0) continue;
                    for (int64_t k = off[v]; k < off[v + 1]; k++)
                        if (__atomic_load_n(&lv[adj[k]], __ATOMIC_RELAXED) == d) {
                            __atomic_store_n(&lv[v], d + 1, __ATOMIC_RELAXED);
                            local.push_back((int32_t)v);
                            break;
                        }
                }
#pragma omp critical
                next.insert(next.end(), local.begin(), local.end());
            }
        } else {
#pragma omp parallel
            {
                std::vector<int32_t> local;
#pragma omp for schedule(dynamic, 64) nowait
                for (int64_t i = 0; i < (int64_t)front.size(); i++) {
                    const int32_t x = front[i];
                    for (int64_t k = off[x]; k < off[x + 1]; k++) {
                        int32_t y = adj[k];
                        int32_t un = -1;
                        if (__atomic_load_n(&lv[y], __ATOMIC_RELAXED) < 0 &&
                            __atomic_compare_exchange_n(&lv[y], &un, d + 1, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                            local.push_back(y);
                    }
                }
#pragma omp critical
                next.insert(next.end(), local.begin(), local.end());
            }
        }
        front.swap(next);
    }
    return omp_get_wtime() - t0;
}

inline int32_t find_root(int32_t* p, int32_t x) {
    while (true) {
        int32_t px = __atomic_load_n(&p[x], __ATOMIC_RELAXED);
        if (px == x) return x;
        int32_t gx = __atomic_load_n(&p[px], __ATOMIC_RELAXED);
        if (gx != px) __atomic_compare_exchange_n(&p[x], &px, gx, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
        x = gx;
    }
}

double cc_all_cores(int64_t n, const int64_t* off, const int32_t* adj, int32_t* lab) {
    const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) lab[v] = (int32_t)v;
#pragma omp parallel for schedule(dynamic, 2048)
    for (int64_t v = 0; v < n; v++) {
        for (int64_t k = off[v]; k < off[v + 1]; k++) {
            const int32_t w = adj[k];
            if (w <= v) continue;   // each undirected edge once
            int32_t a = (int32_t)v, b = w;
            while (true) {
                a = find_root(lab, a);
                b = find_root(lab, b);
                if (a == b) break;
                if (a > b) std::swap(a, b);   // hook the higher root under the lower one
                int32_t expect = b;
                if (__atomic_compare_exchange_n(&lab[b], &expect, a, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < n; v++) lab[v] = find_root(lab, (int32_t)v);
    return omp_get_wtime() - t0;
}

double greedy_color(int64_t n, const int64_t* off, const int32_t* adj, int32_t* col) {
    const double t0 = omp_get_wtime();
    std::vector<int64_t> mark;
    for (int64_t v = 0; v < n; v++) col[v] = -1;
    for (int64_t v = 0; v < n; v++) {
        for (int64_t k = off[v]; k < off[v + 1]; k++) {
            const int32_t c = col[adj[k]];
            if (c >= 0) {
                if (c >= (int32_t)mark.size()) mark.resize((size_t)c + 1, -1);
                mark[c] = v;
            }
        }
        int32_t c = 0;
        while (c < (int32_t)mark.size() && mark[c] == v) c++;
        col[v] = c;
    }
    return omp_get_wtime() - t0;
}

double greedy_mis(int64_t n, const int64_t* off, const int32_t* adj, int32_t* in) {
    const double t0 = omp_get_wtime();
    std::vector<char> blocked((size_t)n, 0);
    for (int64_t v = 0; v < n; v++) {
        in[v] = 0;
        if (blocked[v]) continue;
        in[v] = 1;
        for (int64_t k = off[v]; k < off[v + 1]; k++) blocked[adj[k]] = 1;
    }
    return omp_get_wtime() - t0;
}

}  // namespace

extern "C" {

// Recomputes problem (0 MIS, 1 colouring, 2 BFS from `source`, 3 CC) from scratch into out[n]
// with `threads` OpenMP threads (0: all); returns the elapsed seconds, or -1 for a bad problem.
double orc_cpu_recompute(int problem, int64_t n, const int64_t* off, const int32_t* adj, int32_t source,
                         int threads, int32_t* out) {
    const int before = omp_get_max_threads();
    if (threads > 0) omp_set_num_threads(threads);
    double t = -1.0;
    switch (problem) {
    case 0: t = greedy_mis(n, off, adj, out); break;
    case 1: t = greedy_color(n, off, adj, out); break;
    case 2: t = bfs_all_cores(n, off, adj, source, out); break;
    case 3: t = cc_all_cores(n, off, adj, out); break;
    }
    if (threads > 0) omp_set_num_threads(before);
    return t;
}

int orc_cpu_threads() { return omp_get_max_threads(); }

}  // extern "C"

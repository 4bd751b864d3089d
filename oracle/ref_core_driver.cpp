// ORACLE -- test infrastructure, not product code.
//
// Command driver around the reference's own header-only host code, compiled by
// oracle/build_ref.sh against the headers where they lie in the reference tree
// (core/FlashGraph.h, core/cli_setup.h, core/chunking.h, core/flash_compactor.h). Its output
// is the golden record for the scratchpad row semantics, toggle classification, batch
// parsing, read_ints_fast, the degree-bounded chunking rule and the compactor's bytes.
//
// Usage: ref_core_driver <graph.egr> < commands
//   ins u v | del u v       HybridGraph::insertEdge / removeEdge
//   adj u v                 prints isAdjacent
//   row v                   prints degree and neighbors_into
//   parse <file> <n>        prints parse_batch_file's classified edits (u v ins)
//   ints <file>             prints read_ints_fast
//   chunk cap v1 v2 ...     prints bound_by_cumulative_degree
//   compact <out.egr>       compact_flash_graph + remap + clear
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "FlashGraph.h"
#include "chunking.h"
#include "cli_setup.h"
#include "flash_compactor.h"

int main(int argc, char** argv) {
    if (argc < 2) { std::cerr << "usage: ref_core_driver <graph.egr>\n"; return 2; }
    HybridGraph g;
    g.open(argv[1]);
    std::string line;
    std::vector<int> row;
    while (std::getline(std::cin, line)) {
        std::istringstream is(line);
        std::string cmd;
        if (!(is >> cmd)) continue;
        if (cmd == "ins" || cmd == "del" || cmd == "adj") {
            int u, v;
            is >> u >> v;
            if (cmd == "ins") g.insertEdge(u, v);
            else if (cmd == "del") g.removeEdge(u, v);
            else std::cout << "adj " << u << " " << v << " " << (g.isAdjacent(u, v) ? 1 : 0) << "\n";
        } else if (cmd == "row") {
            int v;
            is >> v;
            g.neighbors_into(v, row);
            std::cout << "row " << v << " " << g.degree(v) << ":";
            for (int x : row) std::cout << " " << x;
            std::cout << "\n";
        } else if (cmd == "parse") {
            std::string f;
            int n;
            is >> f >> n;
            auto b = parse_batch_file(std::filesystem::path(f), g, n);
            std::cout << "parse " << b.size() << "\n";
            for (auto& e : b) std::cout << e.u << " " << e.v << " " << (e.is_insertion ? 1 : 0) << "\n";
        } else if (cmd == "ints") {
            std::string f;
            is >> f;
            auto v = read_ints_fast(f);
            std::cout << "ints " << v.size() << ":";
            for (long long x : v) std::cout << " " << x;
            std::cout << "\n";
        } else if (cmd == "chunk") {
            long long cap;
            is >> cap;
            std::vector<int> cand;
            int x;
            while (is >> x) cand.push_back(x);
            std::cout << "chunk " << bound_by_cumulative_degree(g, cand, cap) << "\n";
        } else if (cmd == "compact") {
            std::string out;
            is >> out;
            compact_flash_graph(g.base, g.delta, out);
            g.base.remap(out.c_str());
            g.delta.clear();
            std::cout << "compacted " << g.base.nodes << " " << g.base.edges << "\n";
        }
    }
    return 0;
}

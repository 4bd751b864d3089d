// scout_main.cpp -- bin/scout_<problem>: the reference's command-line contract over the
// scout-b200 engine (one binary per problem, built with SCOUT_PROBLEM_NAME).
//
//   scout_<p> <graph.egr> <initial_state.txt> <batch_folder> <num_batches> <gpu_id>
//
// Contract kept from the reference: argument handling and usage line (core/cli_setup.h:32-45),
// numeric batch order (64-74), the parse/classification rule (87-103), the initial-state
// decodings of each main(), the stdout lines of core/reporting.h, the MIS output file
// datasets/Final_MISs/<stem>_flash_final_mis.txt (scout_mis.cu:932-947) and the in-place
// compaction of the input .egr unless SCOUT_SKIP_COMPACTION=1 (scout_mis.cu:949-965).
// Environment: SCOUT_NO_MADV_RANDOM, SCOUT_SKIP_COMPACTION, SCOUT_DUMP_TOUCHED=<file>,
// SCOUT_DEVICE_BUDGET_GB (cap on the engine's HBM use). SCOUT_BFS_BOUND, SCOUT_DEFER_FALLBACK,
// SCOUT_NO_MEMO, SCOUT_NO_OVERLAP and SCOUT_FORCE_COPY are accepted; the engine repairs every
// batch exactly, so it has no bound, deferral, memo or zero-copy path for them to switch.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../../include/scout_gpu.h"
#include "../../../include/scout_host.h"

#ifndef SCOUT_PROBLEM_NAME
#define SCOUT_PROBLEM_NAME "bfs"
#endif

namespace fs = std::filesystem;
using clk = std::chrono::high_resolution_clock;

static double ms_since(clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

[[noreturn]] static void die(const std::string& what, const char* detail) {
    std::cerr << "ERROR: " << what << (detail && *detail ? std::string(": ") + detail : std::string()) << std::endl;
    std::exit(1);
}

static int problem_id(const std::string& p) {
    if (p == "mis") return SCOUT_MIS;
    if (p == "coloring") return SCOUT_COLORING;
    if (p == "bfs") return SCOUT_BFS;
    return SCOUT_CC;
}

static bool parse_int(const char* s, int& out) {
    char* e = nullptr;
    long v = std::strtol(s, &e, 10);
    if (e == s) return false;
    out = (int)v;
    return true;
}

// print_batch_result / print_stage_times / print_final_summary (core/reporting.h:35-62)
static void batch_line(int i, int nb, int64_t edges, double ms, const std::vector<std::pair<std::string, std::string>>& kv) {
    std::cout << "Batch " << i << "/" << nb << " | edges=" << edges << " | time=" << std::fixed << std::setprecision(3)
              << ms << "ms";
    for (auto& p : kv) std::cout << " | " << p.first << "=" << p.second;
    std::cout << std::endl;
}
static void stage_line(int i, double fetch, double pack, double h2d, double repair, double commit) {
    std::cout << "[STAGE] batch=" << i << std::fixed << std::setprecision(3) << " fetch_ms=" << fetch
              << " seed_pack_ms=" << pack << " h2d_ms=" << h2d << " repair_ms=" << repair << " commit_ms=" << commit
              << std::endl;
}
static void final_summary(double setup, double proc, const std::string& label, long long init, long long fin) {
    std::cout << "\n=== FINAL SUMMARY ===" << std::endl;
    std::cout << "Setup time:      " << std::fixed << std::setprecision(3) << setup << " ms" << std::endl;
    std::cout << "Processing time: " << std::fixed << std::setprecision(3) << proc << " ms" << std::endl;
    std::cout << "End-to-end time: " << std::fixed << std::setprecision(3) << setup + proc << " ms" << std::endl;
    std::cout << "Initial " << label << ": " << init << std::endl;
    std::cout << "Final " << label << ":   " << fin << std::endl;
}

static long long measure(int problem, const std::vector<int32_t>& sol) {
    long long r = 0;
    if (problem == SCOUT_MIS) {
        for (int32_t x : sol) r += x != 0;
    } else if (problem == SCOUT_COLORING) {
        int32_t mx = -1;
        for (int32_t x : sol) mx = std::max(mx, x);
        r = (long long)mx + 1;
    } else if (problem == SCOUT_BFS) {
        for (int32_t x : sol) r += x >= 0;
    } else {
        std::unordered_set<int32_t> s(sol.begin(), sol.end());
        r = (long long)s.size();
    }
    return r;
}

int main(int argc, char** argv) {
    const std::string pname = SCOUT_PROBLEM_NAME;
    const int problem = problem_id(pname);
    if (argc < 6) {   // parse_scout_cli (cli_setup.h:32-45)
        std::cerr << "Usage: " << argv[0] << " <graph.egr> <initial_" << pname
                  << "_context.txt> <batch_folder> <num_batches> <gpu_device_id>" << std::endl;
        return 1;
    }
    const std::string egr_path = argv[1], state_path = argv[2], batch_dir = argv[3];
    int num_batches = 0, gpu = 0;
    if (!parse_int(argv[4], num_batches) || !parse_int(argv[5], gpu)) die("num_batches and gpu_device_id must be integers", "");

    auto setup0 = clk::now();
    uint64_t budget = 0;
    if (const char* b = std::getenv("SCOUT_DEVICE_BUDGET_GB")) budget = (uint64_t)(std::atof(b) * (1ull << 30));
    scout_ctx* ctx = nullptr;
    if (scout_ctx_create(gpu, budget, &ctx) != SCOUT_OK) die("device setup failed", scout_last_error(nullptr));
    char devname[256] = {0};
    scout_ctx_info(ctx, devname, sizeof devname, nullptr);

    if (problem == SCOUT_BFS || problem == SCOUT_CC)
        std::cout << "[Exact repair] Every batch leaves the exact " << (problem == SCOUT_BFS ? "BFS levels" : "components")
                  << "; no cascade is deferred." << std::endl;
    scout_hgraph* h = nullptr;
    const bool madv = std::getenv("SCOUT_NO_MADV_RANDOM") == nullptr;
    if (scout_hgraph_open(egr_path.c_str(), madv ? 1 : 0, &h) != SCOUT_OK) die("could not open graph", scout_last_error(nullptr));
    const int64_t n = scout_hgraph_nodes(h);
    scout_egr* e = nullptr;
    scout_egr_open(egr_path.c_str(), 0, &e);
    const int64_t edges = e ? scout_egr_edges(e) : 0;
    if (e) scout_egr_close(e);
    const double avg = n > 0 ? (double)edges / (double)n : 0.0;
    // print_run_header (core/reporting.h:22-32)
    std::cout << "=== SCOUT " << pname << " ===" << std::endl;
    std::cout << "Graph: " << egr_path << std::endl;
    std::cout << "  nodes=" << n << " edges=" << edges << " avg_degree=" << std::fixed << std::setprecision(2) << avg
              << std::endl;
    std::cout << "GPU: " << devname << " | discrete (explicit-transfer path)" << std::endl;

    if (scout_fetch_all(h, ctx, 0) != SCOUT_OK) die("loading the graph into HBM failed", scout_last_error(ctx));
    std::vector<int32_t> sol((size_t)n);
    int64_t aux = 0;
    if (scout_load_state(state_path.c_str(), problem, n, sol.data(), &aux) != SCOUT_OK)
        die("could not read the initial state", scout_last_error(nullptr));
    if (scout_state_upload(ctx, problem, sol.data(), n) != SCOUT_OK) die("state upload failed", scout_last_error(ctx));
    if (problem == SCOUT_CC) scout_state_download(ctx, problem, sol.data(), n);
    const long long initial = problem == SCOUT_MIS ? aux : measure(problem, sol);
    const double setup_ms = ms_since(setup0);

    std::vector<std::string> paths;
    {
        std::error_code ec;
        std::vector<std::pair<long long, std::string>> files;
        for (const auto& ent : fs::directory_iterator(batch_dir, ec)) {
            if (!ent.is_regular_file()) continue;
            std::string stem = ent.path().stem().string();
            char* end = nullptr;
            long long k = std::strtoll(stem.c_str(), &end, 10);
            if (end == stem.c_str()) die("batch file without a numeric stem", ent.path().c_str());
            files.emplace_back(k, ent.path().string());
        }
        if (ec) die("could not list the batch folder", batch_dir.c_str());
        std::stable_sort(files.begin(), files.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (auto& f : files) paths.push_back(f.second);
    }
    if ((int)paths.size() > num_batches) paths.resize((size_t)std::max(num_batches, 0));

    // Parse every batch; MIS classifies all of them against the base graph up front
    // (scout_mis.cu:835-842), on the device (a binary search in the sorted HBM rows instead of
    // the reference's linear base-row scan, FlashGraph.h:356-366), after removing repeated
    // identical lines inside a batch.
    std::vector<std::vector<scout_edge>> batches;
    std::vector<std::vector<uint8_t>> ops;
    for (auto& p : paths) {
        int64_t m = 0;
        scout_parse_batch_file(p.c_str(), n, nullptr, 0, &m);
        std::vector<scout_edge> b((size_t)std::max<int64_t>(m, 1));
        if (scout_parse_batch_file(p.c_str(), n, b.data(), (int64_t)b.size(), &m) != SCOUT_OK)
            die("could not read batch", p.c_str());
        b.resize((size_t)m);
        std::vector<uint8_t> op;
        if (problem == SCOUT_MIS) {
            std::unordered_set<uint64_t> seen;
            std::vector<scout_edge> kept;
            for (auto& x : b) {
                uint64_t key = ((uint64_t)(uint32_t)x.u << 32) | (uint32_t)x.v;
                if (seen.insert(key).second) kept.push_back(x);
            }
            b.swap(kept);
            std::vector<uint8_t> ins(b.size());
            if (!b.empty() && scout_classify(ctx, b.data(), (int64_t)b.size(), ins.data()) != SCOUT_OK)
                die("classification failed", scout_last_error(ctx));
            op.resize(b.size());
            for (size_t k = 0; k < b.size(); k++) op[k] = ins[k] == 1 ? SCOUT_OP_INSERT : SCOUT_OP_DELETE;
        }
        batches.push_back(std::move(b));
        ops.push_back(std::move(op));
    }

    std::unordered_set<int32_t> touched;
    const bool dump_touched = std::getenv("SCOUT_DUMP_TOUCHED") != nullptr;
    double proc_ms = 0;
    long long tot_ins = 0, tot_del = 0, tot_conf = 0, tot_rounds = 0, max_rounds = 0;
    long long tot_ins_eff = 0, tot_del_eff = 0, tot_recomputed_del = 0, batches_recomputed = 0;
    double kernel_ms = 0, transfer_ms = 0;
    std::vector<int32_t> before;
    bool hinted = false;   // the current batch was passed to scout_prefetch
    for (size_t i = 0; i < batches.size(); i++) {
        auto& b = batches[i];
        scout_batch_stats st;
        auto t0 = clk::now();
        // the next batch's edits are copied to the device during this repair (and, for a graph
        // beyond the device budget, its cold rows gathered into HBM), as the reference's MIS
        // pipeline prepares batch K+1 while K runs (scout_mis.cu:855-912); the next repair then
        // declares them prefetched (toggle batches: explicit ops are uploaded with the edits)
        scout_sched sd;
        std::memset(&sd, 0, sizeof(sd));
        sd.prefetched = hinted && ops[i].empty() ? 1 : 0;
        hinted = i + 1 < batches.size() && !batches[i + 1].empty();
        if (hinted) scout_prefetch(ctx, batches[i + 1].data(), (int64_t)batches[i + 1].size());
        int rc = scout_repair(ctx, problem, b.data(), ops[i].empty() ? nullptr : ops[i].data(), (int64_t)b.size(),
                              &sd, &st);
        if (rc != SCOUT_OK) die("repair failed", scout_last_error(ctx));
        auto t1 = clk::now();
        if (dump_touched) before = sol;
        int64_t changed = 0;
        if (scout_commit(ctx, problem, sol.data(), n, &changed) != SCOUT_OK) die("commit failed", scout_last_error(ctx));
        double commit_ms = ms_since(t1);
        double batch_ms = std::chrono::duration<double, std::milli>(t1 - t0).count() + commit_ms;
        proc_ms += batch_ms;
        if (dump_touched)
            for (int64_t v = 0; v < n; v++)
                if (before[v] != sol[v]) touched.insert((int32_t)v);
        tot_ins += st.insertions;
        tot_del += st.deletions;
        tot_conf += st.conflicts;
        tot_rounds += st.rounds;
        max_rounds = std::max<long long>(max_rounds, st.rounds);
        tot_ins_eff += st.ins_effective;
        if (st.variant != 0) {   // a whole-batch recompute variant settled this batch's deletions
            batches_recomputed++;
            tot_recomputed_del += problem == SCOUT_BFS ? st.del_effective : st.deletions - st.del_effective;
        } else {
            tot_del_eff += st.del_effective;
        }
        kernel_ms += st.ms_update + st.ms_repair;
        transfer_ms += st.ms_h2d;
        std::vector<std::pair<std::string, std::string>> kv;
        if (problem == SCOUT_COLORING)
            kv = {{"insertions", std::to_string(st.insertions)}, {"conflicts", std::to_string(st.conflicts)},
                  {"rounds", std::to_string(st.rounds)}};
        else if (problem == SCOUT_MIS)
            kv = {{"clusters", std::to_string(st.affected)}};
        else
            kv = {{"insertions", std::to_string(st.insertions)}, {"deletions", std::to_string(st.deletions)},
                  {"fallback", std::to_string(st.recomputes)}};
        batch_line((int)i + 1, problem == SCOUT_MIS ? (int)batches.size() : num_batches, (int64_t)b.size(), batch_ms, kv);
        stage_line((int)i + 1, 0.0, std::max(0.0, st.ms_total - st.ms_h2d - st.ms_update - st.ms_repair), st.ms_h2d,
                   st.ms_update + st.ms_repair, commit_ms);
    }

    const long long final_v = measure(problem, sol);
    const char* label = problem == SCOUT_MIS ? "MIS size" : problem == SCOUT_COLORING ? "colors used"
                        : problem == SCOUT_BFS ? "reached vertices" : "components";
    // End-of-run breakdown lines (scout_bfs.cu:607-613, scout_cc.cu:531-539,
    // scout_coloring.cu:351-357). The batch engine repairs every batch exactly, so nothing is
    // deferred; "fallback" counts the deletions a whole-batch recompute variant settled.
    if (problem == SCOUT_BFS) {
        std::cout << "Insertions: " << tot_ins << " (noop=" << tot_ins - tot_ins_eff << ", repaired=" << tot_ins_eff
                  << ")" << std::endl;
        std::cout << "Deletions:  " << tot_del << " (noop=" << tot_del - tot_del_eff - tot_recomputed_del
                  << ", local=" << tot_del_eff << ", fallback=" << tot_recomputed_del << ", deferred=0)" << std::endl;
        std::cout << "  fallback (batches repaired by a full traversal): " << batches_recomputed
                  << " | deferred catch-up: 0.000 ms | GPU kernel: " << std::fixed << std::setprecision(3) << kernel_ms
                  << " ms | transfer: " << transfer_ms << " ms" << std::endl;
    } else if (problem == SCOUT_CC) {
        std::cout << "Insertions: " << tot_ins << " (noop=" << tot_ins - tot_ins_eff << ", merged=" << tot_ins_eff << ")"
                  << std::endl;
        std::cout << "Deletions:  " << tot_del << " (noop=0, still_connected="
                  << tot_del - tot_del_eff - tot_recomputed_del << ", definitive_split=" << tot_del_eff
                  << ", fallback=" << tot_recomputed_del << ", deferred=0)" << std::endl;
        std::cout << "  fallback (batches repaired by a class recompute): " << batches_recomputed
                  << " | deferred catch-up: 0.000 ms" << std::endl;
    } else if (problem == SCOUT_COLORING) {
        std::cout << "Insertions: " << tot_ins << " (noop=" << tot_ins - tot_conf << ", conflict=" << tot_conf << ")"
                  << std::endl;
        std::cout << "Deletions:  " << tot_del << " (always a structural noop for coloring)" << std::endl;
        std::cout << "Speculative rounds: total=" << tot_rounds << " max_in_single_batch=" << max_rounds << std::endl;
        std::cout << "  GPU kernel: " << std::fixed << std::setprecision(3) << kernel_ms << " ms | transfer: "
                  << transfer_ms << " ms" << std::endl;
    }
    double compact_ms = 0;
    if (problem == SCOUT_MIS) {
        std::string out_dir = "datasets/Final_MISs";
        fs::create_directories(out_dir);
        std::string out = out_dir + "/" + fs::path(egr_path).stem().string() + "_flash_final_mis.txt";
        if (scout_write_state(out.c_str(), SCOUT_MIS, n, sol.data()) == SCOUT_OK)
            std::cout << "Saved final MIS to " << out << std::endl;
        else
            std::cerr << "Warning: Could not open file to save final MIS: " << out << std::endl;
        const char* skip = std::getenv("SCOUT_SKIP_COMPACTION");
        if (!(skip && std::string(skip) == "1")) {
            auto c0 = clk::now();
            // the host scratchpad receives the same edits (applied when consistent), then the
            // input .egr is rewritten in place as the reference does
            for (size_t i = 0; i < batches.size(); i++)
                for (size_t k = 0; k < batches[i].size(); k++) {
                    auto& x = batches[i][k];
                    int adj = scout_hgraph_is_adjacent(h, x.u, x.v);
                    if (ops[i][k] == SCOUT_OP_INSERT && !adj) scout_hgraph_insert(h, x.u, x.v);
                    else if (ops[i][k] == SCOUT_OP_DELETE && adj) scout_hgraph_remove(h, x.u, x.v);
                }
            if (scout_hgraph_compact(h, egr_path.c_str()) != SCOUT_OK) die("compaction failed", scout_last_error(nullptr));
            compact_ms = ms_since(c0);
        } else {
            std::cout << "\n[SCOUT_SKIP_COMPACTION=1] Skipping end-of-cycle compaction — on-disk .egr left untouched."
                      << std::endl;
        }
        std::cout << "\nEnd-of-cycle compaction time (NOT counted in per-batch numbers above): " << std::fixed
                  << std::setprecision(3) << compact_ms << " ms" << std::endl;
    }
    final_summary(setup_ms, proc_ms, label, initial, final_v);
    if (dump_touched) {
        FILE* f = std::fopen(std::getenv("SCOUT_DUMP_TOUCHED"), "wb");
        if (f) {
            std::vector<int32_t> v(touched.begin(), touched.end());
            std::sort(v.begin(), v.end());
            std::fwrite(v.data(), sizeof(int32_t), v.size(), f);
            std::fclose(f);
        }
    }
    std::cout.flush();
    std::fflush(stdout);
    scout_ctx_destroy(ctx);
    scout_hgraph_close(h);
    std::_Exit(0);
}

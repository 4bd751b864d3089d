// union.cu -- one persistent kernel for a round of several problems' union stores.
//
// The batched engine (multi.cu) keeps many streams of ONE problem as a disjoint union in one
// store, so a round over streams of all four problems would be four merges and four
// cooperative repair launches. Here the stores' merges are queued first, each on its own
// context's stream, and ONE cooperative launch then runs their repairs one after the other:
// every block runs the BFS store's phases, then the CC store's, then the colouring and the
// MIS store's, each over its own store and work queues, with its own counters and its own
// bounded grid barrier (zeroed before the launch). Every block takes part in every repair, so
// each repair sees the same grid as when launched alone; the kernel's register count is the
// largest of the four bodies', within the four-blocks-per-SM budget all four already meet.
#include "ctx.cuh"
#include "bfs_dev.cuh"
#include "cc_dev.cuh"
#include "coloring_dev.cuh"
#include "mis_dev.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>

namespace scout {

constexpr int UNION_THREADS = 256;
static_assert(BFS_THREADS == UNION_THREADS && CC_THREADS == UNION_THREADS && COL_THREADS == UNION_THREADS &&
                  MIS_THREADS == UNION_THREADS,
              "the fused repair runs every body with the same block size");

struct UnionRound {
    int has_bfs, has_cc, has_col, has_mis;
    BfsParams bfs;
    CcParams cc;
    ColParams col;
    MisParams mis;
};

__global__ void __launch_bounds__(UNION_THREADS, 4) k_union_round(UnionRound u) {
    if (u.has_bfs) bfs_body(u.bfs);
    if (u.has_cc) cc_body(u.cc);
    if (u.has_col) coloring_body(u.col);
    if (u.has_mis) mis_body(u.mis);
}

// cs[i] holds the union store of problems[i] (distinct problems, one device) with its batch
// merged (queued on its stream). Launches the fused repair on cs[0]'s stream once every merge
// is done; every context's stream then waits for the repair. variants[i]: the repair variant
// (BFS mode, CC variant). cs[0]'s ev_t[4] / ev_t[5] bracket the launch.
int union_launch(scout_ctx* const* cs, const int* problems, const scout_sched* sds, const int* variants, int ne) {
    UnionRound u;
    std::memset(&u, 0, sizeof(u));
    scout_ctx* c0 = cs[0];
    size_t smem = 0;
    for (int i = 0; i < ne; i++) {
        scout_ctx* c = cs[i];
        switch (problems[i]) {
        case SCOUT_BFS: SCOUT_RC(bfs_params(c, variants[i], nullptr, &u.bfs)); u.has_bfs = 1; break;
        case SCOUT_CC:
            SCOUT_RC(cc_params(c, &sds[i], variants[i], nullptr, &u.cc));
            u.has_cc = 1;
            smem = CC_SMEM;
            break;
        case SCOUT_COLORING: SCOUT_RC(coloring_params(c, &u.col)); u.has_col = 1; break;
        case SCOUT_MIS: SCOUT_RC(mis_params(c, &u.mis)); u.has_mis = 1; break;
        default: return c->fail(SCOUT_E_INVALID, "unknown problem");
        }
    }
    for (int i = 1; i < ne; i++) {   // the launch stream waits for every other store's merge
        SCOUT_CU(cs[i], cudaEventRecord(cs[i]->ev_union, cs[i]->s_main));
        SCOUT_CU(c0, cudaStreamWaitEvent(c0->s_main, cs[i]->ev_union, 0));
    }
    for (int i = 0; i < ne; i++)   // every repair's grid barrier starts at zero
        SCOUT_CU(c0, cudaMemsetAsync(&cs[i]->d_bar->count, 0, sizeof(unsigned int), c0->s_main));
    if (smem) {   // the dynamic shared-memory opt-in: once per device
        static std::atomic<unsigned long long> attr_done{0};
        const unsigned long long bit = 1ull << (c0->device & 63);
        if (!(attr_done.load() & bit)) {
            SCOUT_CU(c0, cudaFuncSetAttribute(k_union_round, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_done.fetch_or(bit);
        }
    }
    int per_sm = 0;
    SCOUT_CU(c0, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_union_round, UNION_THREADS, smem));
    if (per_sm < 1) return c0->fail(SCOUT_E_CUDA, "fused repair kernel does not fit on an SM");
    per_sm = std::min(per_sm, c0->tune_blocks_per_sm > 0 ? c0->tune_blocks_per_sm : 4);
    void* args[] = {&u};
    SCOUT_CU(c0, cudaEventRecord(c0->ev_t[4], c0->s_main));
    SCOUT_CU(c0, cudaLaunchCooperativeKernel((const void*)k_union_round, dim3((unsigned)(per_sm * c0->sm_count)),
                                             dim3(UNION_THREADS), args, smem, c0->s_main));
    SCOUT_CU(c0, cudaEventRecord(c0->ev_t[5], c0->s_main));
    c0->nlaunch += 1;
    SCOUT_CU(c0, cudaEventRecord(c0->ev_union, c0->s_main));
    for (int i = 1; i < ne; i++) SCOUT_CU(cs[i], cudaStreamWaitEvent(cs[i]->s_main, c0->ev_union, 0));
    return SCOUT_OK;
}

}  // namespace scout

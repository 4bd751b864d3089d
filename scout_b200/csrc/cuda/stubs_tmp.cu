#include "ctx.cuh"
namespace scout {
int cc_repair(scout_ctx* c, const scout_sched*, scout_batch_stats*) { return c->fail(SCOUT_E_STATE, "cc not built yet"); }
int cc_recompute(scout_ctx* c, scout_batch_stats*) { return c->fail(SCOUT_E_STATE, "cc not built yet"); }
int coloring_repair(scout_ctx* c, scout_batch_stats*) { return c->fail(SCOUT_E_STATE, "coloring not built yet"); }
int mis_repair(scout_ctx* c, scout_batch_stats*) { return c->fail(SCOUT_E_STATE, "mis not built yet"); }
}

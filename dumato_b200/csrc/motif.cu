#include "engine.hpp"
namespace dmb {
size_t motif_scratch_bytes(const MotifPlan&, const LaunchCtx&, int* w) { *w = 0; return 0; }
int motif_launch(const GraphView&, const MotifPlan&, DevCounters*, LaunchCtx&, void*, size_t, dm_stats*) {
  return fail(DM_EINVAL, "motifs not built yet");
}
}
extern "C" int dm_count_motifs(dm_graph*, int32_t, const dm_dictionary*, const dm_opts*, uint64_t*, dm_stats*) {
  return dmb::fail(DM_EINVAL, "motifs not built yet");
}

#include "engine.hpp"
namespace dmb {
int predictor_order(const void*, dm_graph*, int, bool, std::vector<int32_t>&) { return fail(DM_EINVAL, "no predictor yet"); }
}

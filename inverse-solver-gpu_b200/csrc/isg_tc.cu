// Tensor-core engine for the dense leaf stages (near field + L2P, P2M).
#include "isg_context.hpp"

namespace isg {

struct TcPlan {
  int dummy = 0;
};

isg_status tc_setup(isg_ctx *) { return ISG_OK; }
void tc_destroy(isg_ctx *c) {
  delete c->tc;
  c->tc = nullptr;
}
bool tc_available(const isg_ctx *c) { return c->tc != nullptr; }
isg_status tc_p2m(isg_ctx *, const BatchArgs &, float2 *, cudaStream_t) { return ISG_UNSUPPORTED; }
isg_status tc_near(isg_ctx *, const NearArgs &, cudaStream_t) { return ISG_UNSUPPORTED; }

}  // namespace isg

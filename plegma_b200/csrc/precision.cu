// Split-FP16 form (filled in by the tensor-core projection).
#include "ctx.h"

namespace p2 {

p2_status precision_run_batch(p2_ctx* c, const p2_prop*, int, const p2_request*, int) {
  return c->fail(P2_ERR_UNSUPPORTED, "split-FP16 form not built");
}
void precision_release(p2_ctx*) {}

}  // namespace p2

// Learned message-passing preconditioner (filled in by the network kernels).
#include "pd_internal.cuh"

namespace pdb {
bool mpnn_ready(const pd_ctx*) { return false; }
int mpnn_apply(pd_ctx* c, const double*, double*, const double*) {
  c->err = "learned preconditioner not available";
  return PD_ERR_STATE;
}
void mpnn_release(pd_ctx*) {}
}  // namespace pdb

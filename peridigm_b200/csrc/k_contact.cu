// Short-range contact (filled in by the contact kernels).
#include "pd_internal.cuh"

namespace pdb {
void contact_release(pd_ctx*) {}
int contact_prepare(pd_ctx*, int64_t) { return PD_OK; }
int contact_eval(pd_ctx*) { return PD_OK; }
int64_t contact_pairs(const pd_ctx*) { return 0; }
void qs_release(pd_ctx*) {}
}  // namespace pdb

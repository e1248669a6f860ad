// Batched driver: placeholder entry points until the persistent work-queued launch lands.
#include "../../include/pmfmhd.h"

extern "C" {
int pmfmhd_batch_create(pmfmhd_ctx*, const pmfmhd_box*, int, pmfmhd_batch** out) {
  if (out) *out = nullptr;
  return PMFMHD_EUNSUPPORTED;
}
int pmfmhd_batch_step(pmfmhd_batch*, int, void*) { return PMFMHD_EUNSUPPORTED; }
int pmfmhd_batch_query(pmfmhd_batch*, double*, int32_t*, float*) { return PMFMHD_EUNSUPPORTED; }
int pmfmhd_batch_destroy(pmfmhd_batch*) { return PMFMHD_OK; }
}

// pending.cpp — entry points of include/ba_cuda.h whose GPU implementation lands in a later change.
// They validate nothing and report Unsupported, so a caller hands the work to another path.
#include <cstdio>

#include "../../include/ba_cuda.h"

static int32_t pending(omvgba_error* e, const char* what) {
  if (e) {
    e->code = OMVGBA_UNSUPPORTED;
    e->detail = -1;
    std::snprintf(e->message, sizeof(e->message), "%s is not available in this build", what);
  }
  return OMVGBA_UNSUPPORTED;
}

extern "C" {
int32_t omvgba_solve_batched(omvgba_context*, uint64_t, const omvgba_problem*, const omvgba_config*, omvgba_solution*,
                             omvgba_error* error) {
  return pending(error, "omvgba_solve_batched");
}
}

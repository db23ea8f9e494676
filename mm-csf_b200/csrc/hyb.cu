// HB-CSF construction (src/util.h:852-1142, 1786-1885).
#include "format.h"
#include "prims.cuh"

namespace mmcsf {
int build_hyb(mmcsf_format* F, CsfPart& X, cudaStream_t s, int* launches) {
  (void)F; (void)X; (void)s; (void)launches;
  return set_error(MMCSF_ERR_UNSUPPORTED, "HB-CSF (-t 10) construction is not built yet");
}
}  // namespace mmcsf

/* The reference includes <nvToolsExt.h> (solver_functions/cuda_helper.h:4); this image has
 * only the header-only NVTX3 tree, so forward to it. Test infrastructure only. */
#include <nvtx3/nvToolsExt.h>

// Mixed-precision path (placeholder until the FP32 kernels land).
#include "mb_common.cuh"

namespace mb {
int launch_mixed_step(mb_sim *, int, int) { return fail(MB_ERR_UNSUPPORTED, "mixed precision not built yet"); }
int mixed_alloc(mb_sim *) { return fail(MB_ERR_UNSUPPORTED, "mixed precision not built yet"); }
void mixed_free(mb_sim *) {}
int mixed_after_upload(mb_sim *) { return MB_ERR_UNSUPPORTED; }
int mixed_pack_df_rho(mb_sim *) { return MB_ERR_UNSUPPORTED; }
int mixed_kernel_times(mb_sim *, int, float *, float *) { return MB_ERR_UNSUPPORTED; }
} // namespace mb

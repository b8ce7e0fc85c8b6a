// Fused fast path (placeholder until the fused kernels land).
#include "hv_internal.h"

namespace hv {

hv_status fused_prepare(hv_ctx *) { return HV_ERR_UNSUPPORTED; }
hv_status fused_release(hv_ctx *) { return HV_OK; }
hv_status fused_run(hv_ctx *, int, hv_observables *) { return HV_ERR_UNSUPPORTED; }

}  // namespace hv

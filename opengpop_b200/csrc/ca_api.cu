// ca_api.cu -- closest-approach entry points (placeholder until the screen kernels land).
#include "context.h"

extern "C" {
gpop_status gpop_ca_create(gpop_ctx* ctx, const gpop_time*, double, int64_t, const double*,
    const double*, const uint32_t*, gpop_ca** out)
{
    if (out)
        *out = nullptr;
    return ctx ? gpop::fail(ctx, GPOP_ERR_UNSUPPORTED, "closest approach not built yet") : GPOP_ERR_INVALID_ARG;
}
gpop_status gpop_ca_propagate(gpop_ca*, int32_t) { return GPOP_ERR_UNSUPPORTED; }
gpop_status gpop_ca_find(gpop_ca*, double, gpop_ca_record*, int64_t, int64_t*) { return GPOP_ERR_UNSUPPORTED; }
gpop_status gpop_ca_pairs(gpop_ca*, double*, double*, double*, double*, uint32_t*) { return GPOP_ERR_UNSUPPORTED; }
int64_t gpop_ca_num_pairs(const gpop_ca*) { return 0; }
gpop_status gpop_ca_trajectory(gpop_ca*, double*, double*, double*, int32_t*) { return GPOP_ERR_UNSUPPORTED; }
void gpop_ca_destroy(gpop_ca*) { }
}

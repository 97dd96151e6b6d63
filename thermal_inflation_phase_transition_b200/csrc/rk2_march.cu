// Marching (2.5-D blocked) real-field stage kernel.
#include "rk2_march.cuh"
#include "tipt_internal.h"

namespace tipt {

bool march_supported(int, const RealStageParams&) { return false; }

int launch_march(int, const RealStageParams&, int64_t, cudaStream_t) {
    return fail(TIPT_ERR_UNSUPPORTED, "marching kernel not built");
}

}  // namespace tipt

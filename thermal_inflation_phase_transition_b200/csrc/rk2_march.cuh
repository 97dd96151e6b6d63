// Marching (2.5-D blocked) real-field stage kernel -- declarations.
#pragma once

#include "rk2_real.cuh"

namespace tipt {

bool march_supported(int storage, const RealStageParams& p);
int launch_march(int storage, const RealStageParams& p, int64_t smem_table, cudaStream_t st);

}  // namespace tipt

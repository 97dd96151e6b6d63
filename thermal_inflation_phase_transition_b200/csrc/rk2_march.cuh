// Marching (2.5-D blocked) real-field stage kernel -- declarations.
#pragma once

#include "rk2_complex.cuh"

namespace tipt {

bool march_supported(int storage, const RealStageParams& p);
int launch_march(int storage, const RealStageParams& p, int64_t smem_table, cudaStream_t st);

// Batched ensemble: the replicas rids[0..n_rids) of one 3-D shape class on the
// compensated-FP32 marching stage.
bool ensemble_march_supported(int n0, int n1, int n2);
int launch_ensemble_march(const RealStageParams& p, const tipt_replica* reps, const int32_t* rids,
                          int n_rids, const int32_t* n_rids_dev, const int32_t* active,
                          int64_t n_total, const unsigned long long* ctr, long long offset,
                          cudaStream_t st);

// Overdamped / BAOAB passes (mode kOD, kBA1, kBA2) of the real or complex
// field, compensated FP32.
struct AltParams;
bool alt_march_supported(const AltParams& p, bool cplx);
int launch_alt_march(int mode, bool cplx, const AltParams& p, cudaStream_t st);

// Complex field, compensated FP32, Z_N off, V'(rho) polynomial or staged in shared memory.
bool complex_march_supported(const ComplexStageParams& p);
int launch_complex_march(const ComplexStageParams& p, cudaStream_t st);

}  // namespace tipt

// Host-side helpers shared by the translation units of libtipt.so.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "tipt.h"

namespace tipt {

// Record a formatted detail for tipt_last_error() and return `status`.
int fail(int status, const char* fmt, ...);
// Record a CUDA error and return TIPT_ERR_CUDA.
int fail_cuda(cudaError_t e, const char* what);
// Number of SMs of the current device (cached per process).
int num_sms();

// Argument validation shared by the entry points (each records a detail and
// returns a tipt_status on failure, TIPT_OK otherwise).
int check_dims(int64_t nx, int64_t ny, int64_t nz);
int check_storage(int s);
int elem_bytes(int s);
int elem_align(int s);
int check_ptr(const void* p, int align, const char* name);
bool overlap(const void* a, const void* b, int64_t n);
int check_vsource(const tipt_vsource* vp, const char* name);
int check_state(int storage, const void* phi, const void* pi, void* phi_out, void* pi_out,
                int64_t nx, int64_t ny, int64_t nz);
// The same pointer/overlap checks for a packed buffer of `sites` sites (ensembles).
int check_state_sites(int storage, const void* phi, const void* pi, void* phi_out,
                      void* pi_out, int64_t sites);

// Stage kernel selection set by tipt_set_kernel_policy (0 auto, 1 generic, 2 marching).
int kernel_policy();

// Status word of the surrogate kernels' bounded waits (TIPT_ERR_TIMEOUT or 0).
int mlp_status(int* status, int clear);
// Status word of the labeller's bounded union-find loops.
int label_status(int* status, int clear);

struct RealStageParams;
int launch_real_stage(int storage, RealStageParams p, cudaStream_t st);

}  // namespace tipt

// fe_learn.h -- what the engine translation unit and the learned-closure translation unit
// share (internal; not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include "fasteddy_b200.h"
#include "fe_device.cuh"

// record an error message for fe_last_error() and return `code`
int fe_internal_error(int code, const char* msg);
// enqueue the network's stresses for the state `st` of a domain (time-step form): inputs from
// Q.feat (written by the tiled closure kernel) or, with `fromState` or no Q.feat, evaluated from
// the state by the inference kernel itself; returns a CUDA error code of the launch
cudaError_t fe_learn_enqueue_tau(const fe_mlp* m, const fe::Phys& P, const fe::Ptrs& Q, const float* st, cudaStream_t s,
                                 bool fromState);
// device error flag of the network's kernels (1 = a tensor-core wait expired)
int* fe_learn_err_flag(const fe_mlp* m);
int fe_learn_device(const fe_mlp* m);

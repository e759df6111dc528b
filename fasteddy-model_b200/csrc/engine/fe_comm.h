// fe_comm.h -- the stage barrier of a domain decomposed over several processes (one GPU each).
//
// The commits of a slab write its neighbours' halo cells over peer memory; before any slab
// starts the next stage, every slab's commit must be complete. The barrier is a one-element
// NCCL all-reduce on the slab's stream: stream-ordered, capturable in a CUDA graph, and
// complete on a rank only once every rank has reached it. NCCL is loaded at run time
// (libnccl.so.2, the library torch.distributed already loaded when present), so the engine
// library has no link-time NCCL dependency.
#pragma once
#include <cuda_runtime.h>

#include "fasteddy_b200.h"

// Enqueue the barrier on stream s (no host synchronisation).
void fe_comm_barrier(fe_comm* c, cudaStream_t s);

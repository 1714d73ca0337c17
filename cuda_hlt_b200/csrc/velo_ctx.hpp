// Internal link between the chain context (velo_chain.cu) and the scorer trainer
// (velo_mlp_train.cu): device pointers of the last velo_run of a context. Not part of the
// C ABI.
#pragma once
#include <cuda_runtime.h>

#include "velo_kernels.cuh"

struct VeloCtx;

// Pointers of the last run on `ctx` (n_events, hits, windows, tracks of the search) and the
// stream it ran on; false if the context has not run.
bool velo_ctx_last_run(VeloCtx* ctx, velo::ChainPointers* P, cudaStream_t* stream, int* device);

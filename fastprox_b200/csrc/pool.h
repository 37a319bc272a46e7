// Memory for workspaces without device-wide synchronisation.
//
// cudaMalloc/cudaFree and cudaHostAlloc/cudaFreeHost synchronise the whole
// device, so a service that creates a workspace per request (the reference's
// fp_prox with ws = NULL, or one operator per request) would stall every
// other stream twice per request. Workspaces therefore take their device
// memory as one block from a stream-ordered pool per device (kept, not
// returned to the driver, until fp_b200_release_cached), and their pinned
// host memory from a cache of power-of-two blocks.
#pragma once

#include <cuda_runtime_api.h>

#include <cstddef>
#include <functional>

namespace fpb {

// `bytes` of device memory on `device`; `init` may queue work (memsets,
// uploads) on the pool's stream, and all of it has finished on return, so
// the block is ready for any stream.
cudaError_t pool_alloc(int device, size_t bytes, void **p, const std::function<cudaError_t(cudaStream_t)> &init);
// Returns a block to the pool. Every call on a workspace synchronises its
// stream before returning, so nothing of ours still uses the block; the
// caller's own stream may be gone by now and is not touched.
void pool_free(int device, void *p);
// Pinned host memory of at least `bytes` (nullptr when none can be had);
// give it back with the same size.
void *pinned_take(size_t bytes);
void pinned_give(void *p, size_t bytes);
// Releases cached blocks of both kinds (device memory of every pool).
void pool_release_cached();

}  // namespace fpb

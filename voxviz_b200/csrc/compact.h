// compact.h - the page-request compaction (selection mask, histopyramid,
// compaction) in three launches instead of one per pyramid level.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace vv {

// The selection, the histopyramid's counts and exclusive offsets and the
// compaction of `p` (the CompactParams of launch_compact, its `counts` and
// `offsets` used only as scratch), with results identical to launch_select
// followed by launch_compact: the same mask, request order, requests and
// count.  cudaErrorNotSupported (nothing launched) when the frame has too
// few pyramid levels or too many level-5 nodes for one CTA's shared memory;
// the caller then takes the per-level launches.
cudaError_t launch_compact_fused(const CompactParams& p, uint32_t* mask, cudaStream_t s);

}  // namespace vv

// Internal interface between the translation units of libfhtgs (not exported).
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/fhtgs.h"
#include "fhtgs_types.cuh"

namespace fhtgs {

// Message returned by fhtgs_last_error() on the calling thread (fhtgs_host.cu).
void set_last_error(const std::string& msg);

// Checks a frame's arguments as fhtgs_render_views does.
fhtgs_status validate_frame(const fhtgs_primitives* p, const fhtgs_view* views, int n_views, const fhtgs_settings* s);

// Enqueues one frame on `stream` like fhtgs_render_views and, when `host_status` is given
// (pinned, n_views entries), copies the frame's status into it on the same stream.
fhtgs_status enqueue_frame(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                           const fhtgs_settings* s, cudaStream_t stream, FrameStatus* host_status);

// Bytes the context's arena holds after rendering this frame at instance capacity `cap`
// (its current size when that suffices, else the size it grows to).
size_t frame_arena_need(fhtgs_context ctx, const fhtgs_primitives* prims, const fhtgs_view* views, int n_views,
                        const fhtgs_settings* s, int64_t cap);

int64_t default_instance_capacity(int64_t n_prims);
int64_t context_capacity(fhtgs_context ctx);
// Sets the instance slots per view (rounded up to a whole sort tile).
void set_context_capacity(fhtgs_context ctx, int64_t cap);
// Frees the context's arena (synchronises the device, as cudaFree does).
fhtgs_status release_arena(fhtgs_context ctx);

}  // namespace fhtgs

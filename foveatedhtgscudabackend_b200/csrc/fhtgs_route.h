// Routing policy of the replica group (fhtgs_group.cu): which replica's server a new request
// goes to.  Host code with no CUDA dependency, so that it can be compiled and exercised alone.
#pragma once
#include <stdint.h>

namespace fhtgs {

struct ReplicaLoad {
    int device;                // CUDA device the replica renders on
    int64_t outstanding_cost;  // work routed to it and not yet completed (see request_cost)
};

// Estimated work of a request: the pixels of its eyes, scaled by a factor that grows with the
// scene's Gaussians (the instances a frame sorts and blends grow with both).
inline int64_t request_cost(const int64_t* eye_pixels, int n_eyes, int64_t n_gaussians) {
    int64_t px = 0;
    for (int e = 0; e < n_eyes; ++e) px += eye_pixels[e] > 0 ? eye_pixels[e] : 0;
    const int64_t factor = 1 + (n_gaussians > 0 ? n_gaussians : 0) / 262144;
    return (px > 0 ? px : 1) * factor;
}

// The replica a request goes to: among the replicas on `device` (-1: any replica), the one with
// the least outstanding cost; among equals, the first at or after `*cursor` in index order
// (round robin), and the cursor moves past the choice.  -1 when no replica is eligible.
inline int pick_replica(const ReplicaLoad* reps, int n, int device, uint64_t* cursor) {
    int best = -1;
    for (int k = 0; k < n; ++k) {
        const int i = static_cast<int>((*cursor + static_cast<uint64_t>(k)) % static_cast<uint64_t>(n));
        if (device >= 0 && reps[i].device != device) continue;
        if (best < 0 || reps[i].outstanding_cost < reps[best].outstanding_cost) best = i;
    }
    if (best >= 0) *cursor = static_cast<uint64_t>(best) + 1;
    return best;
}

}  // namespace fhtgs

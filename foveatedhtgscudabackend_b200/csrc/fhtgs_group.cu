// Replica group of request servers over several CUDA devices (C ABI in include/fhtgs.h,
// "several GPUs").  Host code only.
//
// Views are independent once their camera is known, and the K-buffer blend cannot combine
// partial results over a split of the Gaussians (the core is quantised to RGBA8 as fragments
// arrive, so the merge is not associative), so the group scales by replication: every replica
// (one fhtgs_server on one device) holds every scene in its own device's HBM, and each request
// is rendered, whole, by one replica chosen by fhtgs::pick_replica (fhtgs_route.h).  Nothing
// crosses devices per frame: scenes are copied once, peer to peer, when they are added.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fhtgs.h"
#include "fhtgs_internal.h"
#include "fhtgs_route.h"

using namespace fhtgs;

namespace {

constexpr int kMaxReplicas = 64;   // group tickets are server ticket * kMaxReplicas + replica

fhtgs_status grp_fail(fhtgs_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

// Bytes of each attribute array of a scene (positions always float32).
struct SceneArrays {
    size_t bytes[6];
};
SceneArrays array_bytes(const fhtgs_primitives& p) {
    const size_t n = static_cast<size_t>(p.n_primitives), s = static_cast<size_t>(p.total_sh_bases);
    const size_t a = p.storage == FHTGS_STORAGE_HALF ? 2 : 4;
    return SceneArrays{{12 * n, 3 * a * n, 4 * a * n, a * n, 3 * a * n, 3 * a * s * n}};
}

size_t background_bytes(const fhtgs_settings& s) {
    if (!s.background_data) return 0;
    if (s.background_type == FHTGS_BACKGROUND_SH) return 16 * 3 * sizeof(float);
    if (s.background_type == FHTGS_BACKGROUND_TEXTURE || s.background_type == FHTGS_BACKGROUND_TEXTURE_RAW)
        return 3ull * s.texture_width * s.texture_height * sizeof(float);
    return 0;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct Replica {
    int device = 0;
    fhtgs_server server = nullptr;
};

struct GroupScene {
    int home_device = 0;
    int64_t n_gaussians = 0;
    std::vector<int32_t> server_scene;   // the scene's id in each replica's server
    std::vector<void*> copy;             // per replica: its device copy (null: the caller's arrays)
    bool live = true;
};

}  // namespace

struct fhtgs_server_group_s {
    std::mutex mu;
    std::vector<Replica> reps;
    std::vector<ReplicaLoad> load;
    std::vector<GroupScene> scenes;
    std::unordered_map<int64_t, int64_t> cost_of;   // group ticket -> routed cost, until polled
    uint64_t cursor = 0;
};

namespace {

void decode(int64_t group_ticket, int* replica, int64_t* server_ticket) {
    *replica = static_cast<int>(group_ticket % kMaxReplicas);
    *server_ticket = group_ticket / kMaxReplicas;
}

// The device of the request's device buffers (-1: it carries none).
fhtgs_status request_device(const fhtgs_request* r, int* device) {
    *device = -1;
    for (int e = 0; e < r->n_eyes; ++e) {
        const fhtgs_eye& eye = r->eyes[e];
        const void* ptrs[4] = {eye.visibility_mask, eye.visibility_mask_area_table, eye.fovea_mask_area_table,
                               eye.image};
        for (const void* p : ptrs) {
            if (!p) continue;
            cudaPointerAttributes a{};
            const cudaError_t err = cudaPointerGetAttributes(&a, p);
            if (err != cudaSuccess) {
                cudaGetLastError();
                return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, std::string("request buffer: ") + cudaGetErrorString(err));
            }
            if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
                return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "request buffers must be device memory");
            if (*device >= 0 && a.device != *device)
                return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "the buffers of one request lie on different devices");
            *device = a.device;
        }
    }
    return FHTGS_OK;
}

// Copies a scene's arrays (and background data) from `home` into one allocation on `device`
// and fills `prims`/`settings` with the copy's pointers.
fhtgs_status replicate(const fhtgs_primitives& src, const fhtgs_settings& src_set, int home, int device,
                       fhtgs_primitives* prims, fhtgs_settings* settings, void** out) {
    const SceneArrays sz = array_bytes(src);
    const size_t bg = background_bytes(src_set);
    size_t total = align256(bg);
    for (size_t b : sz.bytes) total += align256(b);
    cudaError_t e = cudaSetDevice(device);
    char* base = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&base, total > 0 ? total : 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return grp_fail(FHTGS_ERR_OUT_OF_MEMORY, std::string("scene replica: ") + cudaGetErrorString(e));
    }
    cudaStream_t s = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    const void* from[6] = {src.positions, src.scales, src.rotations, src.opacities, src.sh_0, src.sh_rest};
    void* to[6] = {};
    size_t off = 0;
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) {
        to[k] = base + off;
        if (from[k] && sz.bytes[k]) e = cudaMemcpyPeerAsync(to[k], device, from[k], home, sz.bytes[k], s);
        off += align256(sz.bytes[k]);
    }
    void* bg_copy = nullptr;
    if (e == cudaSuccess && bg) {
        bg_copy = base + off;
        e = cudaMemcpyPeerAsync(bg_copy, device, src_set.background_data, home, bg, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the server's streams read the copy
    if (s) cudaStreamDestroy(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(base);
        return grp_fail(FHTGS_ERR_CUDA, std::string("scene replica copy: ") + cudaGetErrorString(e));
    }
    *prims = src;
    prims->positions = static_cast<const float*>(to[0]);
    prims->scales = static_cast<const float*>(to[1]);
    prims->rotations = static_cast<const float*>(to[2]);
    prims->opacities = static_cast<const float*>(to[3]);
    prims->sh_0 = static_cast<const float*>(to[4]);
    prims->sh_rest = src.sh_rest ? static_cast<const float*>(to[5]) : nullptr;
    *settings = src_set;
    if (bg) settings->background_data = static_cast<const float*>(bg_copy);
    *out = base;
    return FHTGS_OK;
}

}  // namespace

extern "C" {

fhtgs_status fhtgs_server_group_create(const int32_t* devices, int32_t n_devices, const fhtgs_server_config* config,
                                       fhtgs_server_group* out) {
    if (!devices || !config || !out) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (n_devices < 1 || n_devices > kMaxReplicas)
        return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "n_devices must be in [1, 64]");
    auto* G = new fhtgs_server_group_s();
    for (int i = 0; i < n_devices; ++i) {
        fhtgs_server_config c = *config;
        c.device = devices[i];
        Replica r;
        r.device = devices[i];
        const fhtgs_status st = fhtgs_server_create(&c, &r.server);
        if (st != FHTGS_OK) {
            const std::string msg = fhtgs_last_error();
            fhtgs_server_group_destroy(G);
            return grp_fail(st, "replica " + std::to_string(i) + " (device " + std::to_string(devices[i]) + "): " + msg);
        }
        G->reps.push_back(r);
        G->load.push_back(ReplicaLoad{devices[i], 0});
    }
    *out = G;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_destroy(fhtgs_server_group G) {
    if (!G) return FHTGS_OK;
    for (Replica& r : G->reps) fhtgs_server_destroy(r.server);  // waits for running frames
    for (GroupScene& sc : G->scenes)
        for (size_t i = 0; i < sc.copy.size(); ++i)
            if (sc.copy[i]) {
                cudaSetDevice(G->reps[i].device);
                cudaFree(sc.copy[i]);
            }
    delete G;
    return FHTGS_OK;
}

int32_t fhtgs_server_group_size(fhtgs_server_group G) { return G ? static_cast<int32_t>(G->reps.size()) : 0; }

fhtgs_status fhtgs_server_group_add_scene(fhtgs_server_group G, int32_t home_device, const fhtgs_primitives* prims,
                                          const fhtgs_settings* settings, int32_t* scene_id) {
    if (!G || !prims || !settings || !scene_id) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(G->mu);   // scenes are added one at a time
    GroupScene sc;
    sc.home_device = home_device;
    sc.n_gaussians = prims->n_primitives;
    bool borrowed = false;
    fhtgs_status st = FHTGS_OK;
    for (size_t i = 0; i < G->reps.size() && st == FHTGS_OK; ++i) {
        fhtgs_primitives p = *prims;
        fhtgs_settings s = *settings;
        void* copy = nullptr;
        if (G->reps[i].device == home_device && !borrowed) {
            borrowed = true;   // the first replica on the home device renders the caller's arrays
        } else {
            st = replicate(*prims, *settings, home_device, G->reps[i].device, &p, &s, &copy);
            if (st != FHTGS_OK) break;
        }
        int32_t id = -1;
        st = fhtgs_server_add_scene(G->reps[i].server, &p, &s, &id);
        if (st != FHTGS_OK) {
            const std::string msg = fhtgs_last_error();
            if (copy) cudaFree(copy);
            st = grp_fail(st, "replica " + std::to_string(i) + ": " + msg);
            break;
        }
        sc.server_scene.push_back(id);
        sc.copy.push_back(copy);
    }
    if (st != FHTGS_OK) {   // undo the replicas already registered
        const std::string msg = fhtgs_last_error();
        for (size_t i = 0; i < sc.server_scene.size(); ++i) {
            fhtgs_server_remove_scene(G->reps[i].server, sc.server_scene[i]);
            fhtgs_server_drain(G->reps[i].server, -1);
            if (sc.copy[i]) {
                cudaSetDevice(G->reps[i].device);
                cudaFree(sc.copy[i]);
            }
        }
        return grp_fail(st, msg);
    }
    *scene_id = static_cast<int32_t>(G->scenes.size());
    G->scenes.push_back(std::move(sc));
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_remove_scene(fhtgs_server_group G, int32_t scene_id) {
    if (!G) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null group");
    std::lock_guard<std::mutex> lk(G->mu);
    if (scene_id < 0 || scene_id >= static_cast<int>(G->scenes.size()) || !G->scenes[scene_id].live)
        return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown scene");
    GroupScene& sc = G->scenes[scene_id];
    sc.live = false;
    for (size_t i = 0; i < G->reps.size(); ++i) fhtgs_server_remove_scene(G->reps[i].server, sc.server_scene[i]);
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_submit(fhtgs_server_group G, const fhtgs_request* request, int64_t* ticket,
                                       int32_t* replica) {
    if (!G || !request || !ticket) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (request->n_eyes < 1 || request->n_eyes > 2) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "n_eyes must be 1 or 2");
    int device = -1;
    fhtgs_status st = request_device(request, &device);
    if (st != FHTGS_OK) return st;
    fhtgs_request routed = *request;
    // the lock is held across the server's submit, so that a concurrent poll that receives the
    // completion finds its cost recorded (poll takes the servers' locks without this one)
    std::lock_guard<std::mutex> lk(G->mu);
    if (request->scene < 0 || request->scene >= static_cast<int>(G->scenes.size()) || !G->scenes[request->scene].live)
        return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown scene");
    const GroupScene& sc = G->scenes[request->scene];
    int64_t px[2] = {0, 0};
    for (int e = 0; e < request->n_eyes; ++e)
        px[e] = static_cast<int64_t>(request->eyes[e].width) * request->eyes[e].height;
    const int64_t cost = request_cost(px, request->n_eyes, sc.n_gaussians);
    uint64_t cursor = G->cursor;
    const int r = pick_replica(G->load.data(), static_cast<int>(G->load.size()), device, &cursor);
    if (r < 0)
        return grp_fail(FHTGS_ERR_INVALID_ARGUMENT,
                        "no replica on device " + std::to_string(device) + ", where the request's buffers lie");
    routed.scene = sc.server_scene[r];
    int64_t t = 0;
    st = fhtgs_server_submit(G->reps[r].server, &routed, &t);
    if (st != FHTGS_OK) return st;
    G->cursor = cursor;
    G->load[r].outstanding_cost += cost;
    *ticket = t * kMaxReplicas + r;
    G->cost_of[*ticket] = cost;
    if (replica) *replica = r;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_poll(fhtgs_server_group G, fhtgs_group_completion* out, int32_t max_completions,
                                     int32_t wait_ms, int32_t* n_out) {
    if (!G || !out || !n_out || max_completions < 1) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "bad poll request");
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(wait_ms > 0 ? wait_ms : 0);
    std::vector<fhtgs_completion> buf(static_cast<size_t>(max_completions));
    int n = 0;
    for (;;) {
        for (size_t i = 0; i < G->reps.size() && n < max_completions; ++i) {
            int32_t k = 0;
            const fhtgs_status st = fhtgs_server_poll(G->reps[i].server, buf.data(), max_completions - n, 0, &k);
            if (st != FHTGS_OK) return st;
            std::lock_guard<std::mutex> lk(G->mu);
            for (int j = 0; j < k; ++j) {
                fhtgs_group_completion& g = out[n++];
                g.completion = buf[j];
                g.completion.ticket = buf[j].ticket * kMaxReplicas + static_cast<int64_t>(i);
                g.replica = static_cast<int32_t>(i);
                g.device = G->reps[i].device;
                auto it = G->cost_of.find(g.completion.ticket);
                if (it != G->cost_of.end()) {
                    G->load[i].outstanding_cost -= it->second;
                    G->cost_of.erase(it);
                }
            }
        }
        if (n > 0 || std::chrono::steady_clock::now() >= deadline) break;
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    *n_out = n;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_release(fhtgs_server_group G, int64_t ticket) {
    if (!G) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null group");
    int r = 0;
    int64_t t = 0;
    decode(ticket, &r, &t);
    if (ticket <= 0 || r >= static_cast<int>(G->reps.size())) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown ticket");
    return fhtgs_server_release(G->reps[r].server, t);
}

fhtgs_status fhtgs_server_group_drain(fhtgs_server_group G, int32_t timeout_ms) {
    if (!G) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null group");
    const auto t0 = std::chrono::steady_clock::now();
    for (Replica& r : G->reps) {
        int32_t left = timeout_ms;
        if (timeout_ms >= 0) {
            const auto spent = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
            left = std::max<int32_t>(0, timeout_ms - static_cast<int32_t>(spent.count()));
        }
        const fhtgs_status st = fhtgs_server_drain(r.server, left);
        if (st != FHTGS_OK) return st;
    }
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_group_get_stats(fhtgs_server_group G, int32_t replica, fhtgs_server_stats* out,
                                          int64_t* outstanding_cost) {
    if (!G || !out) return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    if (replica < 0 || replica >= static_cast<int>(G->reps.size()))
        return grp_fail(FHTGS_ERR_INVALID_ARGUMENT, "replica index out of range");
    const fhtgs_status st = fhtgs_server_get_stats(G->reps[replica].server, out);
    if (st != FHTGS_OK) return st;
    if (outstanding_cost) {
        std::lock_guard<std::mutex> lk(G->mu);
        *outstanding_cost = G->load[replica].outstanding_cost;
    }
    return FHTGS_OK;
}

}  // extern "C"

// Request server of libfhtgs: resident scenes, a request queue, continuous batching over a few
// frame slots, and admission of every frame's device memory against an HBM budget (C ABI in
// include/fhtgs.h, "serving").  Host code only: frames are rendered by the same launches as
// fhtgs_render_views (fhtgs_host.cu); the mask tables come from fhtgs_build_tile_masks.
//
// Threads: callers submit/poll under `mu`; one scheduler thread forms frames and enqueues them
// with `mu` released (a CUDA call such as cudaFree may wait for running frames, whose completion
// callbacks take `mu`); the completion callback (a host function on the slot's stream) only
// records the time and wakes the scheduler.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fhtgs.h"
#include "fhtgs_internal.h"

using namespace fhtgs;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kMaxSlots = 8;
constexpr int kMaxBatchRequests = 64;
constexpr int kMaxFrameViews = 2 * kMaxBatchRequests;
constexpr int kCamFloats = 48;            // M 12 | VPM 16 | VPR_inv 16 | cam 3 | pad 1
constexpr int kMaxAttempts = 4;           // renders of one request before FHTGS_ERR_CAPACITY
constexpr int64_t kDefaultBudget = 150ll * 1000 * 1000 * 1000;

double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

fhtgs_status srv_fail(fhtgs_status s, const std::string& msg) {
    set_last_error(msg);
    return s;
}

int64_t scene_bytes(const fhtgs_primitives& p) {
    const int64_t n = p.n_primitives, s = p.total_sh_bases;
    if (p.storage == FHTGS_STORAGE_HALF) return n * (12 + 2 * (3 + 4 + 1) + 2 * (3 + 3 * s));
    return n * 4 * (3 + 3 + 4 + 1 + 3 + 3 * s);
}

size_t image_bytes(int w, int h) { return 12ull * w * h; }

struct Scene {
    fhtgs_primitives prims{};
    fhtgs_settings settings{};
    int64_t bytes = 0;
    int64_t cap_need = 0;   // instance slots per view a frame of this scene is given
    bool live = false;      // removed scenes stay until their running frames finished
    int in_flight = 0;
};

struct Pending {
    int64_t ticket = 0;
    fhtgs_request req{};
    double t_submit = 0.0;
    double t_launch = 0.0;
    int attempts = 0;
    float* own[2] = {nullptr, nullptr};   // server-owned outputs (eyes with image == NULL)
};

// All-visible tile tables of one resolution.
struct Tables {
    uint32_t* words = nullptr;
    uint32_t* sat = nullptr;
    size_t bytes = 0;
};

struct Slot {
    fhtgs_context ctx = nullptr;
    cudaStream_t stream = nullptr;
    float* h_cam = nullptr;         // pinned [kMaxFrameViews][kCamFloats]
    float* d_cam = nullptr;         // device copy read by the frame
    FrameStatus* h_status = nullptr;   // pinned [kMaxFrameViews]
    std::vector<Pending> batch;
    int scene = -1;
    int n_views = 0;
    int64_t cap = 0;
    size_t arena = 0;               // bytes of the slot's arena (updated by the scheduler)
    bool busy = false;
    bool done = false;              // set by the completion callback
    double t_done = 0.0;
    struct fhtgs_server_s* server = nullptr;
};

}  // namespace

struct fhtgs_server_s {
    fhtgs_server_config cfg{};
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;        // wakes the scheduler
    std::condition_variable cv_done;   // wakes pollers and drain
    std::deque<Pending> queue;
    std::vector<Scene> scenes;
    std::map<std::pair<int, int>, Tables> tables;
    uint32_t* fovea = nullptr;         // standard 49x49 fovea table (+ scratch of its build)
    size_t fixed_bytes = 0;            // camera buffers, tables
    Slot slots[kMaxSlots];
    int n_slots = 0;
    std::deque<fhtgs_completion> completions;
    std::multimap<size_t, float*> free_outputs;          // by bytes
    std::map<int64_t, std::vector<float*>> held_outputs; // ticket -> server-owned images
    std::map<float*, size_t> output_size;
    size_t output_bytes = 0;           // all server-owned outputs (free, held, in frames)
    int64_t next_ticket = 1;
    bool stop = false;
    bool paused = false;
    bool mem_blocked = false;          // a frame waits for running frames to free memory
    fhtgs_server_stats stats{};
    std::thread worker;
};

namespace {

size_t resident_bytes_locked(const fhtgs_server_s* S) {
    size_t b = S->fixed_bytes + S->output_bytes;
    for (const Scene& sc : S->scenes)
        if (sc.live || sc.in_flight > 0) b += static_cast<size_t>(sc.bytes);
    for (int i = 0; i < S->n_slots; ++i) b += S->slots[i].arena;
    return b;
}

void complete_locked(fhtgs_server_s* S, const Pending& p, fhtgs_status st, int frame_views, double t_done,
                     const std::string& msg) {
    fhtgs_completion c{};
    c.ticket = p.ticket;
    c.tag = p.req.tag;
    c.status = st;
    c.frame_views = frame_views;
    c.submit_ms = p.t_submit;
    c.launch_ms = p.t_launch;
    c.done_ms = t_done;
    for (int e = 0; e < p.req.n_eyes; ++e) c.images[e] = p.req.eyes[e].image ? p.req.eyes[e].image : p.own[e];
    std::snprintf(c.message, sizeof(c.message), "%s", msg.c_str());
    std::vector<float*> own;
    for (int e = 0; e < 2; ++e)
        if (p.own[e]) own.push_back(p.own[e]);
    if (st == FHTGS_OK) {
        if (!own.empty()) S->held_outputs[p.ticket] = own;
        ++S->stats.completed;
    } else {
        for (float* o : own) S->free_outputs.emplace(S->output_size[o], o);
        for (int e = 0; e < 2; ++e) c.images[e] = p.req.eyes[e].image;
        ++S->stats.failed;
    }
    S->completions.push_back(c);
}

void CUDART_CB frame_done(void* arg) {
    Slot* slot = static_cast<Slot*>(arg);
    fhtgs_server_s* S = slot->server;
    const double t = ms_since(S->t0);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        slot->done = true;
        slot->t_done = t;
    }
    S->cv.notify_all();
}

// Finished frames: complete their requests, or queue them again after an instance overflow.
void reap_locked(fhtgs_server_s* S) {
    bool any = false;
    for (int i = 0; i < S->n_slots; ++i) {
        Slot& sl = S->slots[i];
        if (!sl.busy || !sl.done) continue;
        any = true;
        Scene& sc = S->scenes[sl.scene];
        unsigned long long need = 0;
        bool failed = false;  // a bounded device wait gave up (sort look-back, attribute staging)
        for (int v = 0; v < sl.n_views; ++v) {
            need = std::max(need, sl.h_status[v].n_instances);
            failed = failed || (sl.h_status[v].overflow & (kFrameErrSortLookback | kFrameErrStaging)) != 0;
        }
        const bool overflow = need > static_cast<unsigned long long>(sl.cap);
        const int64_t grown = static_cast<int64_t>(need + need / 4);
        if (grown > sc.cap_need) sc.cap_need = grown;
        --sc.in_flight;
        ++S->stats.frames;
        S->stats.views += sl.n_views;
        if (failed) {
            for (const Pending& p : sl.batch)
                complete_locked(S, p, FHTGS_ERR_CUDA, sl.n_views, sl.t_done,
                                "a bounded device wait of the frame gave up (sort look-back or attribute staging)");
        } else if (overflow) {
            ++S->stats.retries;
            for (auto it = sl.batch.rbegin(); it != sl.batch.rend(); ++it) {
                Pending p = *it;
                if (++p.attempts >= kMaxAttempts)
                    complete_locked(S, p, FHTGS_ERR_CAPACITY, sl.n_views, sl.t_done,
                                    "instance capacity still insufficient after regrowth");
                else
                    S->queue.push_front(p);
            }
        } else {
            for (const Pending& p : sl.batch) complete_locked(S, p, FHTGS_OK, sl.n_views, sl.t_done, "");
        }
        sl.batch.clear();
        sl.busy = false;
        sl.done = false;
    }
    if (any) {
        S->mem_blocked = false;
        S->cv_done.notify_all();
    }
}

bool any_done_locked(const fhtgs_server_s* S) {
    for (int i = 0; i < S->n_slots; ++i)
        if (S->slots[i].busy && S->slots[i].done) return true;
    return false;
}

// A free slot; the one with the largest arena, so that frames reuse memory already held.
int free_slot_locked(const fhtgs_server_s* S) {
    int best = -1;
    for (int i = 0; i < S->n_slots; ++i)
        if (!S->slots[i].busy && (best < 0 || S->slots[i].arena > S->slots[best].arena)) best = i;
    return best;
}

bool any_busy_locked(const fhtgs_server_s* S) {
    for (int i = 0; i < S->n_slots; ++i)
        if (S->slots[i].busy) return true;
    return false;
}

// Builds the all-visible tables of a resolution (called with `mu` released).
fhtgs_status build_tables(int device, int w, int h, Tables* out) {
    const int gw = (w + 15) / 16, gh = (h + 15) / 16;
    const size_t words = (static_cast<size_t>(gw) * gh + 31) / 32;
    const size_t sat = static_cast<size_t>(gw + 1) * (gh + 1);
    Tables t;
    t.bytes = 4 * (words + sat);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&t.words, t.bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return srv_fail(FHTGS_ERR_OUT_OF_MEMORY, std::string("tile tables: ") + cudaGetErrorString(e));
    }
    t.sat = t.words + words;
    fhtgs_status st = fhtgs_build_tile_masks(nullptr, w, h, t.words, t.sat, nullptr, nullptr);
    if (st == FHTGS_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) st = FHTGS_ERR_CUDA;
    if (st != FHTGS_OK) {
        cudaFree(t.words);
        return srv_fail(st, "tile table build failed");
    }
    *out = t;
    return FHTGS_OK;
}

// Views of a candidate frame (camera pointers into the slot's device buffer).
void frame_views_locked(fhtgs_server_s* S, const Slot& sl, const std::vector<const Pending*>& reqs,
                        std::vector<fhtgs_view>* views) {
    views->clear();
    for (const Pending* p : reqs) {
        for (int e = 0; e < p->req.n_eyes; ++e) {
            const fhtgs_eye& eye = p->req.eyes[e];
            const int v = static_cast<int>(views->size());
            fhtgs_view view{};
            float* cam = sl.d_cam + static_cast<size_t>(v) * kCamFloats;
            view.M = cam;
            view.VPM = cam + 12;
            view.VPR_inv = cam + 28;
            view.cam_position = cam + 44;
            view.gaze_x = eye.gaze_x;
            view.gaze_y = eye.gaze_y;
            if (eye.visibility_mask) {
                view.visibility_mask = eye.visibility_mask;
                view.visibility_mask_area_table = eye.visibility_mask_area_table;
            } else {
                const Tables& t = S->tables[{eye.width, eye.height}];
                view.visibility_mask = t.words;
                view.visibility_mask_area_table = t.sat;
            }
            view.fovea_mask_area_table = eye.fovea_mask_area_table ? eye.fovea_mask_area_table : S->fovea;
            view.width = eye.width;
            view.height = eye.height;
            view.focal_x = eye.focal_x;
            view.focal_y = eye.focal_y;
            view.center_x = eye.center_x;
            view.center_y = eye.center_y;
            view.image = eye.image ? eye.image : p->own[e];
            views->push_back(view);
        }
    }
}

// Output bytes a candidate frame needs beyond the free pool (and which free buffers it takes).
size_t output_need_locked(const fhtgs_server_s* S, const std::vector<const Pending*>& reqs) {
    std::multimap<size_t, float*> pool = S->free_outputs;
    size_t need = 0;
    for (const Pending* p : reqs)
        for (int e = 0; e < p->req.n_eyes; ++e) {
            if (p->req.eyes[e].image || p->own[e]) continue;
            const size_t b = image_bytes(p->req.eyes[e].width, p->req.eyes[e].height);
            auto it = pool.find(b);
            if (it != pool.end()) pool.erase(it);
            else need += b;
        }
    return need;
}

// Launches one frame on a slot (called with `mu` released; the slot is reserved).
fhtgs_status launch_frame(fhtgs_server_s* S, Slot& sl, const Scene& sc, const std::vector<fhtgs_view>& views) {
    for (const Pending& p : sl.batch)
        if (p.req.ready_event) {
            const cudaError_t e = cudaStreamWaitEvent(sl.stream, static_cast<cudaEvent_t>(p.req.ready_event), 0);
            if (e != cudaSuccess) return srv_fail(FHTGS_ERR_CUDA, std::string("ready event: ") + cudaGetErrorString(e));
        }
    int v = 0;
    for (const Pending& p : sl.batch)
        for (int e = 0; e < p.req.n_eyes; ++e, ++v) {
            const fhtgs_eye& eye = p.req.eyes[e];
            float* h = sl.h_cam + static_cast<size_t>(v) * kCamFloats;
            std::memcpy(h, eye.M, 12 * sizeof(float));
            std::memcpy(h + 12, eye.VPM, 16 * sizeof(float));
            std::memcpy(h + 28, eye.VPR_inv, 16 * sizeof(float));
            std::memcpy(h + 44, eye.cam_position, 3 * sizeof(float));
            h[47] = 0.0f;
        }
    cudaError_t e = cudaMemcpyAsync(sl.d_cam, sl.h_cam, sizeof(float) * kCamFloats * v, cudaMemcpyHostToDevice,
                                    sl.stream);
    if (e != cudaSuccess) return srv_fail(FHTGS_ERR_CUDA, std::string("camera upload: ") + cudaGetErrorString(e));
    set_context_capacity(sl.ctx, sl.cap);
    fhtgs_status st = enqueue_frame(sl.ctx, &sc.prims, views.data(), v, &sc.settings, sl.stream, sl.h_status);
    if (st != FHTGS_OK) return st;
    e = cudaLaunchHostFunc(sl.stream, frame_done, &sl);
    if (e != cudaSuccess) return srv_fail(FHTGS_ERR_CUDA, std::string("completion callback: ") + cudaGetErrorString(e));
    return FHTGS_OK;
}

// Forms and launches frames while a slot is free and the queue is not empty.
void schedule_locked(fhtgs_server_s* S, std::unique_lock<std::mutex>& lk) {
    while (!S->queue.empty() && !S->mem_blocked) {
        const int si = free_slot_locked(S);
        if (si < 0) return;
        Slot& sl = S->slots[si];
        const Pending& head = S->queue.front();
        const int scene_id = head.req.scene;
        Scene& sc = S->scenes[scene_id];
        if (!sc.live) {
            Pending p = head;
            S->queue.pop_front();
            complete_locked(S, p, FHTGS_ERR_INVALID_ARGUMENT, 0, ms_since(S->t0), "scene was removed");
            S->cv_done.notify_all();
            continue;
        }
        // tables of resolutions seen for the first time (built with the lock released)
        std::pair<int, int> missing{0, 0};
        for (size_t i = 0; i < S->queue.size() && missing.first == 0; ++i) {
            const fhtgs_request& r = S->queue[i].req;
            if (r.scene != scene_id) continue;
            for (int e = 0; e < r.n_eyes; ++e)
                if (!r.eyes[e].visibility_mask && !S->tables.count({r.eyes[e].width, r.eyes[e].height}))
                    missing = {r.eyes[e].width, r.eyes[e].height};
        }
        if (missing.first) {
            lk.unlock();
            Tables t;
            fhtgs_status st = build_tables(S->cfg.device, missing.first, missing.second, &t);
            lk.lock();
            if (st != FHTGS_OK) {
                // fail every queued request that needs this resolution's tables
                const std::string msg = std::string("tile tables: ") + fhtgs_last_error();
                for (auto it = S->queue.begin(); it != S->queue.end();) {
                    bool needs = false;
                    for (int e = 0; e < it->req.n_eyes; ++e)
                        needs = needs || (!it->req.eyes[e].visibility_mask && it->req.eyes[e].width == missing.first &&
                                          it->req.eyes[e].height == missing.second);
                    if (needs) {
                        complete_locked(S, *it, st, 0, ms_since(S->t0), msg);
                        it = S->queue.erase(it);
                    } else {
                        ++it;
                    }
                }
                S->cv_done.notify_all();
            } else {
                S->tables[missing] = t;
                S->fixed_bytes += t.bytes;
            }
            continue;
        }
        // the frame: the oldest request and the next queued ones of its scene
        std::vector<size_t> idx;
        int views_total = 0;
        for (size_t i = 0; i < S->queue.size() && static_cast<int>(idx.size()) < S->cfg.max_batch_requests; ++i) {
            const fhtgs_request& r = S->queue[i].req;
            if (r.scene != scene_id) continue;
            if (views_total + r.n_eyes > kMaxFrameViews) break;
            idx.push_back(i);
            views_total += r.n_eyes;
        }
        const int64_t cap = std::max<int64_t>(sc.cap_need, 1);
        std::vector<const Pending*> reqs;
        std::vector<fhtgs_view> views;
        size_t extra = 0;
        const size_t resident = resident_bytes_locked(S);
        const size_t budget = static_cast<size_t>(S->cfg.hbm_budget_bytes);
        for (;;) {
            reqs.clear();
            for (size_t i : idx) reqs.push_back(&S->queue[i]);
            frame_views_locked(S, sl, reqs, &views);
            const size_t arena = frame_arena_need(sl.ctx, &sc.prims, views.data(), static_cast<int>(views.size()),
                                                  &sc.settings, cap);
            extra = (arena > sl.arena ? arena - sl.arena : 0) + output_need_locked(S, reqs);
            if (resident + extra <= budget || idx.size() == 1) break;
            idx.pop_back();
        }
        if (resident + extra > budget) {
            // free memory nobody is using: idle slots' arenas, unused output buffers
            bool freed = false;
            std::vector<fhtgs_context> idle;
            for (int i = 0; i < S->n_slots; ++i)
                if (i != si && !S->slots[i].busy && S->slots[i].arena > 0) {
                    idle.push_back(S->slots[i].ctx);
                    S->slots[i].arena = 0;
                    S->slots[i].busy = true;   // reserved while its arena is released
                }
            std::vector<float*> unused;
            for (auto& kv : S->free_outputs) {
                unused.push_back(kv.second);
                S->output_bytes -= kv.first;
                S->output_size.erase(kv.second);
            }
            S->free_outputs.clear();
            if (!idle.empty() || !unused.empty()) {
                lk.unlock();
                for (fhtgs_context c : idle) release_arena(c);
                for (float* o : unused) cudaFree(o);
                lk.lock();
                for (int i = 0; i < S->n_slots; ++i)
                    for (fhtgs_context c : idle)
                        if (S->slots[i].ctx == c) S->slots[i].busy = false;
                freed = true;
            }
            if (freed) continue;
            if (any_busy_locked(S)) {
                S->mem_blocked = true;
                ++S->stats.admission_waits;
                return;
            }
            Pending p = S->queue.front();
            S->queue.pop_front();
            complete_locked(S, p, FHTGS_ERR_OUT_OF_MEMORY, 0, ms_since(S->t0),
                            "request needs " + std::to_string(extra) + " bytes beyond the " +
                                std::to_string(resident) + " resident; budget " + std::to_string(budget));
            S->cv_done.notify_all();
            continue;
        }
        // take the requests out of the queue (in order) and give them output buffers
        sl.batch.clear();
        for (size_t i : idx) sl.batch.push_back(S->queue[i]);
        for (auto it = idx.rbegin(); it != idx.rend(); ++it) S->queue.erase(S->queue.begin() + *it);
        std::vector<std::pair<Pending*, int>> to_alloc;
        for (Pending& p : sl.batch)
            for (int e = 0; e < p.req.n_eyes; ++e) {
                if (p.req.eyes[e].image || p.own[e]) continue;
                const size_t b = image_bytes(p.req.eyes[e].width, p.req.eyes[e].height);
                auto it = S->free_outputs.find(b);
                if (it != S->free_outputs.end()) {
                    p.own[e] = it->second;
                    S->free_outputs.erase(it);
                } else {
                    to_alloc.push_back({&p, e});
                    S->output_bytes += b;   // accounted before the allocation
                }
            }
        sl.busy = true;
        sl.done = false;
        sl.scene = scene_id;
        sl.cap = cap;
        int nv = 0;
        for (const Pending& p : sl.batch) nv += p.req.n_eyes;
        sl.n_views = nv;
        ++sc.in_flight;
        const double t_launch = ms_since(S->t0);
        for (Pending& p : sl.batch) p.t_launch = t_launch;
        S->stats.max_frame_requests = std::max<int64_t>(S->stats.max_frame_requests, static_cast<int64_t>(sl.batch.size()));
        const size_t peak = resident + extra;
        S->stats.peak_resident_bytes = std::max<int64_t>(S->stats.peak_resident_bytes, static_cast<int64_t>(peak));
        const Scene scene_copy = sc;
        lk.unlock();
        fhtgs_status st = FHTGS_OK;
        std::string msg;
        for (auto& pa : to_alloc) {
            const fhtgs_eye& eye = pa.first->req.eyes[pa.second];
            float* o = nullptr;
            cudaError_t e = cudaMalloc(&o, image_bytes(eye.width, eye.height));
            if (e != cudaSuccess) {
                cudaGetLastError();
                st = FHTGS_ERR_OUT_OF_MEMORY;
                msg = std::string("output image: ") + cudaGetErrorString(e);
                break;
            }
            pa.first->own[pa.second] = o;
        }
        std::vector<fhtgs_view> launch_views;
        if (st == FHTGS_OK) {
            std::vector<const Pending*> rs;
            for (const Pending& p : sl.batch) rs.push_back(&p);
            {
                // table lookups read the map; entries are only added by this thread
                frame_views_locked(S, sl, rs, &launch_views);
            }
            st = launch_frame(S, sl, scene_copy, launch_views);
            if (st != FHTGS_OK) msg = fhtgs_last_error();
        }
        const size_t arena_now = fhtgs_context_arena_bytes(sl.ctx);
        // a frame that could not be enqueued gets no completion callback: let whatever part of
        // it was queued finish before its buffers are reused (with `mu` released)
        if (st != FHTGS_OK) cudaStreamSynchronize(sl.stream);
        lk.lock();
        sl.arena = arena_now;
        for (auto& pa : to_alloc) {
            const fhtgs_eye& eye = pa.first->req.eyes[pa.second];
            const size_t b = image_bytes(eye.width, eye.height);
            if (pa.first->own[pa.second]) S->output_size[pa.first->own[pa.second]] = b;
            else S->output_bytes -= b;
        }
        if (st != FHTGS_OK) {
            for (const Pending& p : sl.batch) complete_locked(S, p, st, 0, ms_since(S->t0), msg);
            sl.batch.clear();
            sl.busy = false;
            --S->scenes[scene_id].in_flight;
            S->cv_done.notify_all();
        }
    }
}

void worker_main(fhtgs_server_s* S) {
    cudaSetDevice(S->cfg.device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        // Stopping, the thread waits (with `mu` released) for the running frames' completion
        // callbacks, which take `mu`, and leaves once no frame runs: a predicate that held while
        // frames still ran would keep `mu` locked and the callbacks out for good.
        S->cv.wait(lk, [&] {
            return any_done_locked(S) || (S->stop && !any_busy_locked(S)) ||
                   (!S->stop && !S->paused && !S->queue.empty() && !S->mem_blocked && free_slot_locked(S) >= 0);
        });
        reap_locked(S);
        if (S->stop) {
            // shutting down: requests queued again by the reaping (an instance overflow) fail
            // like the rest of the queue; no new frame is launched
            while (!S->queue.empty()) {
                complete_locked(S, S->queue.front(), FHTGS_ERR_NOT_READY, 0, ms_since(S->t0), "server shut down");
                S->queue.pop_front();
            }
            if (!any_busy_locked(S)) break;
            continue;
        }
        if (!S->paused) schedule_locked(S, lk);
    }
    S->cv_done.notify_all();
}

fhtgs_status check_request(fhtgs_server_s* S, const fhtgs_request* r) {
    if (!r) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null request");
    if (r->n_eyes < 1 || r->n_eyes > 2) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "n_eyes must be 1 or 2");
    for (int e = 0; e < r->n_eyes; ++e) {
        const fhtgs_eye& eye = r->eyes[e];
        if ((eye.visibility_mask == nullptr) != (eye.visibility_mask_area_table == nullptr))
            return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "give both the visibility mask and its area table, or neither");
    }
    // the frame checks of fhtgs_render_views, on stand-in device pointers
    fhtgs_view v[2] = {};
    for (int e = 0; e < r->n_eyes; ++e) {
        const fhtgs_eye& eye = r->eyes[e];
        v[e].M = v[e].VPM = v[e].VPR_inv = v[e].cam_position = S->slots[0].d_cam;
        v[e].visibility_mask = eye.visibility_mask ? eye.visibility_mask : S->fovea;
        v[e].visibility_mask_area_table = eye.visibility_mask_area_table ? eye.visibility_mask_area_table : S->fovea;
        v[e].fovea_mask_area_table = S->fovea;
        v[e].width = eye.width;
        v[e].height = eye.height;
        v[e].image = eye.image ? eye.image : reinterpret_cast<float*>(S->slots[0].d_cam);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (r->scene < 0 || r->scene >= static_cast<int>(S->scenes.size()) || !S->scenes[r->scene].live)
        return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown scene");
    const Scene& sc = S->scenes[r->scene];
    return validate_frame(&sc.prims, v, r->n_eyes, &sc.settings);
}

}  // namespace

extern "C" {

fhtgs_status fhtgs_server_create(const fhtgs_server_config* config, fhtgs_server* out) {
    if (!config || !out) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    fhtgs_server_config cfg = *config;
    if (cfg.max_in_flight == 0) cfg.max_in_flight = 2;
    if (cfg.max_batch_requests == 0) cfg.max_batch_requests = 8;
    if (cfg.hbm_budget_bytes == 0) cfg.hbm_budget_bytes = kDefaultBudget;
    if (cfg.max_in_flight < 1 || cfg.max_in_flight > kMaxSlots)
        return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "max_in_flight must be in [1, 8]");
    if (cfg.max_batch_requests < 1 || cfg.max_batch_requests > kMaxBatchRequests)
        return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "max_batch_requests must be in [1, 64]");
    if (cfg.hbm_budget_bytes < 0) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "negative budget");
    if (cfg.blend_split_permille != 0 && (cfg.blend_split_permille < 50 || cfg.blend_split_permille > 8000))
        return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "blend_split_permille must be 0 (off) or in [50, 8000]");
    int n_dev = 0;
    cudaError_t e = cudaGetDeviceCount(&n_dev);
    if (e != cudaSuccess) return srv_fail(FHTGS_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    if (cfg.device < 0 || cfg.device >= n_dev) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "no such CUDA device");
    e = cudaSetDevice(cfg.device);
    if (e != cudaSuccess) return srv_fail(FHTGS_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));

    auto* S = new fhtgs_server_s();
    S->cfg = cfg;
    S->t0 = Clock::now();
    S->n_slots = cfg.max_in_flight;
    fhtgs_status st = FHTGS_OK;
    auto bail = [&](fhtgs_status s, const std::string& msg) {
        fhtgs_server_destroy(S);  // releases whatever was created so far
        return srv_fail(s, msg);
    };
    // standard fovea table (built once; the words/area outputs of that build are scratch)
    const size_t fovea_words = 49 * 49 + 8 + 16;
    e = cudaMalloc(&S->fovea, 4 * fovea_words);
    if (e != cudaSuccess) { cudaGetLastError(); delete S; return srv_fail(FHTGS_ERR_OUT_OF_MEMORY, "fovea table"); }
    S->fixed_bytes += 4 * fovea_words;
    st = fhtgs_build_tile_masks(nullptr, 16, 16, S->fovea + 49 * 49, S->fovea + 49 * 49 + 8, S->fovea, nullptr);
    if (st != FHTGS_OK || cudaStreamSynchronize(nullptr) != cudaSuccess) return bail(FHTGS_ERR_CUDA, "fovea table build");
    for (int i = 0; i < S->n_slots; ++i) {
        Slot& sl = S->slots[i];
        sl.server = S;
        st = fhtgs_context_create(cfg.device, &sl.ctx);
        if (st != FHTGS_OK) return bail(st, fhtgs_last_error());
        if (cfg.blend_split_permille != 0) {
            st = fhtgs_context_set_blend_split(sl.ctx, static_cast<float>(cfg.blend_split_permille) / 1000.0f, 0);
            if (st != FHTGS_OK) return bail(st, fhtgs_last_error());
        }
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaMallocHost(&sl.h_cam, sizeof(float) * kCamFloats * kMaxFrameViews) != cudaSuccess ||
            cudaMallocHost(&sl.h_status, sizeof(FrameStatus) * kMaxFrameViews) != cudaSuccess ||
            cudaMalloc(&sl.d_cam, sizeof(float) * kCamFloats * kMaxFrameViews) != cudaSuccess) {
            cudaGetLastError();
            return bail(FHTGS_ERR_CUDA, "slot resources");
        }
        S->fixed_bytes += sizeof(float) * kCamFloats * kMaxFrameViews;
    }
    if (static_cast<int64_t>(S->fixed_bytes) > cfg.hbm_budget_bytes)
        return bail(FHTGS_ERR_OUT_OF_MEMORY, "budget below the server's own buffers");
    S->worker = std::thread(worker_main, S);
    *out = S;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_destroy(fhtgs_server S) {
    if (!S) return FHTGS_OK;
    if (S->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stop = true;
            while (!S->queue.empty()) {
                complete_locked(S, S->queue.front(), FHTGS_ERR_NOT_READY, 0, ms_since(S->t0), "server shut down");
                S->queue.pop_front();
            }
        }
        S->cv.notify_all();
        S->worker.join();
    }
    cudaSetDevice(S->cfg.device);
    for (int i = 0; i < S->n_slots; ++i) {
        Slot& sl = S->slots[i];
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.ctx) fhtgs_context_destroy(sl.ctx);
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.h_cam) cudaFreeHost(sl.h_cam);
        if (sl.h_status) cudaFreeHost(sl.h_status);
        if (sl.d_cam) cudaFree(sl.d_cam);
    }
    for (auto& kv : S->tables) cudaFree(kv.second.words);
    for (auto& kv : S->output_size) cudaFree(kv.first);
    if (S->fovea) cudaFree(S->fovea);
    delete S;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_add_scene(fhtgs_server S, const fhtgs_primitives* prims, const fhtgs_settings* settings,
                                    int32_t* scene_id) {
    if (!S || !prims || !settings || !scene_id) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    // the frame checks of fhtgs_render_views for this scene, on a stand-in view
    fhtgs_view v{};
    v.M = v.VPM = v.VPR_inv = v.cam_position = S->slots[0].d_cam;
    v.visibility_mask = v.visibility_mask_area_table = v.fovea_mask_area_table = S->fovea;
    v.width = v.height = 16;
    v.image = S->slots[0].d_cam;
    fhtgs_status st = validate_frame(prims, &v, 1, settings);
    if (st != FHTGS_OK) return st;
    Scene sc;
    sc.prims = *prims;
    sc.settings = *settings;
    sc.bytes = scene_bytes(*prims);
    sc.cap_need = default_instance_capacity(prims->n_primitives);
    sc.live = true;
    std::lock_guard<std::mutex> lk(S->mu);
    const size_t resident = resident_bytes_locked(S);
    if (static_cast<int64_t>(resident) + sc.bytes > S->cfg.hbm_budget_bytes)
        return srv_fail(FHTGS_ERR_OUT_OF_MEMORY, "scene of " + std::to_string(sc.bytes) + " bytes does not fit the budget beside " +
                                                     std::to_string(resident) + " resident bytes");
    *scene_id = static_cast<int32_t>(S->scenes.size());
    S->scenes.push_back(sc);
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_remove_scene(fhtgs_server S, int32_t scene_id) {
    if (!S) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (scene_id < 0 || scene_id >= static_cast<int>(S->scenes.size()) || !S->scenes[scene_id].live)
            return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "unknown scene");
        S->scenes[scene_id].live = false;
    }
    S->cv.notify_all();
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_submit(fhtgs_server S, const fhtgs_request* request, int64_t* ticket) {
    if (!S || !ticket) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    fhtgs_status st = check_request(S, request);
    if (st != FHTGS_OK) return st;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stop) return srv_fail(FHTGS_ERR_NOT_READY, "server is shutting down");
        Pending p;
        p.ticket = S->next_ticket++;
        p.req = *request;
        p.t_submit = ms_since(S->t0);
        S->queue.push_back(p);
        ++S->stats.submitted;
        *ticket = p.ticket;
    }
    S->cv.notify_all();
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_poll(fhtgs_server S, fhtgs_completion* out, int32_t max_completions, int32_t wait_ms,
                               int32_t* n_out) {
    if (!S || !out || !n_out || max_completions < 1) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "bad poll request");
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->completions.empty() && wait_ms > 0)
        S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->completions.empty(); });
    int n = 0;
    while (n < max_completions && !S->completions.empty()) {
        out[n++] = S->completions.front();
        S->completions.pop_front();
    }
    *n_out = n;
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_release(fhtgs_server S, int64_t ticket) {
    if (!S) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->held_outputs.find(ticket);
    if (it == S->held_outputs.end()) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "no server-owned outputs for this ticket");
    for (float* o : it->second) S->free_outputs.emplace(S->output_size[o], o);
    S->held_outputs.erase(it);
    S->mem_blocked = false;
    S->cv.notify_all();
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_set_paused(fhtgs_server S, int32_t paused) {
    if (!S) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null server");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->paused = paused != 0;
    }
    S->cv.notify_all();
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_drain(fhtgs_server S, int32_t timeout_ms) {
    if (!S) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->paused && !S->queue.empty()) return srv_fail(FHTGS_ERR_NOT_READY, "server is paused with requests queued");
    auto idle = [&] { return S->queue.empty() && !any_busy_locked(S); };
    if (timeout_ms < 0) {
        S->cv_done.wait(lk, idle);
        return FHTGS_OK;
    }
    if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle))
        return srv_fail(FHTGS_ERR_NOT_READY, "requests still queued or running");
    return FHTGS_OK;
}

fhtgs_status fhtgs_server_get_stats(fhtgs_server S, fhtgs_server_stats* out) {
    if (!S || !out) return srv_fail(FHTGS_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->queued = static_cast<int64_t>(S->queue.size());
    int64_t running = 0;
    for (int i = 0; i < S->n_slots; ++i)
        if (S->slots[i].busy) running += static_cast<int64_t>(S->slots[i].batch.size());
    out->in_flight = running;
    out->resident_bytes = static_cast<int64_t>(resident_bytes_locked(S));
    return FHTGS_OK;
}

double fhtgs_server_clock_ms(fhtgs_server S) { return S ? ms_since(S->t0) : 0.0; }

}  // extern "C"

// Request server of include/depth_cuda.h (ds_server_*): continuous batching of stereo frames.
//
// Frames are submitted from any thread and queued in arrival order. One worker thread admits the
// queue's head as soon as a slot is free and its cost / path-value volume fits the memory budget,
// enqueues the frame on that slot's stream (host -> device copy of the pair, the frame's kernels,
// device -> host copy of the results) and goes on admitting, so that frames that arrive while others
// are on the GPU overlap with them. A host callback at the end of each slot's stream work timestamps
// the completion and wakes the worker, which releases the slot and hands the completion to
// ds_server_poll.
//
// Memory: each slot keeps one frame handle per (size, parameters) for its small buffers (rectified
// pair, census, outputs); the large volumes belong to the slot (one buffer, reused by every frame the
// slot runs). The sum of the slots' volume buffers never exceeds the budget, so volume memory is what
// admission is decided by.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/depth_cuda.h"
#include "dispatch.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

constexpr size_t kDefaultBudget = size_t{40} << 30;
constexpr float kMaxDepthJump = 4.0f;  // depth::PointParams default (libs/depth/include/einstar/depth/point_image.hpp:43-45)

struct Calib {
    bool present = false;
    float* map[4] = {nullptr, nullptr, nullptr, nullptr};
    int map_w = 0, map_h = 0, raw_w = 0, raw_h = 0;
    bool have_geom = false;
    ds_geometry geom{};
    float min_depth = 0.0f, max_depth = 0.0f;
};

// Frames of one key share a handle per slot.
struct ShapeKey {
    int w = 0, h = 0;
    ds_stereo_params p{};
    bool operator<(const ShapeKey& o) const { return std::memcmp(this, &o, sizeof(ShapeKey)) < 0; }
};
static_assert(sizeof(ShapeKey) == 2 * sizeof(int) + sizeof(ds_stereo_params), "ShapeKey must have no padding");

// Frames that differ only in min_disparity share a handle (it moves the census guards, not the sizes).
ShapeKey key_of(int w, int h, const ds_stereo_params& p) {
    ShapeKey k;
    std::memset(&k, 0, sizeof(k));
    k.w = w;
    k.h = h;
    k.p = p;
    k.p.sgm.min_disparity = 0;
    return k;
}

struct Job {
    uint64_t ticket = 0;
    ds_request r{};
    Clock::time_point t_submit, t_admit, t_done;
    size_t volume = 0;
};

struct Slot {
    ds_server* server = nullptr;
    int index = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void* volume = nullptr;
    size_t volume_cap = 0;
    std::map<ShapeKey, ds_handle*> handles;
    bool busy = false;
    Job job;
};

struct Failure {
    int code;
    std::string what;
};

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Failure{DS_IO, std::string(what) + ": " + cudaGetErrorString(e)};
}

}  // namespace

struct ds_server {
    ds_server_options opt{};
    int device = 0;
    std::mutex m;
    std::condition_variable cv_work;  // worker: submissions, finished slots, stop
    std::condition_variable cv_done;  // pollers: completions
    std::deque<Job> pending;
    std::vector<int> finished;        // slots whose stream work has ended (set by host callbacks)
    std::deque<ds_completion> done;
    std::vector<std::unique_ptr<Slot>> slots;
    std::map<int, Calib> calib;
    std::map<ShapeKey, size_t> key_volume;  // volume bytes of a frame of each key
    bool stop = false;
    bool dirty = false;                     // something to admit may have changed
    bool configuring = false;               // ds_server_reserve owns the slots: admit nothing
    uint64_t next_ticket = 1;
    ds_server_stats stats{};
    // Written by the thread that owns the slots, read by ds_server_get_stats.
    std::atomic<size_t> volume_total{0};    // sum of the slots' volume buffers
    std::atomic<size_t> handle_bytes{0};    // device buffers of the slots' frame handles
    std::string err;
    std::thread worker;

    void set_error(const std::string& e) {
        std::lock_guard<std::mutex> lk(m);
        err = e;
    }
};

namespace {

void CUDART_CB on_slot_done(void* arg) {
    // Runs on a CUDA driver thread: no CUDA calls here.
    auto* slot = static_cast<Slot*>(arg);
    ds_server* s = slot->server;
    std::lock_guard<std::mutex> lk(s->m);
    slot->job.t_done = Clock::now();
    s->finished.push_back(slot->index);
    s->cv_work.notify_one();
}

// A slot's handle for `key`, created (with its device buffers) when the slot first serves the key.
ds_handle* slot_handle(ds_server* s, Slot& sl, const ShapeKey& key) {
    auto it = sl.handles.find(key);
    if (it != sl.handles.end()) return it->second;
    ds_handle* h = nullptr;
    const int rc = ds::create_shared_volume_handle(&key.p, key.w, key.h, &h);
    if (rc != DS_OK) throw Failure{rc, ds_last_global_error()};
    sl.handles.emplace(key, h);
    s->key_volume[key] = ds::volume_bytes(h);
    s->handle_bytes += ds_device_bytes(h);
    return h;
}

Slot& new_slot(ds_server* s) {
    auto sl = std::make_unique<Slot>();
    sl->server = s;
    sl->index = static_cast<int>(s->slots.size());
    check_cuda(cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    check_cuda(cudaEventCreate(&sl->ev0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&sl->ev1), "cudaEventCreate");
    std::lock_guard<std::mutex> lk(s->m);
    s->slots.push_back(std::move(sl));
    return *s->slots.back();
}

// Resizes an idle slot's volume buffer (stream-ordered, so no device-wide synchronisation).
void set_volume(ds_server* s, Slot& sl, size_t bytes) {
    if (sl.volume_cap == bytes) return;
    if (sl.volume) {
        check_cuda(cudaFreeAsync(sl.volume, sl.st), "cudaFreeAsync");
        s->volume_total -= sl.volume_cap;
        sl.volume = nullptr;
        sl.volume_cap = 0;
    }
    if (bytes) {
        check_cuda(cudaMallocAsync(&sl.volume, bytes, sl.st), "cudaMallocAsync");
        sl.volume_cap = bytes;
        s->volume_total += bytes;
    }
}

// Picks (and sizes) an idle slot for a frame of `volume` bytes without letting the slots' volume
// buffers exceed the budget. Returns nullptr when the frame has to wait for running frames.
Slot* pick_slot(ds_server* s, size_t volume) {
    Slot* best = nullptr;
    for (auto& p : s->slots)  // an idle slot that is large enough, the smallest such
        if (!p->busy && p->volume_cap >= volume && (!best || p->volume_cap < best->volume_cap)) best = p.get();
    if (best) return best;
    Slot* grow = nullptr;  // else the largest idle slot, grown
    for (auto& p : s->slots)
        if (!p->busy && (!grow || p->volume_cap > grow->volume_cap)) grow = p.get();
    const size_t budget = s->opt.volume_budget_bytes;
    if (!grow && static_cast<int>(s->slots.size()) < s->opt.max_slots) {
        if (s->volume_total + volume > budget) {
            // reclaim nothing here: no idle slot exists, the running frames hold the memory
            return nullptr;
        }
        grow = &new_slot(s);
    }
    if (!grow) return nullptr;
    if (s->volume_total - grow->volume_cap + volume > budget) {
        for (auto& p : s->slots)  // give back the volumes of other idle slots
            if (!p->busy && p.get() != grow && p->volume) set_volume(s, *p, 0);
        if (s->volume_total - grow->volume_cap + volume > budget) return nullptr;
    }
    set_volume(s, *grow, volume);
    return grow;
}

void launch(ds_server* s, Slot& sl, ds_handle* h, const Calib* c) {
    const ds_request& r = sl.job.r;
    const bool raw = r.calib >= 0;
    if (const int rc = ds::set_frame_params(h, r.params); rc != DS_OK) throw Failure{rc, ds_last_error(h)};
    ds::bind_volumes(h, sl.volume);
    if (raw) {
        const int rc = ds::bind_rectification(h, c->map, c->map_w, c->map_h, c->raw_w, c->raw_h);
        if (rc != DS_OK) throw Failure{rc, ds_last_error(h)};
    }
    const bool depth = r.out.depth && c && c->have_geom;
    if (depth) ds_set_point_params(h, &c->geom, c->min_depth, c->max_depth, kMaxDepthJump);
    uint8_t* in[2];
    ds::input_buffers(h, raw, in);
    const int iw = ds::input_width(h, raw), ih = ds::input_height(h, raw);
    check_cuda(cudaEventRecord(sl.ev0, sl.st), "cudaEventRecord");
    check_cuda(cudaMemcpy2DAsync(in[0], iw, r.left, r.stride, iw, ih, cudaMemcpyHostToDevice, sl.st), "copy left");
    check_cuda(cudaMemcpy2DAsync(in[1], iw, r.right, r.stride, iw, ih, cudaMemcpyHostToDevice, sl.st), "copy right");
    const ds_outputs all = ds::device_outputs(h);
    ds_outputs dev{};
    dev.disparity = r.out.disparity ? all.disparity : nullptr;
    dev.confidence = r.out.confidence ? all.confidence : nullptr;
    dev.disparity_u16 = r.out.disparity_u16 ? all.disparity_u16 : nullptr;
    dev.depth = depth ? all.depth : nullptr;
    const int rc = raw ? ds_compute_raw_device(h, in[0], in[1], &dev, sl.st) : ds_compute_device(h, in[0], in[1], &dev, sl.st);
    if (rc != DS_OK) throw Failure{rc, ds_last_error(h)};
    const size_t n = static_cast<size_t>(r.width) * r.height;
    if (dev.disparity) check_cuda(cudaMemcpyAsync(r.out.disparity, dev.disparity, n * 4, cudaMemcpyDeviceToHost, sl.st), "copy disparity");
    if (dev.confidence) check_cuda(cudaMemcpyAsync(r.out.confidence, dev.confidence, n * 4, cudaMemcpyDeviceToHost, sl.st), "copy confidence");
    if (dev.disparity_u16)
        check_cuda(cudaMemcpyAsync(r.out.disparity_u16, dev.disparity_u16, n * 2, cudaMemcpyDeviceToHost, sl.st), "copy u16");
    if (dev.depth) check_cuda(cudaMemcpyAsync(r.out.depth, dev.depth, n * 4, cudaMemcpyDeviceToHost, sl.st), "copy depth");
    check_cuda(cudaEventRecord(sl.ev1, sl.st), "cudaEventRecord");
    check_cuda(cudaLaunchHostFunc(sl.st, on_slot_done, &sl), "cudaLaunchHostFunc");
}

void push_completion(ds_server* s, const Job& j, int status, double gpu_ms, const std::string& err) {
    ds_completion c{};
    c.ticket = j.ticket;
    c.tag = j.r.tag;
    c.status = status;
    c.queue_ms = status == DS_OK ? ms_between(j.t_submit, j.t_admit) : 0.0;
    c.gpu_ms = gpu_ms;
    c.latency_ms = ms_between(j.t_submit, status == DS_OK ? j.t_done : Clock::now());
    std::lock_guard<std::mutex> lk(s->m);
    s->done.push_back(c);
    if (status == DS_OK) {
        ++s->stats.completed;
    } else {
        ++s->stats.failed;
        s->err = err;
    }
    s->cv_done.notify_all();
}

// Admits queued frames in arrival order while slots and memory allow.
void admit(ds_server* s) {
    for (;;) {
        Job job;
        Calib calib;
        {
            std::lock_guard<std::mutex> lk(s->m);
            if (s->pending.empty() || s->configuring) return;
            job = s->pending.front();
            if (job.r.calib >= 0) calib = s->calib.at(job.r.calib);  // validated at submit
        }
        const ShapeKey key = key_of(job.r.width, job.r.height, job.r.params);
        const Calib* c = job.r.calib >= 0 ? &calib : nullptr;
        Slot* sl = nullptr;
        try {
            auto kv = s->key_volume.find(key);
            if (kv == s->key_volume.end()) {
                // First frame of this key: size it with a handle in an idle slot (or a new one).
                Slot* probe = nullptr;
                for (auto& p : s->slots)
                    if (!p->busy) probe = p.get();
                if (!probe && static_cast<int>(s->slots.size()) < s->opt.max_slots) probe = &new_slot(s);
                if (!probe) return;
                slot_handle(s, *probe, key);
                kv = s->key_volume.find(key);
            }
            const size_t volume = kv->second;
            if (volume > s->opt.volume_budget_bytes) {
                {
                    std::lock_guard<std::mutex> lk(s->m);
                    s->pending.pop_front();
                    --s->stats.pending;
                }
                push_completion(s, job, DS_INVALID_ARGUMENT, 0.0,
                                "frame needs " + std::to_string(volume) + " bytes of volume memory, above the budget of " +
                                    std::to_string(s->opt.volume_budget_bytes));
                continue;
            }
            sl = pick_slot(s, volume);
            if (!sl) return;  // wait for running frames to finish
            ds_handle* h = slot_handle(s, *sl, key);
            job.volume = volume;
            job.t_admit = Clock::now();
            sl->job = job;
            sl->busy = true;
            {
                std::lock_guard<std::mutex> lk(s->m);
                s->pending.pop_front();
                --s->stats.pending;
                ++s->stats.running;
                s->stats.peak_running = std::max(s->stats.peak_running, s->stats.running);
                s->stats.running_volume_bytes += volume;
                s->stats.peak_running_volume_bytes = std::max(s->stats.peak_running_volume_bytes, s->stats.running_volume_bytes);
            }
            launch(s, *sl, h, c);
        } catch (const Failure& f) {
            if (sl && sl->busy) {
                // The slot's stream may hold part of the frame: wait for it before reusing the slot.
                cudaStreamSynchronize(sl->st);
                sl->busy = false;
                std::lock_guard<std::mutex> lk(s->m);
                --s->stats.running;
                s->stats.running_volume_bytes -= job.volume;
            } else {
                std::lock_guard<std::mutex> lk(s->m);
                if (!s->pending.empty() && s->pending.front().ticket == job.ticket) {
                    s->pending.pop_front();
                    --s->stats.pending;
                }
            }
            push_completion(s, job, f.code, 0.0, f.what);
        }
    }
}

void complete(ds_server* s, Slot& sl) {
    float ms = 0.0f;
    const cudaError_t e = cudaEventElapsedTime(&ms, sl.ev0, sl.ev1);
    const Job job = sl.job;
    sl.busy = false;
    {
        std::lock_guard<std::mutex> lk(s->m);
        --s->stats.running;
        s->stats.running_volume_bytes -= job.volume;
    }
    if (e != cudaSuccess)
        push_completion(s, job, DS_IO, 0.0, std::string("frame failed on the device: ") + cudaGetErrorString(e));
    else
        push_completion(s, job, DS_OK, ms, "");
}

void worker_main(ds_server* s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<int> fin;
        {
            std::unique_lock<std::mutex> lk(s->m);
            s->cv_work.wait(lk, [&] { return s->stop || !s->finished.empty() || (s->dirty && !s->pending.empty()); });
            if (s->stop) break;
            fin.swap(s->finished);
            s->dirty = false;
        }
        for (int i : fin) complete(s, *s->slots[i]);
        admit(s);
    }
    // Shutdown: let the frames on the GPU finish, then report them.
    for (auto& p : s->slots)
        if (p->busy) cudaStreamSynchronize(p->st);
    std::vector<int> fin;
    {
        std::lock_guard<std::mutex> lk(s->m);
        fin.swap(s->finished);
    }
    for (int i : fin)
        if (s->slots[i]->busy) complete(s, *s->slots[i]);
}

void release_server(ds_server* s) {
    for (auto& p : s->slots) {
        if (p->st) cudaStreamSynchronize(p->st);
        for (auto& kv : p->handles) ds_destroy(kv.second);
        if (p->volume) cudaFreeAsync(p->volume, p->st);
        if (p->st) {
            cudaStreamSynchronize(p->st);
            cudaStreamDestroy(p->st);
        }
        if (p->ev0) cudaEventDestroy(p->ev0);
        if (p->ev1) cudaEventDestroy(p->ev1);
    }
    s->slots.clear();
    for (auto& kv : s->calib)
        for (auto* m : kv.second.map)
            if (m) cudaFree(m);
    s->calib.clear();
}

}  // namespace

extern "C" {

DS_API int ds_server_create(const ds_server_options* options, ds_server** out) {
    if (!out) return DS_INVALID_ARGUMENT;
    *out = nullptr;
    auto* s = new (std::nothrow) ds_server();
    if (!s) return DS_IO;
    if (options) s->opt = *options;
    if (s->opt.volume_budget_bytes == 0) s->opt.volume_budget_bytes = kDefaultBudget;
    if (s->opt.max_slots <= 0) s->opt.max_slots = 8;
    s->opt.max_slots = std::min(s->opt.max_slots, 256);
    if (s->opt.max_pending <= 0) s->opt.max_pending = 4096;
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        ds::set_global_error("no usable CUDA device");
        delete s;
        return DS_IO;
    }
    try {
        s->worker = std::thread(worker_main, s);
    } catch (...) {
        ds::set_global_error("cannot start the server's worker thread");
        delete s;
        return DS_IO;
    }
    *out = s;
    return DS_OK;
}

DS_API void ds_server_destroy(ds_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    release_server(s);
    delete s;
}

DS_API const char* ds_server_last_error(const ds_server* s) {
    if (!s) return ds_last_global_error();
    return s->err.c_str();
}

DS_API int ds_server_add_calibration(ds_server* s, int calib, const float* lx, const float* ly, const float* rx,
                                     const float* ry, int map_w, int map_h, int raw_w, int raw_h, const ds_geometry* geometry,
                                     float min_depth, float max_depth) {
    if (!s) return DS_INVALID_ARGUMENT;
    if (calib < 0) {
        s->set_error("calibration index must be >= 0");
        return DS_INVALID_ARGUMENT;
    }
    if (!lx || !ly || !rx || !ry || map_w < 1 || map_h < 1 || raw_w < 2 || raw_h < 2 || raw_w > 16384 || raw_h > 16384) {
        s->set_error("invalid remap tables or raw size");
        return DS_INVALID_ARGUMENT;
    }
    // Replacing a calibration in use: wait until no frame is queued or running.
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(s->m);
            if (s->pending.empty() && s->stats.running == 0) break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    Calib c;
    c.present = true;
    c.map_w = map_w;
    c.map_h = map_h;
    c.raw_w = raw_w;
    c.raw_h = raw_h;
    const size_t n = static_cast<size_t>(map_w) * map_h;
    const float* src[4] = {lx, ly, rx, ry};
    for (int i = 0; i < 4; ++i) {
        if (cudaMalloc(&c.map[i], n * 4) != cudaSuccess || cudaMemcpy(c.map[i], src[i], n * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
            for (auto* p : c.map)
                if (p) cudaFree(p);
            s->set_error("cannot upload the remap tables");
            return DS_IO;
        }
    }
    if (geometry) {
        c.have_geom = true;
        c.geom = *geometry;
        c.min_depth = min_depth;
        c.max_depth = max_depth;
    }
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->calib.find(calib);
    if (it != s->calib.end())
        for (auto* p : it->second.map)
            if (p) cudaFree(p);
    s->calib[calib] = c;
    return DS_OK;
}

DS_API int ds_server_reserve(ds_server* s, int width, int height, const ds_stereo_params* params, int calib, int count) {
    if (!s || !params || count < 0) return DS_INVALID_ARGUMENT;
    std::string msg;
    if (const int rc = ds::validate_params(*params, width, height, msg); rc != DS_OK) {
        s->set_error(msg);
        return rc;
    }
    // The worker owns the slots while frames are queued or running: wait until it is idle, then keep
    // it from admitting while this call sizes the slots.
    Calib c;
    for (;;) {
        {
            std::lock_guard<std::mutex> lk(s->m);
            if (calib >= 0 && !s->calib.count(calib)) {
                s->err = "unknown calibration";
                return DS_INVALID_ARGUMENT;
            }
            if (s->pending.empty() && s->stats.running == 0 && !s->configuring) {
                s->configuring = true;
                if (calib >= 0) c = s->calib.at(calib);
                break;
            }
        }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    int result = DS_OK;
    try {
        const ShapeKey key = key_of(width, height, *params);
        count = std::min(count, s->opt.max_slots);
        while (static_cast<int>(s->slots.size()) < count) new_slot(s);
        for (int i = 0; i < count; ++i) {
            Slot& sl = *s->slots[i];
            ds_handle* h = slot_handle(s, sl, key);
            if (calib >= 0) {
                const int rc = ds::bind_rectification(h, c.map, c.map_w, c.map_h, c.raw_w, c.raw_h);
                if (rc != DS_OK) throw Failure{rc, ds_last_error(h)};
            }
            const size_t v = s->key_volume[key];
            if (sl.volume_cap < v) {
                if (s->volume_total - sl.volume_cap + v > s->opt.volume_budget_bytes) break;
                set_volume(s, sl, v);
            }
        }
        for (auto& p : s->slots) check_cuda(cudaStreamSynchronize(p->st), "cudaStreamSynchronize");
    } catch (const Failure& f) {
        s->set_error(f.what);
        result = f.code;
    }
    std::lock_guard<std::mutex> lk(s->m);
    s->configuring = false;
    s->dirty = true;
    s->cv_work.notify_one();
    return result;
}

DS_API int ds_server_submit(ds_server* s, const ds_request* r, uint64_t* ticket) {
    if (!s || !r) return DS_INVALID_ARGUMENT;
    std::string msg;
    if (const int rc = ds::validate_params(r->params, r->width, r->height, msg); rc != DS_OK) {
        s->set_error(msg);
        return rc;
    }
    if (!r->left || !r->right) {
        s->set_error("null image");
        return DS_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(s->m);
    int iw = r->width;
    if (r->calib >= 0) {
        auto it = s->calib.find(r->calib);
        if (it == s->calib.end()) {
            s->err = "unknown calibration " + std::to_string(r->calib);
            return DS_INVALID_ARGUMENT;
        }
        const Calib& c = it->second;
        const bool same = c.map_w == r->width && c.map_h == r->height;
        const bool twice = c.map_w == 2 * r->width && c.map_h == 2 * r->height;
        if (!same && !twice) {
            s->err = "calibration remap size does not match the frame size";
            return DS_INVALID_ARGUMENT;
        }
        if (r->out.depth && !c.have_geom) {
            s->err = "depth needs a calibration with geometry";
            return DS_INVALID_ARGUMENT;
        }
        iw = c.raw_w;
    } else if (r->out.depth) {
        s->err = "depth needs a calibration with geometry";
        return DS_INVALID_ARGUMENT;
    }
    if (r->stride < iw) {
        s->err = "stride smaller than the image width";
        return DS_INVALID_ARGUMENT;
    }
    if (static_cast<int>(s->pending.size()) >= s->opt.max_pending) {
        s->err = "too many pending frames";
        return DS_BUSY;
    }
    Job j;
    j.ticket = s->next_ticket++;
    j.r = *r;
    j.t_submit = Clock::now();
    s->pending.push_back(j);
    ++s->stats.submitted;
    ++s->stats.pending;
    s->dirty = true;
    s->cv_work.notify_one();
    if (ticket) *ticket = j.ticket;
    return DS_OK;
}

DS_API int ds_server_poll(ds_server* s, ds_completion* out, int max, int* n, int timeout_ms) {
    if (!s || (!out && max > 0) || !n) return DS_INVALID_ARGUMENT;
    *n = 0;
    std::unique_lock<std::mutex> lk(s->m);
    auto ready = [&] { return !s->done.empty(); };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (timeout_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    while (*n < max && !s->done.empty()) {
        out[(*n)++] = s->done.front();
        s->done.pop_front();
    }
    return DS_OK;
}

DS_API int ds_server_get_stats(ds_server* s, ds_server_stats* out) {
    if (!s || !out) return DS_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->m);
    *out = s->stats;
    out->slots = static_cast<int>(s->slots.size());
    out->volume_bytes = s->volume_total;
    size_t maps = 0;
    for (auto& kv : s->calib) maps += static_cast<size_t>(kv.second.map_w) * kv.second.map_h * 16;
    out->device_bytes = s->volume_total + s->handle_bytes + maps;
    return DS_OK;
}

}  // extern "C"

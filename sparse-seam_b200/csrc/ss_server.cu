// ss_server.cu -- continuous-batching request loop over the batch route.
//
// One worker thread per server drives four steps in a loop:
//   admit     waiting requests, in arrival order, get image + mask buffers
//             from the device pool (first fit; the head waits when it does
//             not fit yet, so large requests are not starved) and their
//             image copy is enqueued on the copy stream;
//   launch    whenever a batch slot is free, every admitted request not yet
//             launched (up to the slot's image and tile capacity) becomes one
//             batch: plan filled on the host, the slot's stream waits for the
//             copies, the plan is copied in, the route is enqueued, then the
//             masks come back (as bit planes expanded by host threads in a
//             stream-ordered host function when the host masks are unpadded,
//             else as byte copies) and the batch's device status is read back
//             into pinned memory;
//   complete  slots whose last event has fired hand their requests back as
//             completions and return their pool memory;
//   wait      with batches on the device the worker spins (yielding); with
//             nothing to do it sleeps until the next submit.
// Batches of different slots run concurrently on the device (one stream per
// slot), so a request arriving while a batch runs is launched in the next
// batch as soon as a slot frees, without waiting for the first to finish.
//
// No counterpart in the reference, whose harness runs one image per call
// (harness/primary/gpu_common_v0_6.cu:137-206).
#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "sparse_seam.h"
#include "ss_device.cuh"
#include "ss_internal.h"
#include "ss_pool.hpp"

namespace ss {
namespace serve {

static int64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return static_cast<int64_t>(ts.tv_sec) * 1000000000ll + ts.tv_nsec;
}

struct Req {
    uint64_t ticket = 0;
    ss_request r{};
    int64_t submit_ns = 0, admit_ns = 0, launch_ns = 0;
    int64_t tiles = 0;
    bool pooled = false;
    size_t pool_off = 0, pool_bytes = 0;
    const uint8_t* d_img = nullptr;
    uint8_t* d_max = nullptr;
    uint8_t* d_min = nullptr;
    uint32_t* d_bits = nullptr;   // compact read-back: two bit planes
    int32_t d_pitch = 0, d_out_pitch = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t copies_in = nullptr;
    cudaEvent_t done = nullptr;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    void* d_plan = nullptr;
    void* h_plan = nullptr;
    size_t plan_cap = 0;
    Header* h_header = nullptr;   // pinned copy of the status words
    uint32_t* h_bits = nullptr;   // pinned staging of the bit planes
    size_t bits_cap = 0;          // in 32-bit words
    std::vector<Req> reqs;
    bool busy = false;
};

}  // namespace serve
}  // namespace ss

using ss::serve::Req;
using ss::serve::Slot;
using ss::serve::now_ns;

struct ss_server {
    ss_server_config cfg{};
    ss::OffsetPool pool{0};
    uint8_t* d_pool = nullptr;
    cudaStream_t copy_stream = nullptr;
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_submit;
    std::condition_variable cv_done;
    std::deque<Req> submitted;             // guarded by mu
    std::deque<ss_completion> completions; // guarded by mu
    bool stop = false;                     // guarded by mu
    uint64_t next_ticket = 1;              // guarded by mu
    ss_server_stats stats{};               // guarded by mu

    int unpack_threads = 1;                // resolved from the config

    // Worker-only state.
    std::deque<Req> waiting;
    std::deque<Req> admitted;
    std::thread worker;

    ~ss_server() = default;
};

namespace {

int64_t tiles_of(int w, int h, int t) {
    return static_cast<int64_t>((w + t - 1) / t) *
           static_cast<int64_t>((h + t - 1) / t);
}

// Pool bytes of a host request: image and two masks, plus the two bit
// planes of the compact read-back when it applies.
size_t plane_bytes(const ss_request& r) {
    return ss::OffsetPool::round(static_cast<size_t>(r.width) *
                                 static_cast<size_t>(r.height));
}

size_t bit_words(const ss_request& r) {
    return (static_cast<size_t>(r.width) * static_cast<size_t>(r.height) +
            31) / 32;
}

// Requests from this size on come back as bit planes: below it the byte
// copies are shorter than the hand-off to the host function that expands
// the planes (a few hundred microseconds).
constexpr uint64_t kCompactMinPixels = 8ull << 20;

bool compact_readback(const ss_server_config& c, const ss_request& r) {
    return c.unpack_threads >= 0 && !(r.flags & SS_REQUEST_DEVICE) &&
           r.out_pitch == r.width &&
           static_cast<uint64_t>(r.width) * static_cast<uint64_t>(r.height) >=
               kCompactMinPixels;
}

size_t footprint(const ss_server_config& c, const ss_request& r) {
    if (r.flags & SS_REQUEST_DEVICE) {
        return 0;
    }
    size_t bytes = 3 * plane_bytes(r);
    if (compact_readback(c, r)) {
        bytes += ss::OffsetPool::round(2 * 4 * bit_words(r));
    }
    return bytes;
}

void finish(ss_server* s, Slot& slot, ss_status status) {
    const int64_t t = now_ns();
    std::vector<ss_completion> out;
    out.reserve(slot.reqs.size());
    uint64_t pixels = 0;
    for (const Req& q : slot.reqs) {
        ss_completion c{};
        c.ticket = q.ticket;
        c.user = q.r.user;
        c.status = status;
        c.batch_images = static_cast<int32_t>(slot.reqs.size());
        c.submit_ns = q.submit_ns;
        c.admit_ns = q.admit_ns;
        c.launch_ns = q.launch_ns;
        c.done_ns = t;
        out.push_back(c);
        pixels += static_cast<uint64_t>(q.r.width) *
                  static_cast<uint64_t>(q.r.height);
        if (q.pooled) {
            s->pool.release(q.pool_off, q.pool_bytes);
        }
    }
    slot.reqs.clear();
    slot.busy = false;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (const ss_completion& c : out) {
            s->completions.push_back(c);
        }
        s->stats.completed += out.size();
        s->stats.pixels += pixels;
    }
    s->cv_done.notify_all();
}

// Waiting -> admitted: pool memory and the image copy.
bool admit(ss_server* s) {
    bool progress = false;
    while (!s->waiting.empty()) {
        Req& q = s->waiting.front();
        if (q.r.flags & SS_REQUEST_DEVICE) {
            q.d_img = q.r.image;
            q.d_max = q.r.maxima;
            q.d_min = q.r.minima;
            q.d_pitch = q.r.pitch;
            q.d_out_pitch = q.r.out_pitch;
        } else {
            const size_t bytes = footprint(s->cfg, q.r);
            size_t off = 0;
            if (!s->pool.alloc(bytes, &off)) {
                break;   // the head waits for memory; arrival order is kept
            }
            const size_t plane = plane_bytes(q.r);
            q.pooled = true;
            q.pool_off = off;
            q.pool_bytes = bytes;
            uint8_t* base = s->d_pool + off;
            q.d_img = base;
            q.d_max = base + plane;
            q.d_min = base + 2 * plane;
            q.d_bits = compact_readback(s->cfg, q.r)
                           ? reinterpret_cast<uint32_t*>(base + 3 * plane)
                           : nullptr;
            q.d_pitch = q.r.width;
            q.d_out_pitch = q.r.width;
            cudaMemcpy2DAsync(base, q.r.width, q.r.image, q.r.pitch,
                              q.r.width, q.r.height, cudaMemcpyHostToDevice,
                              s->copy_stream);
            std::lock_guard<std::mutex> lock(s->mu);
            s->stats.pool_high_water =
                std::max<uint64_t>(s->stats.pool_high_water,
                                   s->pool.used_bytes());
        }
        q.admit_ns = now_ns();
        s->admitted.push_back(q);
        s->waiting.pop_front();
        progress = true;
    }
    return progress;
}

// Admitted -> one batch per free slot.
bool launch(ss_server* s) {
    bool progress = false;
    for (Slot& slot : s->slots) {
        if (s->admitted.empty()) {
            break;
        }
        if (slot.busy) {
            continue;
        }
        std::vector<ss_image_desc> descs;
        int64_t tiles = 0;
        size_t words = 0;
        while (!s->admitted.empty() &&
               static_cast<int>(slot.reqs.size()) < s->cfg.max_batch_images) {
            const Req q = s->admitted.front();
            const size_t w = q.d_bits ? bit_words(q.r) : 0;
            if (tiles + q.tiles > s->cfg.batch_tiles ||
                2 * (words + w) > slot.bits_cap) {
                break;
            }
            tiles += q.tiles;
            words += w;
            slot.reqs.push_back(q);
            s->admitted.pop_front();
            ss_image_desc d{};
            d.image = q.d_img;
            d.maxima = q.d_max;
            d.minima = q.d_min;
            d.width = q.r.width;
            d.height = q.r.height;
            d.pitch = q.d_pitch;
            d.out_pitch = q.d_out_pitch;
            descs.push_back(d);
        }
        if (slot.reqs.empty()) {
            continue;
        }
        slot.busy = true;
        progress = true;
        size_t plan_bytes = 0;
        size_t ws_need = 0;
        ss_status st = ss_batch_plan_bytes(static_cast<int>(descs.size()),
                                           tiles, &plan_bytes);
        if (st == SS_OK && plan_bytes > slot.plan_cap) {
            st = SS_ERR_TOO_LARGE;
        }
        if (st == SS_OK) {
            st = ss_batch_plan_fill(descs.data(), static_cast<int>(descs.size()),
                                    s->cfg.tile, slot.h_plan, plan_bytes,
                                    &ws_need);
        }
        if (st == SS_OK && ws_need > slot.ws_bytes) {
            st = SS_ERR_WORKSPACE_TOO_SMALL;
        }
        bool ok = st == SS_OK;
        ok = ok && cudaEventRecord(slot.copies_in, s->copy_stream) == cudaSuccess;
        ok = ok && cudaStreamWaitEvent(slot.stream, slot.copies_in, 0) ==
                       cudaSuccess;
        ok = ok && cudaMemcpyAsync(slot.d_plan, slot.h_plan, plan_bytes,
                                   cudaMemcpyHostToDevice, slot.stream) ==
                       cudaSuccess;
        if (ok) {
            ss_launch l{};
            l.persistent = s->cfg.persistent;
            st = ss_extrema_batch_launch(slot.h_plan, slot.d_plan, plan_bytes,
                                         &l, slot.ws, slot.ws_bytes,
                                         slot.stream);
            ok = st == SS_OK;
        } else if (st == SS_OK) {
            st = SS_ERR_CUDA;
        }
        const int64_t t = now_ns();
        size_t staged = 0;   // words of the slot's bit-plane staging used
        for (Req& q : slot.reqs) {
            q.launch_ns = t;
            if (!ok || (q.r.flags & SS_REQUEST_DEVICE)) {
                continue;
            }
            if (q.d_bits) {
                // Compact read-back: pack on the device, copy the planes,
                // expand them into the caller's masks on the host.
                const uint64_t n = static_cast<uint64_t>(q.r.width) *
                                   static_cast<uint64_t>(q.r.height);
                const size_t w = bit_words(q.r);
                uint32_t* hb = slot.h_bits + staged;
                staged += 2 * w;
                ok = ss_pack_masks(q.d_max, q.d_min, n, q.d_bits,
                                   q.d_bits + w, slot.stream) == SS_OK &&
                     cudaMemcpyAsync(hb, q.d_bits, 2 * 4 * w,
                                     cudaMemcpyDeviceToHost,
                                     slot.stream) == cudaSuccess &&
                     ss_enqueue_unpack_masks(hb, hb + w, n, q.r.maxima,
                                             q.r.minima, s->unpack_threads,
                                             slot.stream) == SS_OK;
            } else {
                ok = cudaMemcpy2DAsync(q.r.maxima, q.r.out_pitch, q.d_max,
                                       q.d_out_pitch, q.r.width, q.r.height,
                                       cudaMemcpyDeviceToHost,
                                       slot.stream) == cudaSuccess &&
                     cudaMemcpy2DAsync(q.r.minima, q.r.out_pitch, q.d_min,
                                       q.d_out_pitch, q.r.width, q.r.height,
                                       cudaMemcpyDeviceToHost,
                                       slot.stream) == cudaSuccess;
            }
            if (!ok && st == SS_OK) {
                st = SS_ERR_CUDA;
            }
        }
        // The batch's status words, then a clean error word for the next use.
        ok = ok && cudaMemcpyAsync(slot.h_header, slot.ws, 16,
                                   cudaMemcpyDeviceToHost, slot.stream) ==
                       cudaSuccess;
        ok = ok && cudaMemsetAsync(static_cast<char*>(slot.ws) +
                                       offsetof(ss::Header, error),
                                   0, 2 * sizeof(uint32_t), slot.stream) ==
                       cudaSuccess;
        ok = ok && cudaEventRecord(slot.done, slot.stream) == cudaSuccess;
        if (!ok) {
            // Nothing of this batch may still read or write its buffers when
            // their memory is handed back.
            cudaStreamSynchronize(slot.stream);
            finish(s, slot, st == SS_OK ? SS_ERR_CUDA : st);
            continue;
        }
        std::lock_guard<std::mutex> lock(s->mu);
        s->stats.batches += 1;
        s->stats.max_batch_images_seen = std::max<uint32_t>(
            s->stats.max_batch_images_seen,
            static_cast<uint32_t>(slot.reqs.size()));
        uint32_t busy = 0;
        for (const Slot& o : s->slots) {
            busy += o.busy ? 1u : 0u;
        }
        s->stats.inflight_high_water =
            std::max(s->stats.inflight_high_water, busy);
    }
    return progress;
}

bool complete(ss_server* s) {
    bool progress = false;
    for (Slot& slot : s->slots) {
        if (!slot.busy) {
            continue;
        }
        const cudaError_t e = cudaEventQuery(slot.done);
        if (e == cudaErrorNotReady) {
            continue;
        }
        ss_status st = SS_OK;
        if (e != cudaSuccess) {
            st = SS_ERR_CUDA;
        } else if (slot.h_header->magic != ss::kMagic) {
            st = SS_ERR_WORKSPACE_UNINITIALIZED;
        } else if (slot.h_header->error) {
            st = static_cast<ss_status>(slot.h_header->error);
        }
        finish(s, slot, st);
        progress = true;
    }
    return progress;
}

void worker_main(ss_server* s) {
    cudaSetDevice(s->cfg.device);
    for (;;) {
        bool busy_slots = false;
        for (const Slot& slot : s->slots) {
            busy_slots = busy_slots || slot.busy;
        }
        {
            std::unique_lock<std::mutex> lock(s->mu);
            while (!s->submitted.empty()) {
                s->waiting.push_back(s->submitted.front());
                s->submitted.pop_front();
            }
            const bool idle =
                s->waiting.empty() && s->admitted.empty() && !busy_slots;
            if (idle) {
                if (s->stop) {
                    return;
                }
                s->cv_submit.wait(lock, [s] {
                    return s->stop || !s->submitted.empty();
                });
                continue;
            }
        }
        bool progress = admit(s);
        progress = launch(s) || progress;
        progress = complete(s) || progress;
        if (!progress) {
            std::this_thread::yield();
        }
    }
}

void release_all(ss_server* s) {
    for (Slot& slot : s->slots) {
        if (slot.stream) cudaStreamSynchronize(slot.stream);
        if (slot.copies_in) cudaEventDestroy(slot.copies_in);
        if (slot.done) cudaEventDestroy(slot.done);
        if (slot.stream) cudaStreamDestroy(slot.stream);
        if (slot.ws) cudaFree(slot.ws);
        if (slot.d_plan) cudaFree(slot.d_plan);
        if (slot.h_plan) cudaFreeHost(slot.h_plan);
        if (slot.h_header) cudaFreeHost(slot.h_header);
        if (slot.h_bits) cudaFreeHost(slot.h_bits);
    }
    s->slots.clear();
    if (s->copy_stream) {
        cudaStreamSynchronize(s->copy_stream);
        cudaStreamDestroy(s->copy_stream);
    }
    if (s->d_pool) cudaFree(s->d_pool);
}

// Restores the calling thread's current device on scope exit.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(device);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

ss_status ss_server_create(const ss_server_config* config,
                           ss_server** server) {
    if (!config || !server) {
        return SS_ERR_INVALID_VALUE;
    }
    *server = nullptr;
    const ss_server_config c = *config;
    if (c.tile != 16 && c.tile != 32 && c.tile != 64) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    if (c.device < 0 || c.inflight < 1 || c.inflight > 16 ||
        c.max_batch_images < 1 || c.max_batch_images > (1 << 20) ||
        c.batch_tiles < 1 || c.unpack_threads < -1) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t ws_bytes = 0;
    size_t plan_cap = 0;
    if (!ss::workspace_bytes_for_tiles(c.batch_tiles, c.tile, &ws_bytes) ||
        ss_batch_plan_bytes(c.max_batch_images, c.batch_tiles, &plan_cap) !=
            SS_OK) {
        return SS_ERR_TOO_LARGE;
    }
    ss_server* s = new (std::nothrow) ss_server();
    if (!s) {
        return SS_ERR_HOST_ALLOC;
    }
    s->cfg = c;
    if (c.unpack_threads > 0) {
        s->unpack_threads = c.unpack_threads;
    } else {
        const unsigned hw = std::thread::hardware_concurrency();
        s->unpack_threads = hw > 3 ? static_cast<int>(hw / 2) : 1;
    }
    // Bit-plane staging per slot: two planes for the largest batch.
    const size_t batch_pixels =
        static_cast<size_t>(c.batch_tiles) * c.tile * c.tile;
    const size_t bits_cap =
        c.unpack_threads >= 0 ? 2 * ((batch_pixels + 31) / 32 + 32 *
                                     static_cast<size_t>(c.max_batch_images))
                              : 0;
    DeviceScope scope(c.device);
    bool ok = cudaStreamCreateWithFlags(&s->copy_stream,
                                        cudaStreamNonBlocking) == cudaSuccess;
    if (ok && c.pool_bytes) {
        ok = cudaMalloc(&s->d_pool, c.pool_bytes) == cudaSuccess;
        s->pool = ss::OffsetPool(c.pool_bytes);
    }
    s->slots.resize(static_cast<size_t>(c.inflight));
    for (Slot& slot : s->slots) {
        if (!ok) break;
        slot.ws_bytes = ws_bytes;
        slot.plan_cap = plan_cap;
        slot.bits_cap = bits_cap;
        if (bits_cap) {
            ok = cudaMallocHost(reinterpret_cast<void**>(&slot.h_bits),
                                bits_cap * 4) == cudaSuccess;
        }
        ok = cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking) ==
                 cudaSuccess &&
             cudaEventCreateWithFlags(&slot.copies_in,
                                      cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) ==
                 cudaSuccess &&
             cudaMalloc(&slot.ws, ws_bytes) == cudaSuccess &&
             cudaMalloc(&slot.d_plan, plan_cap) == cudaSuccess &&
             cudaMallocHost(&slot.h_plan, plan_cap) == cudaSuccess &&
             cudaMallocHost(reinterpret_cast<void**>(&slot.h_header),
                            sizeof(ss::Header)) == cudaSuccess;
        ok = ok && ss_workspace_init(slot.ws, ws_bytes, slot.stream) == SS_OK;
    }
    if (ok) {
        for (Slot& slot : s->slots) {
            ok = ok && cudaStreamSynchronize(slot.stream) == cudaSuccess;
        }
    }
    if (!ok) {
        release_all(s);
        delete s;
        return SS_ERR_CUDA;
    }
    s->stats.pool_bytes = s->pool.capacity();
    s->worker = std::thread(worker_main, s);
    *server = s;
    return SS_OK;
}

ss_status ss_server_submit(ss_server* server, const ss_request* request,
                           uint64_t* ticket) {
    if (!server || !request) {
        return SS_ERR_INVALID_VALUE;
    }
    const ss_request& r = *request;
    if (!r.image || !r.maxima || !r.minima || r.width < 1 || r.height < 1 ||
        r.pitch < r.width || r.out_pitch < r.width ||
        (r.flags & ~SS_REQUEST_DEVICE) != 0) {
        return SS_ERR_INVALID_VALUE;
    }
    const int64_t tiles = tiles_of(r.width, r.height, server->cfg.tile);
    if (tiles > server->cfg.batch_tiles ||
        footprint(server->cfg, r) > server->pool.capacity()) {
        return SS_ERR_TOO_LARGE;
    }
    Req q;
    q.r = r;
    q.tiles = tiles;
    q.submit_ns = now_ns();
    {
        std::lock_guard<std::mutex> lock(server->mu);
        if (server->stop) {
            return SS_ERR_INVALID_VALUE;
        }
        q.ticket = server->next_ticket++;
        server->submitted.push_back(q);
        server->stats.submitted += 1;
    }
    server->cv_submit.notify_one();
    if (ticket) {
        *ticket = q.ticket;
    }
    return SS_OK;
}

ss_status ss_server_poll(ss_server* server, ss_completion* out, int capacity,
                         int* count, int timeout_us) {
    if (!server || !out || capacity < 1 || !count || timeout_us < 0) {
        return SS_ERR_INVALID_VALUE;
    }
    std::unique_lock<std::mutex> lock(server->mu);
    if (server->completions.empty() && timeout_us > 0) {
        server->cv_done.wait_for(lock, std::chrono::microseconds(timeout_us),
                                 [server] {
                                     return !server->completions.empty();
                                 });
    }
    int n = 0;
    while (n < capacity && !server->completions.empty()) {
        out[n++] = server->completions.front();
        server->completions.pop_front();
    }
    *count = n;
    return SS_OK;
}

ss_status ss_server_get_stats(ss_server* server, ss_server_stats* stats) {
    if (!server || !stats) {
        return SS_ERR_INVALID_VALUE;
    }
    std::lock_guard<std::mutex> lock(server->mu);
    *stats = server->stats;
    return SS_OK;
}

void ss_server_destroy(ss_server* server) {
    if (!server) {
        return;
    }
    {
        std::lock_guard<std::mutex> lock(server->mu);
        server->stop = true;
    }
    server->cv_submit.notify_all();
    if (server->worker.joinable()) {
        server->worker.join();
    }
    DeviceScope scope(server->cfg.device);
    release_all(server);
    delete server;
}

}  // extern "C"

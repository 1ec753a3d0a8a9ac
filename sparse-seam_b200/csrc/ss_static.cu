// ss_static.cu -- the zero-allocation form of the route.
//
// Some callers cannot allocate device memory: code that runs where the
// allocator must not be entered (inside another allocator's callback, a
// latency-critical loop that may not block on cudaMalloc), or a plug-in whose
// host owns every device allocation.  For them the route's scratch lives in a
// fixed array of this translation unit instead of a caller-provided
// workspace.  The array sits in its own module, so the driver creates it only
// on GPUs where this entry point (or its status read-back) was called, and
// keeps it there until the process exits.
//
// The array's name is a host-side stand-in in host code, not a device
// address; its address is looked up with cudaGetSymbolAddress in the CUDA
// context that is current, and the one-time set-up (a full clear and the
// status header) is done once per context.  No counterpart in the reference,
// which allocates its buffers per image.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "sparse_seam.h"
#include "ss_device.cuh"
#include "ss_internal.h"

namespace {

constexpr size_t kStaticScratchBytes = static_cast<size_t>(32) << 20;
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// cuCtxGetCurrent, found through the runtime so the library needs no link
// against the driver library (CUresult cuCtxGetCurrent(CUcontext*)).
using CtxGetCurrent = int (*)(void**);

CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault,
                                    &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            p = nullptr;
        }
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    return fn;
}

// Contexts whose array has been set up, with the array's address there.
struct Ready {
    void* context;
    int device;
    void* address;
};
constexpr int kMaxContexts = 64;
std::mutex g_mutex;
Ready g_ready[kMaxContexts] = {};

// The current context (falls back to the device ordinal as the key if the
// driver entry point is unavailable) and the array's address in it.
ss_status current(void** context, int* device, void** address) {
    if (cudaGetDevice(device) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    *context = nullptr;
    if (CtxGetCurrent fn = ctx_get_current()) {
        if (fn(context) != 0) {
            return SS_ERR_CUDA;
        }
    }
    *address = nullptr;
    if (cudaGetSymbolAddress(address, g_static_scratch) != cudaSuccess ||
        !*address) {
        return SS_ERR_CUDA;
    }
    return SS_OK;
}

Ready* find_ready(void* context, int device) {
    for (Ready& r : g_ready) {
        if (r.address && r.context == context && r.device == device) {
            return &r;
        }
    }
    return nullptr;
}

}  // namespace

extern "C" {

ss_status ss_extrema_static_scratch(const uint8_t* d_image, int width,
                                    int height, int pitch, int tile,
                                    uint8_t* d_maxima, uint8_t* d_minima,
                                    int out_pitch, void* stream) {
    if (!d_image || !d_maxima || !d_minima || width <= 0 || height <= 0 ||
        pitch < width || out_pitch < width) {
        return SS_ERR_INVALID_VALUE;
    }
    if (tile != 16 && tile != 32 && tile != 64) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    const int64_t tiles =
        static_cast<int64_t>((width + tile - 1) / tile) *
        static_cast<int64_t>((height + tile - 1) / tile);
    size_t needed = 0;
    if (!ss::workspace_bytes_for_tiles(tiles, tile, &needed)) {
        return SS_ERR_TOO_LARGE;
    }
    if (needed > kStaticScratchBytes) {
        return SS_ERR_EXCEEDS_STATIC_SCRATCH;
    }
    void* context = nullptr;
    int device = 0;
    void* scratch = nullptr;
    ss_status st = current(&context, &device, &scratch);
    if (st != SS_OK) {
        return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        Ready* r = find_ready(context, device);
        if (!r || r->address != scratch) {
            // First use in this context: a full clear and the status header,
            // waited for, so later calls on any stream see it.
            st = ss_workspace_init(scratch, kStaticScratchBytes, stream);
            if (st != SS_OK) {
                return st;
            }
            if (cudaStreamSynchronize(s) != cudaSuccess) {
                return SS_ERR_CUDA;
            }
            if (!r) {
                for (Ready& e : g_ready) {
                    if (!e.address) {
                        r = &e;
                        break;
                    }
                }
            }
            if (r) {
                *r = Ready{context, device, scratch};
            }
        }
    }
    // The array keeps the previous call's contents.  What this call needs at
    // zero: the error word and its detail, and the seam-pair counters of
    // this geometry (16 bytes per tile after the header).
    ss::Header* header = static_cast<ss::Header*>(scratch);
    if (cudaMemsetAsync(&header->error, 0, 2 * sizeof(uint32_t), s) !=
            cudaSuccess ||
        cudaMemsetAsync(static_cast<char*>(scratch) + sizeof(ss::Header), 0,
                        static_cast<size_t>(tiles) * 16, s) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    return ss_extrema(d_image, width, height, pitch, tile, d_maxima, d_minima,
                      out_pitch, scratch, kStaticScratchBytes, stream);
}

ss_status ss_static_scratch_read_status(void* stream, ss_stats* stats) {
    void* context = nullptr;
    int device = 0;
    void* scratch = nullptr;
    ss_status st = current(&context, &device, &scratch);
    if (st != SS_OK) {
        return st;
    }
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        Ready* r = find_ready(context, device);
        if (!r || r->address != scratch) {
            return SS_ERR_WORKSPACE_UNINITIALIZED;
        }
    }
    st = ss_read_status(scratch, kStaticScratchBytes, stream, stats);
    if (st == SS_ERR_WORKSPACE_UNINITIALIZED) {
        // The array lost its set-up (its context was replaced by one that
        // reuses the handle and the address): the next call sets it up.
        std::lock_guard<std::mutex> lock(g_mutex);
        if (Ready* r = find_ready(context, device)) {
            *r = Ready{};
        }
    }
    return st;
}

}  // extern "C"

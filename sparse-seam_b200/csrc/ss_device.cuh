// ss_device.cuh -- device-side building blocks of the exact dual
// regional-extrema route for sm_100a.
//
// Work unit: one T x T tile of one image (T = 16, 32 or 64), one CTA of NW
// warps.  A tile is staged with its one-pixel halo into shared memory and its
// equal-valued flat zones are labelled there; zones that stay inside the tile
// are final at once, zones that touch a tile seam become "fragments" in a
// global union-find arena, merged with the fragments of the neighbouring
// tiles and resolved by a second pass.
//
// Lane layout: pixel p = 32*c + lane of the tile (row-major) is handled by
// lane `lane` in chunk c, so one warp instruction covers 32 horizontally
// consecutive pixels and __ballot_sync turns a per-pixel predicate into a row
// bitmask.  Runs of equal pixels inside a row are read off those bitmasks, so
// the tile-local union-find works on runs, not pixels: each run is one node
// (indexed by its first pixel) and exactly one union is issued per pair of
// 8-adjacent equal runs in consecutive rows.
//
// Reference behaviour followed (paths inside the reference repository):
//   - zone flags HAS_GREATER / HAS_SMALLER / TOUCHES_SEAM and the seam test
//     "an equal 8-neighbour outside the tile":
//     harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:43-45, 340-390;
//   - seam fragments numbered per tile, at most 4T slots per tile:
//     snapshot_sparse_seam_cuda_v1_0.cu:40-42, 392-410;
//   - min-root lock-free union (links point to smaller indices):
//     snapshot_sparse_seam_cuda_v1_0.cu:105-160;
//   - cross-seam merging of equal 8-adjacent boundary pixels:
//     snapshot_sparse_seam_cuda_v1_0.cu:508-581;
//   - masks 255 where the resolved zone lacks the flag, else 0:
//     snapshot_sparse_seam_cuda_v1_0.cu:420-430, 502-505.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ss {

constexpr uint32_t kHasGreater = 1u;
constexpr uint32_t kHasSmaller = 2u;
constexpr uint32_t kTouchesSeam = 4u;
constexpr uint32_t kRecordShift = 8u;  // tile-local bits: (record + 1) << 8
constexpr uint32_t kLocalShift = 8u;   // arena bits: own flags << 8
constexpr uint32_t kMagic = 0x53534232u;  // "SSB2"

// Device error codes; the values are the matching ss_status codes.
constexpr uint32_t kErrFragmentOverflow = 7u;
constexpr uint32_t kErrRecordRange = 8u;
constexpr uint32_t kErrInvariant = 9u;
constexpr uint32_t kErrSpinLimit = 10u;
constexpr uint32_t kErrUninitialized = 11u;

// Seam relations of a tile, numbered by the neighbour they join it to.
constexpr int kRelLeft = 0, kRelTop = 1, kRelTopLeft = 2, kRelTopRight = 3,
              kRelRight = 4, kRelBottom = 5, kRelBottomRight = 6,
              kRelBottomLeft = 7;

// Workspace status header (first 256 bytes of every workspace).
struct Header {
    uint32_t magic;
    uint32_t error;          // first device error code, 0 if none
    uint32_t error_detail;
    uint32_t queue_head;     // persistent tile-pass work-queue cursor
    uint32_t resolve_head;   // persistent resolve-pass work-queue cursor
    uint32_t resolve_done;   // resolve CTAs finished in this call
    uint32_t flipped_tiles;  // tiles rewritten by the resolve pass
    uint32_t tile;           // tile edge of the last call
    uint64_t last_tiles;     // tiles of the last call
    uint32_t route;          // 1: the last call ran the row-scan kernels
    uint32_t pad;
    uint64_t reserved[26];
};
static_assert(sizeof(Header) == 256, "header is one 256-byte block");

// One image of a batch (also used, by value, for a single image).
struct __align__(16) PlanImage {
    const uint8_t* image;
    uint8_t* maxima;
    uint8_t* minima;
    int32_t width;
    int32_t height;
    int32_t pitch;
    int32_t out_pitch;
    int32_t tiles_x;
    int32_t tiles_y;
    int64_t tile_base;   // global index of the image's tile (0, 0)
    int32_t levels;      // re-quantise the pixels to this many gray levels
                         //   as they are loaded (2..255), 0 or 256: as is
};
static_assert(sizeof(PlanImage) == 64, "plan entries are 64 bytes");

// The reference's re-quantisation of an 8-bit value to `levels` gray levels
// (harness/quantization_and_scaling/gpu_common_quant_v0_7.cu:479-494):
// bin = (v * levels) >> 8, value = (bin * 255 + (levels - 1) / 2) /
// (levels - 1).
__host__ __device__ __forceinline__ int quantize_level(int v, int levels) {
    const int bin = (v * levels) >> 8;
    return (bin * 255 + (levels - 1) / 2) / (levels - 1);
}

__host__ __device__ __forceinline__ bool levels_active(int levels) {
    return levels >= 2 && levels < 256;
}

// Device plan of a batch: header, image table, tile -> image map.
struct __align__(16) PlanHeader {
    uint32_t magic;
    int32_t count;
    int32_t tile;
    int32_t reserved0;
    int64_t total_tiles;
    int64_t reserved1[5];
};
static_assert(sizeof(PlanHeader) == 64, "plan header is 64 bytes");

// Where a launch finds its (image, tile) work items.
struct Source {
    const PlanImage* images;     // batch image table, or nullptr
    const int32_t* tile_image;   // batch tile -> image map, or nullptr
    PlanImage single;            // the image when images == nullptr
    int64_t total_tiles;
    int32_t group;               // tiles per warp in the row-scan seam and
                                 //   resolve passes (power of two, 1..32)
    int32_t flatten;             // fragment forest flatten schedule of the
                                 //   row-scan flags pass (kFlatten*)
};

// Flatten schedules of the fragment union-find after the seam pass (the
// row-scan route): the flags pass finds each fragment's root with path
// halving (kFlattenHalve); or also points the fragment straight at its root
// (kFlattenCompress), so the resolve pass's finds take one step; or a
// separate pass first points every fragment at its root, as the
// reference's compress_fragment_parents does
// (harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:583-599), and the flags
// pass then finds roots in one step (kFlattenSeparate; one more launch).
constexpr int32_t kFlattenHalve = 0;
constexpr int32_t kFlattenCompress = 1;
constexpr int32_t kFlattenSeparate = 2;
constexpr int32_t kFlattenOnly = 3;      // the separate pass itself

// Device view of the workspace arrays (global tile index g, slot s).
struct Arena {
    Header* header;
    uint32_t* relation;      // [g * 4 + k]: right, bottom, bottom-right,
                             //              bottom-left seam-pair counters
    uint16_t* fragment_count;  // [g]
    uint8_t* border;         // [g * 4T + side * T + i]: fragment record of
                             //   seam-zone border pixels (top, bottom, left,
                             //   right)
    int32_t* parent;         // [g * 4T + record]: fragment union-find
    uint32_t* bits;          // [g * 4T + record]: bits 0-1 zone flags (the
                             //   component's at a root), bits 8-9 own flags
    uint32_t* pending_count; // [g]: run-log entries in bits 0-15, their
                             //   pixels in bits 16-31 (row-scan path)
    uint32_t* pending;       // [g * T * T + e]: run-log entries
    uint32_t* seam_count;    // [g]: seam items (row-scan path)
    uint32_t* seam_items;    // [g * 12T + i]: seam items (row-scan path)
};

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t bits_upto(int i) {
    // Bits 0..i inclusive, for 0 <= i <= 63.
    return (2ull << i) - 1ull;
}

__device__ __forceinline__ int high_bit(uint64_t x) {
    return 63 - __clzll(static_cast<long long>(x));
}

__device__ __forceinline__ int32_t ld_relaxed(const int32_t* p) {
    int32_t v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];"
                 : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];"
                 : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed(int32_t* p, int32_t v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;"
                 :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_cg_u8(const uint8_t* p) {
    return static_cast<uint32_t>(__ldcg(p));
}

__device__ __forceinline__ void raise_error(Header* h, uint32_t code,
                                            uint32_t detail) {
    if (atomicCAS(&h->error, 0u, code) == 0u) {
        atomicExch(&h->error_detail, detail);
    }
}

// ---------------------------------------------------------------------------
// Shared-memory union-find over tile-local pixel indices (run heads).
// Links always point to smaller indices, so a root is the smallest index of
// its set and the final labelling is deterministic.  Path halving writes only
// ancestors into non-root entries, which is safe under concurrent linking.
// ---------------------------------------------------------------------------

template <int BOUND>
__device__ __forceinline__ int smem_find(int32_t* parent_, int x,
                                         uint32_t& err) {
    volatile int32_t* parent = parent_;
#pragma unroll 1
    for (int it = 0; it < BOUND; ++it) {
        const int p = parent[x];
        if (p == x) {
            return x;
        }
        const int gp = parent[p];
        if (gp == p) {
            return p;
        }
        parent[x] = gp;
        x = gp;
    }
    err = kErrSpinLimit;
    return x;
}

template <int BOUND>
__device__ __forceinline__ void smem_union(int32_t* parent, int a, int b,
                                           uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < BOUND; ++it) {
        a = smem_find<BOUND>(parent, a, err);
        b = smem_find<BOUND>(parent, b, err);
        if (a == b || err) {
            return;
        }
        const int hi = a > b ? a : b;
        const int lo = a > b ? b : a;
        const int old = atomicCAS(&parent[hi], hi, lo);
        if (old == hi) {
            return;
        }
        a = old;
        b = lo;
    }
    err = kErrSpinLimit;
}

// ---------------------------------------------------------------------------
// Global fragment union-find with OR-propagated zone flags.
//
// bits[r] & 3 at a root r is the OR of the own flags of every fragment in its
// set once all unions are done.  Protocol (every step is an atomic or a
// relaxed access, separated by fence.sc):
//   link:  CAS parent[hi] hi -> lo; fence; read bits[hi]; OR them into lo.
//   or:    atomicOr bits[r]; fence; re-read parent[r]; if r is no longer a
//          root, continue at its new root.
// Store-buffering with SC fences on both sides means a flag ORed into a root
// concurrently with the root being linked is seen by the linker or sees the
// link, so it always reaches the final root.  A flag that was already present
// has its own propagator, so "already set" ends the walk.
// ---------------------------------------------------------------------------

constexpr int kGlobalBound = 1 << 22;

__device__ __forceinline__ int global_find(int32_t* parent, int x,
                                           uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < kGlobalBound; ++it) {
        const int p = ld_relaxed(parent + x);
        if (p == x) {
            return x;
        }
        if (p < 0 || p > x) {
            err = kErrInvariant;
            return x;
        }
        const int gp = ld_relaxed(parent + p);
        if (gp == p) {
            return p;
        }
        if (gp < 0 || gp > p) {
            err = kErrInvariant;
            return p;
        }
        st_relaxed(parent + x, gp);
        x = gp;
    }
    err = kErrSpinLimit;
    return x;
}

__device__ __forceinline__ void global_or(int32_t* parent, uint32_t* bits,
                                          int x, uint32_t flags,
                                          uint32_t& err) {
    int r = global_find(parent, x, err);
#pragma unroll 1
    for (int it = 0; it < kGlobalBound && !err; ++it) {
        const uint32_t old = atomicOr(bits + r, flags);
        if ((old & flags) == flags) {
            return;
        }
        __threadfence();
        const int p = ld_relaxed(parent + r);
        if (p == r) {
            return;
        }
        r = global_find(parent, p, err);
    }
    if (!err) {
        err = kErrSpinLimit;
    }
}

__device__ __forceinline__ void global_union(int32_t* parent, uint32_t* bits,
                                             int a, int b, uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < kGlobalBound; ++it) {
        a = global_find(parent, a, err);
        b = global_find(parent, b, err);
        if (a == b || err) {
            return;
        }
        const int hi = a > b ? a : b;
        const int lo = a > b ? b : a;
        const int old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) {
            __threadfence();
            const uint32_t flags = ld_relaxed(bits + hi) & 3u;
            if (flags) {
                global_or(parent, bits, lo, flags, err);
            }
            return;
        }
        a = old;
        b = lo;
    }
    err = kErrSpinLimit;
}

// Links the roots of a and b (larger below smaller) without merging flags:
// the row-scan route ORs every fragment's flags into its root in a later
// kernel, after all links are in place.
__device__ __forceinline__ void global_link(int32_t* parent, int a, int b,
                                            uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < kGlobalBound; ++it) {
        a = global_find(parent, a, err);
        b = global_find(parent, b, err);
        if (a == b || err) {
            return;
        }
        const int hi = a > b ? a : b;
        const int lo = a > b ? b : a;
        const int old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) {
            return;
        }
        a = old;
        b = lo;
    }
    err = kErrSpinLimit;
}

}  // namespace ss

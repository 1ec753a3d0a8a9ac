// ss_route.cu -- kernels and C ABI of the exact dual regional-extrema route.
//
// Two kernel families.  The row-scan family (the default at tile edges 32
// and 64; ss_runs.cuh, ss_rowscan.cuh) runs a tile pass, a seam pass, a
// flags pass and a resolve pass.  The CTA-per-tile family (the default at
// tile edge 16, selectable at every edge), defined below, runs two kernels
// per call, for one image or a whole batch:
//
//   tile pass    per (image, tile): label the tile, write both masks (final
//                for zones inside the tile, provisional -- from the tile's own
//                flags -- for seam zones), initialise the tile's seam
//                fragments in the global arena and publish their border
//                records.  Each pair of tiles joined by equal pixels across a
//                seam owns a counter; the second tile of the pair to arrive
//                (it reads 1) unites the pair's fragments, so no tile ever
//                waits for another.
//   resolve pass per tile with fragments: compare every fragment's own flags
//                with its component's; only if one differs, re-label the tile
//                (same deterministic numbering) and rewrite that fragment's
//                pixels.
//
// The kernel boundary is the only global barrier.  Every read of another
// tile's data goes through L2 (relaxed or .cg loads) after a fence-guarded
// counter handshake.  Both tiles of a pair see the same equal pixels across
// their seam (each has the other's border in its halo), so either both or
// neither touch the pair's counter; the resolve pass clears the counters, so
// they are zero between calls.
//
// Reference route replaced (paths inside the reference repository):
//   harness/primary/snapshot_sparse_seam_cuda_v1_0.cu:291-619 (five kernels)
//   harness/primary/gpu_common_v0_6.cu:137-206 (run_sparse_resident)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "sparse_seam.h"
#include "ss_internal.h"
#include "ss_rowscan.cuh"
#include "ss_runs.cuh"
#include "ss_tile.cuh"

namespace ss {

// ---------------------------------------------------------------------------
// Tile pass
// ---------------------------------------------------------------------------

template <int T, int NW>
__device__ __forceinline__ void relation_unions(TileWorker<T, NW>& w,
                                                const Arena& a,
                                                const PlanImage& job,
                                                int64_t g, int r,
                                                int64_t frag_base) {
    constexpr int kH = T + 2;
    constexpr int kSlots = 4 * T;
    TileSmem<T>& s = w.s;
    const int64_t tiles_x = job.tiles_x;
    int64_t ng;
    switch (r) {
        case kRelLeft: ng = g - 1; break;
        case kRelTop: ng = g - tiles_x; break;
        case kRelTopLeft: ng = g - tiles_x - 1; break;
        case kRelTopRight: ng = g - tiles_x + 1; break;
        case kRelRight: ng = g + 1; break;
        case kRelBottom: ng = g + tiles_x; break;
        case kRelBottomRight: ng = g + tiles_x + 1; break;
        default: ng = g + tiles_x - 1; break;
    }
    const uint8_t* nb = a.border + ng * kSlots;
    const int64_t nbase = ng * kSlots;
    auto pix = [&](int lx, int ly) -> int {
        return s.img[(ly + 1) * kH + lx + 1];
    };
    auto own_fragment = [&](int lx, int ly) -> int64_t {
        const uint32_t b = w.zone_word(lx, ly);
        const uint32_t rec1 = b >> kRecordShift;  // record + 1, 0 if none
        if (!(b & kTouchesSeam) || rec1 == 0u ||
            rec1 > static_cast<uint32_t>(kSlots)) {
            return -1;
        }
        return frag_base + static_cast<int64_t>(rec1) - 1;
    };
    auto link = [&](int64_t f, uint32_t rec) {
        if (rec >= static_cast<uint32_t>(kSlots)) {
            w.err = kErrRecordRange;
            return;
        }
        global_union(a.parent, a.bits, static_cast<int>(f),
                     static_cast<int>(nbase + rec), w.err);
    };

    if (r == kRelLeft || r == kRelRight) {
        const int ox = r == kRelLeft ? 0 : T - 1;
        const int nx = r == kRelLeft ? -1 : T;
        const int side = r == kRelLeft ? 3 : 2;  // neighbour's right / left
        for (int y = w.lane; y < w.th; y += 32) {
            const int v = pix(ox, y);
            int64_t f = -2;
            for (int d = -1; d <= 1; ++d) {
                const int y2 = y + d;
                if (y2 < 0 || y2 >= w.th || pix(nx, y2) != v) {
                    continue;
                }
                if (f == -2) {
                    f = own_fragment(ox, y);
                }
                if (f < 0) {
                    w.err = kErrInvariant;
                    break;
                }
                link(f, ld_cg_u8(nb + side * T + y2));
            }
        }
    } else if (r == kRelTop || r == kRelBottom) {
        const int oy = r == kRelTop ? 0 : T - 1;
        const int ny = r == kRelTop ? -1 : T;
        const int side = r == kRelTop ? 1 : 0;  // neighbour's bottom / top
        for (int x = w.lane; x < w.tw; x += 32) {
            const int v = pix(x, oy);
            int64_t f = -2;
            for (int d = -1; d <= 1; ++d) {
                const int x2 = x + d;
                if (x2 < 0 || x2 >= w.tw || pix(x2, ny) != v) {
                    continue;
                }
                if (f == -2) {
                    f = own_fragment(x, oy);
                }
                if (f < 0) {
                    w.err = kErrInvariant;
                    break;
                }
                link(f, ld_cg_u8(nb + side * T + x2));
            }
        }
    } else if (w.lane == 0) {
        int ox, oy, nx, ny, off;
        switch (r) {
            case kRelTopLeft:  // its bottom-right pixel
                ox = 0; oy = 0; nx = -1; ny = -1; off = T + (T - 1); break;
            case kRelTopRight:  // its bottom-left pixel
                ox = T - 1; oy = 0; nx = T; ny = -1; off = T; break;
            case kRelBottomRight:  // its top-left pixel
                ox = T - 1; oy = T - 1; nx = T; ny = T; off = 0; break;
            default:  // bottom-left: its top-right pixel
                ox = 0; oy = T - 1; nx = -1; ny = T; off = T - 1; break;
        }
        if (pix(ox, oy) == pix(nx, ny)) {
            const int64_t f = own_fragment(ox, oy);
            if (f < 0) {
                w.err = kErrInvariant;
            } else {
                link(f, ld_cg_u8(nb + off));
            }
        }
    }
}

template <int T, int NW>
__device__ __forceinline__ void tile_pass_item(TileSmem<T>& s,
                                               const Source& src,
                                               const Arena& a, int64_t item) {
    using W = TileWorker<T, NW>;
    W w(s);
    if (threadIdx.x == 0) {
        s.job = src.images ? src.images[src.tile_image[item]] : src.single;
    }
    __syncthreads();
    const PlanImage job = s.job;
    w.set_tile(job, item - job.tile_base);
    w.load(job);
    __syncthreads();
    w.predicates();
    __syncthreads();
    w.unions();
    __syncthreads();
    w.flatten();
    __syncthreads();
    const int64_t frag_base = item * W::kSlots;
    w.number(&a, frag_base);

    // Masks (provisional for seam zones) and border records.
    uint8_t* border = a.border + item * W::kSlots;
    const int64_t out_pitch = job.out_pitch;
#pragma unroll
    for (int k = 0; k < W::kPerWarp; ++k) {
        const uint32_t pr = w.pred[k];
        if (!(pr & 1u)) {
            continue;
        }
        const int p = W::chunk_of(k, w.warp) * 32 + w.lane;
        const int ly = p >> W::kLog;
        const int lx = p & (T - 1);
        const int head = static_cast<int>((pr >> 8) & 0xFFu);
        const uint32_t b = s.bits[s.parent[ly * T + head]];
        const int64_t o = (w.y0 + ly) * out_pitch + w.x0 + lx;
        job.maxima[o] = (b & kHasGreater) ? 0 : 255;
        job.minima[o] = (b & kHasSmaller) ? 0 : 255;
        if ((b & kTouchesSeam) && (b >> kRecordShift) != 0u) {
            const uint8_t rec = static_cast<uint8_t>((b >> kRecordShift) - 1);
            if (ly == 0) border[lx] = rec;
            if (ly == w.th - 1) border[T + lx] = rec;
            if (lx == 0) border[2 * T + ly] = rec;
            if (lx == w.tw - 1) border[3 * T + ly] = rec;
        }
    }
    if (threadIdx.x == 0) {
        a.fragment_count[item] = static_cast<uint16_t>(s.nfrag);
    }
    // Publish: every thread's arena / border writes, then the counters.
    __threadfence();
    __syncthreads();
    if (threadIdx.x < 8) {
        const int r = static_cast<int>(threadIdx.x);
        if ((s.relations >> r) & 1u) {
            const int64_t tiles_x = job.tiles_x;
            int64_t idx;
            switch (r) {
                case kRelLeft: idx = (item - 1) * 4 + 0; break;
                case kRelTop: idx = (item - tiles_x) * 4 + 1; break;
                case kRelTopLeft: idx = (item - tiles_x - 1) * 4 + 2; break;
                case kRelTopRight: idx = (item - tiles_x + 1) * 4 + 3; break;
                case kRelRight: idx = item * 4 + 0; break;
                case kRelBottom: idx = item * 4 + 1; break;
                case kRelBottomRight: idx = item * 4 + 2; break;
                default: idx = item * 4 + 3; break;
            }
            const uint32_t old = atomicAdd(a.relation + idx, 1u);
            if (old & 1u) {
                __threadfence();
                atomicOr(&s.second, 1u << r);
            }
        }
    }
    __syncthreads();
    const uint32_t second = s.second;
    if (second) {
        __threadfence();
        for (int r = w.warp; r < 8; r += NW) {
            if ((second >> r) & 1u) {
                relation_unions<T, NW>(w, a, job, item, r, frag_base);
            }
        }
    }
    if (w.err) {
        raise_error(a.header, w.err, static_cast<uint32_t>(item));
    }
}

template <int T, int NW, bool kPersistent>
__global__ void __launch_bounds__(NW * 32)
tile_pass_kernel(Source src, Arena a) {
    __shared__ TileSmem<T> s;
    if (a.header->magic != kMagic) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            raise_error(a.header, kErrUninitialized, 0u);
        }
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.header->last_tiles = static_cast<uint64_t>(src.total_tiles);
        a.header->tile = T;
        a.header->route = 0u;
    }
    if constexpr (kPersistent) {
        for (;;) {
            if (threadIdx.x == 0) {
                s.item = atomicAdd(&a.header->queue_head, 1u);
            }
            __syncthreads();
            const int64_t item = s.item;
            __syncthreads();
            if (item >= src.total_tiles) {
                break;
            }
            tile_pass_item<T, NW>(s, src, a, item);
            __syncthreads();
        }
    } else {
        tile_pass_item<T, NW>(s, src, a, blockIdx.x);
    }
}

// ---------------------------------------------------------------------------
// Resolve pass
// ---------------------------------------------------------------------------

template <int T, int NW>
__device__ __forceinline__ void resolve_item(TileSmem<T>& s,
                                             const Source& src,
                                             const Arena& a, int64_t item) {
    using W = TileWorker<T, NW>;
    // The tile pass is complete: clear this tile's seam-pair counters so
    // that every counter is zero again when the call ends.
    if (threadIdx.x < 4) {
        a.relation[item * 4 + threadIdx.x] = 0u;
    }
    const int count = a.fragment_count[item];
    if (count == 0) {
        return;
    }
    if (count > W::kSlots) {
        if (threadIdx.x == 0) {
            raise_error(a.header, kErrFragmentOverflow,
                        static_cast<uint32_t>(item));
        }
        return;
    }
    W w(s);
    const int64_t frag_base = item * W::kSlots;
    if (w.warp == 0) {
        bool any = false;
        for (int r = w.lane; r < count; r += 32) {
            const int f = static_cast<int>(frag_base + r);
            const int root = global_find(a.parent, f, w.err);
            const uint32_t component = ld_relaxed(a.bits + root) & 3u;
            const uint32_t own = (ld_relaxed(a.bits + f) >> kLocalShift) & 3u;
            const bool flip = component != own;
            s.flip[r] = flip ? 1 : 0;
            s.final_flags[r] = static_cast<uint8_t>(component);
            any |= flip;
            if (root != f) {
                st_relaxed(a.parent + f, root);
            }
        }
        any = __any_sync(~0u, any);
        if (w.lane == 0) {
            s.any_flip = any ? 1 : 0;
        }
    }
    if (threadIdx.x == 0) {
        s.job = src.images ? src.images[src.tile_image[item]] : src.single;
    }
    __syncthreads();
    if (!s.any_flip) {
        if (w.err) {
            raise_error(a.header, w.err, static_cast<uint32_t>(item));
        }
        return;
    }
    const PlanImage job = s.job;
    w.set_tile(job, item - job.tile_base);
    w.load(job);
    __syncthreads();
    w.predicates();
    __syncthreads();
    w.unions();
    __syncthreads();
    w.flatten();
    __syncthreads();
    w.number(nullptr, frag_base);
    if (w.err == 0 && s.nfrag != count) {
        w.err = kErrInvariant;
    }
    const int64_t out_pitch = job.out_pitch;
#pragma unroll
    for (int k = 0; k < W::kPerWarp; ++k) {
        const uint32_t pr = w.pred[k];
        if (!(pr & 1u)) {
            continue;
        }
        const int p = W::chunk_of(k, w.warp) * 32 + w.lane;
        const int ly = p >> W::kLog;
        const int lx = p & (T - 1);
        const int head = static_cast<int>((pr >> 8) & 0xFFu);
        const uint32_t b = s.bits[s.parent[ly * T + head]];
        if (!(b & kTouchesSeam)) {
            continue;
        }
        const uint32_t rec = (b >> kRecordShift) - 1;
        if (rec >= static_cast<uint32_t>(count)) {
            w.err = kErrRecordRange;
            continue;
        }
        if (s.flip[rec]) {
            const uint32_t f = s.final_flags[rec];
            const int64_t o = (w.y0 + ly) * out_pitch + w.x0 + lx;
            job.maxima[o] = (f & kHasGreater) ? 0 : 255;
            job.minima[o] = (f & kHasSmaller) ? 0 : 255;
        }
    }
    if (threadIdx.x == 0) {
        atomicAdd(&a.header->flipped_tiles, 1u);
    }
    if (w.err) {
        raise_error(a.header, w.err, static_cast<uint32_t>(item));
    }
}

template <int T, int NW, bool kPersistent>
__global__ void __launch_bounds__(NW * 32)
resolve_pass_kernel(Source src, Arena a) {
    __shared__ TileSmem<T> s;
    if (a.header->magic != kMagic) {
        return;
    }
    if constexpr (kPersistent) {
        for (;;) {
            if (threadIdx.x == 0) {
                s.item = atomicAdd(&a.header->resolve_head, 1u);
            }
            __syncthreads();
            const int64_t item = s.item;
            __syncthreads();
            if (item >= src.total_tiles) {
                break;
            }
            resolve_item<T, NW>(s, src, a, item);
            __syncthreads();
        }
        // The last CTA to finish rewinds both work queues for the next call.
        if (threadIdx.x == 0) {
            __threadfence();
            const uint32_t done = atomicAdd(&a.header->resolve_done, 1u);
            if (done == gridDim.x - 1) {
                atomicExch(&a.header->queue_head, 0u);
                atomicExch(&a.header->resolve_head, 0u);
                atomicExch(&a.header->resolve_done, 0u);
            }
        }
    } else {
        resolve_item<T, NW>(s, src, a, blockIdx.x);
    }
}

__global__ void init_header_kernel(Header* h) {
    h->magic = kMagic;
}

// A kernel that does nothing: the launch-floor measurement's unit.
__global__ void empty_kernel() {}

// ---------------------------------------------------------------------------
// Row-scan kernels: tile pass (T = 32: NW independent warps per CTA, one tile
// each; T = 64: four quadrant warps per tile), seam, flags, resolve passes.
// ---------------------------------------------------------------------------

// Programmatic dependent launch between the row-scan passes.  Each pass
// lets the next one's CTAs be launched once all of its own CTAs have
// started (they then take SM slots as this pass's last CTAs leave, instead
// of after the launch gap), and a pass launched that way waits, before any
// work, until its predecessor grid has completed and its writes are
// visible.  In a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void allow_next_pass() {
    asm volatile("griddepcontrol.launch_dependents;" :::);
}
__device__ __forceinline__ void wait_previous_pass() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Row-scan tile pass: NW independent warps per CTA, one tile each; at most
// 64 registers per thread, so 32 warps fit on an SM (the shared-memory
// limit at 6.6 KB per warp).  The persistent form gets the same budget: at
// 72 registers (28 warps per SM) it measured 3 % slower on the corpus.
template <int NW, bool kPersistent>
__global__ void __launch_bounds__(NW * 32, 32 / NW)
runs_tile_pass_kernel(Source src, Arena a) {
    __shared__ rowscan::RunSmem sm[NW];
    allow_next_pass();
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    if (a.header->magic != kMagic) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            raise_error(a.header, kErrUninitialized, 0u);
        }
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.header->last_tiles = static_cast<uint64_t>(src.total_tiles);
        a.header->tile = rowscan::T;
        a.header->route = 1u;
    }
    if constexpr (kPersistent) {
        // One item per pop: the tiles in flight stay a window of consecutive
        // items, like the grid schedule's, so neighbouring tiles' halo rows
        // and mask sectors meet in L2 (runs of 4 or 16 items per pop spread
        // the window over tens of thousands of tiles and measured slower).
        for (;;) {
            uint32_t item = 0;
            if (lane == 0) {
                item = atomicAdd(&a.header->queue_head, 1u);
            }
            item = __shfl_sync(~0u, item, 0);
            if (static_cast<int64_t>(item) >= src.total_tiles) {
                break;
            }
            rowscan::tile_pass_runs<1>(sm[warp].word, sm[warp].aux, nullptr,
                                       0, src, a, item);
            __syncwarp();
        }
    } else {
        const int64_t item = static_cast<int64_t>(blockIdx.x) * NW + warp;
        if (item < src.total_tiles) {
            rowscan::tile_pass_runs<1>(sm[warp].word, sm[warp].aux, nullptr,
                                       0, src, a, item);
        }
    }
}

// Row-scan tile pass at tile edge 64: one CTA of 4 warps per tile, one warp
// per 32 x 32 quadrant, at most 64 registers per thread (8 CTAs, 32 warps
// per SM; 27 KB of shared memory per CTA).
template <bool kPersistent>
__global__ void __launch_bounds__(128, 8)
runs64_tile_pass_kernel(Source src, Arena a) {
    __shared__ rowscan::RunSmem64 sm;
    __shared__ uint32_t next_item;
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    allow_next_pass();
    if (a.header->magic != kMagic) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            raise_error(a.header, kErrUninitialized, 0u);
        }
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.header->last_tiles = static_cast<uint64_t>(src.total_tiles);
        a.header->tile = 64u;
        a.header->route = 1u;
    }
    if constexpr (kPersistent) {
        for (;;) {
            if (threadIdx.x == 0) {
                next_item = atomicAdd(&a.header->queue_head, 1u);
            }
            __syncthreads();
            const int64_t item = next_item;
            __syncthreads();   // every thread has read next_item
            if (item >= src.total_tiles) {
                break;
            }
            rowscan::tile_pass_runs<4>(sm.word, sm.aux[warp], &sm.cta, warp,
                                       src, a, item);
            __syncthreads();
        }
    } else {
        rowscan::tile_pass_runs<4>(sm.word, sm.aux[warp], &sm.cta, warp, src,
                                   a, blockIdx.x);
    }
}

// Passes after the row-scan tile pass: one CTA of kLaterWarps warps per
// group of src.group consecutive tiles.
template <int TT>
__global__ void __launch_bounds__(rowscan::kLaterWarps * 32)
rowscan_seam_pass_kernel(Source src, Arena a) {
    wait_previous_pass();
    allow_next_pass();
    if (a.header->magic != kMagic) {
        return;
    }
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int64_t first = static_cast<int64_t>(blockIdx.x) * src.group;
    if (first < src.total_tiles) {
        rowscan::seam_pass_group<TT>(src, a, first, warp,
                                     rowscan::kLaterWarps);
    }
}

template <int TT>
__global__ void __launch_bounds__(rowscan::kLaterWarps * 32)
rowscan_flags_pass_kernel(Source src, Arena a) {
    wait_previous_pass();
    allow_next_pass();
    if (a.header->magic != kMagic) {
        return;
    }
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    const int64_t first = static_cast<int64_t>(blockIdx.x) * src.group;
    if (first < src.total_tiles) {
        rowscan::flags_pass_group<TT>(src, a, first, warp,
                                      rowscan::kLaterWarps);
    }
}

template <int TT, bool kPersistent>
__global__ void __launch_bounds__(rowscan::kLaterWarps * 32)
rowscan_resolve_pass_kernel(Source src, Arena a) {
    __shared__ rowscan::ResolveSmem<TT> sm;
    __shared__ uint32_t next_group;
    const int warp = static_cast<int>(threadIdx.x) >> 5;
    wait_previous_pass();
    if (a.header->magic != kMagic) {
        return;
    }
    if constexpr (kPersistent) {
        for (;;) {
            if (threadIdx.x == 0) {
                next_group = atomicAdd(&a.header->resolve_head, 1u);
            }
            __syncthreads();
            const int64_t first =
                static_cast<int64_t>(next_group) * src.group;
            __syncthreads();   // every thread has read next_group
            if (first >= src.total_tiles) {
                break;
            }
            rowscan::resolve_group<TT>(sm, src, a, first, warp,
                                   rowscan::kLaterWarps);
        }
        // The last CTA to finish rewinds both work queues for the next call.
        if (threadIdx.x == 0) {
            __threadfence();
            const uint32_t done = atomicAdd(&a.header->resolve_done, 1u);
            if (done == gridDim.x - 1) {
                atomicExch(&a.header->queue_head, 0u);
                atomicExch(&a.header->resolve_head, 0u);
                atomicExch(&a.header->resolve_done, 0u);
            }
        }
    } else {
        const int64_t first = static_cast<int64_t>(blockIdx.x) * src.group;
        if (first < src.total_tiles) {
            rowscan::resolve_group<TT>(sm, src, a, first, warp,
                                   rowscan::kLaterWarps);
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct Layout {
    size_t relation, count, border, parent, bits, pending_count, pending,
        seam_count, seam_items, total;
};

static size_t round_up(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Every tile needs at least 16 + 2 + 64 + 256 + 256 bytes (T = 16), so a
// workspace of S bytes never holds more than S / 512 tiles.  The seam-pair
// counters of every possible call therefore fit in a fixed region of
// 16 * (S / 512) bytes right after the header, whatever the geometry: reusing
// a workspace for another image size or tile size never reads data of the
// other arrays as counters.  Counters are zero between calls (the resolve
// pass clears each tile's counters after use).
static size_t relation_region_end(size_t workspace_bytes) {
    return round_up(sizeof(Header) + 16 * (workspace_bytes / 512));
}

static bool layout_for(int64_t tiles, int tile, size_t workspace_bytes,
                       Layout* out) {
    if (tiles < 0) {
        return false;
    }
    const int64_t slots = tiles * 4 * tile;
    if (slots >= (int64_t(1) << 31) || tiles >= (int64_t(1) << 32)) {
        return false;  // fragment indices and the work queue are 32-bit
    }
    Layout L;
    L.relation = sizeof(Header);
    size_t off = relation_region_end(workspace_bytes);
    L.count = off;
    off = round_up(off + static_cast<size_t>(tiles) * 2);
    L.border = off;
    off = round_up(off + static_cast<size_t>(slots));
    L.parent = off;
    off = round_up(off + static_cast<size_t>(slots) * 4);
    L.bits = off;
    off = round_up(off + static_cast<size_t>(slots) * 4);
    // The row-scan kernels (T = 32, 64) log pending runs, at most T * T per
    // tile, and up to 12 T seam items per tile.
    const size_t pend = tile >= 32 ? static_cast<size_t>(tiles) : 0;
    const size_t t2 = static_cast<size_t>(tile) * tile;
    L.pending_count = off;
    off = round_up(off + pend * 4);
    L.pending = off;
    off = round_up(off + pend * t2 * 4);
    L.seam_count = off;
    off = round_up(off + pend * 4);
    L.seam_items = off;
    off = round_up(off + pend * 12 * tile * 4);
    L.total = off;
    *out = L;
    return L.total <= workspace_bytes &&
           static_cast<size_t>(tiles) <= workspace_bytes / 512;
}

// Smallest workspace whose layout fits `tiles` tiles of edge `tile`.
static bool workspace_size(int64_t tiles, int tile, size_t* bytes) {
    if (tiles < 0 || tiles * 4 * tile >= (int64_t(1) << 31)) {
        return false;
    }
    const size_t slots = static_cast<size_t>(tiles) * 4 * tile;
    const size_t pend = tile >= 32 ? static_cast<size_t>(tiles) : 0;
    const size_t t2 = static_cast<size_t>(tile) * tile;
    const size_t dirty = round_up(static_cast<size_t>(tiles) * 2) +
                         round_up(slots) + 2 * round_up(slots * 4) +
                         round_up(pend * 4) + round_up(pend * t2 * 4) +
                         round_up(pend * 4) +
                         round_up(pend * 12 * tile * 4);
    size_t s = round_up((dirty + 512) / 31 * 32 + 512);
    Layout L;
    for (int i = 0; i < 1024 && !layout_for(tiles, tile, s, &L); ++i) {
        s += 256;
    }
    if (!layout_for(tiles, tile, s, &L)) {
        return false;
    }
    *bytes = s;
    return true;
}

static Arena arena_at(void* base, const Layout& L) {
    char* b = static_cast<char*>(base);
    Arena a;
    a.header = reinterpret_cast<Header*>(b);
    a.relation = reinterpret_cast<uint32_t*>(b + L.relation);
    a.fragment_count = reinterpret_cast<uint16_t*>(b + L.count);
    a.border = reinterpret_cast<uint8_t*>(b + L.border);
    a.parent = reinterpret_cast<int32_t*>(b + L.parent);
    a.bits = reinterpret_cast<uint32_t*>(b + L.bits);
    a.pending_count = reinterpret_cast<uint32_t*>(b + L.pending_count);
    a.pending = reinterpret_cast<uint32_t*>(b + L.pending);
    a.seam_count = reinterpret_cast<uint32_t*>(b + L.seam_count);
    a.seam_items = reinterpret_cast<uint32_t*>(b + L.seam_items);
    return a;
}

static bool tile_ok(int tile) { return tile == 16 || tile == 32 || tile == 64; }

static int64_t tiles_of(int width, int height, int tile) {
    return static_cast<int64_t>((width + tile - 1) / tile) *
           static_cast<int64_t>((height + tile - 1) / tile);
}

using Kernel = void (*)(Source, Arena);

struct Config {
    int tile;
    int warps;
    Kernel tile_pass[2];
    Kernel resolve_pass[2];
    int items_per_cta;   // tiles one tile-pass CTA handles per launch slot
    Kernel seam_pass;    // between the two passes, or nullptr
    int later_per_cta;   // tiles one seam / resolve CTA handles
    Kernel flags_pass;   // after the seam pass, or nullptr
};

#define SS_CONFIG(T, NW)                                                      \
    Config {                                                                  \
        T, NW, {tile_pass_kernel<T, NW, false>, tile_pass_kernel<T, NW, true>}, \
            {resolve_pass_kernel<T, NW, false>,                               \
             resolve_pass_kernel<T, NW, true>}, 1, nullptr, 1, nullptr        \
    }
// Row-scan configurations are listed with warps = -NW: at tile edge 32 one
// tile per warp, NW warps per CTA; at tile edge 64 (-4) one tile per CTA of
// four quadrant warps.
#define SS_ROWSCAN(NW)                                                        \
    Config {                                                                  \
        32, -(NW),                                                            \
            {runs_tile_pass_kernel<NW, false>,                                \
             runs_tile_pass_kernel<NW, true>},                                \
            {rowscan_resolve_pass_kernel<32, false>,                          \
             rowscan_resolve_pass_kernel<32, true>}, NW,                      \
            rowscan_seam_pass_kernel<32>, 32, rowscan_flags_pass_kernel<32>   \
    }
#define SS_ROWSCAN64()                                                        \
    Config {                                                                  \
        64, -4,                                                               \
            {runs64_tile_pass_kernel<false>, runs64_tile_pass_kernel<true>},  \
            {rowscan_resolve_pass_kernel<64, false>,                          \
             rowscan_resolve_pass_kernel<64, true>}, 1,                       \
            rowscan_seam_pass_kernel<64>, 32, rowscan_flags_pass_kernel<64>   \
    }

static const Config kConfigs[] = {
    SS_CONFIG(16, 2), SS_CONFIG(16, 4), SS_CONFIG(16, 8),
    SS_CONFIG(32, 4), SS_CONFIG(32, 8), SS_CONFIG(32, 16),
    SS_CONFIG(64, 8), SS_CONFIG(64, 16),
    SS_ROWSCAN(2), SS_ROWSCAN(4), SS_ROWSCAN64(),
};
#undef SS_CONFIG
#undef SS_ROWSCAN
#undef SS_ROWSCAN64

// Per tile size, the configuration used by default (index by tile / 16 - 1);
// negative warps select the row-scan kernels.
static std::atomic<int> g_default_warps[4] = {{4}, {-4}, {0}, {-4}};

static const Config* find_config(int tile, int warps) {
    for (const Config& c : kConfigs) {
        if (c.tile == tile && c.warps == warps) {
            return &c;
        }
    }
    return nullptr;
}

static const Config* default_config(int tile) {
    return find_config(tile, g_default_warps[tile / 16 - 1].load());
}

// Persistent grid size per kernel (occupancy x SMs), cached per device.
static int persistent_grid(Kernel k, int threads) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<int, const void*>, int>> cache;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        return 0;
    }
    std::lock_guard<std::mutex> lock(mu);
    for (auto& e : cache) {
        if (e.first.first == device &&
            e.first.second == reinterpret_cast<const void*>(k)) {
            return e.second;
        }
    }
    int sms = 0;
    int per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, reinterpret_cast<const void*>(k), threads, 0) !=
            cudaSuccess) {
        return 0;
    }
    const int grid = std::max(1, sms * std::max(1, per_sm));
    cache.push_back({{device, reinterpret_cast<const void*>(k)}, grid});
    return grid;
}

// Streaming multiprocessors of the current device (cached per device).
static int sm_count() {
    static std::atomic<int> cache[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        return 0;
    }
    if (device >= 0 && device < 64) {
        const int c = cache[device].load();
        if (c > 0) {
            return c;
        }
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) !=
        cudaSuccess) {
        return 0;
    }
    if (device >= 0 && device < 64) {
        cache[device].store(sms);
    }
    return sms;
}

// Tiles per CTA of the row-scan seam, flags and resolve passes: the smallest
// power of two (at most 32) that keeps the grid within 8 CTAs (64 warps) per
// SM.  Small launches (one image) get few tiles per CTA, so each chain of
// dependent global loads is short; large batches get 32, so each warp
// overlaps the round trips of many tiles.
static int later_group(int64_t tiles) {
    const int64_t target = static_cast<int64_t>(std::max(1, sm_count())) * 8;
    int group = 1;
    while (group < 32 && tiles > static_cast<int64_t>(group) * target) {
        group *= 2;
    }
    return group;
}

bool workspace_bytes_for_tiles(int64_t tiles, int tile, size_t* bytes) {
    return tile_ok(tile) && tiles >= 0 && workspace_size(tiles, tile, bytes);
}

// Launches a pass after the row-scan tile pass, allowed to start before its
// predecessor ends (it waits for it on the device).
static void launch_next_pass(Kernel k, unsigned grid, unsigned threads,
                             cudaStream_t stream, const Source& src,
                             const Arena& arena) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(threads);
    lc.dynamicSmemBytes = 0;
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    (void)cudaLaunchKernelEx(&lc, k, src, arena);
}

static ss_status launch_route(const Config& cfg, const Source& src_in,
                              const Arena& arena, int persistent,
                              cudaStream_t stream, int passes = 7,
                              int group = 0, int flatten = kFlattenHalve) {
    if (src_in.total_tiles == 0) {
        return SS_OK;
    }
    // The status reports this call's launches only: drop a result left in
    // the thread's last-error slot by earlier runtime calls (a query that
    // answered cudaErrorNotReady, for instance).  Sticky errors still fail
    // the launches below.
    (void)cudaGetLastError();
    Source src = src_in;
    const int nw = cfg.warps < 0 ? -cfg.warps : cfg.warps;
    const int threads = nw * 32;
    // Tiles per CTA of the passes after the tile pass, and their CTA size.
    int later_per_cta = cfg.later_per_cta;
    int later_threads = threads;
    src.group = 32;
    if (cfg.seam_pass) {
        src.group = group > 0 ? group : later_group(src.total_tiles);
        later_per_cta = src.group;
        later_threads = rowscan::kLaterWarps * 32;
    }
    const int p = persistent ? 1 : 0;
    const int64_t ctas1 =
        (src.total_tiles + cfg.items_per_cta - 1) / cfg.items_per_cta;
    const int64_t ctas2 =
        (src.total_tiles + later_per_cta - 1) / later_per_cta;
    unsigned grid1 = static_cast<unsigned>(ctas1);
    unsigned grid2 = static_cast<unsigned>(ctas2);
    if (p) {
        const int g1 = persistent_grid(cfg.tile_pass[1], threads);
        const int g2 = persistent_grid(cfg.resolve_pass[1], later_threads);
        if (g1 <= 0 || g2 <= 0) {
            return SS_ERR_CUDA;
        }
        grid1 = static_cast<unsigned>(std::min<int64_t>(g1, ctas1));
        grid2 = static_cast<unsigned>(std::min<int64_t>(g2, ctas2));
    }
    if (passes & 1) {
        cfg.tile_pass[p]<<<grid1, threads, 0, stream>>>(src, arena);
    }
    if ((passes & 4) && cfg.seam_pass) {
        launch_next_pass(cfg.seam_pass, static_cast<unsigned>(ctas2),
                         later_threads, stream, src, arena);
        if (cfg.flags_pass) {
            src.flatten = flatten;
            if (flatten == kFlattenSeparate) {
                Source only = src;
                only.flatten = kFlattenOnly;
                launch_next_pass(cfg.flags_pass, static_cast<unsigned>(ctas2),
                                 later_threads, stream, only, arena);
            }
            launch_next_pass(cfg.flags_pass, static_cast<unsigned>(ctas2),
                             later_threads, stream, src, arena);
        }
    }
    if (passes & 2) {
        if (cfg.seam_pass) {
            // Row-scan resolve pass: waits for its predecessor on the device.
            launch_next_pass(cfg.resolve_pass[p], grid2, later_threads,
                             stream, src, arena);
        } else {
            cfg.resolve_pass[p]<<<grid2, later_threads, 0, stream>>>(src,
                                                                     arena);
        }
    }
    return cudaGetLastError() == cudaSuccess ? SS_OK : SS_ERR_CUDA;
}

}  // namespace ss

using namespace ss;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char* ss_status_string(ss_status status) {
    switch (status) {
        case SS_OK: return "SS_OK";
        case SS_ERR_INVALID_VALUE: return "SS_ERR_INVALID_VALUE";
        case SS_ERR_UNSUPPORTED_TILE: return "SS_ERR_UNSUPPORTED_TILE";
        case SS_ERR_WORKSPACE_TOO_SMALL: return "SS_ERR_WORKSPACE_TOO_SMALL";
        case SS_ERR_MISALIGNED: return "SS_ERR_MISALIGNED";
        case SS_ERR_TOO_LARGE: return "SS_ERR_TOO_LARGE";
        case SS_ERR_CUDA: return "SS_ERR_CUDA";
        case SS_ERR_FRAGMENT_OVERFLOW: return "SS_ERR_FRAGMENT_OVERFLOW";
        case SS_ERR_RECORD_RANGE: return "SS_ERR_RECORD_RANGE";
        case SS_ERR_INVARIANT: return "SS_ERR_INVARIANT";
        case SS_ERR_SPIN_LIMIT: return "SS_ERR_SPIN_LIMIT";
        case SS_ERR_WORKSPACE_UNINITIALIZED:
            return "SS_ERR_WORKSPACE_UNINITIALIZED";
        case SS_ERR_HOST_ALLOC: return "SS_ERR_HOST_ALLOC";
        case SS_ERR_EXCEEDS_STATIC_SCRATCH:
            return "SS_ERR_EXCEEDS_STATIC_SCRATCH";
    }
    return "SS_ERR_UNKNOWN";
}

int ss_abi_version(void) { return SS_ABI_VERSION; }

ss_status ss_workspace_bytes(int width, int height, int tile, size_t* bytes) {
    if (!bytes || width <= 0 || height <= 0) {
        return SS_ERR_INVALID_VALUE;
    }
    if (!tile_ok(tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    if (!workspace_size(tiles_of(width, height, tile), tile, bytes)) {
        return SS_ERR_TOO_LARGE;
    }
    return SS_OK;
}

ss_status ss_workspace_init(void* d_workspace, size_t workspace_bytes,
                            void* stream) {
    if (!d_workspace || workspace_bytes < sizeof(Header)) {
        return SS_ERR_INVALID_VALUE;
    }
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256 != 0) {
        return SS_ERR_MISALIGNED;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The header and every seam-pair counter must start at zero.  Where the
    // counters sit depends on the tile size and tile count of later calls,
    // so the whole workspace is cleared.
    if (cudaMemsetAsync(d_workspace, 0, workspace_bytes, st) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    init_header_kernel<<<1, 1, 0, st>>>(static_cast<Header*>(d_workspace));
    return cudaGetLastError() == cudaSuccess ? SS_OK : SS_ERR_CUDA;
}

static ss_status extrema_impl(const uint8_t* d_image, int width, int height,
                              int pitch, int tile, int levels,
                              uint8_t* d_maxima, uint8_t* d_minima,
                              int out_pitch, void* d_workspace,
                              size_t workspace_bytes, void* stream);

ss_status ss_extrema(const uint8_t* d_image, int width, int height, int pitch,
                     int tile, uint8_t* d_maxima, uint8_t* d_minima,
                     int out_pitch, void* d_workspace, size_t workspace_bytes,
                     void* stream) {
    return extrema_impl(d_image, width, height, pitch, tile, 0, d_maxima,
                        d_minima, out_pitch, d_workspace, workspace_bytes,
                        stream);
}

ss_status ss_extrema_levels(const uint8_t* d_image, int width, int height,
                            int pitch, int tile, int levels,
                            uint8_t* d_maxima, uint8_t* d_minima,
                            int out_pitch, void* d_workspace,
                            size_t workspace_bytes, void* stream) {
    if (levels != 0 && (levels < 2 || levels > 256)) {
        return SS_ERR_INVALID_VALUE;
    }
    return extrema_impl(d_image, width, height, pitch, tile, levels,
                        d_maxima, d_minima, out_pitch, d_workspace,
                        workspace_bytes, stream);
}

static ss_status extrema_impl(const uint8_t* d_image, int width, int height,
                              int pitch, int tile, int levels,
                              uint8_t* d_maxima, uint8_t* d_minima,
                              int out_pitch, void* d_workspace,
                              size_t workspace_bytes, void* stream) {
    if (!d_image || !d_maxima || !d_minima || !d_workspace || width <= 0 ||
        height <= 0 || pitch < width || out_pitch < width) {
        return SS_ERR_INVALID_VALUE;
    }
    if (!tile_ok(tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256 != 0) {
        return SS_ERR_MISALIGNED;
    }
    const int64_t tiles = tiles_of(width, height, tile);
    size_t needed = 0;
    if (!workspace_size(tiles, tile, &needed)) {
        return SS_ERR_TOO_LARGE;
    }
    Layout L;
    if (workspace_bytes < needed ||
        !layout_for(tiles, tile, workspace_bytes, &L)) {
        return SS_ERR_WORKSPACE_TOO_SMALL;
    }
    const Config* cfg = default_config(tile);
    if (!cfg) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    Source src{};
    src.images = nullptr;
    src.tile_image = nullptr;
    src.single.image = d_image;
    src.single.maxima = d_maxima;
    src.single.minima = d_minima;
    src.single.width = width;
    src.single.height = height;
    src.single.pitch = pitch;
    src.single.out_pitch = out_pitch;
    src.single.tiles_x = (width + tile - 1) / tile;
    src.single.tiles_y = (height + tile - 1) / tile;
    src.single.tile_base = 0;
    src.single.levels = levels;
    src.total_tiles = tiles;
    return launch_route(*cfg, src, arena_at(d_workspace, L), 0,
                        static_cast<cudaStream_t>(stream));
}

ss_status ss_read_status(void* d_workspace, size_t workspace_bytes,
                         void* stream, ss_stats* stats) {
    if (!d_workspace || workspace_bytes < sizeof(Header)) {
        return SS_ERR_INVALID_VALUE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    Header h;
    if (cudaMemcpy(&h, d_workspace, sizeof(Header), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        return SS_ERR_CUDA;
    }
    if (h.magic != kMagic) {
        return SS_ERR_WORKSPACE_UNINITIALIZED;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->device_error = h.error;
        stats->error_detail = h.error_detail;
        stats->tiles = h.last_tiles;
        stats->flipped_tiles = h.flipped_tiles;
        Layout L;
        if (tile_ok(static_cast<int>(h.tile)) &&
            layout_for(static_cast<int64_t>(h.last_tiles),
                       static_cast<int>(h.tile), workspace_bytes, &L) &&
            h.last_tiles > 0) {
            std::vector<uint16_t> counts(h.last_tiles);
            if (cudaMemcpy(counts.data(),
                           static_cast<char*>(d_workspace) + L.count,
                           counts.size() * sizeof(uint16_t),
                           cudaMemcpyDeviceToHost) != cudaSuccess) {
                return SS_ERR_CUDA;
            }
            uint64_t sum = 0;
            for (uint16_t c : counts) {
                sum += c;
            }
            stats->active_fragments = sum;
            if (h.route == 1u) {
                // Pixels of the logged runs: bits 16-31 of each tile's
                // run-log count.
                std::vector<uint32_t> logs(h.last_tiles);
                if (cudaMemcpy(logs.data(),
                               static_cast<char*>(d_workspace) +
                                   L.pending_count,
                               logs.size() * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost) != cudaSuccess) {
                    return SS_ERR_CUDA;
                }
                uint64_t px = 0;
                for (uint32_t c : logs) {
                    px += c >> 16;
                }
                stats->live_pixels = px;
            }
        }
    }
    // Clear the error word, its detail and the flip counter.
    Header* dh = static_cast<Header*>(d_workspace);
    const uint32_t zeros[2] = {0u, 0u};
    if (cudaMemcpy(&dh->error, zeros, sizeof(zeros), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(&dh->flipped_tiles, zeros, sizeof(uint32_t),
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    return h.error ? static_cast<ss_status>(h.error) : SS_OK;
}

ss_status ss_empty_launches(int count, int grid, int threads, void* stream) {
    if (count < 0 || grid <= 0 || threads <= 0 || threads > 1024) {
        return SS_ERR_INVALID_VALUE;
    }
    (void)cudaGetLastError();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int i = 0; i < count; ++i) {
        empty_kernel<<<static_cast<unsigned>(grid), threads, 0, st>>>();
    }
    return cudaGetLastError() == cudaSuccess ? SS_OK : SS_ERR_CUDA;
}

ss_status ss_set_kernel_config(int tile, int warps) {
    if (!tile_ok(tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    if (!find_config(tile, warps)) {
        return SS_ERR_INVALID_VALUE;
    }
    g_default_warps[tile / 16 - 1].store(warps);
    return SS_OK;
}

ss_status ss_get_kernel_config(int tile, int* warps) {
    if (!warps) {
        return SS_ERR_INVALID_VALUE;
    }
    if (!tile_ok(tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    *warps = g_default_warps[tile / 16 - 1].load();
    return SS_OK;
}

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------

static size_t plan_size(int count, int64_t total_tiles) {
    return round_up(sizeof(PlanHeader) + static_cast<size_t>(count) *
                                             sizeof(PlanImage) +
                    static_cast<size_t>(total_tiles) * sizeof(int32_t));
}

ss_status ss_batch_plan_bytes(int count, int64_t total_tiles, size_t* bytes) {
    if (!bytes || count < 0 || total_tiles < 0) {
        return SS_ERR_INVALID_VALUE;
    }
    *bytes = plan_size(count, total_tiles);
    return SS_OK;
}

ss_status ss_batch_tiles(const ss_image_desc* descs, int count, int tile,
                         int64_t* total_tiles) {
    if (!total_tiles || count < 0 || (count > 0 && !descs)) {
        return SS_ERR_INVALID_VALUE;
    }
    if (!tile_ok(tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    int64_t total = 0;
    for (int i = 0; i < count; ++i) {
        const ss_image_desc& d = descs[i];
        if (!d.image || !d.maxima || !d.minima || d.width <= 0 ||
            d.height <= 0 || d.pitch < d.width || d.out_pitch < d.width) {
            return SS_ERR_INVALID_VALUE;
        }
        total += tiles_of(d.width, d.height, tile);
    }
    *total_tiles = total;
    return SS_OK;
}

ss_status ss_batch_plan_fill(const ss_image_desc* descs, int count, int tile,
                             void* h_plan, size_t plan_bytes,
                             size_t* workspace_bytes) {
    int64_t total = 0;
    ss_status st = ss_batch_tiles(descs, count, tile, &total);
    if (st != SS_OK) {
        return st;
    }
    if (!h_plan) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t needed = 0;
    if (!workspace_size(total, tile, &needed)) {
        return SS_ERR_TOO_LARGE;
    }
    if (plan_bytes < plan_size(count, total)) {
        return SS_ERR_WORKSPACE_TOO_SMALL;
    }
    std::memset(h_plan, 0, plan_size(count, total));
    PlanHeader* ph = static_cast<PlanHeader*>(h_plan);
    ph->magic = kMagic;
    ph->count = count;
    ph->tile = tile;
    ph->total_tiles = total;
    PlanImage* images = reinterpret_cast<PlanImage*>(ph + 1);
    int32_t* map = reinterpret_cast<int32_t*>(images + count);
    int64_t base = 0;
    for (int i = 0; i < count; ++i) {
        const ss_image_desc& d = descs[i];
        PlanImage& pi = images[i];
        pi.image = d.image;
        pi.maxima = d.maxima;
        pi.minima = d.minima;
        pi.width = d.width;
        pi.height = d.height;
        pi.pitch = d.pitch;
        pi.out_pitch = d.out_pitch;
        pi.tiles_x = (d.width + tile - 1) / tile;
        pi.tiles_y = (d.height + tile - 1) / tile;
        pi.tile_base = base;
        const int64_t n = static_cast<int64_t>(pi.tiles_x) * pi.tiles_y;
        for (int64_t t = 0; t < n; ++t) {
            map[base + t] = i;
        }
        base += n;
    }
    if (workspace_bytes) {
        *workspace_bytes = needed;
    }
    return SS_OK;
}

ss_status ss_batch_plan_set_levels(void* h_plan, size_t plan_bytes, int index,
                                   int levels) {
    if (!h_plan || plan_bytes < sizeof(PlanHeader) ||
        (levels != 0 && (levels < 2 || levels > 256))) {
        return SS_ERR_INVALID_VALUE;
    }
    PlanHeader* ph = static_cast<PlanHeader*>(h_plan);
    if (ph->magic != kMagic || index < 0 || index >= ph->count ||
        plan_bytes < plan_size(ph->count, ph->total_tiles)) {
        return SS_ERR_INVALID_VALUE;
    }
    reinterpret_cast<PlanImage*>(ph + 1)[index].levels = levels;
    return SS_OK;
}

static ss_status batch_passes(const void* h_plan, const void* d_plan,
                              size_t plan_bytes, int persistent,
                              void* d_workspace, size_t workspace_bytes,
                              void* stream, int passes, int warps = 0,
                              int group = 0, int flatten = kFlattenHalve) {
    if (!h_plan || !d_plan || !d_workspace ||
        plan_bytes < sizeof(PlanHeader)) {
        return SS_ERR_INVALID_VALUE;
    }
    if (group != 0 && (group < 0 || group > 32 || (group & (group - 1)))) {
        return SS_ERR_INVALID_VALUE;
    }
    if (flatten < kFlattenHalve || flatten > kFlattenSeparate) {
        return SS_ERR_INVALID_VALUE;
    }
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256 != 0 ||
        reinterpret_cast<uintptr_t>(d_plan) % 256 != 0) {
        return SS_ERR_MISALIGNED;
    }
    const PlanHeader* ph = static_cast<const PlanHeader*>(h_plan);
    if (ph->magic != kMagic || ph->count < 0 || ph->total_tiles < 0) {
        return SS_ERR_INVALID_VALUE;
    }
    if (!tile_ok(ph->tile)) {
        return SS_ERR_UNSUPPORTED_TILE;
    }
    if (plan_bytes < plan_size(ph->count, ph->total_tiles)) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t needed = 0;
    if (!workspace_size(ph->total_tiles, ph->tile, &needed)) {
        return SS_ERR_TOO_LARGE;
    }
    Layout L;
    if (workspace_bytes < needed ||
        !layout_for(ph->total_tiles, ph->tile, workspace_bytes, &L)) {
        return SS_ERR_WORKSPACE_TOO_SMALL;
    }
    const Config* cfg =
        warps ? find_config(ph->tile, warps) : default_config(ph->tile);
    if (!cfg) {
        return warps ? SS_ERR_INVALID_VALUE : SS_ERR_UNSUPPORTED_TILE;
    }
    const PlanHeader* dph = static_cast<const PlanHeader*>(d_plan);
    Source src{};
    if (ph->count == 1) {
        // One image: its entry travels in the launch parameters, as for a
        // single call, instead of being looked up per tile.
        src.images = nullptr;
        src.tile_image = nullptr;
        src.single = *reinterpret_cast<const PlanImage*>(ph + 1);
    } else {
        src.images = reinterpret_cast<const PlanImage*>(dph + 1);
        src.tile_image =
            reinterpret_cast<const int32_t*>(src.images + ph->count);
    }
    src.total_tiles = ph->total_tiles;
    return launch_route(*cfg, src, arena_at(d_workspace, L),
                        persistent ? 1 : 0,
                        static_cast<cudaStream_t>(stream), passes, group,
                        flatten);
}

ss_status ss_extrema_batch(const void* h_plan, const void* d_plan,
                           size_t plan_bytes, int persistent,
                           void* d_workspace, size_t workspace_bytes,
                           void* stream) {
    return batch_passes(h_plan, d_plan, plan_bytes, persistent, d_workspace,
                        workspace_bytes, stream, 7);
}

ss_status ss_extrema_batch_launch(const void* h_plan, const void* d_plan,
                                  size_t plan_bytes, const ss_launch* launch,
                                  void* d_workspace, size_t workspace_bytes,
                                  void* stream) {
    ss_launch l{};
    if (launch) {
        l = *launch;
    }
    if (l.passes < 0 || l.passes > 7) {
        return SS_ERR_INVALID_VALUE;
    }
    return batch_passes(h_plan, d_plan, plan_bytes, l.persistent ? 1 : 0,
                        d_workspace, workspace_bytes, stream,
                        l.passes ? l.passes : 7, l.warps, l.group, l.flatten);
}

ss_status ss_extrema_batch_pass(const void* h_plan, const void* d_plan,
                                size_t plan_bytes, int persistent, int pass,
                                void* d_workspace, size_t workspace_bytes,
                                void* stream) {
    if (pass != 1 && pass != 2 && pass != 4) {
        return SS_ERR_INVALID_VALUE;
    }
    return batch_passes(h_plan, d_plan, plan_bytes, persistent, d_workspace,
                        workspace_bytes, stream, pass);
}

// ---------------------------------------------------------------------------
// Host-to-host convenience form
// ---------------------------------------------------------------------------

struct ss_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    uint8_t* d_image = nullptr;
    uint8_t* d_maxima = nullptr;
    uint8_t* d_minima = nullptr;
    size_t pixel_capacity = 0;
    void* d_workspace = nullptr;
    size_t workspace_capacity = 0;
};

ss_status ss_context_create(int device, ss_context** context) {
    if (!context) {
        return SS_ERR_INVALID_VALUE;
    }
    *context = nullptr;
    ss_context* c = new (std::nothrow) ss_context();
    if (!c) {
        return SS_ERR_HOST_ALLOC;
    }
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) !=
            cudaSuccess ||
        cudaEventCreate(&c->start) != cudaSuccess ||
        cudaEventCreate(&c->stop) != cudaSuccess) {
        ss_context_destroy(c);
        return SS_ERR_CUDA;
    }
    *context = c;
    return SS_OK;
}

void ss_context_destroy(ss_context* c) {
    if (!c) {
        return;
    }
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_image);
    cudaFree(c->d_maxima);
    cudaFree(c->d_minima);
    cudaFree(c->d_workspace);
    if (c->start) cudaEventDestroy(c->start);
    if (c->stop) cudaEventDestroy(c->stop);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

ss_status ss_extrema_host(ss_context* c, const uint8_t* h_image, int width,
                          int height, int pitch, int tile, uint8_t* h_maxima,
                          uint8_t* h_minima, int out_pitch, float* elapsed_ms,
                          uint64_t* active_fragments) {
    if (!c || !h_image || !h_maxima || !h_minima || width <= 0 ||
        height <= 0 || pitch < width || out_pitch < width) {
        return SS_ERR_INVALID_VALUE;
    }
    size_t ws = 0;
    ss_status st = ss_workspace_bytes(width, height, tile, &ws);
    if (st != SS_OK) {
        return st;
    }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    const size_t pixels = static_cast<size_t>(width) * height;
    if (pixels > c->pixel_capacity) {
        cudaFree(c->d_image);
        cudaFree(c->d_maxima);
        cudaFree(c->d_minima);
        c->d_image = c->d_maxima = c->d_minima = nullptr;
        c->pixel_capacity = 0;
        if (cudaMalloc(&c->d_image, pixels) != cudaSuccess ||
            cudaMalloc(&c->d_maxima, pixels) != cudaSuccess ||
            cudaMalloc(&c->d_minima, pixels) != cudaSuccess) {
            return SS_ERR_CUDA;
        }
        c->pixel_capacity = pixels;
    }
    if (ws > c->workspace_capacity) {
        cudaFree(c->d_workspace);
        c->d_workspace = nullptr;
        c->workspace_capacity = 0;
        if (cudaMalloc(&c->d_workspace, ws) != cudaSuccess) {
            return SS_ERR_CUDA;
        }
        c->workspace_capacity = ws;
        st = ss_workspace_init(c->d_workspace, ws, c->stream);
        if (st != SS_OK) {
            return st;
        }
    }
    if (cudaMemcpy2DAsync(c->d_image, width, h_image, pitch, width, height,
                          cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
        cudaEventRecord(c->start, c->stream) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    st = ss_extrema(c->d_image, width, height, width, tile, c->d_maxima,
                    c->d_minima, width, c->d_workspace, c->workspace_capacity,
                    c->stream);
    if (st != SS_OK) {
        return st;
    }
    if (cudaEventRecord(c->stop, c->stream) != cudaSuccess ||
        cudaMemcpy2DAsync(h_maxima, out_pitch, c->d_maxima, width, width,
                          height, cudaMemcpyDeviceToHost,
                          c->stream) != cudaSuccess ||
        cudaMemcpy2DAsync(h_minima, out_pitch, c->d_minima, width, width,
                          height, cudaMemcpyDeviceToHost,
                          c->stream) != cudaSuccess) {
        return SS_ERR_CUDA;
    }
    ss_stats stats;
    st = ss_read_status(c->d_workspace, c->workspace_capacity, c->stream,
                        &stats);
    if (st != SS_OK) {
        ss_workspace_init(c->d_workspace, c->workspace_capacity, c->stream);
        return st;
    }
    if (elapsed_ms) {
        if (cudaEventElapsedTime(elapsed_ms, c->start, c->stop) !=
            cudaSuccess) {
            return SS_ERR_CUDA;
        }
    }
    if (active_fragments) {
        *active_fragments = stats.active_fragments;
    }
    return SS_OK;
}

}  // extern "C"

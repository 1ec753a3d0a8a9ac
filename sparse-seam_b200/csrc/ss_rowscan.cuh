// ss_rowscan.cuh -- the row-scan route (tile edge 32, the reference's
// reported setting, and 64): shared definitions and the passes after the
// tile pass, templated on the tile edge.  The tile pass itself (per-row bit
// masks and runs; one warp per 32 x 32 tile or quadrant) is ss_runs.cuh.
//
// Observation the design rests on: a pixel with both a strictly greater and a
// strictly smaller 8-neighbour ("decided" pixel) is in neither mask, and
// neither is any pixel of its flat zone (the zone's flags are the OR of its
// pixels').  On natural images most pixels are decided, so only the others
// need connectivity.  Zones inside a tile are settled by the tile pass; zones
// touching a seam (an equal 8-neighbour outside the tile) whose flags are not
// both set ("live" zones) become fragments: per tile, records 0..k-1, their
// border pixels' records, equal pairs across the seams ("seam items") and a
// log of their pixel runs.
//
// Seam pass, one warp per `group` tiles: every seam item links the two live
//   fragments (union-find over all fragments of the launch), or marks a live
//   fragment whose partner across the seam is decided.
// Flags pass: every fragment ORs its flags into its component's root.
// Resolve pass: every logged run gets its component's verdict; the tile
//   pass left its bytes at 0 in both masks, so only the bytes that become
//   255 are written: byte-parallel for sparse tiles, word ORs for dense.
//
// Reference behaviour followed (paths inside the reference repository):
// zone flags and seam test, harness/primary/snapshot_sparse_seam_cuda_v1_0.cu
// :340-390; per-tile fragment records, :392-410; cross-seam merge of equal
// 8-adjacent border pixels, :508-581; global union-find, :132-160 and its
// flag reduction, :583-619; masks from the resolved flags, :477-506.
#pragma once

#include <type_traits>

#include "ss_device.cuh"

namespace ss {

namespace rowscan {

constexpr int T = 32;                  // the warp's square (a quadrant at
                                       //   tile edge 64)
constexpr int kSlots = 4 * T;          // fragment slots per tile
constexpr int kPendingCap = T * T;     // run-log entries per tile
constexpr int kHaloW = T + 2;          // staged row: columns x0-1 .. x0+T
constexpr int kSeamCap = 12 * T;       // seam items per tile

// Per tile edge TT (32, or 64 = 2 x 2 warp squares): fragment slots (4 TT,
// the reference's SLOTS_PER_TILE), run-log entries and seam items per tile,
// and the row-mask type of the resolve pass.
template <int TT>
struct Edge {
    static constexpr int kSlots = 4 * TT;
    static constexpr int kPendingCap = TT * TT;
    static constexpr int kSeamCap = 12 * TT;
    using Row = typename std::conditional<TT == 64, unsigned long long,
                                          uint32_t>::type;
};
// Loop runs the tile pass lists in the staged tile's shared memory (the
// list's 2-byte entries, then three 32-word row arrays, fit its 2316 bytes).
constexpr int kListCap = 960;
constexpr uint32_t kDeadRecord = 0xFEu;  // border record of a decided zone
constexpr uint32_t kNoRecord = 0xFFu;    // border pixel of an inside zone
// Resolve pass: tiles with at most this many logged runs are written run by
// run; denser tiles row by row.
constexpr uint32_t kSparseRuns = 16u;

// Union-find word of a run head in the tile pass: bits 0-11 parent (XOR
// the word's own index, so an all-zero word is a root), 12-14 zone flags
// (at roots), 15-22 record + 1 (at roots of live seam zones, and at the
// head words of their logged runs).  Indices reach 4095 at tile edge 64.
constexpr uint32_t kParMask = 0xFFFu;
constexpr int kZoneShift = 12;
constexpr int kRecShift = 15;
constexpr uint32_t kDead = kHasGreater | kHasSmaller;

// Seam item of a tile: bits 0-7 own record, 8-14 the neighbour's border
// offset (its record array index), 16-18 neighbour direction (kRel*).

// Run-log entry: bits 0-7 record, 8-13 x, 14-19 y, 20-26 length.
__device__ __forceinline__ uint32_t pending_entry(int rec, int x, int y,
                                                  int len) {
    return static_cast<uint32_t>(rec) | (static_cast<uint32_t>(x) << 8) |
           (static_cast<uint32_t>(y) << 14) |
           (static_cast<uint32_t>(len) << 20);
}

struct TileGeom {
    int x0, y0, tw, th;
};

template <int TT = T>
__device__ __forceinline__ TileGeom tile_geom(const PlanImage& job,
                                              int64_t local) {
    TileGeom g;
    // A 32-bit divide: a launch holds fewer than 2^31 / (4 T) tiles (its
    // workspace refuses more, fragment ids being 32-bit).
    const uint32_t l = static_cast<uint32_t>(local);
    const uint32_t n = static_cast<uint32_t>(job.tiles_x);
    const int ty = static_cast<int>(l / n);
    const int tx = static_cast<int>(l - static_cast<uint32_t>(ty) * n);
    g.x0 = tx * TT;
    g.y0 = ty * TT;
    g.tw = min(TT, job.width - g.x0);
    g.th = min(TT, job.height - g.y0);
    return g;
}

__device__ __forceinline__ PlanImage load_job(const Source& src,
                                              int64_t item) {
    if (!src.images) {
        return src.single;
    }
    const int idx = __ldg(src.tile_image + item);
    return src.images[idx];
}

// Bits 0..x of a 32-bit row mask (x in 0..31).
__device__ __forceinline__ uint32_t le_mask_of(int x) {
    return (2u << x) - 1u;
}

// ---------------------------------------------------------------------------
// Seam and resolve passes: one warp per `group` consecutive tiles (1..32,
// chosen by the launch so the grid fills the GPU), work flattened over the
// tiles so the global round trips of many tiles overlap.
// ---------------------------------------------------------------------------

// Exclusive prefix of `v` over the warp; `total` receives the sum.
__device__ __forceinline__ uint32_t warp_prefix(uint32_t v, uint32_t& total) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t n = __shfl_up_sync(~0u, incl, o);
        if (lane >= o) incl += n;
    }
    total = __shfl_sync(~0u, incl, 31);
    return incl - v;
}

// The lane whose [excl, excl + count) range holds flat index f (all lanes
// call it together; f may differ per lane).
__device__ __forceinline__ int owner_of(uint32_t excl, uint32_t f) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const uint32_t probe = __shfl_sync(~0u, excl, lo + step);
        if (probe <= f) lo += step;
    }
    return lo;
}

__device__ __forceinline__ int64_t neighbour_tile(int64_t g, int dir,
                                                  int64_t tiles_x) {
    switch (dir) {
        case kRelLeft: return g - 1;
        case kRelTop: return g - tiles_x;
        case kRelTopLeft: return g - tiles_x - 1;
        case kRelTopRight: return g - tiles_x + 1;
        case kRelRight: return g + 1;
        case kRelBottom: return g + tiles_x;
        case kRelBottomRight: return g + tiles_x + 1;
        default: return g + tiles_x - 1;
    }
}

// Passes after the tile pass: one CTA of `nwarps` warps per group of
// `src.group` consecutive tiles (lane = tile of the group); the group's work
// is flattened and its 32-wide steps are dealt out to the warps, so a group
// of dense tiles is shared by all the CTA's warps.
template <int TT>
__device__ __forceinline__ void seam_pass_group(const Source& src,
                                                const Arena& a, int64_t first,
                                                int warp, int nwarps) {
    constexpr int kSlots = Edge<TT>::kSlots;
    constexpr int kSeamCap = Edge<TT>::kSeamCap;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int64_t tile = first + lane;
    const bool valid = lane < src.group && tile < src.total_tiles;
    const uint32_t count =
        valid ? min(__ldg(a.seam_count + tile), static_cast<uint32_t>(kSeamCap))
              : 0u;
    uint32_t total = 0;
    const uint32_t excl = warp_prefix(count, total);
    if (total == 0) {
        return;
    }
    int64_t tiles_x = 0;
    if (count) {
        tiles_x = load_job(src, tile).tiles_x;
    }
    uint32_t err = 0;
    for (uint32_t base = 32u * warp; base < total; base += 32u * nwarps) {
        const uint32_t f = base + static_cast<uint32_t>(lane);
        const int owner = owner_of(excl, f);
        const int64_t g = first + owner;
        const int64_t tx = __shfl_sync(~0u, tiles_x, owner);
        const uint32_t j = f - __shfl_sync(~0u, excl, owner);
        // What the item asks for: unite fragment fo with fragment `target`,
        // or (target == -1) OR "both flags" into fo.
        int fo = -1;
        int target = -2;
        if (f < total) {
            const uint32_t it = __ldcg(a.seam_items + g * kSeamCap + j);
            const uint32_t rec = it & 0xFFu;
            const int off = static_cast<int>((it >> 8) & 0xFFu);
            const int dir = static_cast<int>((it >> 16) & 7u);
            const int64_t ng = neighbour_tile(g, dir, tx);
            if (rec >= static_cast<uint32_t>(kSlots) || ng < 0 ||
                ng >= src.total_tiles) {
                err = kErrRecordRange;
            } else {
                const uint32_t rn = __ldg(a.border + ng * kSlots + off);
                if (rn == kDeadRecord) {
                    fo = static_cast<int>(g * kSlots + rec);
                    target = -1;
                } else if (rn < static_cast<uint32_t>(kSlots)) {
                    // Both pixels live: the neighbour tile holds the mirror
                    // item (its pixel is live and equal to this one, and its
                    // streaks keep at least one pair per zone pair and
                    // direction, as this tile's do), so only the items facing
                    // a later tile (right, bottom and the bottom corners)
                    // link; the others would repeat the same unions.
                    if (dir >= kRelRight) {
                        fo = static_cast<int>(g * kSlots + rec);
                        target = static_cast<int>(ng * kSlots + rn);
                    }
                } else {
                    err = kErrInvariant;   // equal across a seam, no seam zone
                }
            }
        }
        // Neighbouring border pixels of one zone pair repeat the same request
        // (items are stored in border order): only the first of a streak
        // acts.
        const int prev_fo = __shfl_up_sync(~0u, fo, 1);
        const int prev_target = __shfl_up_sync(~0u, target, 1);
        const bool repeat = lane > 0 && prev_fo == fo && prev_target == target;
        if (fo >= 0 && !repeat) {
            if (target == -1) {
                // The fragment's own word; the flags pass carries it to the
                // component's root.
                atomicOr(a.bits + fo, kDead);
            } else {
                global_link(a.parent, fo, target, err);
            }
        }
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(first));
    }
}

// Flags pass (after the seam pass, before the resolve pass): every live
// fragment ORs its flags (its zone's flags and the "decided neighbour across
// a seam" marks of the seam pass) into its component's root.  The kernel
// boundaries order it after every link and before every read of a root.
template <int TT>
__device__ __forceinline__ void flags_pass_group(const Source& src,
                                                 const Arena& a, int64_t first,
                                                 int warp, int nwarps) {
    constexpr int kSlots = Edge<TT>::kSlots;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int64_t tile = first + lane;
    const bool valid = lane < src.group && tile < src.total_tiles;
    const uint32_t k =
        valid ? min(static_cast<uint32_t>(a.fragment_count[tile]),
                    static_cast<uint32_t>(kSlots))
              : 0u;
    uint32_t total = 0;
    const uint32_t excl = warp_prefix(k, total);
    uint32_t err = 0;
    for (uint32_t base = 32u * warp; base < total; base += 32u * nwarps) {
        const uint32_t f = base + static_cast<uint32_t>(lane);
        const int owner = owner_of(excl, f);
        const uint32_t r = f - __shfl_sync(~0u, excl, owner);
        if (f < total) {
            const int fr = static_cast<int>((first + owner) * kSlots + r);
            const int root = global_find(a.parent, fr, err);
            if (root != fr) {
                // Pointing a fragment at its root is safe at any time after
                // the links: every reader sees an ancestor either way.
                if (src.flatten != kFlattenHalve) {
                    st_relaxed(a.parent + fr, root);
                }
                if (src.flatten != kFlattenOnly) {
                    const uint32_t own = ld_relaxed(a.bits + fr) & 3u;
                    if (own && (ld_relaxed(a.bits + root) & own) != own) {
                        atomicOr(a.bits + root, own);
                    }
                }
            }
        }
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(first));
    }
}

// Bytes 0x00 / 0xFF of the low 4 bits of `bits` (bit i -> byte i): the
// product adds copies of the 4 bits shifted by 0, 7, 14 and 21, which puts
// bit i at bit 8i (the copies do not overlap, so nothing carries); the mask
// keeps bits 0, 8, 16 and 24, and the multiply by 0xFF fills each byte.
__device__ __forceinline__ uint32_t spread4(uint32_t bits) {
    return (((bits & 15u) * 0x00204081u) & 0x01010101u) * 0xFFu;
}

// Warps per CTA of the seam, flags and resolve passes.
constexpr int kLaterWarps = 8;

template <int TT>
struct __align__(16) ResolveSmem {
    using Row = typename Edge<TT>::Row;
    uint8_t final_flags[32][Edge<TT>::kSlots];  // the group's fragments'
                                                //   verdicts
    uint8_t* maxima[32];
    uint8_t* minima[32];
    int64_t out_origin[32];   // offset of the tile's pixel (0, 0)
    int32_t out_pitch[32];
    int16_t tw[32];
    int16_t th[32];
    // Per warp, one dense tile at a time: the logged pixels per row whose
    // maxima / minima byte is 255.
    Row vmax[kLaterWarps][TT];
    Row vmin[kLaterWarps][TT];
    uint32_t flipped;         // tiles (bits of the group) with a verdict
                              //   other than their tile-local one
};

// Sets the mask bytes of a full tile's logged pixels whose verdict is 255
// (rows and origin on 4-byte boundaries), from per-row bit masks: the tile
// pass left every logged byte at 0, so ORing 0xFF into the bytes of each
// 4-byte word that need it is the whole rewrite, one reduction per word
// with any such byte and no read of the rows.
template <int TT, typename Row>
__device__ __forceinline__ void or_rows(uint8_t* omax, uint8_t* omin,
                                        int64_t pitch, const Row* vmax,
                                        const Row* vmin) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    constexpr int kWords = TT / 4;   // 4-byte words per row
    for (int i = lane; i < TT * kWords; i += 32) {
        const int r = i / kWords;
        const int w = i % kWords;
        const uint32_t bx = static_cast<uint32_t>(vmax[r] >> (4 * w)) & 15u;
        const uint32_t bn = static_cast<uint32_t>(vmin[r] >> (4 * w)) & 15u;
        const int64_t o = static_cast<int64_t>(r) * pitch + 4 * w;
        if (bx) {
            atomicOr(reinterpret_cast<uint32_t*>(omax + o), spread4(bx));
        }
        if (bn) {
            atomicOr(reinterpret_cast<uint32_t*>(omin + o), spread4(bn));
        }
    }
}

// Called by every warp of the CTA with the same `first`; contains
// __syncthreads, so all of the CTA's threads must call it.
template <int TT>
__device__ __forceinline__ void resolve_group(ResolveSmem<TT>& sm,
                                              const Source& src,
                                              const Arena& a, int64_t first,
                                              int warp, int nwarps) {
    using Row = typename Edge<TT>::Row;
    constexpr int kSlots = Edge<TT>::kSlots;
    constexpr int kPendingCap = Edge<TT>::kPendingCap;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int64_t tile = first + lane;
    const bool valid = lane < src.group && tile < src.total_tiles;
    const uint32_t n =
        valid ? min(a.pending_count[tile] & 0xFFFFu,
                    static_cast<uint32_t>(kPendingCap))
              : 0u;
    const uint32_t k = n ? min(static_cast<uint32_t>(a.fragment_count[tile]),
                               static_cast<uint32_t>(kSlots))
                         : 0u;
    uint32_t total_n = 0;
    uint32_t total_k = 0;
    const uint32_t excl_n = warp_prefix(n, total_n);
    const uint32_t excl_k = warp_prefix(k, total_k);
    if (total_n == 0) {
        return;
    }
    uint32_t err = 0;
    if (warp == 0 && n) {
        const PlanImage job = load_job(src, tile);
        const TileGeom g = tile_geom<TT>(job, tile - job.tile_base);
        sm.maxima[lane] = job.maxima;
        sm.minima[lane] = job.minima;
        sm.out_origin[lane] =
            static_cast<int64_t>(g.y0) * job.out_pitch + g.x0;
        sm.out_pitch[lane] = job.out_pitch;
        sm.tw[lane] = static_cast<int16_t>(g.tw);
        sm.th[lane] = static_cast<int16_t>(g.th);
    }
    if (warp == 0 && lane == 0) {
        sm.flipped = 0u;
    }
    __syncthreads();
    // Component flags of every live fragment of these tiles.
    uint32_t flipped = 0u;
    for (uint32_t base = 32u * warp; base < total_k; base += 32u * nwarps) {
        const uint32_t f = base + static_cast<uint32_t>(lane);
        const int owner = owner_of(excl_k, f);
        const uint32_t r = f - __shfl_sync(~0u, excl_k, owner);
        if (f < total_k) {
            const int fr = static_cast<int>((first + owner) * kSlots + r);
            const int root = global_find(a.parent, fr, err);
            const uint32_t comp = ld_relaxed(a.bits + root) & 3u;
            const uint32_t own = (ld_relaxed(a.bits + fr) >> kLocalShift) & 3u;
            sm.final_flags[owner][r] = static_cast<uint8_t>(comp);
            if (comp != own) {
                flipped |= 1u << owner;
            }
        }
    }
    flipped = __reduce_or_sync(~0u, flipped);
    if (lane == 0 && flipped) {
        atomicOr(&sm.flipped, flipped);
    }
    __syncthreads();
    // Tiles with few logged runs: all of the group's runs together, their
    // bytes spread over the lanes (consecutive lanes write consecutive bytes
    // of a run).
    const uint32_t n_sparse = n <= kSparseRuns ? n : 0u;
    uint32_t total_sparse = 0u;
    const uint32_t excl_s = warp_prefix(n_sparse, total_sparse);
    for (uint32_t base = 32u * warp; base < total_sparse;
         base += 32u * nwarps) {
        const uint32_t e = base + static_cast<uint32_t>(lane);
        const int owner = owner_of(excl_s, e);
        const uint32_t j = e - __shfl_sync(~0u, excl_s, owner);
        const uint32_t kown = __shfl_sync(~0u, k, owner);
        uint32_t len = 0u;
        int64_t off = 0;
        uint32_t verdict = 0u;
        if (e < total_sparse) {
            const uint32_t ent =
                __ldcg(a.pending + (first + owner) * kPendingCap + j);
            const uint32_t rec = ent & 0xFFu;
            const int x = static_cast<int>((ent >> 8) & 63u);
            const int y = static_cast<int>((ent >> 14) & 63u);
            const int n_px = static_cast<int>((ent >> 20) & 127u);
            if (rec >= kown || x + n_px > sm.tw[owner] || y >= sm.th[owner] ||
                n_px == 0) {
                err = kErrRecordRange;
            } else {
                const uint32_t fl = sm.final_flags[owner][rec];
                verdict = ((fl & kHasGreater) ? 0u : 0xFFu) |
                          ((fl & kHasSmaller) ? 0u : 0xFF00u);
                off = sm.out_origin[owner] +
                      static_cast<int64_t>(y) * sm.out_pitch[owner] + x;
                // A zone in neither mask keeps the tile pass's placeholder
                // bytes (0, 0): nothing to write.
                len = verdict ? static_cast<uint32_t>(n_px) : 0u;
            }
        }
        uint32_t bytes = 0u;
        const uint32_t excl_len = warp_prefix(len, bytes);
        for (uint32_t b0 = 0; b0 < bytes; b0 += 32) {
            const uint32_t bi = b0 + static_cast<uint32_t>(lane);
            const int src_lane = owner_of(excl_len, bi);
            const int tile_of = __shfl_sync(~0u, owner, src_lane);
            const int64_t o = __shfl_sync(~0u, off, src_lane) +
                              (bi - __shfl_sync(~0u, excl_len, src_lane));
            const uint32_t vd = __shfl_sync(~0u, verdict, src_lane);
            // The tile pass left both bytes at 0: only a 255 is written.
            if (bi < bytes) {
                if (vd & 0xFFu) {
                    sm.maxima[tile_of][o] = 0xFF;
                }
                if (vd & 0xFF00u) {
                    sm.minima[tile_of][o] = 0xFF;
                }
            }
        }
    }
    // Tiles with many logged runs, dealt out to the warps one tile at a
    // time: the pixels whose maxima / minima byte becomes 255 as row masks,
    // then those bytes set.
    const uint32_t dense = __ballot_sync(~0u, n > kSparseRuns);
    Row* vmax_rows = sm.vmax[warp];
    Row* vmin_rows = sm.vmin[warp];
    int rank = 0;
    for (uint32_t d = dense; d; d &= d - 1u, ++rank) {
        if (rank % nwarps != warp) {
            continue;
        }
        const int t = __ffs(d) - 1;
        const uint32_t nt = __shfl_sync(~0u, n, t);
        const uint32_t kt = __shfl_sync(~0u, k, t);
        for (int r = lane; r < TT; r += 32) {
            vmax_rows[r] = 0u;
            vmin_rows[r] = 0u;
        }
        __syncwarp();
        const int tw = sm.tw[t];
        const int th = sm.th[t];
        const uint32_t* plog = a.pending + (first + t) * kPendingCap;
        for (uint32_t e = static_cast<uint32_t>(lane); e < nt; e += 32u) {
            const uint32_t ent = __ldcg(plog + e);
            const uint32_t rec = ent & 0xFFu;
            const int x = static_cast<int>((ent >> 8) & 63u);
            const int y = static_cast<int>((ent >> 14) & 63u);
            const int n_px = static_cast<int>((ent >> 20) & 127u);
            if (rec >= kt || x + n_px > tw || y >= th || n_px == 0) {
                err = kErrRecordRange;
                continue;
            }
            const uint32_t fl = sm.final_flags[t][rec];
            if ((fl & kDead) == kDead) {
                continue;   // in neither mask: the placeholder bytes stand
            }
            const Row R = ((Row(2) << (x + n_px - 1)) - Row(1)) &
                          ~((Row(1) << x) - Row(1));
            if (!(fl & kHasGreater)) {
                atomicOr(&vmax_rows[y], R);
            }
            if (!(fl & kHasSmaller)) {
                atomicOr(&vmin_rows[y], R);
            }
        }
        __syncwarp();
        uint8_t* omax = sm.maxima[t] + sm.out_origin[t];
        uint8_t* omin = sm.minima[t] + sm.out_origin[t];
        const int64_t pitch = sm.out_pitch[t];
        const uint64_t align = reinterpret_cast<uint64_t>(omax) |
                               reinterpret_cast<uint64_t>(omin) |
                               static_cast<uint64_t>(pitch);
        // Whole 4-byte words only inside a full tile: a partial tile's last
        // word may reach past the image's row (and buffer) end.
        if ((align & 3u) == 0 && tw == TT && th == TT) {
            or_rows<TT>(omax, omin, pitch, vmax_rows, vmin_rows);
        } else {
            for (int r = 0; r < th; ++r) {
                for (int x = lane; x < TT; x += 32) {
                    const int64_t o = static_cast<int64_t>(r) * pitch + x;
                    if ((vmax_rows[r] >> x) & 1u) {
                        omax[o] = 255;
                    }
                    if ((vmin_rows[r] >> x) & 1u) {
                        omin[o] = 255;
                    }
                }
            }
        }
        __syncwarp();
    }
    if (warp == 0 && lane == 0 && sm.flipped) {
        atomicAdd(&a.header->flipped_tiles, __popc(sm.flipped));
    }
    // The shared arrays may be reused by the CTA's next group.
    __syncthreads();
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(first));
    }
}

}  // namespace rowscan

}  // namespace ss

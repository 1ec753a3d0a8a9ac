// ss_rowscan.cuh -- the T = 32 route (the reference's reported tile size):
// a warp-per-tile tile pass, a seam pass and a list-driven resolve pass.
//
// Observation the design rests on: a pixel with both a strictly greater and a
// strictly smaller 8-neighbour ("decided" pixel) is in neither mask, and
// neither is any pixel of its flat zone (the zone's flags are the OR of its
// pixels').  On natural images most pixels are decided, so only the others
// need connectivity.
//
// Tile pass, one warp per 32 x 32 tile:
//   prologue  the tile and its one-pixel halo are loaded (all loads in
//             flight at once) and staged in shared memory as int16, -1
//             outside the image;
//   phase A   row scan, lane = column: greater / smaller flags from sliding
//             3 x 3 row maxima / minima (a signed max and an unsigned min
//             both ignore -1); decided pixels get both masks 0 at once; the
//             others ("listed") are appended in pixel order to a per-warp
//             list; per row, ballots record which pixels are listed and which
//             continue a listed run of equal pixels from the left;
//   phase C   dense over the list: flags, "seam" (an equal 8-neighbour outside
//             the tile), "dead" (an equal decided neighbour inside the tile:
//             the zone is decided too), and links.  A run member's parent is
//             its run head; one union per pair of 8-adjacent equal runs in
//             consecutive rows, issued at the first column of the pair's
//             contact (three cases, see phase C);
//   phase D   flatten; zone flags ORed into the roots, one atomic per root
//             and warp step (lanes grouped by root with __match_any_sync);
//   phase E   in pixel order: live seam zones (touching a seam, flags not
//             both set) get fragment records 0..k-1 and are logged as runs;
//             the other listed pixels get their masks;
//   phase F   border records: each border pixel's fragment record, or
//             kDeadRecord when its zone is decided; and the equalities across
//             this tile's right and bottom seams, for the seam pass.
// Seam pass, one warp per tile: every equal pair across the seams the tile
//   owns (right, bottom, bottom-right, bottom-left) unites the two live
//   fragments, or ORs "both flags" into a live fragment whose partner is dead.
// Resolve pass, one warp per tile: looks up every live fragment's component
//   flags and writes the logged runs; every mask byte is written once.
//
// Reference behaviour followed (paths inside the reference repository):
// zone flags and seam test, harness/primary/snapshot_sparse_seam_cuda_v1_0.cu
// :340-390; per-tile fragment records, :392-410; cross-seam merge of equal
// 8-adjacent border pixels, :508-581; masks from the resolved flags, :477-506.
#pragma once

#include "ss_device.cuh"

namespace ss {

namespace rowscan {

constexpr int T = 32;
constexpr int kSlots = 4 * T;          // fragment slots per tile
constexpr int kPendingCap = T * T;     // run-log entries per tile
constexpr int kHaloW = T + 2;          // staged row: columns x0-1 .. x0+T
constexpr int kSeamCap = 12 * T;       // seam items per tile
constexpr uint32_t kDeadRecord = 0xFEu;  // border record of a decided zone
constexpr uint32_t kNoRecord = 0xFFu;    // border pixel of an inside zone
// Resolve pass: tiles with at most this many logged runs are written run by
// run; denser tiles row by row.
constexpr uint32_t kSparseRuns = 16u;

// Per-pixel shared word: bits 0-9 parent, 10-12 zone flags (at roots),
// 13-20 record + 1 (at roots of live seam zones), 21-23 own flags.
constexpr uint32_t kParMask = 0x3FFu;
constexpr int kZoneShift = 10;
constexpr int kRecShift = 13;
constexpr int kOwnShift = 21;
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

struct __align__(16) WarpSmem {
    uint32_t word[T * T];
    uint16_t list[T * T];          // listed pixels, in pixel order
    uint32_t listed[T];            // per row: listed pixels
    uint32_t cont[T];              // per row: listed run continuations
    int16_t img[kHaloW * kHaloW];  // tile + halo, -1 outside the image
};

struct TileGeom {
    int x0, y0, tw, th;
};

__device__ __forceinline__ TileGeom tile_geom(const PlanImage& job,
                                              int64_t local) {
    TileGeom g;
    const int ty = static_cast<int>(local / job.tiles_x);
    const int tx =
        static_cast<int>(local - static_cast<int64_t>(ty) * job.tiles_x);
    g.x0 = tx * T;
    g.y0 = ty * T;
    g.tw = min(T, job.width - g.x0);
    g.th = min(T, job.height - g.y0);
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

// Find with path halving, used while linking (phase C): then a non-root
// word changes only in its parent bits, and halving rewrites those bits with
// an ancestor, which is safe under concurrent linking and halving.
__device__ __forceinline__ int wfind(volatile uint32_t* w, int x,
                                     uint32_t& err) {
#pragma unroll 1
    for (int it = 0; it < T * T; ++it) {
        const uint32_t wx = w[x];
        const int p = static_cast<int>(wx & kParMask);
        if (p == x) {
            return x;
        }
        const int gp = static_cast<int>(w[p] & kParMask);
        if (gp == p) {
            return p;
        }
        w[x] = (wx & ~kParMask) | static_cast<uint32_t>(gp);
        x = gp;
    }
    err = kErrSpinLimit;
    return x;
}

// Links the larger root below the smaller one (CAS on the whole word).
__device__ __forceinline__ void wunion(uint32_t* w_, int a, int b,
                                       uint32_t& err) {
    volatile uint32_t* w = w_;
#pragma unroll 1
    for (int it = 0; it < 4 * T * T; ++it) {
        a = wfind(w, a, err);
        b = wfind(w, b, err);
        if (a == b || err) {
            return;
        }
        const int hi = a > b ? a : b;
        const int lo = a > b ? b : a;
        const uint32_t cur = w[hi];
        if (static_cast<int>(cur & kParMask) != hi) {
            continue;
        }
        const uint32_t next = (cur & ~kParMask) | static_cast<uint32_t>(lo);
        if (atomicCAS(w_ + hi, cur, next) == cur) {
            return;
        }
    }
    err = kErrSpinLimit;
}

// ---------------------------------------------------------------------------
// Tile pass (one warp, one tile)
// ---------------------------------------------------------------------------

__device__ __forceinline__ void tile_pass_warp(WarpSmem& sm, const Source& src,
                                               const Arena& a, int64_t item) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t le_mask = lt_mask | (1u << lane);
    uint32_t err = 0;

    const PlanImage job = load_job(src, item);
    const TileGeom g = tile_geom(job, item - job.tile_base);
    const uint8_t* __restrict__ img = job.image;
    const int64_t pitch = job.pitch;
    const int width = job.width;
    const int height = job.height;
    const int64_t out_pitch = job.out_pitch;
    uint8_t* __restrict__ omax = job.maxima;
    uint8_t* __restrict__ omin = job.minima;

    // -- prologue: stage the tile and its halo --------------------------------
    // Staged row r holds image row y0 - 1 + r, staged column c image column
    // x0 - 1 + c.
    {
        const int gx = g.x0 + lane;
        const bool col_ok = lane < g.tw;
        int vals[T + 2];
#pragma unroll
        for (int r = 0; r < T + 2; ++r) {
            const int gy = g.y0 + r - 1;
            vals[r] = (col_ok && static_cast<unsigned>(gy) <
                                     static_cast<unsigned>(height))
                          ? static_cast<int>(__ldg(img + gy * pitch + gx))
                          : -1;
        }
        const int xl = g.x0 - 1;
        const int xr = g.x0 + T;
        const int gy0 = g.y0 - 1 + lane;
        const int gy1 = g.y0 + 31 + lane;
        const bool ok0 =
            static_cast<unsigned>(gy0) < static_cast<unsigned>(height);
        const bool ok1 = lane < 2 && static_cast<unsigned>(gy1) <
                                         static_cast<unsigned>(height);
        const int hl0 = (xl >= 0 && ok0)
                            ? static_cast<int>(__ldg(img + gy0 * pitch + xl))
                            : -1;
        const int hr0 = (xr < width && ok0)
                            ? static_cast<int>(__ldg(img + gy0 * pitch + xr))
                            : -1;
        const int hl1 = (xl >= 0 && ok1)
                            ? static_cast<int>(__ldg(img + gy1 * pitch + xl))
                            : -1;
        const int hr1 = (xr < width && ok1)
                            ? static_cast<int>(__ldg(img + gy1 * pitch + xr))
                            : -1;
#pragma unroll
        for (int r = 0; r < T + 2; ++r) {
            sm.img[r * kHaloW + lane + 1] = static_cast<int16_t>(vals[r]);
        }
        sm.img[lane * kHaloW] = static_cast<int16_t>(hl0);
        sm.img[lane * kHaloW + kHaloW - 1] = static_cast<int16_t>(hr0);
        if (lane < 2) {
            sm.img[(32 + lane) * kHaloW] = static_cast<int16_t>(hl1);
            sm.img[(32 + lane) * kHaloW + kHaloW - 1] =
                static_cast<int16_t>(hr1);
        }
    }
    __syncwarp();

    // -- phase A: flags, decided pixels, list, runs ----------------------------
    const bool col_ok = lane < g.tw;
    const int16_t* scol = sm.img + lane;   // staged columns lane .. lane + 2
    int Lc = scol[kHaloW];
    int vc = scol[kHaloW + 1];
    int Rc = scol[kHaloW + 2];
    int hmax_p = max(max(static_cast<int>(scol[0]), static_cast<int>(scol[1])),
                     static_cast<int>(scol[2]));
    unsigned hmin_p = min(min(static_cast<unsigned>(scol[0]),
                              static_cast<unsigned>(scol[1])),
                          static_cast<unsigned>(scol[2]));
    int hmax_c = max(max(Lc, vc), Rc);
    unsigned hmin_c = min(min(static_cast<unsigned>(Lc), static_cast<unsigned>(vc)),
                          static_cast<unsigned>(Rc));
    int nlist = 0;
    uint8_t* omax_row =
        omax + static_cast<int64_t>(g.y0) * out_pitch + g.x0 + lane;
    uint8_t* omin_row =
        omin + static_cast<int64_t>(g.y0) * out_pitch + g.x0 + lane;
#pragma unroll 2
    for (int y = 0; y < g.th; ++y) {
        const int16_t* nrow = scol + (y + 2) * kHaloW;
        const int Ln = nrow[0];
        const int vn = nrow[1];
        const int Rn = nrow[2];
        const int hmax_n = max(max(Ln, vn), Rn);
        const unsigned hmin_n =
            min(min(static_cast<unsigned>(Ln), static_cast<unsigned>(vn)),
                static_cast<unsigned>(Rn));
        const int mx = max(max(hmax_p, hmax_n), max(Lc, Rc));
        const unsigned mn = min(min(hmin_p, hmin_n),
                                min(static_cast<unsigned>(Lc),
                                    static_cast<unsigned>(Rc)));
        const bool gt = mx > vc;
        const bool lt = mn < static_cast<unsigned>(vc);
        const bool decided = col_ok && gt && lt;
        if (decided) {
            *omax_row = 0;
            *omin_row = 0;
        }
        omax_row += out_pitch;
        omin_row += out_pitch;
        const bool listed = col_ok && !decided;
        const uint32_t b = __ballot_sync(~0u, listed);
        if (listed) {
            // Entry: pixel index, then its greater / smaller flags.
            sm.list[nlist + __popc(b & lt_mask)] = static_cast<uint16_t>(
                (y * T + lane) | (gt ? 1u << 10 : 0u) | (lt ? 1u << 11 : 0u));
        }
        nlist += __popc(b);
        const bool cont = listed && lane > 0 && Lc == vc &&
                          ((b >> (lane - 1)) & 1u);
        const uint32_t cb = __ballot_sync(~0u, cont);
        if (lane == 0) {
            sm.listed[y] = b;
            sm.cont[y] = cb;
        }
        hmax_p = hmax_c;
        hmin_p = hmin_c;
        hmax_c = hmax_n;
        hmin_c = hmin_n;
        vc = vn;
        Lc = Ln;
        Rc = Rn;
    }
    __syncwarp();

    // -- phase C: flags, seam, dead, links of listed pixels -------------------
    // Run R (value v) in row y is 8-adjacent to every listed run of row y-1
    // with a pixel equal to v in columns [head - 1, end + 1]; those pixels form
    // one segment per such run, and each segment's first column is hit by
    // exactly one of: (a) a pixel x of R with eq-up and not eq-up-left, (b)
    // the head of R with eq-up-left, (c) the end of R with eq-up-right and not
    // eq-up ("eq" meaning equal and listed).
    // The 3 x 3 window is handled as bit sets, bit n = 3 * (dy + 1) + (dx + 1)
    // (centre bit 4 unused): which neighbours are equal, which lie outside
    // the tile, which are listed.
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        const bool active = i < nlist;
        int p = 0;
        int t1 = -1;
        int t2 = -1;
        if (active) {
            const uint32_t ent = sm.list[i];
            p = static_cast<int>(ent & 1023u);
            const int x = p & 31;
            const int y = p >> 5;
            const int16_t* w0 = sm.img + y * kHaloW + x;   // (x-1, y-1)
            const int v = w0[kHaloW + 1];
            uint32_t eq = 0u;
#pragma unroll
            for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    if (dy == 1 && dx == 1) continue;
                    eq |= (static_cast<int>(w0[dy * kHaloW + dx]) == v)
                              ? 1u << (dy * 3 + dx) : 0u;
                }
            }
            const uint64_t up = y > 0 ? sm.listed[y - 1] : 0u;
            const uint64_t cur = sm.listed[y];
            const uint64_t dn = y + 1 < g.th ? sm.listed[y + 1] : 0u;
            // Column x - 1 .. x + 1 of a row mask as 3 bits (column -1 and
            // column 32 read as unlisted).
            const uint32_t lw =
                static_cast<uint32_t>(((up << 1) >> x) & 7u) |
                (static_cast<uint32_t>(((cur << 1) >> x) & 7u) << 3) |
                (static_cast<uint32_t>(((dn << 1) >> x) & 7u) << 6);
            const uint32_t outside = (x == 0 ? 0x049u : 0u) |
                                     (x == T - 1 ? 0x124u : 0u) |
                                     (y == 0 ? 0x007u : 0u) |
                                     (y == T - 1 ? 0x1C0u : 0u);
            const bool seam = (eq & outside) != 0u;
            const bool dead = (eq & ~outside & ~lw) != 0u;
            const uint32_t eql = eq & lw & ~outside;   // equal and listed
            const bool eUL = eql & 1u;
            const bool eU = (eql >> 1) & 1u;
            const bool eUR = (eql >> 2) & 1u;
            const uint32_t cont_row = sm.cont[y];
            const uint32_t heads = static_cast<uint32_t>(cur) & ~cont_row;
            const int head = 31 - __clz(heads & le_mask_of(x));
            const bool is_end = x == T - 1 || !((cont_row >> (x + 1)) & 1u);
            if (eU && !eUL) {
                t1 = p - T;
            } else if (x == head && eUL) {
                t1 = p - T - 1;
            }
            if (is_end && eUR && !eU) {
                t2 = p - T + 1;
            }
            const int parent = x == head ? p : y * T + head;
            const uint32_t own = ((ent >> 10) & 3u) | (dead ? kDead : 0u) |
                                 (seam ? kTouchesSeam : 0u);
            sm.word[p] = static_cast<uint32_t>(parent) | (own << kOwnShift);
        }
        __syncwarp();
        if (__any_sync(~0u, t1 >= 0 || t2 >= 0)) {
            if (t1 >= 0) wunion(sm.word, p, t1, err);
            if (t2 >= 0) wunion(sm.word, p, t2, err);
        }
        __syncwarp();
    }

    // -- phase D: flatten, zone flags -----------------------------------------
    volatile uint32_t* vw = sm.word;
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        const bool active = i < nlist;
        int root = -1 - lane;   // inactive lanes form groups of their own
        uint32_t own = 0;
        if (active) {
            const int p = sm.list[i] & 1023;
            root = p;
#pragma unroll 1
            for (int it = 0; it < T * T; ++it) {
                const int upp = static_cast<int>(vw[root] & kParMask);
                if (upp == root) break;
                root = upp;
            }
            const uint32_t wp = vw[p];
            own = (wp >> kOwnShift) & 7u;
            if (root != p) {
                // p is not a root: no other lane writes its word now.
                vw[p] = (wp & ~kParMask) | static_cast<uint32_t>(root);
            }
        }
        const uint32_t group = __match_any_sync(~0u, root);
        uint32_t agg = 0u;
        agg |= (__ballot_sync(~0u, own & 1u) & group) ? 1u : 0u;
        agg |= (__ballot_sync(~0u, own & 2u) & group) ? 2u : 0u;
        agg |= (__ballot_sync(~0u, own & 4u) & group) ? 4u : 0u;
        if (active && lane == __ffs(group) - 1) {
            const uint32_t zf = (vw[root] >> kZoneShift) & 7u;
            if ((zf & agg) != agg) {
                atomicOr(sm.word + root, agg << kZoneShift);
            }
        }
    }
    __syncwarp();

    // -- phase E: records, masks of listed pixels, run log --------------------
    const int64_t frag_base = item * kSlots;
    uint32_t* plog = a.pending + item * kPendingCap;
    int nrec = 0;
    int nlog = 0;
    for (int base = 0; base < nlist; base += 32) {
        const int i = base + lane;
        const bool active = i < nlist;
        int p = 0;
        int root = 0;
        uint32_t z = 0;
        if (active) {
            p = sm.list[i] & 1023;
            root = static_cast<int>(vw[p] & kParMask);
            z = (vw[root] >> kZoneShift) & 7u;
        }
        const bool live =
            active && (z & kTouchesSeam) && (z & kDead) != kDead;
        const bool first = live && root == p;
        const uint32_t fb = __ballot_sync(~0u, first);
        if (first) {
            const int rec = nrec + __popc(fb & lt_mask);
            if (rec < kSlots) {
                atomicOr(sm.word + p, static_cast<uint32_t>(rec + 1)
                                          << kRecShift);
                const int64_t gi = frag_base + rec;
                a.parent[gi] = static_cast<int32_t>(gi);
                a.bits[gi] = (z & 3u) | ((z & 3u) << kLocalShift);
            } else {
                err = kErrFragmentOverflow;
            }
        }
        nrec += __popc(fb);
        __syncwarp();
        const int x = p & 31;
        const int y = p >> 5;
        if (active && !live) {
            const int64_t o = (g.y0 + y) * out_pitch + g.x0 + x;
            omax[o] = (z & kHasGreater) ? 0 : 255;
            omin[o] = (z & kHasSmaller) ? 0 : 255;
        }
        uint32_t rec1 = 0;
        if (live) {
            rec1 = (vw[root] >> kRecShift) & 0xFFu;
        }
        const bool logged = live && rec1 != 0u;
        // Run continuation: the previous lane holds the left neighbour in
        // the same zone (roots are equal exactly when zones are).
        const int prev_p = __shfl_up_sync(~0u, p, 1);
        const int prev_root = __shfl_up_sync(~0u, root, 1);
        const bool prev_logged = __shfl_up_sync(~0u, logged, 1);
        const bool cont = logged && lane > 0 && prev_logged &&
                          prev_p == p - 1 && x != 0 && prev_root == root;
        const bool head = logged && !cont;
        const uint32_t stops = __ballot_sync(~0u, !cont);
        const uint32_t hb = __ballot_sync(~0u, head);
        if (head) {
            const uint32_t later = stops & ~le_mask;
            const int end = later ? __ffs(later) - 1 : 32;
            plog[nlog + __popc(hb & lt_mask)] =
                pending_entry(static_cast<int>(rec1 - 1u), x, y, end - lane);
        }
        nlog += __popc(hb);
    }
    __syncwarp();

    // -- phase F: border records, seam items -----------------------------------
    uint8_t* border = a.border + item * kSlots;
    auto record_of = [&](int x, int y) -> uint32_t {
        if (!((sm.listed[y] >> x) & 1u)) {
            return kDeadRecord;   // a decided pixel
        }
        const int root = static_cast<int>(vw[y * T + x] & kParMask);
        const uint32_t w = vw[root];
        const uint32_t z = (w >> kZoneShift) & 7u;
        if ((z & kDead) == kDead) {
            return kDeadRecord;
        }
        const uint32_t r1 = (w >> kRecShift) & 0xFFu;
        return r1 ? r1 - 1u : kNoRecord;
    };
    // Staged pixel (x, y) of the tile, x and y in -1 .. T.
    auto px = [&](int x, int y) -> int {
        return sm.img[(y + 1) * kHaloW + x + 1];
    };
    // Seam items: every equal pair across a seam with a live pixel on this
    // side, as (own record, neighbour direction, neighbour border offset).
    // Pairs live on both sides are listed by both tiles; uniting twice is
    // harmless.  Corner pairs are listed by the top and bottom rows.
    uint32_t* items = a.seam_items + item * kSeamCap;
    int nitems = 0;
    auto emit = [&](bool ok, uint32_t rec, int dir, int off) {
        const uint32_t bal = __ballot_sync(~0u, ok);
        if (ok) {
            items[nitems + __popc(bal & lt_mask)] =
                rec | (static_cast<uint32_t>(off) << 8) |
                (static_cast<uint32_t>(dir) << 16);
        }
        nitems += __popc(bal);
    };
    {
        const int x = lane;
        const bool in_row = x < g.tw;
        const uint32_t rt = in_row ? record_of(x, 0) : kNoRecord;
        const uint32_t rb = in_row ? record_of(x, g.th - 1) : kNoRecord;
        if (in_row) {
            border[x] = static_cast<uint8_t>(rt);
            border[T + x] = static_cast<uint8_t>(rb);
        }
        const bool live_t = rt < static_cast<uint32_t>(kSlots);
        const bool live_b = rb < static_cast<uint32_t>(kSlots) &&
                            g.th == T && g.y0 + T < height;
        const int vt = px(x, 0);
        const int vb = px(x, T - 1);
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
            const int x2 = x + d;
            // Top row: neighbour row -1 of the top, top-left or top-right tile.
            const int dir_t = x2 < 0 ? kRelTopLeft
                                     : (x2 >= T ? kRelTopRight : kRelTop);
            const int off_t = T + (x2 < 0 ? T - 1 : (x2 >= T ? 0 : x2));
            emit(live_t && px(x2, -1) == vt, rt, dir_t, off_t);
            // Bottom row: neighbour row T of the lower tiles.
            const int dir_b = x2 < 0 ? kRelBottomLeft
                                     : (x2 >= T ? kRelBottomRight : kRelBottom);
            const int off_b = x2 < 0 ? T - 1 : (x2 >= T ? 0 : x2);
            emit(live_b && px(x2, T) == vb, rb, dir_b, off_b);
        }
    }
    {
        const int y = lane;
        const bool in_col = y < g.th;
        const uint32_t rl = in_col ? record_of(0, y) : kNoRecord;
        const uint32_t rr = in_col ? record_of(g.tw - 1, y) : kNoRecord;
        if (in_col) {
            border[2 * T + y] = static_cast<uint8_t>(rl);
            border[3 * T + y] = static_cast<uint8_t>(rr);
        }
        const bool live_l = rl < static_cast<uint32_t>(kSlots);
        const bool live_r = rr < static_cast<uint32_t>(kSlots) &&
                            g.tw == T && g.x0 + T < width;
        const int vl = px(0, y);
        const int vr = px(T - 1, y);
#pragma unroll
        for (int d = -1; d <= 1; ++d) {
            const int y2 = y + d;
            const bool inside = y2 >= 0 && y2 < g.th;   // corners: rows above
            emit(live_l && inside && px(-1, y2) == vl, rl, kRelLeft,
                 3 * T + y2);
            emit(live_r && inside && px(T, y2) == vr, rr, kRelRight,
                 2 * T + y2);
        }
    }
    if (lane == 0) {
        a.fragment_count[item] = static_cast<uint16_t>(min(nrec, kSlots));
        a.pending_count[item] = static_cast<uint32_t>(nlog);
        a.seam_count[item] = static_cast<uint32_t>(nitems);
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(item));
    }
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

__device__ __forceinline__ void seam_pass_warp32(const Source& src,
                                                 const Arena& a,
                                                 int64_t first) {
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
    for (uint32_t base = 0; base < total; base += 32) {
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
            const int off = static_cast<int>((it >> 8) & 0x7Fu);
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
                    fo = static_cast<int>(g * kSlots + rec);
                    target = static_cast<int>(ng * kSlots + rn);
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
__device__ __forceinline__ void flags_pass_warp32(const Source& src,
                                                  const Arena& a,
                                                  int64_t first) {
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
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t f = base + static_cast<uint32_t>(lane);
        const int owner = owner_of(excl, f);
        const uint32_t r = f - __shfl_sync(~0u, excl, owner);
        if (f < total) {
            const int fr = static_cast<int>((first + owner) * kSlots + r);
            const int root = global_find(a.parent, fr, err);
            if (root != fr) {
                const uint32_t own = ld_relaxed(a.bits + fr) & 3u;
                if (own && (ld_relaxed(a.bits + root) & own) != own) {
                    atomicOr(a.bits + root, own);
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

struct __align__(16) ResolveSmem {
    uint8_t final_flags[32][kSlots];
    uint8_t* maxima[32];
    uint8_t* minima[32];
    int64_t out_origin[32];   // offset of the tile's pixel (0, 0)
    int32_t out_pitch[32];
    int16_t tw[32];
    int16_t th[32];
    uint32_t live[T];         // one tile at a time: logged pixels per row,
    uint32_t vmax[T];         //   and those whose maxima / minima byte is 255
    uint32_t vmin[T];
};

// Rewrites the logged pixels of a full tile (32 x 32, rows and origins
// aligned to `vec` = 16, 8 or 4 bytes) from per-row bit masks: each lane
// takes one `vec`-byte piece of a row (32 / vec lanes per row, vec rows per
// step), loads it unless every byte is logged, replaces the logged bytes and
// stores it back.
__device__ __forceinline__ uint32_t merge4(uint32_t cur, uint32_t live,
                                          uint32_t verdict) {
    const uint32_t m = spread4(live);
    return (cur & ~m) | (spread4(verdict) & m);
}

__device__ __forceinline__ void merge_rows(uint8_t* omax, uint8_t* omin,
                                           int64_t pitch,
                                           const uint32_t* live,
                                           const uint32_t* vmax,
                                           const uint32_t* vmin, int vec) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int per_row = T / vec;
    const int c = lane % per_row;
    const int rr = lane / per_row;
    const uint32_t full = (vec == 16) ? 0xFFFFu : (vec == 8) ? 0xFFu : 0xFu;
    for (int r0 = 0; r0 < T; r0 += vec) {
        const int r = r0 + rr;
        const uint32_t lv = (live[r] >> (c * vec)) & full;
        if (lv == 0u) {
            continue;
        }
        const uint32_t bx = vmax[r] >> (c * vec);
        const uint32_t bn = vmin[r] >> (c * vec);
        const int64_t o = static_cast<int64_t>(r) * pitch + c * vec;
        const bool all = lv == full;
        if (vec == 16) {
            uint4* px = reinterpret_cast<uint4*>(omax + o);
            uint4* pn = reinterpret_cast<uint4*>(omin + o);
            const uint4 cx = all ? make_uint4(0u, 0u, 0u, 0u) : *px;
            const uint4 cn = all ? make_uint4(0u, 0u, 0u, 0u) : *pn;
            *px = make_uint4(merge4(cx.x, lv, bx), merge4(cx.y, lv >> 4, bx >> 4),
                             merge4(cx.z, lv >> 8, bx >> 8),
                             merge4(cx.w, lv >> 12, bx >> 12));
            *pn = make_uint4(merge4(cn.x, lv, bn), merge4(cn.y, lv >> 4, bn >> 4),
                             merge4(cn.z, lv >> 8, bn >> 8),
                             merge4(cn.w, lv >> 12, bn >> 12));
        } else if (vec == 8) {
            uint2* px = reinterpret_cast<uint2*>(omax + o);
            uint2* pn = reinterpret_cast<uint2*>(omin + o);
            const uint2 cx = all ? make_uint2(0u, 0u) : *px;
            const uint2 cn = all ? make_uint2(0u, 0u) : *pn;
            *px = make_uint2(merge4(cx.x, lv, bx), merge4(cx.y, lv >> 4, bx >> 4));
            *pn = make_uint2(merge4(cn.x, lv, bn), merge4(cn.y, lv >> 4, bn >> 4));
        } else {
            uint32_t* px = reinterpret_cast<uint32_t*>(omax + o);
            uint32_t* pn = reinterpret_cast<uint32_t*>(omin + o);
            *px = merge4(all ? 0u : *px, lv, bx);
            *pn = merge4(all ? 0u : *pn, lv, bn);
        }
    }
}

__device__ __forceinline__ void resolve_warp32(ResolveSmem& sm,
                                               const Source& src,
                                               const Arena& a, int64_t first) {
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int64_t tile = first + lane;
    const bool valid = lane < src.group && tile < src.total_tiles;
    const uint32_t n =
        valid ? min(a.pending_count[tile], static_cast<uint32_t>(kPendingCap))
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
    if (n) {
        const PlanImage job = load_job(src, tile);
        const TileGeom g = tile_geom(job, tile - job.tile_base);
        sm.maxima[lane] = job.maxima;
        sm.minima[lane] = job.minima;
        sm.out_origin[lane] =
            static_cast<int64_t>(g.y0) * job.out_pitch + g.x0;
        sm.out_pitch[lane] = job.out_pitch;
        sm.tw[lane] = static_cast<int16_t>(g.tw);
        sm.th[lane] = static_cast<int16_t>(g.th);
    }
    // Component flags of every live fragment of these tiles.
    uint32_t flipped = 0u;
    for (uint32_t base = 0; base < total_k; base += 32) {
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
    __syncwarp();
    // Tiles with few logged runs: all of the group's runs together, their
    // bytes spread over the lanes (consecutive lanes write consecutive bytes
    // of a run).
    const uint32_t n_sparse = n <= kSparseRuns ? n : 0u;
    uint32_t total_sparse = 0u;
    const uint32_t excl_s = warp_prefix(n_sparse, total_sparse);
    for (uint32_t base = 0; base < total_sparse; base += 32) {
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
                len = static_cast<uint32_t>(n_px);
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
            if (bi < bytes) {
                sm.maxima[tile_of][o] = static_cast<uint8_t>(vd);
                sm.minima[tile_of][o] = static_cast<uint8_t>(vd >> 8);
            }
        }
    }
    // Tiles with many logged runs, one at a time: their pixels and verdicts
    // as row masks, then the tile's rows rewritten (logged bytes replaced,
    // the others kept).
    for (int t = 0; t < src.group; ++t) {
        const uint32_t nt = __shfl_sync(~0u, n, t);
        if (nt <= kSparseRuns) {
            continue;
        }
        const uint32_t kt = __shfl_sync(~0u, k, t);
        sm.live[lane] = 0u;
        sm.vmax[lane] = 0u;
        sm.vmin[lane] = 0u;
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
            const uint32_t R = ((2u << (x + n_px - 1)) - 1u) & ~((1u << x) - 1u);
            atomicOr(&sm.live[y], R);
            if (!(fl & kHasGreater)) {
                atomicOr(&sm.vmax[y], R);
            }
            if (!(fl & kHasSmaller)) {
                atomicOr(&sm.vmin[y], R);
            }
        }
        __syncwarp();
        uint8_t* omax = sm.maxima[t] + sm.out_origin[t];
        uint8_t* omin = sm.minima[t] + sm.out_origin[t];
        const int64_t pitch = sm.out_pitch[t];
        const uint64_t align = reinterpret_cast<uint64_t>(omax) |
                               reinterpret_cast<uint64_t>(omin) |
                               static_cast<uint64_t>(pitch);
        int vec = (align & 15u) == 0 ? 16 : (align & 7u) == 0 ? 8
                : (align & 3u) == 0 ? 4 : 1;
        if (tw < T || th < T) {
            vec = 1;
        }
        if (vec > 1) {
            merge_rows(omax, omin, pitch, sm.live, sm.vmax, sm.vmin, vec);
        } else {
            for (int r = 0; r < th; ++r) {
                if ((sm.live[r] >> lane) & 1u) {
                    const int64_t o = static_cast<int64_t>(r) * pitch + lane;
                    omax[o] = ((sm.vmax[r] >> lane) & 1u) ? 255 : 0;
                    omin[o] = ((sm.vmin[r] >> lane) & 1u) ? 255 : 0;
                }
            }
        }
        __syncwarp();
    }
    if (lane == 0 && flipped) {
        atomicAdd(&a.header->flipped_tiles, __popc(flipped));
    }
    if (err) {
        raise_error(a.header, err, static_cast<uint32_t>(first));
    }
}

}  // namespace rowscan

}  // namespace ss
